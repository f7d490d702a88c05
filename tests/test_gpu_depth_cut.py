"""Depth cut-off of the P-SV band (dsm_set_depth_cutoff).

The reference factors every (omega, l) band from the centre
(src/SGTpsv/SGTpsv-MPI.f90:658-662).  With the cut-off, rows where a WKB bound
on the solution's amplitude relative to the source falls below `bound` leave
the system; the outputs then change by about bound^2 relative.  These tests
run the FP64 path with and without the cut-off (so only the cut-off
differs), on the small model and on the 2048-frequency benchmark grid, and
check the bound's validation.  The mixed path's default (cut-off on) is
measured against the FP64 path by tests/test_gpu_scale.py."""
import os
import sys

import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small
from conftest import rel_l2

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

TOL = 1e-12


def _compare(setup, freqs, bound, fb):
    a = dsmsgt.Context(setup, precision=dsmsgt.DSM_PREC_FP64, freq_batch=fb)
    want = a.run(freqs)
    a.close()
    b = dsmsgt.Context(setup, precision=dsmsgt.DSM_PREC_FP64, freq_batch=fb)
    b.set_depth_cutoff(bound)
    got = b.run(freqs)
    b.close()
    assert list(got[3]) == list(want[3])
    errs = []
    for x, y in zip(got[:3], want[:3]):
        assert np.all(np.isfinite(x))
        for i in range(len(freqs)):
            errs.append(rel_l2(x[i], y[i]))
    return max(errs)


@pytest.mark.gpu
def test_cut_changes_small_model_below_tolerance(built):
    s = dsmsgt.Setup(psv_small(r0=6071.0, rdelta=250.0), "psv")
    assert _compare(s, [1, 16, 40, 64], 1e-20, 4) <= TOL


@pytest.mark.gpu
def test_cut_changes_benchmark_grid_below_tolerance(built):
    job, _ = bench.workload("psv2048")
    w = bench.WORKLOADS["psv2048"]
    job = dsmsgt.Job(job.param_text.replace(f"0.0 180.0 {w['thdelta']!r}\n", "0.0 180.0 30.0\n"),
                     job.conf_text, job.model_text)
    s = dsmsgt.Setup(job, "psv")
    assert s.n_unknowns == 33560
    assert _compare(s, [3, 700, 1400, 2048], 1e-20, 4) <= TOL


@pytest.mark.gpu
def test_cut_bound_validation(built):
    c = dsmsgt.Context(dsmsgt.Setup(psv_small(), "psv"))
    for bad in (-1.0, 1.0, 2.0, float("nan")):
        with pytest.raises(dsmsgt.DsmError) as ei:
            c.set_depth_cutoff(bad)
        assert ei.value.code == dsmsgt.DSM_ERR_INVALID
    c.set_depth_cutoff(0.0)
    c.close()
    h = dsmsgt.Context(dsmsgt.Setup(sh_small(), "sh"))
    with pytest.raises(dsmsgt.DsmError):
        h.set_depth_cutoff(1e-20)
    h.close()


@pytest.mark.gpu
def test_mixed_row_tiles_stop_at_last_nonzero_order(built):
    """With the cut a deep receiver's fields are exactly zero above an order
    that grows with its radius; the mixed contraction's row tiles (a few
    neighbouring receivers each) stop at their rows' last nonzero order.
    On the benchmark grid that leaves well under the dense products, the
    outputs still match the FP64 path to the mixed path's tolerance, also
    without the cut (where only fields that underflow FP32 are zero), and
    the executed products never exceed the dense ones padded to whole
    64-order blocks."""
    job, _ = bench.workload("psv2048")
    w = bench.WORKLOADS["psv2048"]
    job = dsmsgt.Job(job.param_text.replace(f"0.0 180.0 {w['thdelta']!r}\n", "0.0 180.0 30.0\n"),
                     job.conf_text, job.model_text)
    s = dsmsgt.Setup(job, "psv")
    freqs = [700, 2048]
    ref = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_FP64, freq_batch=2)
    want = ref.run(freqs)
    ref.close()
    c = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED, freq_batch=2)
    c.set_profiling(True)
    got = c.run(freqs)
    st = c.stats()
    assert st.lsum_flops > 0 and st.lsum_flops_exec < 0.8 * st.lsum_flops, (st.lsum_flops_exec, st.lsum_flops)
    assert list(got[3]) == list(want[3])
    for x, y in zip(got[:3], want[:3]):
        for i in range(len(freqs)):
            assert rel_l2(x[i], y[i]) <= 1e-6
    assert st.lsum_flops_exec <= 1.05 * st.lsum_flops
    c.set_depth_cutoff(0.0)
    got = c.run(freqs)
    st = c.stats()
    assert 0 < st.lsum_flops_exec <= 1.05 * st.lsum_flops
    assert list(got[3]) == list(want[3])
    for x, y in zip(got[:3], want[:3]):
        for i in range(len(freqs)):
            assert rel_l2(x[i], y[i]) <= 1e-6
    c.close()
