"""Parity at the benchmark's model and grid sizes.

* FP64 GPU path against the oracle on the P-SV benchmark model and grid of
  the 1024-frequency band (16 788 band rows, 201 receivers, cutoffs up to
  about 3 700), with the epicentral grid cut to 7 distances so that the
  oracle (its own set-up, all host threads) finishes in seconds.  Bar:
  1e-10 relative L2 per array and identical cutoffs.
* Mixed-precision path against the FP64 GPU path on the 2048-frequency band
  (33 560 band rows, 1 441 distances), on frequencies up to the top of the
  band (cutoffs near 7 000).  Bar: 1e-6 relative L2 per output component,
  identical cutoffs, finite outputs."""
import os
import sys

import numpy as np
import pytest

import dsmsgt
from conftest import rel_l2
from test_gpu_mixed import per_component

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from oracle import driver_setup, oracle as orc  # noqa: E402

TOL_FP64 = 1e-10
TOL_MIXED = 1e-6


def _cut_thetas(job, name, delta):
    w = bench.WORKLOADS[name]
    text = job.param_text.replace(f"0.0 180.0 {w['thdelta']!r}\n", f"0.0 180.0 {delta!r}\n")
    return dsmsgt.Job(text, job.conf_text, job.model_text)


@pytest.mark.gpu
def test_fp64_matches_oracle_on_benchmark_model_and_grid(built):
    job = _cut_thetas(bench.workload("psv1024")[0], "psv1024", 30.0)
    freqs = [1, 512, 1024]
    s = dsmsgt.Setup(job, "psv")
    assert s.n_unknowns == 16788 and s.theta_n == 7 and s.r_n == 201
    ctx = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_FP64, freq_batch=3)
    t, r, y, llog = ctx.run(freqs)
    ctx.close()
    threads = len(os.sched_getaffinity(0))
    ot, orr, oy, ollog, _, _ = orc.run_threads(driver_setup.psv_setup(job), freqs, threads)
    assert list(llog) == list(ollog), (llog, ollog)
    assert max(llog) > 3000
    for k, (a, b) in (("tsgt", (t, ot)), ("rsgt", (r, orr)), ("synn", (y, oy))):
        for i in range(len(freqs)):
            e = rel_l2(a[i], b[i])
            assert e <= TOL_FP64, (k, freqs[i], e)


@pytest.mark.gpu
def test_mixed_matches_fp64_to_the_top_of_the_2048_band(built):
    job, desc = bench.workload("psv2048")
    s = dsmsgt.Setup(job, "psv")
    assert s.theta_n == 1441 and s.n_unknowns == 33560
    freqs = [3, 700, 1400, 2048]
    c64 = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_FP64, freq_batch=len(freqs))
    t, r, y, llog = c64.run(freqs)
    c64.close()
    cm = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED, freq_batch=len(freqs))
    tm, rm, ym, llm = cm.run(freqs)
    cm.close()
    assert list(llm) == list(llog)
    assert max(llog) > 6000, llog
    for a in (tm, rm, ym):
        assert np.all(np.isfinite(a))
    for k, (a, b) in (("tsgt", (tm, t)), ("rsgt", (rm, r)), ("synn", (ym, y))):
        for i in range(len(freqs)):
            e = max(per_component(a[i:i + 1], b[i:i + 1]))
            assert e <= TOL_MIXED, (k, freqs[i], e)
