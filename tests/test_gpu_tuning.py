"""Run-time tile shapes (dsm_set_tuning, dsm_autotune) and requests of
several contexts run together (dsm_run_request).

The tile shapes change how the work is staged, not the arithmetic of an
(omega, l) system, so FP64 outputs are bit-identical across them.  A
request runs each context on its own host thread and streams; every
context's outputs equal those of the same context run alone, bit for bit.
Neither has a counterpart in the reference, which runs one model and one
depth per MPI job (src/SGTpsv/SGTpsv-MPI.f90, src/SGTsh/SGTsh-MPI.f90)."""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small


def _same(a, b):
    assert list(a[3]) == list(b[3])
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_fp64_outputs_identical_across_tile_shapes(built):
    s = dsmsgt.Setup(psv_small(), "psv")
    freqs = [1, 20, 47, 64]
    ctx = dsmsgt.Context(s, freq_batch=3)
    t0 = ctx.tuning()
    assert t0["fac_rows"] == 16 and t0["fld_orders"] == 32 and t0["fwd_merge"] == 1
    want = ctx.run(freqs)
    for fr in (8, 16):
        for fo in (16, 32):
            for fm in (0, 1):
                ctx.set_tuning(fac_rows=fr, fld_orders=fo, fwd_merge=fm)
                _same(ctx.run(freqs), want)
    ctx.close()


@pytest.mark.gpu
def test_set_tuning_rejects_other_shapes(built):
    ctx = dsmsgt.Context(dsmsgt.Setup(psv_small(), "psv"))
    for bad in ({"fac_rows": 12}, {"fld_orders": 64}, {"tc_orders": 16}, {"fwd_merge": 2}):
        with pytest.raises(dsmsgt.DsmError) as ei:
            ctx.set_tuning(**bad)
        assert ei.value.code == dsmsgt.DSM_ERR_INVALID
    assert ctx.tuning()["fac_rows"] == 16
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [dsmsgt.DSM_PREC_FP64, dsmsgt.DSM_PREC_MIXED])
def test_autotune_keeps_a_valid_shape(built, prec):
    s = dsmsgt.Setup(psv_small(), "psv")
    freqs = [3, 30, 60]
    ctx = dsmsgt.Context(s, precision=prec, freq_batch=2)
    ref = dsmsgt.Context(s, freq_batch=2)
    want = ref.run(freqs)
    ref.close()
    t, ms = ctx.autotune(freqs, reps=1)
    assert ms > 0.0
    assert t == ctx.tuning()
    assert t["fac_rows"] in (8, 16) and t["fld_orders"] in (16, 32) and t["tc_orders"] in (32, 64)
    assert t["fwd_merge"] in (0, 1)
    got = ctx.run(freqs)
    ctx.close()
    assert list(got[3]) == list(want[3])
    tol = 0.0 if prec == dsmsgt.DSM_PREC_FP64 else 1e-5
    for a, b in zip(got[:3], want[:3]):
        err = np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2))
        assert err <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [dsmsgt.DSM_PREC_FP64, dsmsgt.DSM_PREC_MIXED])
def test_request_equals_contexts_run_alone(built, prec):
    psv_depths = [dsmsgt.Setup(psv_small(r0=r0), "psv") for r0 in (6361.0, 5771.0)]
    psv_other = dsmsgt.Setup(psv_small(seed=2), "psv")
    sh = dsmsgt.Setup(sh_small(seed=1), "sh")
    fl_psv, fl_sh = [2, 31, 64], [1, 9, 17, 32]

    def contexts():
        return [dsmsgt.MultiSourceContext(psv_depths, precision=prec, freq_batch=2),
                dsmsgt.Context(psv_other, precision=prec, freq_batch=2),
                dsmsgt.Context(sh, precision=prec, freq_batch=2)]

    lists = [fl_psv, fl_psv, fl_sh]
    alone = contexts()
    want = [alone[0].run(fl_psv), [alone[1].run(fl_psv)], [alone[2].run(fl_sh)]]
    for c in alone:
        c.close()
    together = contexts()
    got = dsmsgt.run_request(together, lists)
    for c in together:
        c.close()
    assert len(got) == 3 and len(got[0]) == 2
    for g, w in zip(got, want):
        for gs, ws in zip(g, w):
            _same(gs, ws)


@pytest.mark.gpu
def test_request_rejects_a_context_twice(built):
    ctx = dsmsgt.Context(dsmsgt.Setup(sh_small(), "sh"))
    with pytest.raises(dsmsgt.DsmError) as ei:
        dsmsgt.run_request([ctx, ctx], [[1], [2]])
    assert ei.value.code == dsmsgt.DSM_ERR_INVALID
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["psv", "sh"])
def test_mixed_outputs_identical_across_lsum_groups(built, mode, monkeypatch):
    """The mixed l-sum runs in frequency groups (split, tensor-core
    contraction and epilogue of different groups on three streams); the
    grouping changes only the order of the launches, so the outputs are
    bit-identical for any group count, with and without complex64 records."""
    s = dsmsgt.Setup(psv_small() if mode == "psv" else sh_small(), mode)
    freqs = [1, 9, 20, 33, 47, 64]
    runs = []
    for g in ("1", "2", "4", "8"):
        monkeypatch.setenv("DSM_LSUM_GROUPS", g)
        ctx = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED, freq_batch=6)
        runs.append((ctx.run(freqs), ctx.run(freqs, want32=True)))
        ctx.close()
    for r, r32 in runs[1:]:
        _same(r, runs[0][0])
        _same(r32[:4], runs[0][1][:4])
        for x, y in zip(r32[4], runs[0][1][4]):
            assert np.array_equal(x, y)
