"""Error paths of the engine through the C-ABI: non-finite values and the
bounded device waits.

The reference's band solvers print a message and carry on when a pivot is
tiny (src/SGTsh/dclib.f90:36-40, src/SGTpsv/dcsymbdl.f90:47-50), so their
outputs silently turn into Inf/NaN.  The library returns DSM_ERR_NONFINITE
instead and stays usable.  The NaN is planted in the set-up on the host;
nothing here faults or hangs the GPU: the tensor-core stall test withholds
one stage's copies so a bounded (20 ms) wait runs out, and the kernel
returns its error word."""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small
from conftest import rel_l2


def _plant_nan(setup, field, index):
    getattr(setup.s, field)[index] = float("nan")


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [dsmsgt.DSM_PREC_FP64, dsmsgt.DSM_PREC_MIXED])
def test_psv_nan_in_setup_returns_nonfinite(built, prec):
    s = dsmsgt.Setup(psv_small(), "psv")
    # the mass integral of a mantle element: its band rows, every pivot above
    # them and the cutoff probe become NaN
    _plant_nan(s, "solid_el", s.s.n_sel - 40)
    ctx = dsmsgt.Context(s, precision=prec)
    with pytest.raises(dsmsgt.DsmError) as ei:
        ctx.run([5, 9])
    assert ei.value.code == dsmsgt.DSM_ERR_NONFINITE, str(ei.value)
    assert "frequency index" in str(ei.value)
    # the context answers the next call with the same code (no stale state,
    # no hang), and a fresh context on a clean set-up works
    with pytest.raises(dsmsgt.DsmError) as ei:
        ctx.run([7])
    assert ei.value.code == dsmsgt.DSM_ERR_NONFINITE
    ctx.close()
    good = dsmsgt.Setup(psv_small(), "psv")
    c2 = dsmsgt.Context(good, precision=prec)
    t, r, y, llog = c2.run([5, 9])
    c2.close()
    assert np.all(np.isfinite(t)) and llog.min() > 0


@pytest.mark.gpu
def test_sh_nan_in_setup_returns_nonfinite(built):
    s = dsmsgt.Setup(sh_small(), "sh")
    _plant_nan(s, "t", 4 * (s.s.nnlayer // 2))
    ctx = dsmsgt.Context(s)
    with pytest.raises(dsmsgt.DsmError) as ei:
        ctx.run([3, 11])
    assert ei.value.code == dsmsgt.DSM_ERR_NONFINITE, str(ei.value)
    ctx.close()


@pytest.mark.gpu
def test_psv_nan_in_receiver_weights_is_caught_in_the_outputs(built):
    # a NaN that never reaches the cutoff probe (one receiver's position in
    # its interpolation stencil): the solves finish, the epilogue's check
    # of the outputs reports it
    s = dsmsgt.Setup(psv_small(), "psv")
    _plant_nan(s, "rrsta", 3 * 2 + 1)
    ctx = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_FP64)
    with pytest.raises(dsmsgt.DsmError) as ei:
        ctx.run([5])
    assert ei.value.code == dsmsgt.DSM_ERR_NONFINITE, str(ei.value)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["psv", "sh"])
def test_tensor_core_wait_times_out_and_context_recovers(built, mode):
    s = dsmsgt.Setup(psv_small() if mode == "psv" else sh_small(), mode)
    freqs = [4, 13]
    ctx = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED)
    want = ctx.run(freqs)
    ctx.debug_set("tc_stall", 1)
    with pytest.raises(dsmsgt.DsmError) as ei:
        ctx.run(freqs)
    assert ei.value.code == dsmsgt.DSM_ERR_TIMEOUT, str(ei.value)
    # the hook lasts one run: the same context computes the same results again
    got = ctx.run(freqs)
    ctx.close()
    assert list(got[3]) == list(want[3])
    for a, b in zip(got[:3], want[:3]):
        assert rel_l2(a, b) == 0.0


@pytest.mark.gpu
def test_debug_hook_rejects_fp64_and_unknown_names(built):
    s = dsmsgt.Setup(sh_small(), "sh")
    ctx = dsmsgt.Context(s)
    for name in ("tc_stall", "no_such_hook"):
        with pytest.raises(dsmsgt.DsmError) as ei:
            ctx.debug_set(name, 1)
        assert ei.value.code == dsmsgt.DSM_ERR_INVALID
    ctx.close()
