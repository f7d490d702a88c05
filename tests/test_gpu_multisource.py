"""Several source depths in one P-SV context (dsm_psv_create_multi): the band
of each (omega, l) is factored once and solved for every source.  Every
source's outputs must equal those of a context of that source alone, bit for
bit (the same operations run on the same numbers), and match the oracle run
on that source's own set-up; the reference takes one depth per run
(src/SGTpsv/others.f90:52-54)."""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small
from conftest import rel_l2

DEPTHS_R0 = (6361.0, 6071.0, 5771.0)  # 10, 300 and 600 km deep


def _setups(**kw):
    return [dsmsgt.Setup(psv_small(r0=r0, **kw), "psv") for r0 in DEPTHS_R0]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [dsmsgt.DSM_PREC_FP64, dsmsgt.DSM_PREC_MIXED])
def test_multisource_equals_single_source_contexts(built, prec):
    """Bit for bit without the depth cut-off (the mixed default is turned
    off on both sides: a context cuts at the deepest of its sources)."""
    setups = _setups()
    freqs = [2, 17, 40]
    mc = dsmsgt.MultiSourceContext(setups, precision=prec, freq_batch=2)
    mc.set_depth_cutoff(0.0)
    got = mc.run(freqs)
    mc.close()
    for s, g in zip(setups, got):
        c = dsmsgt.Context(s, precision=prec, freq_batch=2)
        c.set_depth_cutoff(0.0)
        want = c.run(freqs)
        c.close()
        assert list(g[3]) == list(want[3])
        for a, b in zip(g[:3], want[:3]):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_multisource_with_depth_cut_close_to_single_source_contexts(built):
    """With the mixed path's default cut-off, the shared cut (from the
    deepest source) moves each source's outputs by far less than the path's
    tolerance."""
    setups = _setups()
    freqs = [2, 17, 40]
    mc = dsmsgt.MultiSourceContext(setups, precision=dsmsgt.DSM_PREC_MIXED, freq_batch=2)
    got = mc.run(freqs)
    mc.close()
    for s, g in zip(setups, got):
        c = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED, freq_batch=2)
        want = c.run(freqs)
        c.close()
        assert list(g[3]) == list(want[3])
        for a, b in zip(g[:3], want[:3]):
            assert rel_l2(a, b) <= 1e-10


@pytest.mark.gpu
def test_multisource_matches_oracle(built):
    from oracle import driver_setup, oracle as orc
    setups = _setups(rdelta=700.0)
    freqs = [5, 33]
    mc = dsmsgt.MultiSourceContext(setups)
    got = mc.run(freqs)
    mc.close()
    for s, g in zip(setups, got):
        ot, orr, oy, ollog = orc.run(driver_setup.psv_setup(s.job), freqs, threads=8)
        assert list(g[3]) == list(ollog)
        for a, b in zip(g[:3], (ot, orr, oy)):
            assert rel_l2(a, b) <= 1e-10


@pytest.mark.gpu
def test_multisource_rejects_other_grids_and_single_run_call(built):
    a = dsmsgt.Setup(psv_small(r0=6071.0), "psv")
    b = dsmsgt.Setup(psv_small(r0=6071.0, seed=1), "psv")  # another model
    with pytest.raises(dsmsgt.DsmError) as ei:
        dsmsgt.MultiSourceContext([a, b])
    assert ei.value.code == dsmsgt.DSM_ERR_INVALID
    mc = dsmsgt.MultiSourceContext([a, dsmsgt.Setup(psv_small(r0=5771.0), "psv")])
    L = dsmsgt.lib()
    fl = np.array([3], np.int32)
    out = dsmsgt.Out()
    import ctypes as C
    rc = L.dsm_run_freqs(mc.h, fl.ctypes.data_as(C.POINTER(C.c_int)), 1, C.byref(out))
    assert rc == dsmsgt.DSM_ERR_INVALID
    mc.close()
