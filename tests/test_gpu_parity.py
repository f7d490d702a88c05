"""CUDA engine vs the FP64 oracle (the CPU restatement of the reference).

The plain FP64 path must match the oracle to 1e-10 relative L2 per output
array, with an identical realised cutoff (llog) per frequency.  The oracle
runs on its own set-up (oracle/driver_setup.py), built from the same job as
the engine's.
"""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small
from conftest import rel_l2

TOL_FP64 = 1e-10


def _compare(setup, freqs, ctx_kwargs=None, tol=TOL_FP64):
    from oracle import driver_setup, oracle as orc
    ctx = dsmsgt.Context(setup, **(ctx_kwargs or {}))
    t, r, y, llog = ctx.run(freqs)
    ot, orr, oy, ollog = orc.run(driver_setup.setup(setup.job, setup.mode), freqs, threads=8)
    assert list(llog) == list(ollog)
    errs = {"tsgt": rel_l2(t, ot), "rsgt": rel_l2(r, orr), "synn": rel_l2(y, oy)}
    for k, v in errs.items():
        assert v <= tol, (k, v, errs)
    assert np.all(np.isfinite(t))
    ctx.close()
    return errs


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sh_small_seed0", "psv_small_seed0", "psv_deep_seed1"])
def test_fp64_matches_golden(built, name):
    """The FP64 engine against the committed oracle fixtures."""
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_golden
    import cases
    mode, fn, kw, freqs = make_golden.CASES[name]
    g = np.load(os.path.join(here, "golden", name + ".npz"))
    s = dsmsgt.Setup(getattr(cases, fn)(**kw), mode)
    ctx = dsmsgt.Context(s)
    t, r, y, llog = ctx.run(freqs)
    ctx.close()
    assert list(llog) == list(g["llog"])
    for k, v in (("tsgt", t), ("rsgt", r), ("synn", y)):
        assert rel_l2(v, g[k]) <= TOL_FP64, k


@pytest.mark.gpu
def test_sh_fp64_matches_oracle(built):
    s = dsmsgt.Setup(sh_small(), "sh")
    errs = _compare(s, [1, 7, 16, 31])
    print(errs)


@pytest.mark.gpu
def test_sh_fp64_small_chunks(built):
    """Several speculative l chunks per frequency must give the same result."""
    s = dsmsgt.Setup(sh_small(seed=3), "sh")
    _compare(s, [5, 20], {"l_chunk": 64, "freq_batch": 2})


@pytest.mark.gpu
def test_psv_fp64_matches_oracle(built):
    """Solid inner core, fluid outer core (fluid receivers), mantle; poles included."""
    s = dsmsgt.Setup(psv_small(), "psv")
    errs = _compare(s, [1, 17, 50])
    print(errs)


@pytest.mark.gpu
def test_psv_fp64_deep_source_small_chunks(built):
    s = dsmsgt.Setup(psv_small(seed=2, r0=5771.0, rdelta=700.0), "psv")
    _compare(s, [4, 33], {"l_chunk": 64, "freq_batch": 1})


@pytest.mark.gpu
def test_psv_fp64_order_capacity_growth(built):
    """A coarse grid (imax = 16) with the top receiver 71 km below the source
    needs ~15 000 orders before the cutoff fires: the engine must grow its
    order capacity several times and still match the oracle."""
    s = dsmsgt.Setup(psv_small(imax=16, thdelta=45.0), "psv")
    _compare(s, [6], {"l_chunk": 1024, "freq_batch": 1})


@pytest.mark.gpu
def test_psv_fp64_receivers_all_solid(built):
    """Receivers in the mantle only (no fluid receiver rows in the field
    matrices) must match the oracle as well."""
    s = dsmsgt.Setup(psv_small(seed=1, rmin=3800.0, rdelta=400.0), "psv")
    _compare(s, [3, 29])
