"""The catalogue-consumer oracle (KernelMaker's rdsgtomega / clsgt /
vectorFFT_double restatement) against identities that pin it without the
Fortran: the DFT definition for the restated cdft, hand-derived single-line
spectra, interpolation at catalogue nodes, the KernelMaker example's
transform length; plus the C-ABI's argument checks (no device needed)."""
import ctypes as C

import numpy as np
import pytest

import dsmsgt
from oracle import catalogue as cat


@pytest.mark.parametrize("N", [2, 4, 8, 32, 256, 4096])
def test_restated_cdft_is_the_unnormalised_inverse_dft(N):
    rng = np.random.default_rng(N)
    x = rng.standard_normal((3, N)) + 1j * rng.standard_normal((3, N))
    k = np.arange(N)
    dft = x @ np.exp(2j * np.pi * np.outer(k, k) / N)          # X_k = sum_n x_n e^{+2 pi i n k / N}
    got = cat.cdft(x)
    assert np.abs(got - dft).max() <= 1e-12 * np.abs(dft).max()


def test_transform_length_of_the_kernelmaker_example():
    # kernel.inf.in of the single-kernel example: 2 Hz, window 400-460 s;
    # catalogue tlen 3276.8 s, imax 2048
    np1, shz, s0, s1 = cat.transform_length(3276.8, 2048, 2.0, 400.0, 460.0)
    assert (np1, s0, s1) == (2048, 500, 575) and shz == 1.25
    np1, shz, s0, s1 = cat.transform_length(1638.4, 256, 20.0, 0.0, 100.0)
    assert np1 == 256 * 64 and shz == 2 * np1 / 1638.4


def test_c_abi_transform_length_matches(built):
    for args in [(3276.8, 2048, 2.0, 400.0, 460.0), (1638.4, 256, 20.0, 0.0, 100.0),
                 (3276.8, 1000, 5.0, 10.0, 1200.0), (100.0, 1, 1.0, 0.0, 1.0)]:
        assert dsmsgt.cat_np1(*args) == cat.transform_length(*args)


def test_find_idelta_region_clips_at_both_ends():
    assert cat.find_idelta_region(1, 10, 100) == (1, 21)
    assert cat.find_idelta_region(100, 10, 100) == (80, 100)
    assert cat.find_idelta_region(50, 10, 100) == (40, 60)
    assert cat.find_idelta_region(5, 10, 12) == (1, 12)


def _params(**kw):
    p = dict(num=4, theta_n=41, theta_min=10.0, theta_delta=0.5, fmin=0, fmax=32, np1=32, tlen=409.6,
             omegai=np.log(100.0) / 409.6, ipdistance=4.0, c_red_reci=0.0, iwin_start=0, iwin_end=63)
    p.update(kw)
    return p


def test_single_frequency_line_gives_a_damped_cosine():
    """Records nonzero only at index i0 and constant over distance: the
    interpolation returns the constant; the Hermitian extension makes the
    transform 2 Re(a e^{2 pi i i0 t / N}); the window multiplies by
    exp(omegai t / sHz) / tlen * 1e3."""
    p = _params()
    i0, a = 5, 0.75 - 0.4j
    nf, N = p["fmax"] - p["fmin"] + 1, 2 * p["np1"]
    rec = np.zeros((nf, p["theta_n"], p["num"]), np.complex64)
    rec[i0 - p["fmin"], :, 2] = a
    out = cat.series(p, [(rec, np.arange(4), np.ones(4))], [17.3])
    t = np.arange(p["iwin_start"], p["iwin_end"] + 1)
    shz = N / p["tlen"]
    a32 = complex(np.complex64(a)) * 1e-21
    want = 2 * np.real(a32 * np.exp(2j * np.pi * i0 * t / N)) * np.exp(p["omegai"] * t / shz) / p["tlen"] * 1e3
    assert np.abs(out[0, 2] - want).max() <= 1e-12 * np.abs(want).max()
    assert np.abs(out[0, [0, 1, 3]]).max() == 0.0


def test_interpolation_at_a_node_returns_the_record_and_cancels_the_reduction_phase():
    p = _params(c_red_reci=12.5)
    rng = np.random.default_rng(3)
    nf = p["fmax"] - p["fmin"] + 1
    rec = (rng.standard_normal((nf, p["theta_n"], 4)) + 1j * rng.standard_normal((nf, p["theta_n"], 4)))
    theta = p["theta_min"] + np.arange(p["theta_n"]) * p["theta_delta"]
    om = cat.omega_sgt([(rec, np.arange(4), np.ones(4))], 4, p["fmin"], p["fmax"], theta, p["tlen"],
                       p["c_red_reci"])
    k = 23
    f = cat.clsgt(theta[k], om, p["fmin"], p["theta_min"], p["theta_delta"], p["ipdistance"], p["tlen"],
                  p["c_red_reci"])
    want = rec[:, k, :] * 1e-21
    want[0] = 0.0                      # index 0 is never read
    assert np.abs(f - want).max() <= 1e-13 * np.abs(want).max()


def test_rdsgtomega_maps_and_halvings():
    assert list(np.nonzero(cat.kind_scale(cat.SYNN_PSV, 10) != 1)[0]) == [1, 7, 8, 9]
    assert list(np.nonzero(cat.kind_scale(cat.SYNN_SH, 5) != 1)[0]) == [2, 3, 4]
    assert list(cat.kind_dst(cat.TSGT_SH, 10)) == [6] + list(range(11, 20))
    assert list(cat.kind_dst(cat.RSGT_SH, 5)) == [5, 6, 7, 8, 9]


def test_hermitian_extension_rule():
    """vectorFFT_double writes cvec(np1+i) = conj(cvec(np1-i)) for
    i = imin..np1-1 in order; with imin = 0 index np1 is conjugated in place."""
    np1 = 8
    cc = np.arange(1, 10) + 1j * np.arange(11, 20)        # imin 0 .. imax 8 = np1
    x = cat.hermitian_extend(cc, 0, 8, np1)
    assert x[np1] == np.conj(cc[8])
    assert all(x[np1 + i] == np.conj(x[np1 - i]) for i in range(1, np1))
    cc2 = np.arange(1, 6) + 1j                             # imin 3 .. imax 7
    x2 = cat.hermitian_extend(cc2, 3, 7, np1)
    assert np.all(x2[np1:np1 + 3] == 0)                     # np1, np1+1, np1+2 stay zero
    assert all(x2[np1 + i] == np.conj(x2[np1 - i]) for i in range(3, np1))


def test_c_abi_rejects_bad_parameters_without_a_device(built):
    import torch
    L = dsmsgt.lib()
    base = dict(_params(), device=0)
    bad = [dict(np1=48), dict(np1=16), dict(iwin_end=64), dict(iwin_start=-1), dict(num=33),
           dict(fmin=5, fmax=4), dict(theta_delta=0.0), dict(ipdistance=600.0)]
    for b in bad:
        q = dict(base, **b)
        h = C.c_void_p()
        rc = L.dsm_cat_create(C.byref(dsmsgt.CatParams(**q)), C.byref(h))
        assert rc == 1, (b, rc)
        assert h.value is None
    if not torch.cuda.is_available():
        h = C.c_void_p()
        rc = L.dsm_cat_create(C.byref(dsmsgt.CatParams(**base)), C.byref(h))
        assert rc == 7 and b"device" in L.dsm_cat_last_error(None)
