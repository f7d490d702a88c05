"""The oracle of KernelMaker's per-point isotropic kernels (calculateKernel's
isovpfreq / isovsfreq with bwfilt's Butterworth band-pass and the
trapezoid sum), pinned by identities that need no Fortran:

* the restated bpcoeff / rekurs is a band-pass with gain 1/sqrt(2) at both
  corner frequencies and 1 between them for even orders (the reference's
  single-precision pole casts move this by ~1e-7), and equals scipy's second-order-section
  filter with sections (a, 0, -a; 1, b1, b2);
* the frequency products: an isotropic (pressure) pair gives no Q_mu
  product and the P / S products of the strain-trace formulas; a pure
  shear pair gives -2 x^2 (S) and -4 x^2 jacobian (Q_mu);
* the kernel value is the trapezoid rule of coeff x filtered series over
  nt1..nt2, and the filtered series is rekurs of vectorFFT_double of the
  products."""
import numpy as np
import pytest
from scipy import signal

from oracle import catalogue as cat


@pytest.mark.parametrize("npoles", [2, 4, 6, 8, 10])
def test_bpcoeff_is_a_band_pass_with_half_power_corners(npoles):
    """Even orders (an odd order keeps one pole of a conjugate pair: the
    reference's sections are then not a Butterworth response)."""
    fs = 4.0
    f1, f2 = 0.05, 0.4
    a, b1, b2 = cat.bpcoeff(f1, f2, npoles, 1.0 / fs)
    sos = np.array([[a[i], 0.0, -a[i], 1.0, b1[i], b2[i]] for i in range(npoles)])
    # the bilinear transform's centre: the analogue corners are prewarped
    fc = fs / np.pi * np.arctan(np.sqrt(np.tan(np.pi * f1 / fs) * np.tan(np.pi * f2 / fs)))
    _, h = signal.sosfreqz(sos, worN=[f1, f2, fc], fs=fs)
    g = np.abs(h)
    assert abs(g[0] - 2 ** -0.5) < 2e-6 and abs(g[1] - 2 ** -0.5) < 2e-6, g
    assert abs(g[2] - 1.0) < 2e-6, g
    _, h = signal.sosfreqz(sos, worN=[f1 / 20, min(0.5 * fs * 0.99, f2 * 4)], fs=fs)
    assert np.all(np.abs(h) < 0.2)


def test_rekurs_equals_second_order_sections():
    a, b1, b2 = cat.bpcoeff(0.01, 0.05, 4, 0.5)
    x = np.random.default_rng(0).standard_normal((3, 400))
    y = cat.rekurs(x, a, b1, b2)
    sos = np.array([[a[i], 0.0, -a[i], 1.0, b1[i], b2[i]] for i in range(4)])
    ref = signal.sosfilt(sos, x)
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


def test_bpcoeff_rounds_the_poles_through_single_precision():
    """The reference's cmplx() casts: coefficients close to, but not equal
    to, a design with every pole in double precision."""
    a, b1, b2 = cat.bpcoeff(0.01, 0.05, 4, 0.5)
    d2 = 4.0
    w1, w2 = d2 * np.tan(2 * np.pi * 0.01 / d2), d2 * np.tan(2 * np.pi * 0.05 / d2)
    w0 = 0.5 * (w2 - w1)
    s = []
    for n in range(1, 5):
        p = np.exp(1j * (2 * n - 1 + 4) * np.pi / 8)
        t1 = p * w0
        t2 = np.sqrt(t1 * t1 - w1 * w2)
        s += [t1 + t2, t1 - t2]
    ad = np.array([2 * d2 * w0 / (d2 * d2 - d2 * 2 * z.real + abs(z) ** 2) for z in s[:4]])
    rel = np.abs(a - ad) / np.abs(ad)
    assert rel.max() > 0 and rel.max() < 1e-6


def _iso(x):
    h = np.zeros((6, x.size), np.complex128)
    h[0] = h[1] = h[2] = x
    return h


def test_products_of_pressure_and_shear_pairs():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    y = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    jac = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    u = cat.iso_products(_iso(x), _iso(y), jac, 3)
    assert np.allclose(u[0], -9.0 * x * y * 1e3, rtol=1e-14)      # -(3x)(3y)
    assert np.allclose(u[1], 6.0 * x * y * 1e3, rtol=1e-14)       # x (2y) three times
    assert np.abs(u[2]).max() <= 1e-12 * np.abs(u[1]).max()        # trace-free: no Q_mu term
    h3 = np.zeros((6, 16), np.complex128)
    h4 = np.zeros((6, 16), np.complex128)
    h3[3] = x
    h4[3] = y
    u = cat.iso_products(h3, h4, jac, 3)
    assert np.abs(u[0]).max() == 0.0
    assert np.allclose(u[1], -2.0 * x * y * 1e3, rtol=1e-14)
    assert np.allclose(u[2], -4.0 * x * y * jac * 1e3, rtol=1e-14)
    # types select the series
    assert cat.iso_products(h3, h4, jac, 1).shape == (1, 16)
    assert cat.iso_products(h3, h4, jac, 2).shape == (2, 16)


def _kparams(p, nr, nfilter, types, rng):
    nwin = p["iwin_end"] - p["iwin_start"] + 1
    nf = p["fmax"] - p["fmin"] + 1
    fs = 2 * p["np1"] / p["tlen"]
    return dict(types=types, nfilter=nfilter,
                fclp=[fs * 0.02 * (k + 1) for k in range(nfilter + 1)],
                fchp=[fs * 0.2 + fs * 0.02 * k for k in range(nfilter + 1)],
                npoles=4, sampling_hz=fs,
                nt1=[p["iwin_start"] + 5 + k for k in range(nfilter + 1)],
                nt2=[p["iwin_end"] - 7 - 2 * k for k in range(nfilter + 1)],
                nr=nr, nktype=8,
                coeff=rng.standard_normal((nwin, nr, 8, nfilter + 1)),
                jacobian=rng.standard_normal((nf, nr)) + 1j * rng.standard_normal((nf, nr)))


P = dict(fmin=0, fmax=48, np1=64, tlen=819.2, omegai=np.log(100.0) / 819.2, iwin_start=3, iwin_end=120)


def test_kernel_is_the_trapezoid_of_coeff_times_the_filtered_series():
    rng = np.random.default_rng(11)
    nf = P["fmax"] - P["fmin"] + 1
    kp = _kparams(P, 3, 1, 3, rng)
    ir = np.array([2, 0, 1, 2])
    h3 = rng.standard_normal((4, 6, nf)) + 1j * rng.standard_normal((4, 6, nf))
    h4 = rng.standard_normal((4, 6, nf)) + 1j * rng.standard_normal((4, 6, nf))
    ker, filt = cat.iso_kernels(P, kp, ir, h3, h4)
    assert ker.shape == (4, 2, 9) and filt.shape == (4, 3, 2, 118)
    jac = kp["jacobian"].T[ir]
    spec = cat.iso_products(h3, h4, jac, 3)
    du = cat.vector_fft_double(spec, P["fmin"], P["fmax"], P["np1"], P["omegai"], P["tlen"],
                               P["iwin_start"], P["iwin_end"])
    iws = P["iwin_start"]
    for f in range(2):
        a, b1, b2 = cat.bpcoeff(kp["fclp"][f], kp["fchp"][f], 4, 1.0 / kp["sampling_hz"])
        y = cat.rekurs(du, a, b1, b2)
        assert np.array_equal(filt[:, :, f], y)
        t1, t2 = kp["nt1"][f] - iws, kp["nt2"][f] - iws
        for pt in range(4):
            for s, ks in enumerate([(1, 3, 4), (5, 7), (8,)]):
                for k in ks:
                    c = kp["coeff"][:, ir[pt], k - 1, f]
                    want = np.trapezoid(c[t1:t2 + 1] * y[pt, s, t1:t2 + 1])
                    assert abs(ker[pt, f, k] - want) <= 1e-12 * max(1.0, abs(want))
        for k in (0, 2, 6):
            assert np.all(ker[:, f, k] == 0.0)


def _angles(rng, n):
    ph = rng.uniform(0, 2 * np.pi, (n, 3))            # phirq, phisq, phiqs
    cols = []
    for k in range(3):
        cols += [np.cos(ph[:, k]), np.sin(ph[:, k]), np.cos(2 * ph[:, k]), np.sin(2 * ph[:, k])]
    return np.stack(cols, axis=1)                       # crq, srq, crq2, srq2, csq, ..., sqs2


@pytest.mark.parametrize("compo", ["Z", "R", "T"])
def test_c_abi_h3h4_matrices_reproduce_the_reference_formulas(built, compo):
    """dsm_cat_h3h4_coef (host code, no device) against the oracle's
    rsgt2h3freq / tsgt2h4freq applied to spectra: the matrices times the
    components equal the formulas."""
    import dsmsgt
    rng = np.random.default_rng(ord(compo))
    ang = _angles(rng, 5)
    mt = rng.standard_normal(6)
    c3, c4 = dsmsgt.cat_h3h4_coef(ang, compo, mt)
    assert c3.shape == (5, 6, 10) and c4.shape == (5, 6, 20)
    for p in range(5):
        r = rng.standard_normal((10, 33)) + 1j * rng.standard_normal((10, 33))
        t = rng.standard_normal((20, 33)) + 1j * rng.standard_normal((20, 33))
        w3 = cat.rsgt2h3freq(r, ang[p], compo)
        w4 = cat.tsgt2h4freq(t, ang[p], mt)
        assert np.abs(c3[p] @ r - w3).max() <= 1e-13 * np.abs(w3).max()
        assert np.abs(c4[p] @ t - w4).max() <= 1e-13 * np.abs(w4).max()
    # each h4 row is linear in the moment tensor
    mt2 = rng.standard_normal(6)
    _, a = dsmsgt.cat_h3h4_coef(ang, compo, mt2)
    _, b = dsmsgt.cat_h3h4_coef(ang, compo, mt + 2.0 * mt2)
    assert np.abs(b - (c4 + 2.0 * a)).max() <= 1e-13 * np.abs(b).max()


def test_c_abi_h3h4_rejects_bad_arguments(built):
    import dsmsgt
    ang = _angles(np.random.default_rng(0), 2)
    with pytest.raises(dsmsgt.DsmError, match="compo"):
        dsmsgt.cat_h3h4_coef(ang, "X")
    bad = ang.copy()
    bad[1, 3] = np.inf
    with pytest.raises(dsmsgt.DsmError, match="non-finite"):
        dsmsgt.cat_h3h4_coef(bad, "Z")
