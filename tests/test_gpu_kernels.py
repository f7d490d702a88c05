"""Per-point isotropic kernels on the device (dsm_cat_set_kernel_params,
dsm_cat_kernels: calculateKernel's isovpfreq / isovsfreq, the Butterworth
filter of bwfilt and the trapezoid sum) against the oracle restatement.

Bar: 1e-10 relative L2 on every point's tmpker and on the filtered series
(FP64 throughout; the differences are the transform's rounding carried
through the recursive filter).  Cases: both kernel families and each alone,
several filters with their own integration windows (nt1 = nt2 included),
1, 4 and 10 filter sections, points at several radii, host and device
spectra and outputs, batches split by the buffer limit (identical results),
the composition with dsm_cat_spectra on a record set, a larger transform,
and argument checks that leave the handle usable."""
import numpy as np
import pytest

import dsmsgt
from conftest import rel_l2

TOL = 1e-10


def _params(**kw):
    p = dict(num=20, theta_n=61, theta_min=0.0, theta_delta=0.5, fmin=0, fmax=48, np1=64, tlen=819.2,
             omegai=np.log(100.0) / 819.2, ipdistance=5.0, c_red_reci=0.0, iwin_start=3, iwin_end=120)
    p.update(kw)
    return p


def _kparams(p, nr, nfilter, types, rng, npoles=4):
    nwin = p["iwin_end"] - p["iwin_start"] + 1
    nf = p["fmax"] - p["fmin"] + 1
    fs = 2 * p["np1"] / p["tlen"]
    nt1 = [p["iwin_start"] + 5 + k for k in range(nfilter + 1)]
    nt2 = [p["iwin_end"] - 7 - 2 * k for k in range(nfilter + 1)]
    if nfilter >= 2:
        nt2[2] = nt1[2]                     # a one-sample window: both half weights
    return dict(types=types, nfilter=nfilter,
                fclp=[fs * 0.02 * (k + 1) for k in range(nfilter + 1)],
                fchp=[fs * 0.2 + fs * 0.02 * k for k in range(nfilter + 1)],
                npoles=npoles, sampling_hz=fs, nt1=nt1, nt2=nt2,
                coeff=rng.standard_normal((nwin, nr, 8, nfilter + 1)),
                jacobian=rng.standard_normal((nf, nr)) + 1j * rng.standard_normal((nf, nr)))


def _spectra(rng, npoint, nf):
    shp = (npoint, 6, nf)
    return (rng.standard_normal(shp) + 1j * rng.standard_normal(shp),
            rng.standard_normal(shp) + 1j * rng.standard_normal(shp))


def _oracle(p, kp, ir, h3, h4):
    from oracle import catalogue as cat
    q = dict(kp, nr=kp["coeff"].shape[1], nktype=kp["coeff"].shape[2])
    return cat.iso_kernels(p, q, ir, h3, h4)


def _device(p, kp, ir, h3, h4, batch_bytes=None):
    c = dsmsgt.Catalogue(p)
    if batch_bytes:
        c.set_batch_bytes(batch_bytes)
    c.set_kernel_params(kp["types"], kp["nfilter"], kp["fclp"], kp["fchp"], kp["npoles"], kp["sampling_hz"],
                        kp["nt1"], kp["nt2"], kp["coeff"], kp["jacobian"])
    ker, filt = c.kernels(ir, h3, h4, filtered=True)
    c.close()
    return ker, filt


def _check(got, want):
    ker, filt = got
    wk, wf = want
    assert ker.shape == wk.shape and filt.shape == wf.shape
    assert rel_l2(filt, wf) <= TOL
    assert rel_l2(ker, wk) <= TOL
    for k in range(ker.shape[0]):
        assert rel_l2(ker[k], wk[k]) <= TOL, k
    assert np.all(ker[wk == 0.0] == 0.0)     # types not computed stay zero


@pytest.mark.gpu
@pytest.mark.parametrize("types", [1, 2, 3])
@pytest.mark.parametrize("npoles", [1, 4, 10])
def test_kernels_match_oracle(built, types, npoles):
    rng = np.random.default_rng(100 + 10 * types + npoles)
    p = _params()
    nf = p["fmax"] - p["fmin"] + 1
    kp = _kparams(p, 4, 2, types, rng, npoles)
    ir = np.array([0, 3, 1, 1, 2, 3, 0])
    h3, h4 = _spectra(rng, ir.size, nf)
    _check(_device(p, kp, ir, h3, h4), _oracle(p, kp, ir, h3, h4))


@pytest.mark.gpu
def test_kernels_partial_spectrum_and_batches(built):
    rng = np.random.default_rng(7)
    p = _params(fmin=5, fmax=64, iwin_start=0, iwin_end=127)
    nf = p["fmax"] - p["fmin"] + 1
    kp = _kparams(p, 2, 1, 3, rng)
    ir = rng.integers(0, 2, 37)
    h3, h4 = _spectra(rng, ir.size, nf)
    want = _oracle(p, kp, ir, h3, h4)
    one = _device(p, kp, ir, h3, h4)
    _check(one, want)
    # one point per batch: the same kernels and series, bit for bit
    small = _device(p, kp, ir, h3, h4, batch_bytes=1 << 20)
    assert np.array_equal(one[0], small[0]) and np.array_equal(one[1], small[1])


@pytest.mark.gpu
def test_kernels_device_pointers_and_spectra_composition(built):
    import torch
    rng = np.random.default_rng(9)
    p = _params(c_red_reci=6.0)
    nf = p["fmax"] - p["fmin"] + 1
    rec = (rng.standard_normal((nf, p["theta_n"], 20)) + 1j * rng.standard_normal((nf, p["theta_n"], 20)))
    dist = np.array([1.3, 7.25, 12.0, 29.0])
    coef3 = rng.standard_normal((dist.size, 6, 20))
    coef4 = rng.standard_normal((dist.size, 6, 20))
    c = dsmsgt.Catalogue(p)
    c.add(rec.astype(np.complex64))
    h3 = c.spectra(dist, coef3)
    h4 = c.spectra(dist, coef4)
    kp = _kparams(p, 3, 0, 3, rng)
    c.set_kernel_params(kp["types"], kp["nfilter"], kp["fclp"], kp["fchp"], kp["npoles"], kp["sampling_hz"],
                        kp["nt1"], kp["nt2"], kp["coeff"], kp["jacobian"])
    ir = np.array([2, 0, 1, 2])
    host = c.kernels(ir, h3, h4, filtered=True)
    _check(host, _oracle(p, kp, ir, h3, h4))
    d3 = torch.from_numpy(h3).cuda()
    d4 = torch.from_numpy(h4).cuda()
    dev = c.kernels(ir, d3, d4, filtered=True)
    assert np.array_equal(host[0], dev[0]) and np.array_equal(host[1], dev[1])
    # device outputs through the C-ABI directly
    ko = torch.zeros(host[0].shape, dtype=torch.float64, device="cuda")
    fo = torch.zeros(host[1].shape, dtype=torch.float64, device="cuda")
    irr = np.ascontiguousarray(ir, np.int32)
    rc = dsmsgt.lib().dsm_cat_kernels(c.h, ir.size, dsmsgt._ptr(irr, dsmsgt._ip), d3.data_ptr(), d4.data_ptr(), 1,
                                      ko.data_ptr(), fo.data_ptr(), 1)
    assert rc == 0
    assert np.array_equal(ko.cpu().numpy(), host[0]) and np.array_equal(fo.cpu().numpy(), host[1])
    c.close()


@pytest.mark.gpu
def test_kernels_larger_transform(built):
    rng = np.random.default_rng(21)
    p = _params(fmax=700, np1=1024, tlen=3276.8, omegai=np.log(100.0) / 3276.8, iwin_start=100,
                iwin_end=1800)
    nf = p["fmax"] - p["fmin"] + 1
    kp = _kparams(p, 5, 3, 3, rng)
    ir = rng.integers(0, 5, 96)
    h3, h4 = _spectra(rng, ir.size, nf)
    _check(_device(p, kp, ir, h3, h4), _oracle(p, kp, ir, h3, h4))


@pytest.mark.gpu
def test_kernels_reject_bad_calls_and_stay_usable(built):
    rng = np.random.default_rng(4)
    p = _params()
    nf = p["fmax"] - p["fmin"] + 1
    kp = _kparams(p, 2, 0, 3, rng)
    h3, h4 = _spectra(rng, 2, nf)
    c = dsmsgt.Catalogue(p)
    with pytest.raises(dsmsgt.DsmError, match="set_kernel_params has not been called"):
        c._ker_shape, c._ker_ns = (1, 9), 3
        c.kernels([0, 1], h3, h4)

    def setp(**kw):
        q = dict(kp)
        q.update(kw)
        c.set_kernel_params(q["types"], q["nfilter"], q["fclp"], q["fchp"], q["npoles"], q["sampling_hz"],
                            q["nt1"], q["nt2"], q["coeff"], q["jacobian"])

    with pytest.raises(dsmsgt.DsmError, match="npoles"):
        setp(npoles=11)
    with pytest.raises(dsmsgt.DsmError, match="nt1/nt2"):
        setp(nt1=[p["iwin_start"] - 1])
    with pytest.raises(dsmsgt.DsmError, match="nt1/nt2"):
        setp(nt1=[50], nt2=[40])
    with pytest.raises(dsmsgt.DsmError, match="jacobianFuji"):
        setp(jacobian=None)
    bad = kp["coeff"].copy()
    bad[3, 1, 4, 0] = np.nan
    with pytest.raises(dsmsgt.DsmError, match="non-finite coeff"):
        setp(coeff=bad)
    setp()
    with pytest.raises(dsmsgt.DsmError, match="radius index"):
        c.kernels([0, 2], h3, h4)
    ker, filt = c.kernels([1, 0], h3, h4, filtered=True)
    want = _oracle(p, kp, np.array([1, 0]), h3, h4)
    _check((ker, filt), want)
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("compo", ["Z", "T"])
def test_calculate_kernel_end_to_end(built, compo):
    """calculateKernel for points of one radius from the records: the RSGT
    catalogue interpolated at each point's receiver distance with the
    rsgt2h3freq matrices, the TSGT catalogue at its source distance with the
    tsgt2h4freq matrices (dsm_cat_h3h4_coef), then dsm_cat_kernels; against
    the oracle's clsgt, rsgt2h3freq, tsgt2h4freq and iso_kernels."""
    from oracle import catalogue as cat
    rng = np.random.default_rng(55)
    pr = _params(num=10, c_red_reci=4.0)
    pt = _params(num=20, c_red_reci=4.0)
    nf = pr["fmax"] - pr["fmin"] + 1
    shp = (nf, pr["theta_n"])
    rrec = (rng.standard_normal(shp + (10,)) + 1j * rng.standard_normal(shp + (10,))).astype(np.complex64)
    trec = (rng.standard_normal(shp + (20,)) + 1j * rng.standard_normal(shp + (20,))).astype(np.complex64)
    npt = 6
    deltar = rng.uniform(2.0, 28.0, npt)
    deltas = rng.uniform(2.0, 28.0, npt)
    ph = rng.uniform(0, 2 * np.pi, (npt, 3))
    ang = np.stack([f(m * ph[:, k]) for k in range(3) for m, f in ((1, np.cos), (1, np.sin), (2, np.cos), (2, np.sin))],
                   axis=1)
    mt = rng.standard_normal(6)
    c3, c4 = dsmsgt.cat_h3h4_coef(ang, compo, mt)
    cr = dsmsgt.Catalogue(pr)
    cr.add(rrec)
    ct = dsmsgt.Catalogue(pt)
    ct.add(trec)
    h3 = cr.spectra(deltar, c3)
    h4 = ct.spectra(deltas, c4)
    kp = _kparams(pt, 2, 1, 3, rng)
    ct.set_kernel_params(kp["types"], kp["nfilter"], kp["fclp"], kp["fchp"], kp["npoles"], kp["sampling_hz"],
                         kp["nt1"], kp["nt2"], kp["coeff"], kp["jacobian"])
    ir = rng.integers(0, 2, npt)
    got = ct.kernels(ir, h3, h4, filtered=True)
    cr.close()
    ct.close()
    theta = pr["theta_min"] + np.arange(pr["theta_n"]) * pr["theta_delta"]
    omr = cat.omega_sgt([(rrec, np.arange(10), np.ones(10))], 10, pr["fmin"], pr["fmax"], theta, pr["tlen"], 4.0)
    omt = cat.omega_sgt([(trec, np.arange(20), np.ones(20))], 20, pt["fmin"], pt["fmax"], theta, pt["tlen"], 4.0)
    w3, w4 = [], []
    for k in range(npt):
        fr = cat.clsgt(float(deltar[k]), omr, pr["fmin"], pr["theta_min"], pr["theta_delta"], pr["ipdistance"],
                       pr["tlen"], 4.0)
        ft = cat.clsgt(float(deltas[k]), omt, pt["fmin"], pt["theta_min"], pt["theta_delta"], pt["ipdistance"],
                       pt["tlen"], 4.0)
        w3.append(cat.rsgt2h3freq(fr.T, ang[k], compo))
        w4.append(cat.tsgt2h4freq(ft.T, ang[k], mt))
    w3, w4 = np.stack(w3), np.stack(w4)
    assert rel_l2(h3, w3) <= TOL and rel_l2(h4, w4) <= TOL
    _check(got, _oracle(pt, kp, ir, w3, w4))


@pytest.mark.gpu
def test_kernels_without_series_mixed_segment_counts(built):
    """Without the filtered output an item runs only up to its filter's
    nt2, so filters whose windows end early run as one segment and the
    others as several; the kernels match the oracle either way."""
    rng = np.random.default_rng(31)
    p = _params(fmax=200, np1=256, tlen=1638.4, omegai=np.log(100.0) / 1638.4, iwin_start=10, iwin_end=500)
    nf = p["fmax"] - p["fmin"] + 1
    kp = _kparams(p, 3, 3, 3, rng)
    kp["nt1"] = [12, 14, 20, 11]
    kp["nt2"] = [30, 200, 490, 11]          # 21, 191, 481 and 2 samples from the window start
    ir = rng.integers(0, 3, 23)
    h3, h4 = _spectra(rng, ir.size, nf)
    c = dsmsgt.Catalogue(p)
    c.set_kernel_params(kp["types"], kp["nfilter"], kp["fclp"], kp["fchp"], kp["npoles"], kp["sampling_hz"],
                        kp["nt1"], kp["nt2"], kp["coeff"], kp["jacobian"])
    ker = c.kernels(ir, h3, h4)
    ker2, _ = c.kernels(ir, h3, h4, filtered=True)
    c.close()
    wk, _ = _oracle(p, kp, ir, h3, h4)
    assert rel_l2(ker, wk) <= TOL and rel_l2(ker2, wk) <= TOL
    for f in range(4):
        assert rel_l2(ker[:, f], wk[:, f]) <= TOL, f


@pytest.mark.gpu
def test_calculate_rsgt_video_series(built):
    """calculateRSGT (calculateK.f90:1-64): the RSGT catalogue at each
    point's receiver distance, the rsgt2h3freq combinations transformed
    (dsm_cat_series with the dsm_cat_h3h4_coef matrices) and filtered by
    every filter (dsm_cat_filter); against the oracle's clsgt,
    rsgt2h3freq, vectorFFT_double and rekurs.  Device pointers give the
    same values."""
    import torch
    from oracle import catalogue as cat
    rng = np.random.default_rng(77)
    p = _params(num=10, c_red_reci=3.0)
    nf = p["fmax"] - p["fmin"] + 1
    shp = (nf, p["theta_n"], 10)
    rec = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
    npt = 5
    dist = rng.uniform(2.0, 28.0, npt)
    ph = rng.uniform(0, 2 * np.pi, (npt, 3))
    ang = np.stack([f(m * ph[:, k]) for k in range(3) for m, f in ((1, np.cos), (1, np.sin), (2, np.cos), (2, np.sin))],
                   axis=1)
    c3, _ = dsmsgt.cat_h3h4_coef(ang, "R")
    c = dsmsgt.Catalogue(p)
    c.add(rec)
    kp = _kparams(p, 1, 2, 3, rng, npoles=6)
    c.set_kernel_params(kp["types"], kp["nfilter"], kp["fclp"], kp["fchp"], kp["npoles"], kp["sampling_hz"],
                        kp["nt1"], kp["nt2"], kp["coeff"], kp["jacobian"])
    ser = c.series(dist, c3)                                   # [point][6][nwin]
    got = c.filter(ser)                                        # [point][6][3][nwin]
    din = torch.from_numpy(ser).cuda()
    dout = torch.zeros(got.shape, dtype=torch.float64, device="cuda")
    rc = dsmsgt.lib().dsm_cat_filter(c.h, npt * 6, din.data_ptr(), dout.data_ptr(), 1)
    assert rc == 0
    assert np.array_equal(dout.cpu().numpy(), got)
    c.close()
    theta = p["theta_min"] + np.arange(p["theta_n"]) * p["theta_delta"]
    om = cat.omega_sgt([(rec, np.arange(10), np.ones(10))], 10, p["fmin"], p["fmax"], theta, p["tlen"], 3.0)
    want = np.empty_like(got)
    for k in range(npt):
        fr = cat.clsgt(float(dist[k]), om, p["fmin"], p["theta_min"], p["theta_delta"], p["ipdistance"],
                       p["tlen"], 3.0)
        h3 = cat.rsgt2h3freq(fr.T, ang[k], "R")
        du = cat.vector_fft_double(h3, p["fmin"], p["fmax"], p["np1"], p["omegai"], p["tlen"],
                                   p["iwin_start"], p["iwin_end"])
        for f in range(3):
            a, b1, b2 = cat.bpcoeff(kp["fclp"][f], kp["fchp"][f], 6, 1.0 / kp["sampling_hz"])
            want[k, :, f] = cat.rekurs(du, a, b1, b2)
    assert rel_l2(got, want) <= TOL
    for k in range(npt):
        assert rel_l2(got[k], want[k]) <= TOL, k
