"""Device catalogue consumer (dsm_cat_*) against the oracle restatement of
KernelMaker's rdsgtomega / clsgt / vectorFFT_double.

Every case must match the oracle to 1e-10 relative L2 (FP64 throughout; the
differences are the transform's and sin/cos rounding).  Cases cover: points
on catalogue nodes, between nodes, at and beyond both ends of the distance
grid (window clipping); fmin > 0 (partial Hermitian extension) and
fmax = np1 (the self-conjugated middle sample); complex64 and complex128
records; two record sets with the SH -> P-SV component map and halvings; a
reducing slowness; a per-point combination matrix; batches split by the
buffer limit; device pointers; and the full-size workload (1441 distances,
2049 frequencies) on sampled points plus linearity."""
import numpy as np
import pytest

import dsmsgt
from conftest import rel_l2

TOL = 1e-10


def _records(p, ncomp, seed, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    nf = p["fmax"] - p["fmin"] + 1
    shp = (nf, p["theta_n"], ncomp)
    return (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(dtype)


def _params(**kw):
    p = dict(num=20, theta_n=61, theta_min=0.0, theta_delta=0.5, fmin=0, fmax=48, np1=64, tlen=819.2,
             omegai=np.log(100.0) / 819.2, ipdistance=5.0, c_red_reci=0.0, iwin_start=3, iwin_end=120)
    p.update(kw)
    return p


DIST = [0.0, 0.26, 2.0, 7.5, 15.13, 29.9, 30.0, 31.2]


def _oracle(p, sets, dist, coef=None):
    from oracle import catalogue as cat
    return cat.series(p, sets, dist, coef)


def _run(p, sets, dist, coef=None, batch_bytes=None):
    c = dsmsgt.Catalogue(p)
    if batch_bytes:
        c.set_batch_bytes(batch_bytes)
    for rec, dst, scale in sets:
        c.add(rec, dst, scale)
    out = c.series(dist, coef)
    c.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("c_red", [0.0, 12.5])
def test_catalogue_components_match_oracle(built, c_red):
    p = _params(c_red_reci=c_red)
    sets = [(_records(p, 20, 1), None, None)]
    got = _run(p, sets, DIST)
    want = _oracle(p, [(sets[0][0], np.arange(20), np.ones(20))], DIST)
    assert got.shape == (len(DIST), 20, 118)
    assert rel_l2(got, want) <= TOL
    for k in range(len(DIST)):                       # every point, not only the sum
        assert rel_l2(got[k], want[k]) <= TOL, k


@pytest.mark.gpu
def test_catalogue_combination_matrix_matches_oracle(built):
    p = _params(c_red_reci=7.0)
    rng = np.random.default_rng(5)
    coef = rng.standard_normal((len(DIST), 6, 20))
    rec = _records(p, 20, 2)
    got = _run(p, [(rec, None, None)], DIST, coef)
    want = _oracle(p, [(rec, np.arange(20), np.ones(20))], DIST, coef)
    assert got.shape == (len(DIST), 6, 118)
    assert rel_l2(got, want) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("fmin,fmax,win", [(5, 64, (0, 127)), (0, 64, (60, 70)), (33, 40, (0, 0))])
def test_catalogue_two_sets_partial_spectrum(built, fmin, fmax, win):
    """P-SV TSGT (complex64) plus SH TSGT (complex128, halved, mapped into
    components 7 and 12-20 as rdsgtomega does)."""
    from oracle import catalogue as cat
    p = _params(fmin=fmin, fmax=fmax, iwin_start=win[0], iwin_end=win[1])
    psv = _records(p, 20, 3)
    sh = _records(p, 10, 4, np.complex128)
    dst = cat.kind_dst(cat.TSGT_SH, 10)
    scale = np.linspace(0.5, 1.5, 10)
    got = _run(p, [(psv, None, None), (sh, dst, scale)], DIST)
    want = _oracle(p, [(psv, np.arange(20), np.ones(20)), (sh, dst, scale)], DIST)
    assert rel_l2(got, want) <= TOL


@pytest.mark.gpu
def test_catalogue_batches_and_device_pointers(built):
    import torch
    p = _params(np1=8192, iwin_end=300)
    rng = np.random.default_rng(9)
    dist = rng.uniform(-1.0, 31.0, 40)
    coef = rng.standard_normal((40, 5, 20))
    rec = _records(p, 20, 6)
    one = _run(p, [(rec, None, None)], dist, coef)
    split = _run(p, [(rec, None, None)], dist, coef, batch_bytes=1 << 20)   # one point per batch
    assert rel_l2(split, one) <= 1e-13
    c = dsmsgt.Catalogue(p)
    drec = torch.from_numpy(rec).cuda()
    c.add(drec)
    dout = torch.empty((40, 5, p["iwin_end"] - p["iwin_start"] + 1), dtype=torch.float64, device="cuda")
    c.series(dist, coef, out=dout)
    torch.cuda.synchronize()
    assert np.array_equal(dout.cpu().numpy(), one)
    c.clear()
    with pytest.raises(dsmsgt.DsmError, match="no record set"):
        c.series(dist, coef)
    c.close()
    want = _oracle(p, [(rec, np.arange(20), np.ones(20))], dist[:6], coef[:6])
    assert rel_l2(one[:6], want) <= TOL


def _full_params():
    np1, shz, s0, s1 = dsmsgt.cat_np1(3276.8, 2048, 2.0, 400.0, 1000.0)
    return dict(num=20, theta_n=1441, theta_min=0.0, theta_delta=0.125, fmin=0, fmax=2048, np1=np1,
                tlen=3276.8, omegai=np.log(100.0) / 3276.8, ipdistance=10.0, c_red_reci=0.0,
                iwin_start=s0, iwin_end=s1)


@pytest.mark.gpu
def test_catalogue_full_size_sampled_points_and_linearity(built):
    """1441 distances x 2049 frequencies x 20 components, 1681 points, 6
    outputs each: three interior points against the oracle (run on the 81
    catalogue distances around each), and linearity in the records."""
    import torch
    p = _full_params()
    rng = np.random.default_rng(11)
    P = 1681
    dist = np.sort(rng.uniform(30.0, 90.0, P))
    coef = rng.standard_normal((P, 6, 20))
    g = torch.Generator(device="cuda").manual_seed(0)
    shp = (p["fmax"] + 1, p["theta_n"], 20)
    r1 = torch.randn(shp, dtype=torch.complex128, device="cuda", generator=g)
    r2 = torch.randn(shp, dtype=torch.complex128, device="cuda", generator=g)
    out = {}
    for name, recs in (("a", [r1]), ("b", [r2]), ("ab", [r1 + 2.0 * r2])):
        c = dsmsgt.Catalogue(p)
        for r in recs:
            c.add(r)
        out[name] = c.series(dist, coef)
        c.close()
    assert np.all(np.isfinite(out["ab"]))
    assert rel_l2(out["ab"], out["a"] + 2.0 * out["b"]) <= 1e-12
    r1h = r1.cpu().numpy()
    for k in (0, P // 2, P - 1):
        ids = int(dist[k] / p["theta_delta"]) - 40         # window of +-40 catalogue distances (0-based)
        q = dict(p, theta_n=81, theta_min=ids * p["theta_delta"])
        sub = r1h[:, ids:ids + 81, :]
        want = _oracle(q, [(sub, np.arange(20), np.ones(20))], [dist[k]], coef[k:k + 1])
        assert rel_l2(out["a"][k:k + 1], want) <= TOL, k


@pytest.mark.gpu
def test_catalogue_rejects_bad_calls_and_stays_usable(built):
    """Errors come back as codes with a message, and the handle still works
    afterwards: a fifth record set, a destination outside the components,
    two record components on one destination, non-finite distances and
    coefficients, more than 64 outputs."""
    p = _params()
    rec = _records(p, 20, 7)
    c = dsmsgt.Catalogue(p)
    for _ in range(4):
        c.add(rec)
    with pytest.raises(dsmsgt.DsmError, match="at most 4"):
        c.add(rec)
    c.clear()
    with pytest.raises(dsmsgt.DsmError, match="out of range"):
        c.add(rec[:, :, :2], dst=[0, 20])
    with pytest.raises(dsmsgt.DsmError, match="one destination"):
        c.add(rec[:, :, :2], dst=[3, 3])
    c.add(rec)
    with pytest.raises(dsmsgt.DsmError, match="non-finite distance"):
        c.series([1.0, float("nan")])
    coef = np.ones((2, 3, 20))
    coef[1, 2, 5] = np.inf
    with pytest.raises(dsmsgt.DsmError, match="non-finite coefficient"):
        c.series([1.0, 2.0], coef)
    with pytest.raises(dsmsgt.DsmError, match="nout"):
        c.series([1.0], np.ones((1, 65, 20)))
    got = c.series(DIST)
    c.close()
    want = _oracle(p, [(rec, np.arange(20), np.ones(20))], DIST)
    assert rel_l2(got, want) <= TOL


@pytest.mark.gpu
def test_catalogue_long_transform_and_many_frequencies(built):
    """A transform of 2^19 samples (np1 = 2^18) over 70 001 frequencies: more
    frequency blocks and more frequencies than one grid dimension of 65 535
    holds, on a small catalogue (9 distances, 4 components, 2 points)."""
    p = _params(num=4, theta_n=9, theta_min=10.0, fmin=0, fmax=70000, np1=1 << 18, tlen=1000.0,
                omegai=np.log(100.0) / 1000.0, ipdistance=2.0, iwin_start=100, iwin_end=160)
    rec = _records(p, 4, 8)
    dist = [11.3, 12.75]
    got = _run(p, [(rec, None, None)], dist)
    want = _oracle(p, [(rec, np.arange(4), np.ones(4))], dist)
    assert got.shape == (2, 4, 61)
    assert rel_l2(got, want) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("fmin,c_red", [(0, 0.0), (5, 9.0)])
def test_catalogue_spectra_and_transform_match_oracle(built, fmin, c_red):
    """dsm_cat_spectra against the oracle's clsgt plus combination,
    dsm_cat_transform against its vectorFFT_double (random spectra whose
    index-0 value is nonzero too), and their composition against
    dsm_cat_series."""
    from oracle import catalogue as cat
    p = _params(fmin=fmin, fmax=64, c_red_reci=c_red)
    rec = _records(p, 20, 12)
    rng = np.random.default_rng(13)
    coef = rng.standard_normal((len(DIST), 6, 20))
    c = dsmsgt.Catalogue(p)
    c.add(rec)
    spec = c.spectra(DIST, coef)
    series = c.series(DIST, coef)
    theta = p["theta_min"] + np.arange(p["theta_n"]) * p["theta_delta"]
    om = cat.omega_sgt([(rec, np.arange(20), np.ones(20))], 20, p["fmin"], p["fmax"], theta, p["tlen"],
                       p["c_red_reci"])
    want = np.stack([coef[k] @ cat.clsgt(d, om, p["fmin"], p["theta_min"], p["theta_delta"], p["ipdistance"],
                                         p["tlen"], p["c_red_reci"]).T for k, d in enumerate(DIST)])
    assert spec.shape == want.shape
    assert rel_l2(spec, want) <= TOL
    assert rel_l2(c.transform(spec), series) <= 1e-12
    x = rng.standard_normal((5, 65 - fmin)) + 1j * rng.standard_normal((5, 65 - fmin))
    got = c.transform(x)
    c.close()
    ref = cat.vector_fft_double(x, p["fmin"], p["fmax"], p["np1"], p["omegai"], p["tlen"], p["iwin_start"],
                                p["iwin_end"])
    assert got.shape == ref.shape
    assert rel_l2(got, ref) <= TOL


@pytest.mark.gpu
def test_catalogue_rejects_misaligned_device_outputs(built):
    """Device outputs are written with 16-byte (spectra) or 8-byte (series)
    stores: a pointer off that alignment is rejected before anything runs.
    The calls ask for zero points, so even without the check no kernel would
    touch the pointer."""
    import ctypes as C
    import torch
    p = _params()
    c = dsmsgt.Catalogue(p)
    c.add(_records(p, 20, 3))
    buf = torch.empty(64, dtype=torch.complex128, device="cuda")
    d = np.zeros(1)
    L = dsmsgt.lib()
    rc = L.dsm_cat_spectra(c.h, 0, d.ctypes.data_as(C.POINTER(C.c_double)), 20, None,
                           C.c_void_p(buf.data_ptr() + 8), 1)
    assert rc == dsmsgt.DSM_ERR_INVALID and b"misaligned" in L.dsm_cat_last_error(c.h)
    rc = L.dsm_cat_series(c.h, 0, d.ctypes.data_as(C.POINTER(C.c_double)), 20, None,
                          C.c_void_p(buf.data_ptr() + 4), 1)
    assert rc == dsmsgt.DSM_ERR_INVALID and b"misaligned" in L.dsm_cat_last_error(c.h)
    rc = L.dsm_cat_spectra(c.h, 0, d.ctypes.data_as(C.POINTER(C.c_double)), 20, None,
                           C.c_void_p(buf.data_ptr() + 16), 1)
    assert rc == dsmsgt.DSM_OK
    got = c.series(DIST)
    c.close()
    assert rel_l2(got, _oracle(p, [(_records(p, 20, 3), np.arange(20), np.ones(20))], DIST)) <= TOL
