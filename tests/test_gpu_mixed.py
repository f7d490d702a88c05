"""Mixed-precision path (split 16-bit tensor-core l-sum with FP32
accumulation) against the plain FP64 GPU path on the same inputs.

Target: relative L2 <= 1e-6 per output component with fp16 pieces; the
realised cutoff is the plain method's (the solves are unchanged).  bf16
pieces carry ~16 significant bits and are held to a looser bound."""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small
from conftest import rel_l2

TOL_F16 = 1e-6
TOL_BF16 = 1e-4


def per_component(a, b):
    """rel-L2 of each output component over frequencies, radii, distances.

    Components that vanish identically for the path (SH has no radial
    displacement, so some TSGT/RSGT/SYNN entries are pure round-off, 1e-16
    of the others) are measured against the norm of the whole array."""
    tot = np.sqrt(np.sum(np.abs(b) ** 2))
    out = []
    for c in range(a.shape[-1]):
        nc = np.sqrt(np.sum(np.abs(b[..., c]) ** 2))
        if nc < 1e-10 * tot:
            out.append(float(np.sqrt(np.sum(np.abs(a[..., c] - b[..., c]) ** 2)) / tot))
        else:
            out.append(rel_l2(a[..., c], b[..., c]))
    return out


def _mixed_vs_fp64(setup, freqs, prec):
    c64 = dsmsgt.Context(setup, precision=dsmsgt.DSM_PREC_FP64)
    t, r, y, llog = c64.run(freqs)
    c64.close()
    cm = dsmsgt.Context(setup, precision=prec)
    tm, rm, ym, llogm = cm.run(freqs)
    cm.close()
    assert list(llog) == list(llogm)
    assert np.all(np.isfinite(tm)) and np.all(np.isfinite(rm))
    errs = {"tsgt": per_component(tm, t), "rsgt": per_component(rm, r), "synn": per_component(ym, y)}
    return errs


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(dsmsgt.DSM_PREC_MIXED, TOL_F16), (dsmsgt.DSM_PREC_MIXED_BF16, TOL_BF16)])
def test_sh_mixed_close_to_fp64(built, prec, tol):
    s = dsmsgt.Setup(sh_small(), "sh")
    errs = _mixed_vs_fp64(s, [1, 7, 16, 31], prec)
    print(prec, {k: max(v) for k, v in errs.items()})
    for k, v in errs.items():
        assert max(v) <= tol, (k, v)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(dsmsgt.DSM_PREC_MIXED, TOL_F16), (dsmsgt.DSM_PREC_MIXED_BF16, TOL_BF16)])
def test_psv_mixed_close_to_fp64(built, prec, tol):
    s = dsmsgt.Setup(psv_small(), "psv")
    errs = _mixed_vs_fp64(s, [1, 17, 50], prec)
    print(prec, {k: max(v) for k, v in errs.items()})
    for k, v in errs.items():
        assert max(v) <= tol, (k, v)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [dsmsgt.DSM_PREC_FP64, dsmsgt.DSM_PREC_MIXED])
def test_records_match_outputs_when_copied_in_groups(prec):
    # ten frequencies in one batch: the complex64 records leave in groups on
    # the copy stream while later groups run; each must be the complex64 cast
    # of the same run's complex128 output, in record order [r][theta][comp]
    s = dsmsgt.Setup(psv_small(), "psv")
    freqs = [3, 5, 8, 11, 14, 17, 20, 23, 26, 29]
    ctx = dsmsgt.Context(s, precision=prec, freq_batch=len(freqs))
    t, r, y, llog, (t32, r32, y32) = ctx.run(freqs, want32=True)
    ctx.close()
    assert np.array_equal(t32, np.transpose(t, (0, 2, 1, 3)).astype(np.complex64))
    assert np.array_equal(r32, np.transpose(r, (0, 2, 1, 3)).astype(np.complex64))
    assert np.array_equal(y32, y.astype(np.complex64))


@pytest.mark.gpu
def test_psv_mixed_receivers_all_solid():
    # no fluid receiver rows: the second row group holds only U' and l(l+1)V/lsq
    s = dsmsgt.Setup(psv_small(seed=1, rmin=3800.0, rdelta=400.0), "psv")
    errs = _mixed_vs_fp64(s, [3, 17, 29], dsmsgt.DSM_PREC_MIXED)
    for k, v in errs.items():
        assert max(v) <= TOL_F16, (k, v)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["psv", "sh"])
def test_library_accuracy_report_matches_host_comparison(built, mode):
    # dsm_set_fp64_check: the library recomputes every second frequency of
    # the request in FP64 and reports the per-component relative L2; it must
    # equal the same comparison made on the host from the two contexts'
    # outputs, and leave the mixed outputs unchanged
    s = dsmsgt.Setup(psv_small() if mode == "psv" else sh_small(), mode)
    freqs = [2, 9, 17, 25, 30]
    c64 = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_FP64, freq_batch=2)
    ref = c64.run(freqs)
    cm = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED, freq_batch=4)
    plain = cm.run(freqs)
    cm.set_fp64_check(c64, 2)
    got = cm.run(freqs)
    acc = cm.accuracy()
    cm.set_fp64_check(None)
    cm.close()
    c64.close()
    for a, b in zip(got, plain):
        assert np.array_equal(a, b)
    sel = [0, 2, 4]
    assert acc["nfreq"] == 3 and acc["llog_equal"]
    for k, (a, b) in (("tsgt", (got[0], ref[0])), ("rsgt", (got[1], ref[1])), ("synn", (got[2], ref[2]))):
        host = per_component(a[sel], b[sel])
        lib_ = acc[k]
        assert len(lib_) == len(host)
        for x, y in zip(lib_, host):
            assert abs(x - y) <= 1e-6 * max(y, 1e-300) + 1e-300, (k, lib_, host)
        assert acc[k + "_max"] == max(lib_)
        assert max(lib_) <= TOL_F16


@pytest.mark.gpu
def test_accuracy_check_rejects_mismatched_context(built):
    s = dsmsgt.Setup(sh_small(), "sh")
    cm = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED)
    other = dsmsgt.Context(s, precision=dsmsgt.DSM_PREC_MIXED)
    with pytest.raises(dsmsgt.DsmError) as ei:
        cm.set_fp64_check(other, 1)
    assert ei.value.code == dsmsgt.DSM_ERR_INVALID
    p = dsmsgt.Setup(psv_small(), "psv")
    c64 = dsmsgt.Context(p, precision=dsmsgt.DSM_PREC_FP64)
    with pytest.raises(dsmsgt.DsmError):
        cm.set_fp64_check(c64, 1)
    for c in (cm, other, c64):
        c.close()
