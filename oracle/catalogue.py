"""Oracle (test infrastructure only): FP64 numpy restatement of KernelMaker's
catalogue consumer, for checking the device catalogue kernels.  Only tests,
``__graft_entry__.smoke()`` and the CPU leg of ``bench.py`` may import it.

Steps restated (paths inside the DSM Kernel Suite):
  * transform length: ``lsmoothfinder`` (src/KernelMaker/others.f90:288-308)
    and the np1 / samplingHz / window set-up of
    src/KernelMaker/KernelMaker-1.0.0.f90:311-330;
  * ``rdsgtomega`` (src/KernelMaker/fourier.f90:1-123): complex64 records
    widened to complex128, the per-kind halvings (:78-85), times
    exp(-2 pi i f/tlen * (-thetaD c_red_reci)) * 1e-21 (:91-101), summed into
    the frequency-domain SGT with the SH -> P-SV component map (:103-116);
  * ``clsgt`` (fourier.f90:128-162) with ``findIdeltaRegion`` (:165-190):
    normalised sinc interpolation in distance and the slowness-reduction
    phase;
  * ``vectorFFT_double`` (fourier.f90:418-450): Hermitian extension, the
    length-2 np1 transform of ``cdft`` / ``bitrv2`` (:492-600) and the
    exp(omegai t) / tlen * 1e3 window.

The transform is restated step for step (radix-2 decimation in frequency
with the reference's twiddle recurrence, then the bit-reversal
permutation), vectorised over series; ``test_cpu_catalogue_oracle`` pins it
against the DFT definition X_k = sum_n x_n exp(+2 pi i n k / N).

Parity status: the restatement is pinned by the DFT identity and by
hand-derivable cases (a single frequency line, a point on a catalogue
node); the reference itself (Fortran) cannot be built here.
"""
from __future__ import annotations

import cmath
import math
from functools import lru_cache

import numpy as np

PI = 3.1415926535897932          # src/KernelMaker/module.f90:54
PI_FFT = 3.141592653589793       # the local constant of vectorFFT_double (fourier.f90:425)

# reference kind codes of rdsgtomega (fourier.f90:13-16)
SYNN_SH, SYNN_PSV, RSGT_SH, RSGT_PSV, TSGT_SH, TSGT_PSV = 1, 2, 10, 20, 100, 200


def lsmoothfinder(tlen: float, np0: int, freq: float) -> int:
    """src/KernelMaker/others.f90:288-308."""
    np_ = 1
    while np_ < np0:
        np_ *= 2
    lsmooth = int(0.5 * tlen * freq / float(np_))
    i = 1
    while i < lsmooth:
        i *= 2
    return i


def transform_length(tlen: float, fmax: int, sampling_hz: float, start: float, end: float):
    """np1, the redefined samplingHz and the window sample range
    (KernelMaker-1.0.0.f90:311-330)."""
    lsmooth = lsmoothfinder(tlen, fmax, sampling_hz)
    i = 1
    while i < lsmooth:
        i *= 2
    lsmooth = i
    np1 = 1
    while np1 < fmax:
        np1 *= 2
    np1 *= lsmooth
    shz = float(2 * np1) / tlen
    return np1, shz, int(start * shz), int(end * shz)


def kind_scale(kind: int, num: int) -> np.ndarray:
    """Per-component factor rdsgtomega applies to one record set
    (fourier.f90:78-85): SYNN_SH halves components 3..5, SYNN_PSV halves 2
    and 8..10 (1-based)."""
    s = np.ones(num)
    if kind == SYNN_SH:
        s[2:5] = 0.5
    elif kind == SYNN_PSV:
        s[1] = 0.5
        s[7:10] = 0.5
    return s


def kind_dst(kind: int, num: int) -> np.ndarray:
    """0-based destination component of each record component in the P-SV
    sized frequency-domain arrays (fourier.f90:103-116)."""
    if kind in (SYNN_SH, RSGT_SH):
        return np.arange(5, 5 + num)
    if kind == TSGT_SH:
        return np.array([6] + list(range(11, 11 + num - 1)))
    return np.arange(num)


def omega_sgt(sets, num: int, fmin: int, fmax: int, theta, tlen: float, c_red_reci: float):
    """rdsgtomega for a list of record sets; each set is (records, dst, scale)
    with records [fmax-fmin+1][theta_n][ncomp] complex64 or complex128.
    Returns the frequency-domain SGT [nf][theta_n][num] complex128.  The
    record of frequency index 0 is never read (fourier.f90:28)."""
    theta = np.asarray(theta, np.float64)
    nf = fmax - fmin + 1
    out = np.zeros((nf, theta.size, num), np.complex128)
    for rec, dst, scale in sets:
        rec = np.asarray(rec)
        assert rec.shape[:2] == (nf, theta.size)
        for k in range(nf):
            i = fmin + k
            if i == 0:
                continue
            sd = rec[k].astype(np.complex128) * np.asarray(scale)[None, :]
            redtime = -theta * c_red_reci
            arg = -2.0 * PI * float(i) / tlen * redtime
            ph = np.cos(arg) + 1j * np.sin(arg)
            sd = sd * ph[:, None] * 1e-21
            out[k][:, np.asarray(dst)] += sd
    return out


def find_idelta_region(ix: int, nhalf: int, nmax: int):
    """fourier.f90:165-190 (1-based indices)."""
    istart, iend = ix - nhalf, ix + nhalf
    if istart < 1:
        iend += 1 - istart
        istart = 1
    if iend > nmax:
        istart -= iend - nmax
        iend = nmax
    istart = max(istart, 1)
    iend = min(iend, nmax)
    return istart, iend


def sinc_weights(distance: float, theta_min: float, theta_delta: float, theta_n: int,
                 ipdistance: float):
    """Window [idstart, idend] (0-based, inclusive), its weights and their
    sum, in the operation order of clsgt (fourier.f90:136-155)."""
    thetaD = lambda i: theta_min + float(i - 1) * theta_delta  # noqa: E731 (KernelMaker-1.0.0.f90:247)
    idelta = 1 + int((distance - thetaD(1)) / theta_delta)
    nhregion = int(ipdistance / theta_delta / 2.0)
    ids, ide = find_idelta_region(idelta, nhregion, theta_n)
    w = []
    norm = 0.0
    for kk in range(ids, ide + 1):
        t = PI * ((distance - thetaD(ids)) / theta_delta - float(kk - ids))
        if t == 0.0:
            w.append(1.0)
            norm = norm + 1.0
        else:
            w.append(math.sin(t) / t)
            norm = norm + math.sin(t) / t
    return ids - 1, ide - 1, np.array(w), norm


def clsgt(distance: float, omega, fmin: int, theta_min: float, theta_delta: float,
          ipdistance: float, tlen: float, c_red_reci: float):
    """Interpolated SGT at one distance: [nf][num] complex128."""
    omega = np.asarray(omega)
    ids, ide, w, norm = sinc_weights(distance, theta_min, theta_delta, omega.shape[1], ipdistance)
    acc = np.zeros((omega.shape[0], omega.shape[2]), np.complex128)
    for q, kk in enumerate(range(ids, ide + 1)):
        acc = acc + w[q] * omega[:, kk, :]   # a weight of exactly 1 adds the term unscaled
    j = np.arange(fmin, fmin + omega.shape[0], dtype=np.float64)
    arg = -2.0 * PI * j / tlen * distance * c_red_reci
    ph = np.cos(arg) + 1j * np.sin(arg)
    return acc / norm * ph[:, None]


@lru_cache(maxsize=16)
def _cdft_twiddles(N: int):
    """Twiddles of each stage of cdft (fourier.f90:492-560) for N complex
    points: a list of (half, w[half]) with w[q] the factor of the q-th
    difference in a block, produced by the reference's recurrence."""
    wmr, wmi = math.cos(PI_FFT / N), math.sin(PI_FFT / N)
    stages = []
    M = N
    while M > 2:
        half = M // 2
        w = np.empty(half, np.complex128)
        wkr, wki = 1.0, 0.0
        wdr = 1 - 2 * wmi * wmi
        wdi = 2 * wmi * wmr
        ss = 2 * wdi
        wmr, wmi = wdr, wdi
        w[0] = 1.0
        if half > 1:
            w[1] = complex(wdr, wdi)
        for q in range(2, half, 2):
            wkr = wkr - ss * wdi
            wki = wki + ss * wdr
            wdr = wdr - ss * wki
            wdi = wdi + ss * wkr
            w[q] = complex(wkr, wki)
            w[q + 1] = complex(wdr, wdi)
        stages.append((half, w))
        M = half
    return stages


@lru_cache(maxsize=16)
def _bit_reverse(N: int) -> np.ndarray:
    bits = N.bit_length() - 1
    idx = np.arange(N)
    rev = np.zeros(N, np.int64)
    for b in range(bits):
        rev |= ((idx >> b) & 1) << (bits - 1 - b)
    return rev


def cdft(c: np.ndarray) -> np.ndarray:
    """The complex transform of cdft(2 N, cos(pi/N), sin(pi/N), c) applied to
    the last axis of c (N complex points, a power of two >= 2): radix-2
    decimation in frequency with twiddles from the reference recurrence
    (complex butterflies written with the reference's real operations),
    a last twiddle-free radix-2 stage, then the bit-reversal permutation."""
    a = np.array(c, np.complex128, copy=True)
    N = a.shape[-1]
    lead = a.shape[:-1]
    for half, w in _cdft_twiddles(N):
        blk = a.reshape(lead + (N // (2 * half), 2, half))
        lo, hi = blk[..., 0, :].copy(), blk[..., 1, :].copy()
        xr, xi = lo.real - hi.real, lo.imag - hi.imag
        blk[..., 0, :] = (lo.real + hi.real) + 1j * (lo.imag + hi.imag)
        blk[..., 1, :] = (w.real * xr - w.imag * xi) + 1j * (w.real * xi + w.imag * xr)
        a = blk.reshape(lead + (N,))
    blk = a.reshape(lead + (N // 2, 2))
    lo, hi = blk[..., 0].copy(), blk[..., 1].copy()
    blk[..., 0] = (lo.real + hi.real) + 1j * (lo.imag + hi.imag)
    blk[..., 1] = (lo.real - hi.real) + 1j * (lo.imag - hi.imag)
    a = blk.reshape(lead + (N,))
    if N > 2:
        a = a[..., _bit_reverse(N)]
    return a


def hermitian_extend(ccvec: np.ndarray, fmin: int, fmax: int, np1: int) -> np.ndarray:
    """cvec of vectorFFT_double (fourier.f90:430-439) for series on the last
    axis of ccvec ([..., fmax-fmin+1])."""
    lead = ccvec.shape[:-1]
    cvec = np.zeros(lead + (2 * np1,), np.complex128)
    cvec[..., fmin:fmax + 1] = ccvec
    for i in range(fmin, np1):
        cvec[..., np1 + i] = np.conj(cvec[..., np1 - i])
    return cvec


def vector_fft_double(ccvec, fmin: int, fmax: int, np1: int, omegai: float, tlen: float,
                      iws: int, iwe: int) -> np.ndarray:
    """Windowed real time series of each series on the last axis."""
    cvec = cdft(hermitian_extend(np.asarray(ccvec, np.complex128), fmin, fmax, np1))
    shz = float(2 * np1) / tlen
    i = np.arange(iws, iwe + 1, dtype=np.float64)
    return cvec[..., iws:iwe + 1].real * np.exp(omegai * i / shz) / tlen * 1.0e3


def series(p: dict, sets, distances, coef=None) -> np.ndarray:
    """Time series [npoint][nout][nwin] of the catalogue consumer.

    p: num, theta_n, theta_min, theta_delta, fmin, fmax, np1, tlen, omegai,
       ipdistance, c_red_reci, iwin_start, iwin_end.
    sets: list of (records, dst, scale) as in omega_sgt.
    coef: [npoint][nout][num] real combination applied after clsgt (as
       rsgt2h3freq / tsgt2h4freq / synn2h3freq do), or None for the
       components themselves."""
    theta = p["theta_min"] + np.arange(p["theta_n"], dtype=np.float64) * p["theta_delta"]
    om = omega_sgt(sets, p["num"], p["fmin"], p["fmax"], theta, p["tlen"], p["c_red_reci"])
    outs = []
    for k, d in enumerate(distances):
        f = clsgt(float(d), om, p["fmin"], p["theta_min"], p["theta_delta"], p["ipdistance"],
                  p["tlen"], p["c_red_reci"])                       # [nf][num]
        h = f.T if coef is None else np.asarray(coef[k]) @ f.T    # [nout][nf]
        outs.append(vector_fft_double(h, p["fmin"], p["fmax"], p["np1"], p["omegai"], p["tlen"],
                                      p["iwin_start"], p["iwin_end"]))
    return np.stack(outs)


# ---------------------------------------------------------------------------
# Per-point isotropic kernels: calculateKernel's isovpfreq / isovsfreq with
# the Butterworth filter of bwfilt.f90 and the trapezoid sum over nt1..nt2.
# ---------------------------------------------------------------------------

def _f32(x: float) -> float:
    """A real rounded to single precision (Fortran cmplx() without a kind)."""
    return float(np.float32(x))


def bpcoeff(f1: float, f2: float, npoles: int, dt: float):
    """bpcoeff (src/KernelMaker/bwfilt.f90:124-166): coefficients a, b1, b2
    of the npoles second-order sections of the recursive band-pass.

    The reference forms the poles through single-precision complex values:
    cexp(cmplx(0, phase)) is a single-precision exponential (here cos and
    sin rounded to single), and cmplx(w0, 0), cmplx(w1 w2, 0) round their
    real parts to single.  Only s(1..npoles) of the 2 npoles roots enter
    the coefficients (:154-162)."""
    if npoles > 10:
        raise ValueError("npoles greater than 10")
    pi = 3.141592653589793
    d2 = 2.0 / dt
    w1 = d2 * math.tan(2.0 * pi * f1 / d2)
    w2 = d2 * math.tan(2.0 * pi * f2 / d2)
    w0 = 0.5 * (w2 - w1)
    s = []
    for n in range(1, npoles + 1):
        ph = _f32(float(2 * n - 1 + npoles) * pi / float(2 * npoles))
        p = complex(_f32(math.cos(ph)), _f32(math.sin(ph)))
        t1 = p * complex(_f32(w0), 0.0)
        t2 = cmath.sqrt(t1 * t1 - complex(_f32(w1 * w2), 0.0))
        s += [t1 + t2, t1 - t2]
    a = np.zeros(npoles)
    b1 = np.zeros(npoles)
    b2 = np.zeros(npoles)
    for n in range(npoles):
        ssum = 2.0 * s[n].real
        sprod = (s[n] * s[n].conjugate()).real
        fact1 = d2 * d2 - d2 * ssum + sprod
        fact2 = 2.0 * (sprod - d2 * d2)
        fact3 = d2 * d2 + d2 * ssum + sprod
        a[n] = 2.0 * d2 * w0 / fact1
        b1[n] = fact2 / fact1
        b2[n] = fact3 / fact1
    return a, b1, b2


def rekurs(x: np.ndarray, a, b1, b2) -> np.ndarray:
    """rekurs (bwfilt.f90:54-117), forward pass only (irek = 0, as
    calculateK.f90 calls bwfilt), vectorised over the leading axes of x
    (samples on the last axis)."""
    x = np.asarray(x, np.float64)
    npoles = len(a)
    lead = x.shape[:-1]
    z1 = [np.zeros(lead) for _ in range(npoles)]
    z2 = [np.zeros(lead) for _ in range(npoles)]
    x1 = np.zeros(lead)
    x2 = np.zeros(lead)
    y = np.empty_like(x)
    for n in range(x.shape[-1]):
        z = [None] * npoles
        z[0] = a[0] * (x[..., n] - x2) - b1[0] * z1[0] - b2[0] * z2[0]
        for i in range(1, npoles):
            z[i] = a[i] * (z[i - 1] - z2[i - 1]) - b1[i] * z1[i] - b2[i] * z2[i]
        x2 = x1
        x1 = x[..., n]
        z2 = z1
        z1 = z
        y[..., n] = z[npoles - 1]
    return y


def iso_products(h3: np.ndarray, h4: np.ndarray, jac=None, types: int = 3):
    """The frequency products of isovpfreq (calculateK.f90:261-265) and
    isovsfreq (:367-374, :395-403) for h3, h4 [..., 6, nf]; jac [..., nf]
    is jacobianFuji at the point's radius.  Returns the spectra in the
    order P (du), S (du), S (duq) of the types present."""
    out = []
    if types & 1:
        out.append(-(h3[..., 0, :] + h3[..., 1, :] + h3[..., 2, :])
                   * (h4[..., 0, :] + h4[..., 1, :] + h4[..., 2, :]) * 1.0e3)
    if types & 2:
        p4 = h3[..., 3, :] * h4[..., 3, :]
        p5 = h3[..., 4, :] * h4[..., 4, :]
        p6 = h3[..., 5, :] * h4[..., 5, :]
        c1 = h3[..., 0, :] * (h4[..., 1, :] + h4[..., 2, :])
        c2 = h3[..., 1, :] * (h4[..., 0, :] + h4[..., 2, :])
        c3 = h3[..., 2, :] * (h4[..., 0, :] + h4[..., 1, :])
        du = (-2.0 * (p4 + p5 + p6) + c1 + c2 + c3) * 1.0e3
        d1 = h3[..., 0, :] * h4[..., 0, :]
        d2 = h3[..., 1, :] * h4[..., 1, :]
        d3 = h3[..., 2, :] * h4[..., 2, :]
        duq = (-(4.0 * (p4 + p5 + p6)) + 2.0 / 3.0 * (c1 + c2 + c3) - 4.0 / 3.0 * (d1 + d2 + d3))
        duq = duq * jac * 1.0e3
        out += [du, duq]
    return np.stack(out, axis=-2)


# (series, coeff type) pairs whose trapezoid sums fill tmpker: P du -> 1, 3, 4;
# S du -> 5, 7; S duq -> 8 (calculateK.f90:302-321, :497-513)
def _series_types(types: int):
    st = []
    if types & 1:
        st.append((1, 3, 4))
    if types & 2:
        st += [(5, 7), (8,)]
    return st


def iso_kernels(p: dict, kp: dict, ir, h3, h4):
    """tmpker [point][nfilter+1][nktype+1] and the filtered series
    [point][series][nfilter+1][nwin] of calculateKernel's isotropic part.

    p: the catalogue parameters (fmin, fmax, np1, tlen, omegai, iwin_start,
       iwin_end); kp: types, nfilter, fclp, fchp, npoles, sampling_hz, nt1,
       nt2, nr, nktype, coeff (Fortran order, as a flat array), jacobian
       (Fortran order, complex128 flat)."""
    ir = np.asarray(ir)
    h3 = np.asarray(h3, np.complex128)
    h4 = np.asarray(h4, np.complex128)
    nf = p["fmax"] - p["fmin"] + 1
    iws, iwe = p["iwin_start"], p["iwin_end"]
    nwin = iwe - iws + 1
    nfl, nkt, nr = kp["nfilter"] + 1, kp["nktype"], kp["nr"]
    jac = None
    if kp["types"] & 2:
        jac = np.asarray(kp["jacobian"], np.complex128).reshape(nf, nr).T[ir]   # [point][nf]
    spec = iso_products(h3, h4, jac, kp["types"])                            # [point][series][nf]
    du = vector_fft_double(spec, p["fmin"], p["fmax"], p["np1"], p["omegai"], p["tlen"], iws, iwe)
    coeff = np.asarray(kp["coeff"], np.float64).reshape(nwin, nr, nkt, nfl)   # [t][ir][k-1][ift]
    npt, ns = du.shape[0], du.shape[1]
    filt = np.empty((npt, ns, nfl, nwin))
    ker = np.zeros((npt, nfl, nkt + 1))
    dt = 1.0 / kp["sampling_hz"]
    st = _series_types(kp["types"])
    for f in range(nfl):
        a, b1, b2 = bpcoeff(kp["fclp"][f], kp["fchp"][f], kp["npoles"], dt)
        y = rekurs(du, a, b1, b2)                                             # [point][series][nwin]
        filt[:, :, f, :] = y
        t1, t2 = kp["nt1"][f] - iws, kp["nt2"][f] - iws
        for s, ks in enumerate(st):
            for k in ks:
                c = coeff[:, ir, k - 1, f].T                                  # [point][nwin]
                acc = np.zeros(npt)
                acc = acc + c[:, t1] * y[:, s, t1] / 2.0
                for t in range(t1 + 1, t2):
                    acc = acc + c[:, t] * y[:, s, t]
                acc = acc + c[:, t2] * y[:, s, t2] / 2.0
                ker[:, f, k] = acc
    return ker, filt


def rsgt2h3freq(rsgtF, ang, compo: str):
    """rsgt2h3freq (src/KernelMaker/fourier.f90:278-320) on interpolated
    RSGT spectra rsgtF [10][nf] at one point; ang = (crq, srq, crq2, srq2,
    ...) as the angles module holds them.  h3 [6][nf] in the order rr, tt,
    pp, rt, rp, tp.  For compo 'T' the reference's h3(3) = -h3(3) (:314)
    negates the previous point's value; the transverse pp entry is -tt."""
    F = lambda k: rsgtF[k - 1]
    crq, srq, crq2, srq2 = ang[0], ang[1], ang[2], ang[3]
    h = np.zeros((6,) + np.shape(rsgtF[0]), np.complex128)
    if compo == "Z":
        h[0] = F(1)
        h[1] = F(3) * crq2 - F(4)
        h[2] = -F(3) * crq2 - F(4)
        h[3] = 2.0 * F(2) * crq
        h[4] = 2.0 * F(2) * srq
        h[5] = 2.0 * F(3) * srq2
    elif compo == "R":
        h[0] = F(5)
        h[1] = -(F(7)) * crq2 - F(6)
        h[2] = (F(7)) * crq2 - F(6)
        h[3] = 4.0 * (F(9)) * crq
        h[4] = 4.0 * (F(9)) * srq
        h[5] = -2.0 * (F(7)) * srq2
    else:
        h[1] = (F(8)) * srq2
        h[2] = -h[1]
        h[3] = 2.0 * (F(10)) * srq
        h[4] = -2.0 * (F(10)) * crq
        h[5] = -2.0 * (F(8)) * crq2
    return h


def tsgt2h4freq(tsgtF, ang, mt):
    """tsgt2h4freq (src/KernelMaker/fourier.f90:322-415) on interpolated
    TSGT spectra tsgtF [20][nf] at one point: the 4th-order TSGT double-
    dotted with the moment tensor mt(1..6); h4 [6][nf]."""
    F = lambda k: tsgtF[k - 1]
    csq, ssq, csq2, ssq2, cqs, sqs, cqs2, sqs2 = ang[4:12]
    m = mt
    t01 = F(7) * cqs; t02 = F(7) * sqs; t03 = F(8) * csq; t04 = F(8) * ssq
    t05 = F(9) * cqs2; t06 = F(10) * csq2; t07 = F(11) * csq2; t08 = F(11) * ssq2
    t09 = F(12) * cqs2; t10 = F(12) * sqs2
    t11 = F(13) * (csq * cqs - ssq * sqs); t12 = F(13) * (ssq * cqs + csq * sqs)
    t13 = F(14) * (csq * cqs + ssq * sqs); t14 = F(14) * (ssq * cqs - csq * sqs)
    t15 = F(15) * (csq2 * cqs - ssq2 * sqs); t16 = F(15) * (ssq2 * cqs + csq2 * sqs)
    t17 = F(17) * (csq * cqs2 - ssq * sqs2); t18 = F(17) * (ssq * cqs2 + csq * sqs2)
    t19 = F(19) * (csq2 * cqs2 - ssq2 * sqs2); t20 = F(19) * (ssq2 * cqs2 + csq2 * sqs2)
    t21 = F(20) * (csq2 * cqs2 + ssq2 * sqs2); t22 = F(20) * (ssq2 * cqs2 - csq2 * sqs2)
    t23 = F(16) * (csq2 * cqs + ssq2 * sqs); t24 = F(16) * (ssq2 * cqs - csq2 * sqs)
    t25 = F(18) * (csq * cqs2 + ssq * sqs2); t26 = F(18) * (ssq * cqs2 - csq * sqs2)
    h = np.zeros((6,) + np.shape(tsgtF[0]), np.complex128)
    h[0] = (F(1) * m[0] + (t05 - F(2)) * m[1] + (-t05 - F(2)) * m[2]
            - F(5) * (cqs * m[3] + sqs * m[4]) + F(9) * sqs2 * m[5])
    h[1] = ((t06 - F(3)) * m[0] + (t21 + t19 - t07 - t09 + F(4)) * m[1]
            + (-t21 - t19 - t07 + t09 + F(4)) * m[2] + (t23 - t15 + t01) * m[3]
            + (-t24 - t16 + t02) * m[4] + (-t22 + t20 - t10) * m[5])
    h[2] = ((-t06 - F(3)) * m[0] + (-t21 - t19 + t07 - t09 + F(4)) * m[1]
            + (t21 + t19 + t07 + t09 + F(4)) * m[2] + (-t23 + t15 + t01) * m[3]
            + (t24 + t16 + t02) * m[4] + (t22 - t20 - t10) * m[5])
    h[3] = (-F(6) * csq * m[0] + (t25 - t17 + t03) * m[1] + (-t25 + t17 + t03) * m[2]
            + (-t13 + t11) * m[3] + (t14 + t12) * m[4] + (-t26 - t18) * m[5])
    h[4] = ((-F(6) * ssq) * m[0] + (t26 - t18 + t04) * m[1] + (-t26 + t18 + t04) * m[2]
            + (-t14 + t12) * m[3] + (-t13 - t11) * m[4] + (t25 + t17) * m[5])
    h[5] = (F(10) * ssq2 * m[0] + (t22 + t20 - t08) * m[1] + (-t22 - t20 - t08) * m[2]
            + (t24 - t16) * m[3] + (t23 + t15) * m[4] + (t21 - t19) * m[5])
    return h
