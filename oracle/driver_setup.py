"""Oracle set-up -- test infrastructure only.

An independent restatement, in numpy, of the part of the reference's P-SV
and SH drivers that runs once before the frequency loop: input parsing,
radial grid, receivers, source position and the element integrals
(src/SGTpsv/SGTpsv-MPI.f90:39-477 with the routines of src/SGTpsv/others.f90
and src/SGTpsv/calmat.f90:1-404; src/SGTsh/SGTsh-MPI.f90:33-347 with
src/SGTsh/others.f90:380-742 and src/SGTsh/calmat.f90:1-160).  It fills the
engine's C-ABI set-up structs (include/dsmsgt.h, dsm_psv_setup_t and
dsm_sh_setup_t) from its own arrays, so the oracle's frequency loops
(liboracle.so) and the CPU baseline run without the product library.  Tests
compare it element by element with the product's driver-side set-up
(host/setup.cpp), which pins that set-up to a second, separately written
restatement of the Fortran.

Layer loops are vectorised per zone; every element keeps the Fortran
operation order (numpy performs one IEEE operation per element, without
fused multiply-adds), so both restatements agree to the last bit.

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py use this
module; the product never imports it.  Parity status: unpinned against the
Fortran itself (no Fortran compiler is available to run the reference).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

PI = 3.1415926535897932

# packing orders of dsm_psv_setup_t.solid_el / hm_el (include/dsmsgt.h)
SOLID_ORDER = ("t", "h1x", "h2L", "h2N", "h3ay", "h4aL", "h4aN", "h5ay", "h6aL", "h6aN", "h7y", "h7z", "h8L",
               "h8N", "h3y", "h4L", "h4N", "h5y", "h6L", "h6N")
HM_ORDER = ("h3my", "h5my", "h4m1L", "h4m2N", "h6m1N", "h6m2L")


# ------------------------------------------------------------------ input
def _records(text: str) -> list[str]:
    """Records kept by pinput / readDSMconf / readpsvmodel: '#' lines are
    dropped and reading stops at a record starting with 'end'
    (src/SGTpsv/others.f90:27-34, 90-97, 117-126)."""
    out = []
    for line in text.splitlines():
        if line[:1] == "#":
            continue
        if line[:3] == "end":
            break
        out.append(line)
    return out


def _fnum(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


class _ListRead:
    """Fortran list-directed READ: one statement consumes whole records until
    it has its values; the rest of its last record is skipped."""

    def __init__(self, records):
        self.rec = list(records)
        self.pos = 0

    def line(self) -> str:
        s = self.rec[self.pos]
        self.pos += 1
        return s

    def values(self, n: int) -> list[str]:
        got = []
        while len(got) < n:
            got.extend(self.line().replace(",", " ").split())
        return got[:n]


def parse_params(text: str) -> dict:
    """pinput (src/SGTpsv/others.f90:1-72)."""
    rd = _ListRead(_records(text))
    p = {"dsmconf": rd.line().strip(), "outdir": rd.line().strip(), "model": rd.line().strip(),
         "modelname": rd.line().strip()}
    p["tlen"] = _fnum(rd.values(1)[0])
    p["rmin_"], p["rmax_"], p["rdelta_"] = (_fnum(v) for v in rd.values(3))
    p["r0min"] = _fnum(rd.values(1)[0])
    p["thetamin"], p["thetamax"], p["thetadelta"] = (_fnum(v) for v in rd.values(3))
    p["imin"], p["imax"] = (int(v) for v in rd.values(2))
    p["rsgt"], p["tsgt"], p["synn"], p["psgt"] = (int(v) for v in rd.values(4))
    return p


def parse_conf(text: str) -> dict:
    """readDSMconf (src/SGTpsv/others.f90:74-111)."""
    rd = _ListRead(_records(text))
    re_, ratc, ratl, omegai = (_fnum(rd.values(1)[0]) for _ in range(4))
    return {"re": re_, "ratc": ratc, "ratl": ratl, "omegai": omegai, "maxlmax": int(rd.values(1)[0])}


def parse_model(text: str) -> dict:
    """The model read of src/SGTpsv/SGTpsv-MPI.f90:100-105: nzone, then per
    zone vrmin, vrmax, rho(4), vpv(4), vph(4), vsv(4), vsh(4), eta(4), qmu,
    qkappa.  Coefficient arrays are [4][nzone] (Fortran (4, nzone))."""
    rd = _ListRead(_records(text))
    nz = int(rd.values(1)[0])
    m = {"nzone": nz, "vrmin": np.zeros(nz), "vrmax": np.zeros(nz), "qmu": np.zeros(nz), "qkappa": np.zeros(nz)}
    for k in ("rho", "vpv", "vph", "vsv", "vsh", "eta"):
        m[k] = np.zeros((4, nz))
    for z in range(nz):
        v = [_fnum(t) for t in rd.values(28)]
        m["vrmin"][z], m["vrmax"][z] = v[0], v[1]
        for i, k in enumerate(("rho", "vpv", "vph", "vsv", "vsh", "eta")):
            m[k][:, z] = v[2 + 4 * i: 6 + 4 * i]
        m["qmu"][z], m["qkappa"][z] = v[26], v[27]
    return m


def _poly_at(c4, r, rmax):
    """Sum of c(j) (r/rmax)^(j-1), j = 1..4, accumulated as the reference does
    (coef = coef * (r/rmax) each step)."""
    x = r / rmax
    coef = 1.0
    s = 0.0 + c4[0] * coef
    for j in range(1, 4):
        coef = coef * x
        s = s + c4[j] * coef
    return s


# ------------------------------------------------------------ grid (others.f90)
def calgrid_psv(m: dict, rmin: float, rmax: float, imax: int, lmin: int, tlen: float):
    """calgrid, src/SGTpsv/others.f90:374-450 (fluid zones use Vp)."""
    nz = m["nzone"]
    vmin, gridpar, dzpar = np.zeros(nz), np.zeros(nz), np.zeros(nz)
    for z in range(nz):
        v = m["vpv"][:, z] if m["vsv"][0, z] == 0.0 else m["vsv"][:, z]
        vs1 = vs2 = 0.0
        c1 = c2 = 1.0
        for j in range(4):
            if j > 0:
                c1 = c1 * (m["vrmin"][z] / rmax)
                c2 = c2 * (m["vrmax"][z] / rmax)
            vs1 = vs1 + v[j] * c1
            vs2 = vs2 + v[j] * c2
        rh = m["vrmax"][z] - m["vrmin"][z]
        omega = 2.0 * PI * float(imax) / tlen
        vmin[z] = vs2 if vs1 >= vs2 else vs1
        amax = m["vrmax"][z]
        g = (omega * omega) / (vmin[z] * vmin[z]) - ((lmin + 0.5) * (lmin + 0.5)) / (amax * amax)
        if g > 0.0:
            dzpar[z] = math.sqrt(1.0 / g)
            gridpar[z] = rh / dzpar[z]
    g = 0.0
    for z in range(nz):
        g = g + gridpar[z]
    for z in range(nz):
        if gridpar[z] > 0.0:
            gridpar[z] = gridpar[z] / g
        else:
            gridpar[z] = (m["vrmax"][z] - m["vrmin"][z]) / (rmax - rmin) * 0.1
    g = 0.0
    for z in range(nz):
        g = g + gridpar[z]
    gridpar = gridpar / g
    return vmin, gridpar, dzpar


def layers_psv(m: dict, dzpar, re_: float) -> np.ndarray:
    """calra_psv, src/SGTpsv/others.f90:1292-1340: layers per zone, at least 5."""
    nnl = np.zeros(m["nzone"], np.int64)
    for z in range(m["nzone"]):
        rh = m["vrmax"][z] - m["vrmin"][z]
        if dzpar[z] == 0.0:
            n = 1
        else:
            n = int(math.sqrt(3.3 / re_) * rh / dzpar[z] / 2.0 / PI / 7.0e-1 + 1)
        nnl[z] = max(n, 5)
    return nnl


def node_radii(m: dict, nnl, rmin: float) -> np.ndarray:
    """First loop of calra2_psv (src/SGTpsv/others.f90:1344-1374): ra[0] = rmin,
    then vrmin + rh i / n for i = 1..n of every zone (0-based array)."""
    out = [rmin]
    for z in range(m["nzone"]):
        rh = m["vrmax"][z] - m["vrmin"][z]
        i = np.arange(1, nnl[z] + 1, dtype=np.float64)
        out.extend((m["vrmin"][z] + rh * i / float(nnl[z])).tolist())
    return np.asarray(out)


# ------------------------------------------------- element integrals (calmat.f90)
def _pinteg_seg(p, x1, x2, c0, c1, v0, v1):
    """pinteg (src/SGTpsv/calmat.f90:86-124) over one structure segment
    [v0, v1] on which con is linear (c0 -> c1), for polynomials p[k] (k-th
    coefficient, arrays over layers): pmulti by (q1 + q2 x) then polint
    (:128-161) from x1 to x2."""
    n = len(p)
    q2 = (c1 - c0) / (v1 - v0)
    q1 = -(q2 * v0) + c0
    # pmulti(n, p, 2, q, n+1, pq): pq(i+j-1) += p(i) q(j), i outer, j inner
    pq = [np.zeros_like(x1) for _ in range(n + 1)]
    for i in range(n):
        pq[i] = pq[i] + p[i] * q1
        pq[i + 1] = pq[i + 1] + p[i] * q2
    # polint(n+1, pq, x1, x2)
    a = [np.ones_like(x1)]
    b = [np.ones_like(x1)]
    for i in range(1, n + 1):
        a.append(a[-1] * x1)
        b.append(b[-1] * x2)
    dx = x2 - x1
    pint = np.zeros_like(x1)
    for i in range(1, n + 2):
        xx = np.zeros_like(x1)
        for j in range(1, i + 1):
            xx = xx + a[j - 1] * b[i - j] / float(i)
        pint = pint + pq[i - 1] * dx * xx
    return pint


class _Zone:
    """Nodes and structure points of one zone: node radii x[0..nl], structure
    values con at the same points (the zone's own copies)."""

    def __init__(self, x, cons):
        self.x = x
        self.lo, self.hi = x[:-1], x[1:]
        self.cons = cons


def calmatc(zone: _Zone, con, rpow: int, w1dn: int, w2dn: int, symmetrise: bool = False) -> np.ndarray:
    """calmatc, src/SGTpsv/calmat.f90:1-62: 4 entries per layer,
    (j, k) = (1,1), (1,2), (2,1), (2,2), of the integral of
    r^rpow con W_j^(w1dn) W_k^(w2dn) over the layer.  The SH version
    (src/SGTsh/calmat.f90:1-83) symmetrises when w1dn /= w2dn: diagonal
    entries doubled, both off-diagonal entries their sum."""
    lo, hi = zone.lo, zone.hi
    rh = hi - lo
    zero = np.zeros_like(rh)

    def basis(dn):  # a(1..2, j) for j = 1, 2: constant and linear coefficients
        if dn == 0:
            return [(hi / rh, -1.0 / rh), (-(lo / rh), 1.0 / rh)]
        return [(-1.0 / rh, zero), (1.0 / rh, zero)]

    A, B = basis(w1dn), basis(w2dn)
    c0, c1 = con[:-1], con[1:]
    out = np.empty((len(rh), 4))
    for j in range(2):
        for k in range(2):
            a, b = A[j], B[k]
            # pmulti(2, a, 2, b, 3, c)
            c = [zero + a[0] * b[0], (zero + a[0] * b[1]) + a[1] * b[0], zero + a[1] * b[1]]
            c = c + [zero, zero]
            if rpow > 0:
                c = [zero] * rpow + c[:3] + [zero] * (2 - rpow)
            out[:, 2 * j + k] = _pinteg_seg(c, lo, hi, c0, c1, lo, hi)
    if symmetrise and w1dn != w2dn:
        off = out[:, 1] + out[:, 2]
        out = np.stack([2.0 * out[:, 0], off, off, 2.0 * out[:, 3]], axis=1)
    return out.reshape(-1)


def _lumped(zone: _Zone, con, mass: bool) -> np.ndarray:
    """caltl (mass, r^2, :165-195) and calhl (rigidity, :200-224): the two
    half-layer integrals on the diagonal, zeros off it."""
    lo, hi = zone.lo, zone.hi
    mid = (lo + hi) / 2.0
    c0, c1 = con[:-1], con[1:]
    zero = np.zeros_like(lo)
    p = [zero, zero, zero + 1.0] if mass else [zero + 1.0]
    out = np.zeros((len(lo), 4))
    out[:, 0] = _pinteg_seg(p, lo, mid, c0, c1, lo, hi)
    out[:, 3] = _pinteg_seg(p, mid, hi, c0, c1, lo, hi)
    return out.reshape(-1)


def calt(tl, tc):
    """calt, :231-241."""
    return (tl + tc) / 2.0


def calh5(zone: _Zone, con) -> np.ndarray:
    """calh5, :246-277."""
    r0, r1, c0, c1 = zone.lo, zone.hi, con[:-1], con[1:]
    out = np.empty((len(r0), 4))
    out[:, 0] = -(3.0 / 8.0 * c0 * r0) - 1.0 / 8.0 * c1 * r1
    out[:, 1] = -out[:, 0]
    out[:, 2] = -(1.0 / 8.0 * c0 * r0) - 3.0 / 8.0 * c1 * r1
    out[:, 3] = -out[:, 2]
    return out.reshape(-1)


def mtrnp(a: np.ndarray) -> np.ndarray:
    """mtrnp, :363-386: the transpose of each 2x2 layer block."""
    b = a.reshape(-1, 4).copy()
    b[:, 1], b[:, 2] = a.reshape(-1, 4)[:, 2], a.reshape(-1, 4)[:, 1]
    return b.reshape(-1)


def calhm1(zone: _Zone, con) -> np.ndarray:
    """calhm1, :282-318: hm1(-1:2, 1:nl+1) as [col][4] (row index -1..2)."""
    x, nl = zone.x, len(zone.x) - 1
    h = np.zeros((nl + 1, 4))
    t = lambda a, c, r: a / 12.0 * c * r  # noqa: E731  (a/12) con r, left to right
    h[0, 1] = 0.0 - t(7.0, con[0], x[0])
    h[0, 2] = 0.0 + t(8.0, con[0], x[0])
    h[0, 3] = 0.0 - t(1.0, con[0], x[0])
    i = np.arange(1, nl - 1)
    h[i, 0] = 0.0 - t(5.0, con[i], x[i])
    h[i, 1] = 0.0 - t(3.0, con[i], x[i])
    h[i, 2] = 0.0 + t(9.0, con[i], x[i])
    h[i, 3] = 0.0 - t(1.0, con[i], x[i])
    k = nl - 1
    h[k, 0] = 0.0 - t(5.0, con[k], x[k])
    h[k, 1] = 0.0 - t(3.0, con[k], x[k])
    h[k, 2] = 0.0 + t(8.0, con[k], x[k])
    k = nl
    h[k, 0] = 0.0 - t(5.0, con[k], x[k])
    h[k, 1] = 0.0 + t(5.0, con[k], x[k])
    return h


def calhm2(zone: _Zone, con) -> np.ndarray:
    """calhm2, :322-358: hm2(-2:1, 1:nl+1) as [col][4] (row index -2..1)."""
    x, nl = zone.x, len(zone.x) - 1
    h = np.zeros((nl + 1, 4))
    t = lambda a, c, r: a / 12.0 * c * r  # noqa: E731
    h[0, 2] = 0.0 - t(5.0, con[0], x[0])
    h[0, 3] = 0.0 + t(5.0, con[0], x[0])
    h[1, 1] = 0.0 - t(8.0, con[1], x[1])
    h[1, 2] = 0.0 + t(3.0, con[1], x[1])
    h[1, 3] = 0.0 + t(5.0, con[1], x[1])
    i = np.arange(2, nl)
    h[i, 0] = 0.0 + t(1.0, con[i], x[i])
    h[i, 1] = 0.0 - t(9.0, con[i], x[i])
    h[i, 2] = 0.0 + t(3.0, con[i], x[i])
    h[i, 3] = 0.0 + t(5.0, con[i], x[i])
    k = nl
    h[k, 0] = 0.0 + t(1.0, con[k], x[k])
    h[k, 1] = 0.0 - t(8.0, con[k], x[k])
    h[k, 2] = 0.0 + t(7.0, con[k], x[k])
    return h


def mtrnp2(h1: np.ndarray, p: int, q: int) -> np.ndarray:
    """mtrnp2, :390-404: hm2(i, j) = hm1(-i, i + j) for i = -q..p where the
    column exists; h1 holds rows -p..q, the result rows -q..p."""
    ncol = h1.shape[0]
    h2 = np.zeros_like(h1)
    for i in range(-q, p + 1):
        for j in range(ncol):
            n = i + j
            if 0 <= n < ncol:
                h2[j, i + q] = h1[n, -i + p]
    return h2


# ---------------------------------------------------------------- P-SV set-up
class PsvOracleSetup:
    """The P-SV set-up struct filled from this module's own arrays; the
    attributes mirror what oracle.run and the tests read from a set-up."""

    mode = "psv"
    num = (20, 10, 10)

    def __init__(self, param_text: str, conf_text: str, model_text: str):
        from dsmsgt import PsvSetup  # the ctypes layout of the C-ABI struct only
        par, conf, m = parse_params(param_text), parse_conf(conf_text), parse_model(model_text)
        nz = m["nzone"]
        rmin, rmax = m["vrmin"][0], m["vrmax"][nz - 1]
        tlen = par["tlen"]
        omegai = -math.log(conf["omegai"]) / tlen
        r_n = int((par["rmax_"] - par["rmin_"]) / par["rdelta_"]) + 1
        r_ = np.array([par["rmin_"] + float(i) * par["rdelta_"] for i in range(r_n)])
        # calstg_for_stackpoints (src/SGTpsv/others.f90:687-762): A and
        # Qkappa at each receiver (the last zone containing it wins)
        lam, qkp = np.zeros(r_n), np.zeros(r_n)
        for ir in range(r_n):
            for z in range(nz):
                if m["vrmin"][z] < r_[ir] <= m["vrmax"][z]:
                    trho = _poly_at(m["rho"][:, z], r_[ir], rmax)
                    tvph = _poly_at(m["vph"][:, z], r_[ir], rmax)
                    lam[ir] = trho * tvph * tvph
                    qkp[ir] = m["qkappa"][z]
        theta_n = int((par["thetamax"] - par["thetamin"]) / par["thetadelta"]) + 1
        theta = np.array([par["thetamin"] + float(i) * par["thetadelta"] for i in range(theta_n)])
        r0 = par["r0min"]
        # calnl (:348-368)
        iphase = np.array([2 if np.all(m["vsv"][:, z] == 0.0) else 1 for z in range(nz)], np.int32)
        if not np.any(iphase == 1):
            raise ValueError("PSV: model has no solid zone")
        if r0 < rmin or r0 > rmax:
            raise ValueError("Location of the source is improper.")
        vmin, gridpar, dzpar = calgrid_psv(m, rmin, rmax, par["imax"], 1, tlen)
        nlayer = layers_psv(m, dzpar, conf["re"])
        nslay = int(nlayer[iphase == 1].sum())
        nllay = int(nlayer[iphase == 2].sum())
        nnlayer = int(nlayer.sum())
        ra = node_radii(m, nlayer, rmin)  # 0-based: ra[k] = Fortran ra(k+1)
        # isp: first node of each zone (calsp, :455-522), 1-based
        isp = np.ones(nz, np.int32)
        for z in range(1, nz):
            isp[z] = isp[z - 1] + nlayer[z - 1]
        # receiver bracketing (second loop of calra2_psv, :1376-1416)
        rrsta = np.zeros((r_n, 3))
        iista = np.zeros((r_n, 3), np.int32)
        istazone = np.zeros(r_n, np.int32)
        itmp = 0
        for z in range(nz):
            for i in range(1, nlayer[z] + 1):
                hit = (ra[itmp] < r_) & (r_ <= ra[itmp + 1])
                for ista in np.nonzero(hit)[0]:
                    istazone[ista] = z + 1
                    g0, l0 = (itmp, i) if i != nlayer[z] else (itmp - 1, i - 1)
                    rrsta[ista] = ra[g0:g0 + 3]
                    iista[ista] = [l0, l0 + 1, l0 + 2]
                itmp += 1
        if np.any(istazone == 0):
            raise ValueError("PSV: receiver outside the grid")
        # stack points of the element arrays (calsp)
        nsl, nll = int((iphase == 1).sum()), int((iphase == 2).sum())
        issp, ilsp, jssp = np.ones(nz, np.int32), np.ones(nz, np.int32), np.ones(nz, np.int32)
        isl = ill = 0
        for z in range(nz - 1):
            if iphase[z] == 1:
                isl += 1
                if isl != nsl:
                    issp[isl] = issp[isl - 1] + 4 * nlayer[z]
                    jssp[isl] = jssp[isl - 1] + nlayer[z] + 1
            else:
                ill += 1
                if ill != nll:
                    ilsp[ill] = ilsp[ill - 1] + 4 * nlayer[z]
        isdr = int(issp[nsl - 1]) - 1 + 4 * int(nlayer[nz - 1])
        jsdr = int(jssp[nsl - 1]) - 1 + int(nlayer[nz - 1]) + 1
        ildr = 4 * nllay
        # calspo (:527-584)
        if r0 == rmax:
            spo = float(nnlayer) - 0.01
            r0 = ra[nnlayer - 1] + (spo - float(nnlayer - 1)) * (ra[nnlayer] - ra[nnlayer - 1])
        else:
            k = 2
            while not (r0 < ra[k - 1]):
                k += 1
            spo = float(k - 2) + (r0 - ra[k - 2]) / (ra[k - 1] - ra[k - 2])
            if spo - float(k - 2) < 0.01:
                spo = float(k - 2) + 0.01
                r0 = ra[k - 2] + (spo - float(k - 2)) * (ra[k - 1] - ra[k - 2])
            if spo - float(k - 2) > 0.99:
                spo = float(k - 2) + 0.99
                r0 = ra[k - 2] + (spo - float(k - 2)) * (ra[k - 1] - ra[k - 2])
        spn = 0
        for z in range(nz):
            spn += 1
            if r0 <= m["vrmax"][z]:
                if iphase[z] == 2:
                    raise ValueError("The source is in the liquid layer.(calspo)")
                break
        spo = spo - float(isp[spn - 1] - 1)
        # structure points (calstg, :590-682): each zone's nodes with its own
        # polynomial values; zone boundaries appear twice
        zones, ecs = [], {}
        for z in range(nz):
            x = ra[isp[z] - 1: isp[z] - 1 + nlayer[z] + 1]
            ev = {k: np.array([_poly_at(m[k][:, z], xi, rmax) for xi in x])
                  for k in ("rho", "vpv", "vph", "vsv", "vsh", "eta")}
            rho = ev["rho"]
            ecL = rho * ev["vsv"] * ev["vsv"]
            ecN = rho * ev["vsh"] * ev["vsh"]
            ecA = rho * ev["vph"] * ev["vph"]
            ecC = rho * ev["vpv"] * ev["vpv"]
            ecF = ev["eta"] * (ecA - 2.0 * ecL)
            kappa = (4.0 * ecA + ecC + 4.0 * ecF - 4.0 * ecN) / 9.0
            cons = {"rho": rho, "kappa": kappa, "ecKx": ecA - 4.0 / 3.0 * ecN, "ecKy": ecF + 2.0 / 3.0 * ecN,
                    "ecKz": (ecC + 2.0 * ecF) / 3.0, "ecL": ecL, "ecN": ecN,
                    "rhoinv": 1.0 / rho, "kappainv": 1.0 / kappa}  # calinv (:835-847)
            zones.append(_Zone(x, cons))
        # elastic constants at the source (end of calstg)
        src = {k: _poly_at(m[k][:, spn - 1], r0, rmax) for k in ("rho", "vpv", "vph", "vsv", "vsh", "eta")}
        ecL0 = src["rho"] * src["vsv"] * src["vsv"]
        ecA0 = src["rho"] * src["vph"] * src["vph"]
        ecC0 = src["rho"] * src["vpv"] * src["vpv"]
        ecF0 = src["eta"] * (ecA0 - 2.0 * ecL0)
        # element integrals (src/SGTpsv/SGTpsv-MPI.f90:383-477)
        n_sel, n_fel, n_hm = 8 * nslay, 8 * max(nllay, 1), 2 * (nslay + nz)
        S = {k: np.zeros(n_sel) for k in SOLID_ORDER}
        p1, p2, p3 = np.zeros(n_fel), np.zeros(n_fel), np.zeros(n_fel)
        hm = {k: np.zeros((n_hm, 4)) for k in HM_ORDER}
        elem, hmoff = np.zeros(nz, np.int32), np.zeros(nz, np.int32)
        isl = ill = 0
        for z in range(nz):
            zn, cs, nl = zones[z], zones[z].cons, int(nlayer[z])
            if iphase[z] == 1:
                isl += 1
                o = isdr + int(issp[isl - 1]) - 1
                sl = slice(o, o + 4 * nl)
                elem[z] = o + 1
                S["t"][sl] = calt(calmatc(zn, cs["rho"], 2, 0, 0), _lumped(zn, cs["rho"], True))
                h1 = {}
                for k, key in (("ecKx", "h1x"), ("ecKy", "h1y"), ("ecKz", "h1z"), ("ecL", "h2L"), ("ecN", "h2N")):
                    h1[key] = calt(calmatc(zn, cs[k], 0, 0, 0), _lumped(zn, cs[k], False))
                for key in ("h1x", "h2L", "h2N"):
                    S[key][sl] = h1[key]
                h5a = {k: calmatc(zn, cs[k], 1, 0, 1) for k in ("ecKx", "ecKy", "ecKz", "ecL", "ecN")}
                S["h5ay"][sl], S["h6aL"][sl], S["h6aN"][sl] = h5a["ecKy"], h5a["ecL"], h5a["ecN"]
                S["h3ay"][sl], S["h4aL"][sl], S["h4aN"][sl] = mtrnp(h5a["ecKy"]), mtrnp(h5a["ecL"]), mtrnp(h5a["ecN"])
                S["h7y"][sl] = calmatc(zn, cs["ecKy"], 2, 1, 1)
                S["h7z"][sl] = calmatc(zn, cs["ecKz"], 2, 1, 1)
                S["h8L"][sl] = calmatc(zn, cs["ecL"], 2, 1, 1)
                S["h8N"][sl] = calmatc(zn, cs["ecN"], 2, 1, 1)
                # modified first-derivative operator (:439-477): submat, mtrnp
                h5y = h5a["ecKy"] - calh5(zn, cs["ecKy"])
                h6L = h5a["ecL"] - calh5(zn, cs["ecL"])
                h6N = h5a["ecN"] - calh5(zn, cs["ecN"])
                S["h5y"][sl], S["h6L"][sl], S["h6N"][sl] = h5y, h6L, h6N
                S["h3y"][sl], S["h4L"][sl], S["h4N"][sl] = mtrnp(h5y), mtrnp(h6L), mtrnp(h6N)
                col = jsdr + int(jssp[isl - 1])
                hmoff[z] = col
                cols = slice(col - 1, col - 1 + nl + 1)
                h5my = calhm1(zn, cs["ecKy"])
                h6m1L, h6m1N = calhm1(zn, cs["ecL"]), calhm1(zn, cs["ecN"])
                h6m2L, h6m2N = calhm2(zn, cs["ecL"]), calhm2(zn, cs["ecN"])
                hm["h5my"][cols] = h5my
                hm["h6m1N"][cols] = h6m1N
                hm["h6m2L"][cols] = h6m2L
                hm["h3my"][cols] = mtrnp2(h5my, 1, 2)
                hm["h4m2N"][cols] = mtrnp2(h6m1N, 1, 2)
                hm["h4m1L"][cols] = mtrnp2(h6m2L, 2, 1)
            else:
                ill += 1
                o = ildr + int(ilsp[ill - 1]) - 1
                sl = slice(o, o + 4 * nl)
                elem[z] = o + 1
                p1[sl] = calmatc(zn, cs["rhoinv"], 2, 1, 1)
                p2[sl] = calt(calmatc(zn, cs["rhoinv"], 0, 0, 0), _lumped(zn, cs["rhoinv"], False))
                p3[sl] = calt(calmatc(zn, cs["kappainv"], 2, 0, 0), _lumped(zn, cs["kappainv"], True))
        # calspdr (:870-898), nn (:628) and the source rows (:557-558, :636-641)
        kkdr = np.ones(nz, np.int32)
        for z in range(nz - 1):
            if iphase[z] == 1:
                kkdr[z + 1] = kkdr[z] + (2 * nlayer[z] if iphase[z + 1] == 1 else 2 * (nlayer[z] + 1))
            else:
                kkdr[z + 1] = kkdr[z] + (nlayer[z] + 1 if iphase[z + 1] == 1 else nlayer[z])
        nn = int(kkdr[nz - 1] + 2 * nlayer[nz - 1] + 1)
        ispo = int(spo)
        mtmp = int(isp[spn - 1]) + ispo
        jtmp = int(kkdr[spn - 1]) + 2 * ispo
        if spo == float(ispo):
            mtmp -= 1
            jtmp -= 2
        # keep every array alive as long as the struct that points into it
        self._keep = []

        def dp(a):
            a = np.ascontiguousarray(a, np.float64)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def ip(a):
            a = np.ascontiguousarray(a, np.int32)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int))

        s = PsvSetup()
        s.nzone = nz
        s.iphase, s.nlayer, s.isp, s.kkdr = ip(iphase), ip(nlayer), ip(isp), ip(kkdr)
        s.elem, s.hmoff = ip(elem), ip(hmoff)
        s.vrmin, s.vrmax, s.qmu, s.qkappa = dp(m["vrmin"]), dp(m["vrmax"]), dp(m["qmu"]), dp(m["qkappa"])
        s.vsv = dp(m["vsv"].T.reshape(-1))
        s.nn, s.rmin, s.rmax = nn, rmin, rmax
        s.n_sel, s.n_fel, s.n_hm = n_sel, n_fel, n_hm
        self.solid = np.concatenate([S[k] for k in SOLID_ORDER])
        self.fluid = np.concatenate([p1, p2, p3])
        self.hm = np.concatenate([hm[k].reshape(-1) for k in HM_ORDER])
        s.solid_el, s.fluid_el, s.hm_el = dp(self.solid), dp(self.fluid), dp(self.hm)
        s.spn, s.spo, s.r0 = spn, spo, r0
        s.ecC0, s.ecF0, s.ecL0 = ecC0, ecF0, ecL0
        s.ra_src[0], s.ra_src[1] = ra[mtmp - 1], ra[mtmp]
        for i, k in enumerate(("rho", "vpv", "vph", "vsv", "vsh", "eta")):
            for j in range(4):
                s.src_poly[4 * i + j] = m[k][j, spn - 1]
        s.jsrc = jtmp
        s.r_n = r_n
        s.r, s.rrsta, s.iista = dp(r_), dp(rrsta.reshape(-1)), ip(iista.reshape(-1))
        s.istazone, s.lambda_, s.qkp = ip(istazone), dp(lam), dp(qkp)
        s.theta_n, s.theta = theta_n, dp(theta)
        s.tlen, s.omegai, s.ratl, s.maxlmax = tlen, omegai, conf["ratl"], conf["maxlmax"]
        s.imin, s.imax = par["imin"], par["imax"]
        s.rsgt_switch, s.tsgt_switch, s.synn_switch = par["rsgt"], par["tsgt"], par["synn"]
        s._owner = self  # the struct points into arrays this object holds
        self.s = s
        self.ptr = C.pointer(s)
        self.n_nodes, self.n_unknowns = nnlayer + 1, nn

    @property
    def r_n(self) -> int:
        return self.s.r_n

    @property
    def theta_n(self) -> int:
        return self.s.theta_n

    def out_shapes(self, n: int):
        nt, nr, ns = self.num
        return ((n, self.theta_n, self.r_n, nt), (n, self.theta_n, self.r_n, nr), (n, self.theta_n, ns))


def psv_setup(job) -> PsvOracleSetup:
    """The oracle's P-SV set-up of a job (parameter file, DSM.config, model)."""
    return PsvOracleSetup(job.param_text, job.conf_text, job.model_text)


# ---------------------------------------------------------------- SH set-up
class ShOracleSetup:
    """The SH set-up struct (dsm_sh_setup_t) filled from this module's own
    arrays (src/SGTsh/SGTsh-MPI.f90:33-347)."""

    mode = "sh"
    num = (10, 5, 5)

    def __init__(self, param_text: str, conf_text: str, model_text: str):
        from dsmsgt import ShSetup  # the ctypes layout of the C-ABI struct only
        par, conf, full = parse_params(param_text), parse_conf(conf_text), parse_model(model_text)
        # the outer-core cut (:83-102, :123-133): zones above the last fluid
        # zone (ioutercore = 0 when there is none)
        iout = 0
        for z in range(full["nzone"]):
            if np.all(full["vsv"][:, z] == 0.0):
                iout = z + 1
        nz = full["nzone"] - iout
        if nz <= 0:
            raise ValueError("SH: no solid zone above the outer core")
        m = {k: (v[iout:] if v.ndim == 1 else v[:, iout:]) for k, v in full.items() if k != "nzone"}
        m["nzone"] = nz
        rmin, rmax = m["vrmin"][0], m["vrmax"][nz - 1]
        tlen = par["tlen"]
        omegai = -math.log(conf["omegai"]) / tlen
        # receivers above rmin (:152-179)
        rmin_, rdelta_ = par["rmin_"], par["rdelta_"]
        r_n = int((par["rmax_"] - rmin_) / rdelta_) + 1
        ir_ = 0
        for i in range(1, r_n + 1):
            if rmin_ + float(i - 1) * rdelta_ <= rmin:
                ir_ = i
        r_n -= ir_
        rmin_ = rmin_ + float(ir_) * rdelta_
        if r_n <= 0:
            raise ValueError("SH: no receiver above rmin")
        r_ = np.array([rmin_ + float(i) * rdelta_ for i in range(r_n)])
        theta_n = int((par["thetamax"] - par["thetamin"]) / par["thetadelta"]) + 1
        theta = np.array([par["thetamin"] + float(i) * par["thetadelta"] for i in range(theta_n)])
        r0 = par["r0min"]
        # calgrid (SH: Vs in every zone, src/SGTsh/others.f90:380-459)
        msh = dict(m, vpv=m["vsv"])
        _, _, dzpar = calgrid_psv(msh, rmin, rmax, par["imax"], 1, tlen)
        nlayer = layers_psv(m, dzpar, conf["re"])  # calra (:463-495): same rule
        nnlayer = int(nlayer.sum())
        ra = node_radii(m, nlayer, rmin)
        # receiver bracketing, calra2 (:500-563): global node indices
        rrsta = np.zeros((r_n, 3))
        iista = np.zeros((r_n, 3), np.int32)
        itmp = 0
        for z in range(nz):
            for i in range(1, nlayer[z] + 1):
                hit = (ra[itmp] < r_) & (r_ <= ra[itmp + 1])
                for ista in np.nonzero(hit)[0]:
                    b = itmp if i != nlayer[z] else itmp - 1
                    rrsta[ista] = ra[b:b + 3]
                    iista[ista] = [b + 1, b + 2, b + 3]
                itmp += 1
        if np.any(iista[:, 0] <= 0):
            raise ValueError("SH: receiver outside the grid")
        # calsp (:569-584)
        isp, jsp = np.ones(nz, np.int32), np.ones(nz, np.int32)
        for z in range(1, nz):
            isp[z] = isp[z - 1] + nlayer[z - 1]
            jsp[z] = jsp[z - 1] + 4 * nlayer[z - 1]
        # calspo (:588-631) and calgra (:637-647)
        ndc = nz - 1
        if r0 < rmin or r0 > rmax:
            raise ValueError("The source location is improper.(calspo)")
        if r0 == rmax:
            spo = float(nnlayer) - 0.01
            r0 = ra[nnlayer - 1] + (spo - float(nnlayer - 1)) * (ra[nnlayer] - ra[nnlayer - 1])
        else:
            k = 2
            while k <= ndc + nnlayer + 2 and not (r0 < ra[k - 1]):
                k += 1
            spo = float(k - 2) + (r0 - ra[k - 2]) / (ra[k - 1] - ra[k - 2])
            if spo - float(k - 2) < 0.01:
                spo = float(k - 2) + 0.01
                r0 = ra[k - 2] + (spo - float(k - 2)) * (ra[k - 1] - ra[k - 2])
            if spo - float(k - 2) > 0.99:
                spo = float(k - 2) + 0.99
                r0 = ra[k - 2] + (spo - float(k - 2)) * (ra[k - 1] - ra[k - 2])
        spn = 0
        for z in range(nz):
            spn += 1
            if r0 <= m["vrmax"][z]:
                break
        spo = spo - float(isp[spn - 1] - 1)
        igr = int(isp[spn - 1]) + int(math.trunc(spo))
        gra = np.array([ra[igr - 1], r0, ra[igr]])

        def structure(z, x):  # calstg (:651-694) / calgstg (:699-742)
            rho = np.array([_poly_at(m["rho"][:, z], xi, rmax) for xi in x])
            vsv = np.array([_poly_at(m["vsv"][:, z], xi, rmax) for xi in x])
            vsh = np.array([_poly_at(m["vsh"][:, z], xi, rmax) for xi in x])
            return {"rho": rho, "ecL": rho * vsv * vsv, "ecN": rho * vsh * vsh}

        # element integrals (:314-339)
        t, h1, h2, h3, h4 = (np.zeros(4 * nnlayer) for _ in range(5))

        def integrals(zn, cs):
            return (calt(calmatc(zn, cs["rho"], 2, 0, 0), _lumped(zn, cs["rho"], True)),
                    calmatc(zn, cs["ecL"], 2, 1, 1),
                    calmatc(zn, cs["ecL"], 1, 1, 0, symmetrise=True),
                    calt(calmatc(zn, cs["ecL"], 0, 0, 0), _lumped(zn, cs["ecL"], False)),
                    calt(calmatc(zn, cs["ecN"], 0, 0, 0), _lumped(zn, cs["ecN"], False)))

        for z in range(nz):
            x = ra[isp[z] - 1: isp[z] - 1 + nlayer[z] + 1]
            sl = slice(jsp[z] - 1, jsp[z] - 1 + 4 * nlayer[z])
            t[sl], h1[sl], h2[sl], h3[sl], h4[sl] = integrals(_Zone(x, None), structure(z, x))
        gcs = structure(spn - 1, gra)
        mu0 = gcs["ecL"][1]
        gt, gh1, gh2, gh3, gh4 = integrals(_Zone(gra, None), gcs)
        ns = int(isp[spn - 1]) + int(math.trunc(spo))
        ins = 4 * ns - 3

        self._keep = []

        def dp(a):
            a = np.ascontiguousarray(a, np.float64)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def ip(a):
            a = np.ascontiguousarray(a, np.int32)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int))

        s = ShSetup()
        s.nzone = nz
        s.vrmin, s.vrmax, s.vsv, s.qmu = dp(m["vrmin"]), dp(m["vrmax"]), dp(m["vsv"].T.reshape(-1)), dp(m["qmu"])
        s.nlayer, s.isp, s.jsp = ip(nlayer), ip(isp), ip(jsp)
        s.nnlayer = nnlayer
        s.t, s.h1, s.h2, s.h3, s.h4 = dp(t), dp(h1), dp(h2), dp(h3), dp(h4)
        s.spn, s.spo, s.r0, s.mu0, s.ins = spn, spo, r0, mu0, ins
        s.gt, s.gh1, s.gh2, s.gh3, s.gh4 = dp(gt), dp(gh1), dp(gh2), dp(gh3), dp(gh4)
        s.r_n, s.r, s.rrsta, s.iista = r_n, dp(r_), dp(rrsta.reshape(-1)), ip(iista.reshape(-1))
        s.theta_n, s.theta = theta_n, dp(theta)
        s.tlen, s.omegai, s.ratl, s.maxlmax = tlen, omegai, conf["ratl"], conf["maxlmax"]
        s.imin, s.imax = par["imin"], par["imax"]
        s.rsgt_switch, s.tsgt_switch, s.synn_switch = par["rsgt"], par["tsgt"], par["synn"]
        s._owner = self  # the struct points into arrays this object holds
        self.s = s
        self.ptr = C.pointer(s)
        self.n_nodes = self.n_unknowns = nnlayer + 1

    @property
    def r_n(self) -> int:
        return self.s.r_n

    @property
    def theta_n(self) -> int:
        return self.s.theta_n

    def out_shapes(self, n: int):
        nt, nr, ns = self.num
        return ((n, self.theta_n, self.r_n, nt), (n, self.theta_n, self.r_n, nr), (n, self.theta_n, ns))


def sh_setup(job) -> ShOracleSetup:
    """The oracle's SH set-up of a job (parameter file, DSM.config, model)."""
    return ShOracleSetup(job.param_text, job.conf_text, job.model_text)


def setup(job, mode: str):
    """The oracle's set-up of a job for mode "psv" or "sh"."""
    return psv_setup(job) if mode == "psv" else sh_setup(job)
