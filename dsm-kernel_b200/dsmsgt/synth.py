"""Seeded synthetic inputs in the reference's file formats.

Writes 1-D polynomial models in the ``*.psv.model`` layout read by
``src/SGTpsv/SGTpsv-MPI.f90:100-105`` (header ``nzone``, then per zone the
radii, four coefficients each of rho, Vpv, Vph, Vsv, Vsh, eta in
x = r / rmax, then Qmu and Qkappa; ``#`` comments; ``end`` terminator), the
stdin parameter file of ``pinput`` (``src/SGTpsv/others.f90:1-72``) and
``DSM.config`` (``readDSMconf``, ``:74-111``).

No public benchmark models are used.  Profiles are quadratic in x with
seed-drawn end values and curvature inside the ranges below (see the
synthetic-model table of the project design notes).
"""
from __future__ import annotations

import numpy as np

RMAX = 6371.0


def _quad_coeffs(rb: float, rt: float, vb: float, vt: float, curv: float) -> list[float]:
    """Coefficients (c0, c1, c2, 0) of v(x) = vb + (vt-vb)(x-xb)/(xt-xb) + curv (x-xb)(x-xt)."""
    xb, xt = rb / RMAX, rt / RMAX
    s = (vt - vb) / (xt - xb)
    c2 = curv
    c1 = s - curv * (xb + xt)
    c0 = vb - s * xb + curv * xb * xt
    return [c0, c1, c2, 0.0]


def _zone_block(rb, rt, rho, vpv, vph, vsv, vsh, eta, qmu, qkappa) -> str:
    def row(c):
        return "".join(f"{v:19.11e}" for v in c)
    # every record stays within the 120 characters of the reference's a120 read
    lines = [f"{rb:10.3f}{rt:10.3f}" + row(rho)]
    for c in (vpv, vph, vsv, vsh):
        lines.append(" " * 20 + row(c))
    lines.append(" " * 20 + row(eta) + f"{qmu:11.3f}{qkappa:11.3f}")
    return "\n".join(lines)


def _profile(rng, radii, top, bottom, jitter, curv_scale):
    """End values per zone along a monotone profile bottom -> top."""
    n = len(radii) - 1
    r = np.asarray(radii, dtype=float)
    frac = (r - r[0]) / (r[-1] - r[0])
    base = bottom + (top - bottom) * frac
    vals = base + rng.uniform(-jitter, jitter, size=base.shape)
    out = []
    for i in range(n):
        curv = rng.uniform(-curv_scale, curv_scale)
        out.append(_quad_coeffs(r[i], r[i + 1], vals[i], vals[i + 1], curv))
    return out


def sh_mantle_model(seed: int = 0) -> str:
    """SH model: 5 solid zones 3480-6371 km; Vs 7.2 -> 6.0 km/s, rho 5.5 ->
    3.3 g/cc (bottom -> top), Qmu in [80, 600]."""
    rng = np.random.default_rng(seed)
    inner = np.sort(rng.uniform(3480.0 + 150, RMAX - 150, size=4))
    radii = [3480.0, *inner.tolist(), RMAX]
    vs = _profile(rng, radii, 6.0, 7.2, 0.05, 0.3)
    rho = _profile(rng, radii, 3.3, 5.5, 0.05, 0.3)
    blocks = []
    for i in range(5):
        vsc = vs[i]
        vpc = [1.8 * c for c in vsc]
        q = float(rng.uniform(80.0, 600.0))
        blocks.append(_zone_block(radii[i], radii[i + 1], rho[i], vpc, vpc, vsc, vsc,
                                  [1.0, 0.0, 0.0, 0.0], q, 57823.0))
    head = (f"# synthetic SH mantle model, seed {seed}\n"
            "    5   nzone\n")
    return head + "\n".join(blocks) + "\nend\n"


def psv_earth_model(seed: int = 0) -> str:
    """PSV model: solid inner core (0-1221.5 km), fluid outer core
    (1221.5-3480 km, Vs = 0, Qmu = -1) and 6 mantle/crust zones.  Ranges:
    Vp 5.8-13.7, Vs 0-7.3 km/s, rho 2.6-13.0 g/cc."""
    rng = np.random.default_rng(seed)
    blocks = []
    # inner core
    ic = (0.0, 1221.5)
    blocks.append(_zone_block(
        *ic,
        _quad_coeffs(*ic, 13.0, 12.76, rng.uniform(-0.1, 0.1)),
        _quad_coeffs(*ic, 11.26, 11.02, rng.uniform(-0.1, 0.1)),
        _quad_coeffs(*ic, 11.26, 11.02, 0.0),
        _quad_coeffs(*ic, 3.67, 3.50, rng.uniform(-0.05, 0.05)),
        _quad_coeffs(*ic, 3.67, 3.50, 0.0),
        [1.0, 0.0, 0.0, 0.0], 84.6, 1327.7))
    # outer core (fluid: all four Vs coefficients exactly zero)
    oc = (1221.5, 3480.0)
    vp_oc = _quad_coeffs(*oc, 10.36, 8.06, rng.uniform(-0.5, 0.5))
    blocks.append(_zone_block(
        *oc,
        _quad_coeffs(*oc, 12.17, 9.90, rng.uniform(-0.5, 0.5)),
        vp_oc, vp_oc, [0.0] * 4, [0.0] * 4,
        [1.0, 0.0, 0.0, 0.0], -1.0, 57823.0))
    # mantle and crust
    inner = np.sort(rng.uniform(3480.0 + 100, RMAX - 60, size=4))
    radii = [3480.0, *inner.tolist(), RMAX - 25.0, RMAX]
    vp = _profile(rng, radii[:-1], 8.1, 13.7, 0.1, 0.5)
    vs = _profile(rng, radii[:-1], 4.5, 7.3, 0.05, 0.3)
    rho = _profile(rng, radii[:-1], 3.4, 5.5, 0.05, 0.3)
    for i in range(5):
        q = float(rng.uniform(80.0, 600.0))
        blocks.append(_zone_block(radii[i], radii[i + 1], rho[i], vp[i], vp[i], vs[i], vs[i],
                                  [1.0, 0.0, 0.0, 0.0], q, 57823.0))
    crust = (radii[-2], radii[-1])
    blocks.append(_zone_block(
        *crust,
        _quad_coeffs(*crust, 2.9, 2.6, 0.0),
        _quad_coeffs(*crust, 6.8, 5.8, 0.0), _quad_coeffs(*crust, 6.8, 5.8, 0.0),
        _quad_coeffs(*crust, 3.9, 3.2, 0.0), _quad_coeffs(*crust, 3.9, 3.2, 0.0),
        [1.0, 0.0, 0.0, 0.0], 600.0, 57823.0))
    head = (f"# synthetic PSV Earth model, seed {seed}\n"
            f"    {len(blocks)}   nzone\n")
    return head + "\n".join(blocks) + "\nend\n"


def dsm_config(re: float = 1.0e-2, ratc: float = 1.0e-10, ratl: float = 1.0e-5,
               omegai: float = 1.0e-2, maxlmax: int = 80000) -> str:
    """DSM.config in the layout of etc/DSMconfiguration/DSM.config."""
    return (f"# DSM configuration (synthetic run)\n# 1. re\n{re!r}\n# 2. ratc\n{ratc!r}\n"
            f"# 3. ratl\n{ratl!r}\n# 4. omegai attenuation\n{omegai!r}\n"
            f"# 5. maxlmax\n{maxlmax}\nend\n")


def param_file(*, tlen: float, rmin: float, rmax: float, rdelta: float, r0: float,
               thmin: float, thmax: float, thdelta: float, imin: int, imax: int,
               modelname: str = "synthetic", outdir: str = "./out",
               conf: str = "DSM.config", model: str = "model.psv.model",
               switches=(1, 1, 1, 0)) -> str:
    """Parameter file read from stdin by pinput (9 items)."""
    sw = " ".join(str(int(s)) for s in switches)
    return (f"# 0. DSM configuration file\n{conf}\n# 1. outputDir\n{outdir}\n"
            f"# 2. psvmodel\n{model}\n# 3. modelname\n{modelname}\n"
            f"# 4. tlen\n{tlen!r}d0\n# 5. r min, max, delta (km)\n{rmin!r} {rmax!r} {rdelta!r}\n"
            f"# 6. source radius (km)\n{r0!r}\n# 7. theta min, max, delta (deg)\n"
            f"{thmin!r} {thmax!r} {thdelta!r}\n# 8. imin imax\n{imin} {imax}\n"
            f"# 9. rsgt tsgt synn psgt switches\n{sw}\nend\n")
