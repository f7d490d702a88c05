"""Driver-side set-up (grid, element integrals, receivers) against closed
forms, on CPU.  The element integrals restate calmatc/caltl/calhl/pinteg of
the reference (src/SGTsh/calmat.f90, src/SGTpsv/calmat.f90); sums over the
elements are integrals of polynomial profiles that numpy evaluates exactly."""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small

P = np.polynomial.polynomial
RMAX = 6371.0


def zones_of(model_text):
    """Zone radii and coefficient rows of a *.model text (reference layout)."""
    lines = [ln for ln in model_text.splitlines() if not ln.startswith("#")]
    nz = int(lines[0].split()[0])
    zs = []
    for z in range(nz):
        blk = lines[1 + 6 * z: 7 + 6 * z]

        def co(ln):
            return [float(ln[20 + 19 * k: 39 + 19 * k]) for k in range(4)]
        zs.append(dict(rb=float(blk[0][0:10]), rt=float(blk[0][10:20]), rho=co(blk[0]),
                       vpv=co(blk[1]), vsv=co(blk[3]), eta=co(blk[5])))
    return zs


def in_r(c):
    """Coefficients in x = r/rmax -> coefficients in r."""
    return np.asarray(c) / RMAX ** np.arange(len(c))


def integral(c, a, b):
    i = P.polyint(c)
    return P.polyval(b, i) - P.polyval(a, i)


def arr(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


@pytest.fixture(scope="module")
def sh(built):
    job = sh_small()
    return job, dsmsgt.Setup(job, "sh")


@pytest.fixture(scope="module")
def psv(built):
    job = psv_small()
    return job, dsmsgt.Setup(job, "psv")


def test_params_parsed(sh):
    job, s = sh
    p = s.params
    assert p.tlen == pytest.approx(1638.4)
    assert s.r_n == len(np.arange(3500.0, 6300.0 + 1e-9, 350.0))
    assert s.theta_n == 13
    th = arr(s.s.theta, s.theta_n)
    assert np.allclose(th, np.arange(0, 181, 15.0))


def test_sh_mass_matrix_integrates_rho_r2(sh):
    """Each linear element's 2x2 mass matrix sums to its integral of rho r^2."""
    job, s = sh
    t = arr(s.s.t, 4 * s.s.nnlayer)
    exact = sum(integral(P.polymul(in_r(z["rho"]), [0, 0, 1]), z["rb"], z["rt"])
                for z in zones_of(job.model_text))
    assert t.sum() == pytest.approx(exact, rel=1e-8)


def test_sh_stiffness_annihilates_constants(sh):
    """Derivative-derivative elements (h1) have zero rows; the symmetrised
    mixed elements (h2) sum to zero per element."""
    _, s = sh
    n = s.s.nnlayer
    h1 = arr(s.s.h1, 4 * n).reshape(n, 4)
    h2 = arr(s.s.h2, 4 * n).reshape(n, 4)
    assert np.abs(h1[:, 0] + h1[:, 1]).max() <= 1e-12 * np.abs(h1).max()
    assert np.abs(h1[:, 2] + h1[:, 3]).max() <= 1e-12 * np.abs(h1).max()
    assert np.abs(h2.sum(axis=1)).max() <= 1e-12 * np.abs(h2).max()


def test_sh_rigidity_integral(sh):
    """h3 sums to the integral of mu = rho Vs^2 (quadrature of the
    reference's profile interpolation: agreement to ~1e-6)."""
    job, s = sh
    h3 = arr(s.s.h3, 4 * s.s.nnlayer)
    mu = sum(integral(P.polymul(in_r(z["rho"]), P.polymul(in_r(z["vsv"]), in_r(z["vsv"]))), z["rb"], z["rt"])
             for z in zones_of(job.model_text))
    assert h3.sum() == pytest.approx(mu, rel=1e-5)


def test_sh_receivers_bracketed(sh):
    _, s = sh
    r = arr(s.s.r, s.r_n)
    rr = arr(s.s.rrsta, 3 * s.r_n).reshape(s.r_n, 3)
    assert np.all(np.diff(rr, axis=1) > 0)
    assert np.all((rr[:, 0] <= r + 1e-9) & (r <= rr[:, 2] + 1e-9))


def test_psv_mass_matrix_integrates_rho_r2(psv):
    job, s = psv
    S = s.s
    sel = arr(S.solid_el, 20 * S.n_sel).reshape(20, S.n_sel)
    solid = [z for z in zones_of(job.model_text) if any(c != 0.0 for c in z["vsv"])]
    exact = sum(integral(P.polymul(in_r(z["rho"]), [0, 0, 1]), z["rb"], z["rt"]) for z in solid)
    assert sel[0].sum() == pytest.approx(exact, rel=1e-8)


def test_psv_fluid_gradient_annihilates_constants(psv):
    _, s = psv
    S = s.s
    fel = arr(S.fluid_el, 3 * S.n_fel).reshape(3, S.n_fel)
    assert abs(fel[0].sum()) <= 1e-12 * max(1.0, np.abs(fel[0]).max())


def test_psv_layout(psv):
    """Unknown count nn = kkdr(nzone) + 2 nlayer(nzone) (solid top zone),
    phases follow the model (solid inner core, fluid outer core)."""
    job, s = psv
    S = s.s
    nz = S.nzone
    ph = arr(S.iphase, nz)
    assert ph[0] == 1 and ph[1] == 2 and np.all(ph[2:] == 1)
    kk = arr(S.kkdr, nz)
    nl = arr(S.nlayer, nz)
    assert S.nn == kk[-1] + 2 * nl[-1] + 1
    assert np.all(np.diff(kk) > 0)
