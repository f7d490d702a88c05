"""The oracle's own set-ups (oracle/driver_setup.py, a numpy restatement of
the reference's grid, receiver, source and element-integral routines)
against the product's driver-side set-up (host/setup.cpp through
dsm_psv_setup_build / dsm_sh_setup_build), field by field and bit for bit:
two separately written restatements of src/SGTpsv/SGTpsv-MPI.f90:39-477 and
src/SGTsh/SGTsh-MPI.f90:33-347 pin each other.  Also: the oracle's P-SV
frequency loop gives the same values on any number of threads."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import dsmsgt
from cases import psv_small, sh_small

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402  (the benchmark workloads' jobs)
from oracle import driver_setup, oracle as orc  # noqa: E402

INT_FIELDS = ("nzone", "nn", "n_sel", "n_fel", "n_hm", "spn", "jsrc", "r_n", "theta_n", "maxlmax", "imin", "imax",
              "rsgt_switch", "tsgt_switch", "synn_switch")
REAL_FIELDS = ("rmin", "rmax", "spo", "r0", "ecC0", "ecF0", "ecL0", "tlen", "omegai", "ratl")


def _arr(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy()


def _diffs(a, b):
    bad = [f for f in INT_FIELDS + REAL_FIELDS if getattr(a, f) != getattr(b, f)]
    bad += ["ra_src"] * any(a.ra_src[k] != b.ra_src[k] for k in range(2))
    bad += ["src_poly"] * any(a.src_poly[k] != b.src_poly[k] for k in range(24))
    nz, R = a.nzone, a.r_n
    arrays = (("iphase", nz), ("nlayer", nz), ("isp", nz), ("kkdr", nz), ("elem", nz), ("hmoff", nz),
              ("iista", 3 * R), ("istazone", R), ("vrmin", nz), ("vrmax", nz), ("qmu", nz), ("qkappa", nz),
              ("vsv", 4 * nz), ("r", R), ("rrsta", 3 * R), ("lambda_", R), ("qkp", R), ("theta", a.theta_n),
              ("solid_el", 20 * a.n_sel), ("fluid_el", 3 * a.n_fel), ("hm_el", 24 * a.n_hm))
    for f, n in arrays:
        if not np.array_equal(_arr(getattr(a, f), n), _arr(getattr(b, f), n)):
            bad.append(f)
    return bad


JOBS = {
    "psv_small": lambda: psv_small(),
    "psv_small_solid_receivers": lambda: psv_small(seed=1, rmin=3800.0, rdelta=400.0),
    "psv_small_deep_source": lambda: psv_small(seed=2, r0=5771.0),
    "psv1024": lambda: bench.workload("psv1024")[0],
    "psv2048": lambda: bench.workload("psv2048")[0],
}


@pytest.mark.parametrize("name", sorted(JOBS))
def test_oracle_setup_equals_product_setup(built, name):
    job = JOBS[name]()
    prod = dsmsgt.Setup(job, "psv")
    own = driver_setup.psv_setup(job)
    assert _diffs(prod.s, own.s) == []
    assert (own.n_nodes, own.n_unknowns) == (prod.n_nodes, prod.n_unknowns)


def test_oracle_setup_parses_the_reference_formats(built):
    job = psv_small()
    p = driver_setup.parse_params(job.param_text)
    assert p["tlen"] == 1638.4 and (p["imin"], p["imax"]) == (0, 64) and p["model"] == "model.psv.model"
    c = driver_setup.parse_conf(job.conf_text)
    assert c["maxlmax"] == 80000 and c["ratl"] == 1e-5
    m = driver_setup.parse_model(job.model_text)
    assert m["nzone"] == 8 and m["vrmax"][-1] == 6371.0 and np.all(m["vsv"][:, 1] == 0.0)


def test_threaded_oracle_gives_identical_values(built):
    s = driver_setup.psv_setup(psv_small())
    freqs = [3, 20, 41]
    ref = orc.run(s, freqs)
    for th in (2, 5):
        got = orc.run_threads(s, freqs, th)
        for a, b in zip(got[:4], ref[:4]):
            assert np.array_equal(a, b)
        assert np.all(got[4] > 0) and np.all(got[5] >= got[4])


def test_oracle_on_its_own_setup_matches_the_product_setup_run(built):
    job = psv_small(seed=1, rmin=3800.0, rdelta=400.0)
    a = orc.run(dsmsgt.Setup(job, "psv"), [5, 17])
    b = orc.run(driver_setup.psv_setup(job), [5, 17])
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


SH_INT = ("nzone", "nnlayer", "spn", "ins", "r_n", "theta_n", "maxlmax", "imin", "imax", "rsgt_switch",
          "tsgt_switch", "synn_switch")
SH_REAL = ("spo", "r0", "mu0", "tlen", "omegai", "ratl")

SH_JOBS = {
    "sh_small": lambda: sh_small(),
    "sh_small_seed1": lambda: sh_small(seed=1),
    "sh256": lambda: bench.workload("sh256")[0],
    # the outer-core cut and the receivers at or below the CMB dropped
    "sh_on_the_psv_earth": lambda: psv_small(),
}


@pytest.mark.parametrize("name", sorted(SH_JOBS))
def test_oracle_sh_setup_equals_product_setup(built, name):
    job = SH_JOBS[name]()
    prod = dsmsgt.Setup(job, "sh")
    own = driver_setup.sh_setup(job)
    a, b = prod.s, own.s
    bad = [f for f in SH_INT + SH_REAL if getattr(a, f) != getattr(b, f)]
    nz, R, nl = a.nzone, a.r_n, a.nnlayer
    for f, n in (("vrmin", nz), ("vrmax", nz), ("vsv", 4 * nz), ("qmu", nz), ("nlayer", nz), ("isp", nz),
                 ("jsp", nz), ("t", 4 * nl), ("h1", 4 * nl), ("h2", 4 * nl), ("h3", 4 * nl), ("h4", 4 * nl),
                 ("gt", 8), ("gh1", 8), ("gh2", 8), ("gh3", 8), ("gh4", 8), ("r", R), ("rrsta", 3 * R),
                 ("iista", 3 * R), ("theta", a.theta_n)):
        if not np.array_equal(_arr(getattr(a, f), n), _arr(getattr(b, f), n)):
            bad.append(f)
    assert bad == []
