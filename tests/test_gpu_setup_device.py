"""P-SV element integrals built on the device (dsm_psv_setup_build_device)
against the host builder, field by field and bit for bit, on the small
parity models and the benchmark grids (16 788 and 33 560 band rows); the
engine run on either set-up gives the same outputs."""
import time

import numpy as np
import pytest

import dsmsgt
from cases import psv_small
from test_cpu_oracle_setup import JOBS, _diffs


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(JOBS))
def test_device_integrals_equal_host_integrals(built, name):
    job = JOBS[name]()
    t0 = time.perf_counter()
    host = dsmsgt.Setup(job, "psv")
    t1 = time.perf_counter()
    dev = dsmsgt.Setup(job, "psv", device=0)
    t2 = time.perf_counter()
    print(f"{name}: host set-up {1e3 * (t1 - t0):.1f} ms, device integrals {1e3 * (t2 - t1):.1f} ms")
    assert _diffs(host.s, dev.s) == []


@pytest.mark.gpu
def test_engine_on_device_setup(built):
    job = psv_small(seed=2, r0=5771.0)
    a = dsmsgt.Context(dsmsgt.Setup(job, "psv")).run([6, 30])
    b = dsmsgt.Context(dsmsgt.Setup(job, "psv", device=0)).run([6, 30])
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
