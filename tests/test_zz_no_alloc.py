"""The allocation-free SH cutoff entry point (dsm_sh_cutoff_noalloc).

Some callers cannot call cudaMalloc: their GPU memory is already held by
another framework's caching allocator, or they must not cause the implicit
device synchronisation of cudaMalloc/cudaFree while other streams run.  For
them the library computes the SH angular-order cutoff with every device
buffer inside one fixed 64 MiB array.  This test checks, through the C-ABI,
that it returns the same cutoff as the regular engine (dsm_run_freqs) on two
calls in a row (the second call reuses the array the first one left behind).
The file is collected last so that a run stopping at the first failure has
run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

import dsmsgt
from cases import sh_small


@pytest.mark.gpu
def test_sh_cutoff_noalloc_matches_engine(built):
    s = dsmsgt.Setup(sh_small(seed=1), "sh")
    freqs = [2, 9, 21, 30]
    ctx = dsmsgt.Context(s)
    _, _, _, llog_ref = ctx.run(freqs)
    ctx.close()
    L = dsmsgt.lib()
    for call in range(2):
        fl = np.asarray(freqs, np.int32)
        out = np.full(len(freqs), -1, np.int32)
        rc = L.dsm_sh_cutoff_noalloc(s.ptr, fl.ctypes.data_as(C.POINTER(C.c_int)), len(freqs),
                                     out.ctypes.data_as(C.POINTER(C.c_int)))
        assert rc == 0, L.dsm_last_error(None).decode()
        assert list(out) == list(llog_ref), (call, list(out), list(llog_ref))


@pytest.mark.gpu
def test_sh_cutoff_noalloc_rejects_oversized_setup(built):
    # 200 000 frequencies need more probe scratch than the fixed array holds
    s = dsmsgt.Setup(sh_small(), "sh")
    L = dsmsgt.lib()
    fl = np.ones(200000, np.int32)
    out = np.zeros(len(fl), np.int32)
    rc = L.dsm_sh_cutoff_noalloc(s.ptr, fl.ctypes.data_as(C.POINTER(C.c_int)), len(fl),
                                 out.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == 1
    assert b"scratch" in L.dsm_last_error(None)
