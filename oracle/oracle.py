"""Oracle loader -- test infrastructure only.

ctypes wrapper of ``oracle/build/liboracle.so``, the CPU FP64 restatement of
the SGTsh / SGTpsv frequency loops; its set-ups come from
``oracle/driver_setup.py`` (the oracle's own restatement of the drivers'
set-up), so an oracle run maps no product library.  Only tests/,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may import this
module; the product (``dsm-kernel_b200``) never does.  Parity status:
unpinned (the Fortran reference cannot be built here and ships no test
vectors).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "liboracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        for name in ("oracle_sh_run", "oracle_psv_run"):
            getattr(L, name).argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        for name in ("oracle_sh_run_parallel", "oracle_psv_run_parallel"):
            getattr(L, name).argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_int]
        L.oracle_psv_run_threads.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def run(setup, freqs, threads: int = 1):
    """Runs the oracle on a dsmsgt.Setup; returns (tsgt, rsgt, synn, llog)
    in the same array layout as dsmsgt.Context.run."""
    from dsmsgt import alloc_outputs  # the harness package, not the product path
    fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
    n = len(fl)
    t, r, y, llog = alloc_outputs(setup, n)
    L = lib()
    ip = fl.ctypes.data_as(C.POINTER(C.c_int))
    lp = llog.ctypes.data_as(C.POINTER(C.c_int))
    sp = C.cast(setup.ptr, C.c_void_p)
    args = (sp, ip, n, t.ctypes.data, r.ctypes.data, y.ctypes.data, lp)
    if setup.mode == "sh":
        if threads > 1:
            L.oracle_sh_run_parallel(*args, threads)
        else:
            L.oracle_sh_run(*args)
    else:
        if threads > 1:
            L.oracle_psv_run_parallel(*args, threads)
        else:
            L.oracle_psv_run(*args)
    return t, r, y, llog


def run_threads(setup, freqs, threads: int):
    """P-SV oracle with each frequency spread over ``threads`` host threads
    (the same values as run()); returns (tsgt, rsgt, synn, llog, t_theta,
    t_total), the last two per frequency in seconds: the time of the parts
    proportional to the number of epicentral distances and the whole time."""
    from dsmsgt import alloc_outputs
    assert setup.mode == "psv"
    fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
    n = len(fl)
    t, r, y, llog = alloc_outputs(setup, n)
    tth, ttot = np.zeros(n), np.zeros(n)
    lib().oracle_psv_run_threads(C.cast(setup.ptr, C.c_void_p), fl.ctypes.data_as(C.POINTER(C.c_int)), n,
                                 t.ctypes.data, r.ctypes.data, y.ctypes.data,
                                 llog.ctypes.data_as(C.POINTER(C.c_int)), threads, tth.ctypes.data,
                                 ttot.ctypes.data)
    return t, r, y, llog, tth, ttot
