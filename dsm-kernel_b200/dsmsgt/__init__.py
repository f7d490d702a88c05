"""ctypes harness of the SGT engine (tests and benchmarks only).

The product is the C-ABI library ``lib/libdsmsgt.so`` declared in
``include/dsmsgt.h`` (engine) and ``include/dsmsgt_host.h`` (driver-side
set-up helpers).  This module loads it, mirrors the structs, and offers
numpy-returning wrappers.  It never computes anything itself: when the
library is missing every call fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import synth  # noqa: F401  (re-export)

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)                 # dsm-kernel_b200/
REPO = os.path.dirname(ROOT)
LIB_PATH = os.path.join(ROOT, "lib", "libdsmsgt.so")

DSM_PREC_FP64 = 0
DSM_PREC_MIXED = 1
DSM_PREC_MIXED_BF16 = 2

SH_NUM = (10, 5, 5)
PSV_NUM = (20, 10, 10)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)


class ShSetup(C.Structure):
    _fields_ = [
        ("nzone", C.c_int), ("vrmin", _dp), ("vrmax", _dp), ("vsv", _dp), ("qmu", _dp),
        ("nlayer", _ip), ("isp", _ip), ("jsp", _ip), ("nnlayer", C.c_int),
        ("t", _dp), ("h1", _dp), ("h2", _dp), ("h3", _dp), ("h4", _dp),
        ("spn", C.c_int), ("spo", C.c_double), ("r0", C.c_double), ("mu0", C.c_double),
        ("ins", C.c_int), ("gt", _dp), ("gh1", _dp), ("gh2", _dp), ("gh3", _dp), ("gh4", _dp),
        ("r_n", C.c_int), ("r", _dp), ("rrsta", _dp), ("iista", _ip),
        ("theta_n", C.c_int), ("theta", _dp),
        ("tlen", C.c_double), ("omegai", C.c_double), ("ratl", C.c_double),
        ("maxlmax", C.c_int), ("imin", C.c_int), ("imax", C.c_int),
        ("rsgt_switch", C.c_int), ("tsgt_switch", C.c_int), ("synn_switch", C.c_int),
    ]


class PsvSetup(C.Structure):
    _fields_ = [
        ("nzone", C.c_int), ("iphase", _ip), ("nlayer", _ip), ("isp", _ip), ("kkdr", _ip),
        ("elem", _ip), ("hmoff", _ip),
        ("vrmin", _dp), ("vrmax", _dp), ("qmu", _dp), ("qkappa", _dp), ("vsv", _dp),
        ("nn", C.c_int), ("rmin", C.c_double), ("rmax", C.c_double),
        ("n_sel", C.c_int), ("n_fel", C.c_int), ("n_hm", C.c_int),
        ("solid_el", _dp), ("fluid_el", _dp), ("hm_el", _dp),
        ("spn", C.c_int), ("spo", C.c_double), ("r0", C.c_double),
        ("ecC0", C.c_double), ("ecF0", C.c_double), ("ecL0", C.c_double),
        ("ra_src", C.c_double * 2), ("src_poly", C.c_double * 24), ("jsrc", C.c_int),
        ("r_n", C.c_int), ("r", _dp), ("rrsta", _dp), ("iista", _ip), ("istazone", _ip),
        ("lambda_", _dp), ("qkp", _dp),
        ("theta_n", C.c_int), ("theta", _dp),
        ("tlen", C.c_double), ("omegai", C.c_double), ("ratl", C.c_double),
        ("maxlmax", C.c_int), ("imin", C.c_int), ("imax", C.c_int),
        ("rsgt_switch", C.c_int), ("tsgt_switch", C.c_int), ("synn_switch", C.c_int),
    ]


class Params(C.Structure):
    _fields_ = [
        ("dsmconf", C.c_char * 256), ("outdir", C.c_char * 256), ("model", C.c_char * 256),
        ("modelname", C.c_char * 128),
        ("tlen", C.c_double), ("rmin_", C.c_double), ("rmax_", C.c_double),
        ("rdelta_", C.c_double), ("r0min", C.c_double),
        ("thetamin", C.c_double), ("thetamax", C.c_double), ("thetadelta", C.c_double),
        ("imin", C.c_int), ("imax", C.c_int),
        ("rsgt_switch", C.c_int), ("tsgt_switch", C.c_int), ("synn_switch", C.c_int),
        ("psgt_switch", C.c_int),
    ]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("use_lmax_predictor", C.c_int),
                ("l_chunk", C.c_int), ("freq_batch", C.c_int)]


class Out(C.Structure):
    _fields_ = [("tsgt", _dp), ("rsgt", _dp), ("synn", _dp),
                ("tsgt32", _fp), ("rsgt32", _fp), ("synn32", _fp), ("llog", _ip)]


class KStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("ms", C.c_double), ("launches", C.c_longlong),
                ("alg_bytes", C.c_double), ("alg_flops", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_solve", C.c_double), ("ms_lsum", C.c_double),
                ("ms_pack", C.c_double), ("ms_h2d", C.c_double), ("ms_d2h", C.c_double),
                ("launches", C.c_longlong), ("systems", C.c_longlong),
                ("orders_used", C.c_longlong), ("orders_padded", C.c_longlong),
                ("lsum_flops", C.c_double), ("solve_bytes", C.c_double),
                ("nk", C.c_int), ("kern", KStat * 24), ("solve_rounds", C.c_longlong),
                ("freqs_extended", C.c_longlong), ("lsum_flops_exec", C.c_double)]

    def kernels(self):
        return {self.kern[i].name.decode(): (self.kern[i].ms, self.kern[i].launches,
                                             self.kern[i].alg_bytes, self.kern[i].alg_flops)
                for i in range(self.nk)}


DSM_OK = 0
DSM_ERR_INVALID = 1
DSM_ERR_CUDA = 2
DSM_ERR_NONFINITE = 3
DSM_ERR_LMAX = 4
DSM_ERR_TIMEOUT = 5
DSM_ERR_NOMEM = 6
DSM_ERR_NODEVICE = 7


class Tuning(C.Structure):
    _fields_ = [("fac_rows", C.c_int), ("fld_orders", C.c_int), ("tc_orders", C.c_int), ("fwd_merge", C.c_int)]


class Accuracy(C.Structure):
    _fields_ = [("nfreq", C.c_int), ("llog_equal", C.c_int), ("tsgt", C.c_double * 20),
                ("rsgt", C.c_double * 10), ("synn", C.c_double * 10), ("tsgt_max", C.c_double),
                ("rsgt_max", C.c_double), ("synn_max", C.c_double)]


class DsmError(RuntimeError):
    """A failed library call; ``code`` is its DSM_ERR_* return code (0 when
    the failure was found on the Python side)."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class CatParams(C.Structure):
    _fields_ = [("num", C.c_int), ("theta_n", C.c_int), ("theta_min", C.c_double),
                ("theta_delta", C.c_double), ("fmin", C.c_int), ("fmax", C.c_int), ("np1", C.c_int),
                ("tlen", C.c_double), ("omegai", C.c_double), ("ipdistance", C.c_double),
                ("c_red_reci", C.c_double), ("iwin_start", C.c_int), ("iwin_end", C.c_int),
                ("device", C.c_int)]


class CatKernelParams(C.Structure):
    _fields_ = [("types", C.c_int), ("nfilter", C.c_int), ("fclp", C.POINTER(C.c_double)),
                ("fchp", C.POINTER(C.c_double)), ("npoles", C.c_int), ("sampling_hz", C.c_double),
                ("nt1", C.POINTER(C.c_int)), ("nt2", C.POINTER(C.c_int)), ("nr", C.c_int), ("nktype", C.c_int),
                ("coeff", C.POINTER(C.c_double)), ("jacobian", C.c_void_p)]


KER_VP, KER_VS = 1, 2

_lib = None


def lib() -> C.CDLL:
    """Loads libdsmsgt.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DsmError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
        L = C.CDLL(LIB_PATH)
        L.dsm_parse_params.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.dsm_sh_setup_build.argtypes = [C.POINTER(Params), C.c_char_p, C.c_char_p,
                                         C.POINTER(C.c_void_p), C.POINTER(C.POINTER(ShSetup))]
        L.dsm_psv_setup_build.argtypes = [C.POINTER(Params), C.c_char_p, C.c_char_p,
                                          C.POINTER(C.c_void_p), C.POINTER(C.POINTER(PsvSetup))]
        L.dsm_psv_setup_build_device.argtypes = [C.POINTER(Params), C.c_char_p, C.c_char_p, C.c_int,
                                                 C.POINTER(C.c_void_p), C.POINTER(C.POINTER(PsvSetup))]
        L.dsm_bundle_free.argtypes = [C.c_void_p]
        L.dsm_bundle_info.argtypes = [C.c_void_p, _ip, _ip]
        L.dsm_host_last_error.restype = C.c_char_p
        L.dsm_sh_create.argtypes = [C.POINTER(ShSetup), C.POINTER(Options), C.POINTER(C.c_void_p)]
        L.dsm_psv_create.argtypes = [C.POINTER(PsvSetup), C.POINTER(Options), C.POINTER(C.c_void_p)]
        L.dsm_run_freqs.argtypes = [C.c_void_p, _ip, C.c_int, C.POINTER(Out)]
        L.dsm_psv_create_multi.argtypes = [C.POINTER(C.POINTER(PsvSetup)), C.c_int, C.POINTER(Options),
                                           C.POINTER(C.c_void_p)]
        L.dsm_run_freqs_multi.argtypes = [C.c_void_p, _ip, C.c_int, C.POINTER(Out), C.c_int]
        L.dsm_run_request.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(_ip), _ip,
                                      C.POINTER(C.POINTER(Out)), _ip]
        L.dsm_set_depth_cutoff.argtypes = [C.c_void_p, C.c_double]
        L.dsm_get_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
        L.dsm_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
        L.dsm_autotune.argtypes = [C.c_void_p, _ip, C.c_int, C.c_int, C.POINTER(Tuning), _dp]
        L.dsm_run_freqs_device.argtypes = [C.c_void_p, _ip, C.c_int, C.POINTER(C.c_void_p),
                                           C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), _ip]
        L.dsm_ctx_destroy.argtypes = [C.c_void_p]
        L.dsm_last_error.argtypes = [C.c_void_p]
        L.dsm_last_error.restype = C.c_char_p
        L.dsm_strerror.restype = C.c_char_p
        L.dsm_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.dsm_set_profiling.argtypes = [C.c_void_p, C.c_int]
        L.dsm_debug_set.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.dsm_set_fp64_check.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.dsm_get_accuracy.argtypes = [C.c_void_p, C.POINTER(Accuracy)]
        L.dsm_sh_cutoff_noalloc.argtypes = [C.POINTER(ShSetup), _ip, C.c_int, _ip]
        _f = C.POINTER(C.c_float)
        L.dsm_lmax_features.argtypes = [C.c_void_p, _ip, C.c_int, _f]
        L.dsm_cutoffs.argtypes = [C.c_void_p, _ip, C.c_int, _ip]
        L.dsm_lmax_init.argtypes = [_f, _f, C.c_int, C.c_uint, _f]
        L.dsm_lmax_train.argtypes = [_f, _f, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint, _f,
                                     _f, C.c_int]
        L.dsm_lmax_grad.argtypes = [_f, _f, _f, C.c_int, _f, _f, C.c_int]
        L.dsm_set_lmax_model.argtypes = [C.c_void_p, _f]
        L.dsm_lmax_predict.argtypes = [C.c_void_p, _ip, C.c_int, _f]
        L.dsm_cat_np1.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, _ip, _dp,
                                  _ip, _ip]
        L.dsm_cat_create.argtypes = [C.POINTER(CatParams), C.POINTER(C.c_void_p)]
        L.dsm_cat_add.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, _ip, _dp, C.c_int]
        L.dsm_cat_clear.argtypes = [C.c_void_p]
        L.dsm_cat_series.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, _dp, C.c_void_p, C.c_int]
        L.dsm_cat_spectra.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, _dp, C.c_void_p, C.c_int]
        L.dsm_cat_transform.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.dsm_cat_h3h4_coef.argtypes = [C.c_int, _dp, C.c_char, _dp, C.c_void_p, C.c_void_p]
        L.dsm_cat_filter.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.dsm_cat_set_kernel_params.argtypes = [C.c_void_p, C.POINTER(CatKernelParams)]
        L.dsm_cat_kernels.argtypes = [C.c_void_p, C.c_int, _ip, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_int]
        L.dsm_cat_set_profiling.argtypes = [C.c_void_p, C.c_int]
        L.dsm_cat_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.dsm_cat_set_batch_bytes.argtypes = [C.c_void_p, C.c_size_t]
        L.dsm_cat_destroy.argtypes = [C.c_void_p]
        L.dsm_cat_last_error.argtypes = [C.c_void_p]
        L.dsm_cat_last_error.restype = C.c_char_p
        L.dsm_fp64_peak.argtypes = [C.c_int, _dp]
        L.dsm_fp64_mma_peak.argtypes = [C.c_int, _dp]
        _lib = L
    return _lib


_selftest = None


def _selftest_lib() -> C.CDLL:
    """The test-only library of the contraction's self-test (built beside
    the engine's, linked against it)."""
    global _selftest
    if _selftest is None:
        lib()
        path = os.path.join(os.path.dirname(LIB_PATH), "libdsmsgt_selftest.so")
        if not os.path.exists(path):
            raise DsmError(f"{path} is missing: run __graft_entry__.build() first")
        _selftest = C.CDLL(path)
        _selftest.dsm_tc_selftest.restype = C.c_int
        _selftest.dsm_tc_selftest.argtypes = [C.c_int] * 10 + [C.POINTER(C.c_double)]
    return _selftest


def tc_selftest(M: int, N: int, K: int, nfreq: int = 1, fmt: int = 0, bk: int = 32, reps: int = 0,
                check: bool = True, flags: int = 1, chunk: int = 2) -> dict:
    """Runs the tensor-core split contraction on seeded pieces (fmt 0 fp16,
    1 bf16) and, with check, compares it with an FP64 sum of the same piece
    products.  flags: 1 high-to-low order; chunk: stages per hi*hi chunk
    summed in FP64 (0: one chunk per tile).
    Returns max |error|, max |reference|, ms per launch and the tensor
    flops of one launch."""
    L = lib()
    T = _selftest_lib()
    res = (C.c_double * 4)()
    rc = T.dsm_tc_selftest(M, N, K, nfreq, fmt, bk, flags, chunk, reps, int(check), res)
    if rc:
        raise DsmError(f"dsm_tc_selftest failed ({rc}): {L.dsm_last_error(None).decode()}")
    return {"max_err": res[0], "ref_max": res[1], "ms": res[2], "flops": res[3]}


LMAX_NFEAT = 11
LMAX_WIDTH = 128
LMAX_NPARAM = 34713


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


def lmax_init(X, T, seed: int = 0) -> np.ndarray:
    """Parameter block: standardisation from (X, T) and He-initialised weights."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    P = np.zeros(LMAX_NPARAM, np.float32)
    rc = lib().dsm_lmax_init(_fptr(X), _fptr(T), len(T), seed, _fptr(P))
    if rc:
        raise DsmError("dsm_lmax_init failed")
    return P


def lmax_train(X, T, params, epochs: int = 200, batch: int = 256, lr: float = 1e-3, seed: int = 0,
               device: int = 0, weight_decay: float = 0.0):
    """Adam on the GPU with the project's forward/backward kernels; returns
    (trained parameters, per-epoch loss)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    P = np.ascontiguousarray(params, dtype=np.float32).copy()
    losses = np.zeros(epochs, np.float32)
    rc = lib().dsm_lmax_train(_fptr(X), _fptr(T), len(T), epochs, batch, lr, weight_decay, seed, _fptr(P),
                              _fptr(losses), device)
    if rc:
        raise DsmError(f"dsm_lmax_train failed ({rc}): {lib().dsm_last_error(None).decode()}")
    return P, losses


def lmax_grad(params, X, T, device: int = 0):
    """Loss and gradient of the network on (X, T) from the GPU kernels."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    P = np.ascontiguousarray(params, dtype=np.float32)
    G = np.zeros(LMAX_NPARAM, np.float32)
    loss = np.zeros(1, np.float32)
    rc = lib().dsm_lmax_grad(_fptr(P), _fptr(X), _fptr(T), len(T), _fptr(G), _fptr(loss), device)
    if rc:
        raise DsmError(f"dsm_lmax_grad failed ({rc}): {lib().dsm_last_error(None).decode()}")
    return G, float(loss[0])


def _ptr(a: np.ndarray, typ):
    return a.ctypes.data_as(typ)


@dataclass
class Job:
    """Inputs of one run: parameter file, DSM.config and model contents."""
    param_text: str
    conf_text: str
    model_text: str


class Setup:
    """Driver-side set-up (grid and element integrals) built by the library."""

    def __init__(self, job: Job, mode: str, device: int | None = None):
        """device: build the P-SV element integrals on that CUDA device
        (dsm_psv_setup_build_device) instead of the host."""
        L = lib()
        self.mode = mode
        self.job = job
        self.params = Params()
        rc = L.dsm_parse_params(job.param_text.encode(), C.byref(self.params))
        if rc:
            raise DsmError(L.dsm_host_last_error().decode())
        self._bundle = C.c_void_p()
        if mode == "sh":
            self.ptr = C.POINTER(ShSetup)()
            rc = L.dsm_sh_setup_build(C.byref(self.params), job.conf_text.encode(),
                                      job.model_text.encode(), C.byref(self._bundle),
                                      C.byref(self.ptr))
            self.num = SH_NUM
        elif mode == "psv":
            self.ptr = C.POINTER(PsvSetup)()
            if device is None:
                rc = L.dsm_psv_setup_build(C.byref(self.params), job.conf_text.encode(),
                                           job.model_text.encode(), C.byref(self._bundle),
                                           C.byref(self.ptr))
            else:
                rc = L.dsm_psv_setup_build_device(C.byref(self.params), job.conf_text.encode(),
                                                  job.model_text.encode(), device, C.byref(self._bundle),
                                                  C.byref(self.ptr))
            self.num = PSV_NUM
        else:
            raise ValueError(mode)
        if rc:
            raise DsmError(L.dsm_host_last_error().decode())
        self.s = self.ptr.contents
        nodes, unk = C.c_int(), C.c_int()
        L.dsm_bundle_info(self._bundle, C.byref(nodes), C.byref(unk))
        self.n_nodes, self.n_unknowns = nodes.value, unk.value

    @property
    def r_n(self) -> int:
        return self.s.r_n

    @property
    def theta_n(self) -> int:
        return self.s.theta_n

    def out_shapes(self, n: int):
        nt, nr, ns = self.num
        return ((n, self.theta_n, self.r_n, nt), (n, self.theta_n, self.r_n, nr),
                (n, self.theta_n, ns))

    def __del__(self):
        try:
            if getattr(self, "_bundle", None) and self._bundle.value:
                lib().dsm_bundle_free(self._bundle)
                self._bundle = C.c_void_p()
        except Exception:
            pass


def alloc_outputs(setup: Setup, n: int):
    """Complex128 outputs in the reference's column-major order, returned as
    C-order arrays [k][itheta][ir][comp] (same memory layout)."""
    st, sr, ss = setup.out_shapes(n)
    return (np.zeros(st, np.complex128), np.zeros(sr, np.complex128),
            np.zeros(ss, np.complex128), np.zeros(n, np.int32))


class Context:
    """A device context of the engine (dsm_sh_create / dsm_psv_create)."""

    def __init__(self, setup: Setup, precision: int = DSM_PREC_FP64, device: int = 0,
                 use_lmax_predictor: int = 0, l_chunk: int = 0, freq_batch: int = 0):
        L = lib()
        self.setup = setup
        self.opt = Options(precision, device, use_lmax_predictor, l_chunk, freq_batch)
        self.h = C.c_void_p()
        fn = L.dsm_sh_create if setup.mode == "sh" else L.dsm_psv_create
        rc = fn(setup.ptr, C.byref(self.opt), C.byref(self.h))
        if rc:
            msg = L.dsm_last_error(self.h).decode() if self.h.value else L.dsm_strerror(rc).decode()
            raise DsmError(f"create failed ({rc}): {msg}", rc)

    def run(self, freqs, want32: bool = False):
        L = lib()
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        n = len(fl)
        t, r, y, llog = alloc_outputs(self.setup, n)
        out = Out()
        out.tsgt = t.ctypes.data_as(_dp)
        out.rsgt = r.ctypes.data_as(_dp)
        out.synn = y.ctypes.data_as(_dp)
        out.llog = llog.ctypes.data_as(_ip)
        t32 = r32 = y32 = None
        if want32:
            nt, nr, ns = self.setup.num
            t32 = np.zeros((n, self.setup.r_n, self.setup.theta_n, nt), np.complex64)
            r32 = np.zeros((n, self.setup.r_n, self.setup.theta_n, nr), np.complex64)
            y32 = np.zeros((n, self.setup.theta_n, ns), np.complex64)
            out.tsgt32 = t32.ctypes.data_as(_fp)
            out.rsgt32 = r32.ctypes.data_as(_fp)
            out.synn32 = y32.ctypes.data_as(_fp)
        rc = L.dsm_run_freqs(self.h, _ptr(fl, _ip), n, C.byref(out))
        if rc:
            raise DsmError(f"dsm_run_freqs failed ({rc}): {L.dsm_last_error(self.h).decode()}", rc)
        if want32:
            return t, r, y, llog, (t32, r32, y32)
        return t, r, y, llog

    def set_profiling(self, on: bool):
        lib().dsm_set_profiling(self.h, 1 if on else 0)

    def set_fp64_check(self, ref, stride: int = 1):
        """Attaches an FP64 context of the same set-up (None detaches): later
        runs recompute every stride-th frequency in FP64 and report the
        per-component relative L2 (dsm_set_fp64_check)."""
        rc = lib().dsm_set_fp64_check(self.h, ref.h if ref is not None else None, stride)
        if rc:
            raise DsmError(f"dsm_set_fp64_check failed ({rc}): {lib().dsm_last_error(self.h).decode()}", rc)
        self._check_ref = ref  # keeps it alive while attached

    def accuracy(self) -> dict:
        """Accuracy report of the last run (dsm_get_accuracy)."""
        a = Accuracy()
        lib().dsm_get_accuracy(self.h, C.byref(a))
        nt, nr, ns = self.setup.num
        return {"nfreq": a.nfreq, "llog_equal": bool(a.llog_equal), "tsgt": list(a.tsgt[:nt]),
                "rsgt": list(a.rsgt[:nr]), "synn": list(a.synn[:ns]), "tsgt_max": a.tsgt_max,
                "rsgt_max": a.rsgt_max, "synn_max": a.synn_max}

    def set_depth_cutoff(self, bound: float):
        """Amplitude bound of the P-SV depth cut-off (dsm_set_depth_cutoff;
        0 = the whole band)."""
        rc = lib().dsm_set_depth_cutoff(self.h, float(bound))
        if rc:
            raise DsmError(f"dsm_set_depth_cutoff failed ({rc}): {lib().dsm_last_error(self.h).decode()}", rc)

    def tuning(self) -> dict:
        t = Tuning()
        lib().dsm_get_tuning(self.h, C.byref(t))
        return {"fac_rows": t.fac_rows, "fld_orders": t.fld_orders, "tc_orders": t.tc_orders,
                "fwd_merge": t.fwd_merge}

    def set_tuning(self, fac_rows: int = 16, fld_orders: int = 32, tc_orders: int = 64, fwd_merge: int = 1):
        t = Tuning(fac_rows, fld_orders, tc_orders, fwd_merge)
        rc = lib().dsm_set_tuning(self.h, C.byref(t))
        if rc:
            raise DsmError(f"dsm_set_tuning failed ({rc}): {lib().dsm_last_error(self.h).decode()}", rc)

    def autotune(self, freqs, reps: int = 2):
        """Measures the tile shapes on this request and keeps the fastest
        (dsm_autotune); returns (tuning dict, ms per request)."""
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        t, ms = Tuning(), C.c_double()
        rc = lib().dsm_autotune(self.h, _ptr(fl, _ip), len(fl), reps, C.byref(t), C.byref(ms))
        if rc:
            raise DsmError(f"dsm_autotune failed ({rc}): {lib().dsm_last_error(self.h).decode()}", rc)
        return {"fac_rows": t.fac_rows, "fld_orders": t.fld_orders, "tc_orders": t.tc_orders,
                "fwd_merge": t.fwd_merge}, ms.value

    def debug_set(self, name: str, value: int = 1):
        """Test hook of the library's error paths (dsm_debug_set)."""
        rc = lib().dsm_debug_set(self.h, name.encode(), value)
        if rc:
            raise DsmError(f"dsm_debug_set failed ({rc}): {lib().dsm_last_error(self.h).decode()}", rc)

    def run_device(self, freqs):
        """Runs with outputs left on the device; returns llog."""
        L = lib()
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        llog = np.zeros(len(fl), np.int32)
        dt, dr, ds = C.c_void_p(), C.c_void_p(), C.c_void_p()
        rc = L.dsm_run_freqs_device(self.h, _ptr(fl, _ip), len(fl), C.byref(dt), C.byref(dr),
                                    C.byref(ds), _ptr(llog, _ip))
        if rc:
            raise DsmError(f"dsm_run_freqs_device failed ({rc}): {L.dsm_last_error(self.h).decode()}", rc)
        return llog

    def run_host32(self, freqs, t32, r32, y32, llog):
        """Runs with complex64 catalogue outputs copied into caller buffers
        (addresses of pinned host memory)."""
        L = lib()
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        out = Out()
        out.tsgt32 = C.cast(C.c_void_p(t32), _fp)
        out.rsgt32 = C.cast(C.c_void_p(r32), _fp) if r32 else None
        out.synn32 = C.cast(C.c_void_p(y32), _fp) if y32 else None
        out.llog = _ptr(llog, _ip)
        rc = L.dsm_run_freqs(self.h, _ptr(fl, _ip), len(fl), C.byref(out))
        if rc:
            raise DsmError(f"dsm_run_freqs failed ({rc}): {L.dsm_last_error(self.h).decode()}", rc)

    def cutoffs(self, freqs):
        """Realised cutoffs (llog) only: banded solves and the amplitude
        test, no l-sum (dsm_cutoffs)."""
        L = lib()
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        llog = np.zeros(len(fl), np.int32)
        rc = L.dsm_cutoffs(self.h, _ptr(fl, _ip), len(fl), _ptr(llog, _ip))
        if rc:
            raise DsmError(f"dsm_cutoffs failed ({rc}): {L.dsm_last_error(self.h).decode()}", rc)
        return llog

    def lmax_features(self, freqs):
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        f = np.zeros((len(fl), LMAX_NFEAT), np.float32)
        rc = lib().dsm_lmax_features(self.h, _ptr(fl, _ip), len(fl), _fptr(f))
        if rc:
            raise DsmError("dsm_lmax_features failed")
        return f

    def set_lmax_model(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == LMAX_NPARAM
        rc = lib().dsm_set_lmax_model(self.h, _fptr(p))
        if rc:
            raise DsmError(f"dsm_set_lmax_model failed ({rc}): {lib().dsm_last_error(self.h).decode()}")

    def lmax_predict(self, freqs):
        """log(lmax) predicted by the attached network."""
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        out = np.zeros(len(fl), np.float32)
        rc = lib().dsm_lmax_predict(self.h, _ptr(fl, _ip), len(fl), _fptr(out))
        if rc:
            raise DsmError(f"dsm_lmax_predict failed ({rc}): {lib().dsm_last_error(self.h).decode()}")
        return out

    def stats(self) -> Stats:
        s = Stats()
        lib().dsm_get_stats(self.h, C.byref(s))
        return s

    def close(self):
        if self.h.value:
            lib().dsm_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MultiSourceContext:
    """Several source depths of one P-SV model in one context
    (dsm_psv_create_multi): each (omega, l) band is factored once and solved
    for every source."""

    def __init__(self, setups, precision: int = DSM_PREC_FP64, device: int = 0, use_lmax_predictor: int = 0,
                 l_chunk: int = 0, freq_batch: int = 0):
        L = lib()
        self.setups = list(setups)
        assert all(s.mode == "psv" for s in self.setups)
        self.opt = Options(precision, device, use_lmax_predictor, l_chunk, freq_batch)
        arr = (C.POINTER(PsvSetup) * len(self.setups))(*[s.ptr for s in self.setups])
        self.h = C.c_void_p()
        rc = L.dsm_psv_create_multi(arr, len(self.setups), C.byref(self.opt), C.byref(self.h))
        if rc:
            raise DsmError(f"dsm_psv_create_multi failed ({rc}): {L.dsm_last_error(None).decode()}", rc)

    def run(self, freqs):
        """[(tsgt, rsgt, synn, llog)] per source, as Context.run returns."""
        L = lib()
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        n = len(fl)
        res, outs = [], (Out * len(self.setups))()
        for k, s in enumerate(self.setups):
            t, r, y, llog = alloc_outputs(s, n)
            res.append((t, r, y, llog))
            outs[k].tsgt = t.ctypes.data_as(_dp)
            outs[k].rsgt = r.ctypes.data_as(_dp)
            outs[k].synn = y.ctypes.data_as(_dp)
            outs[k].llog = llog.ctypes.data_as(_ip)
        rc = L.dsm_run_freqs_multi(self.h, _ptr(fl, _ip), n, outs, len(self.setups))
        if rc:
            raise DsmError(f"dsm_run_freqs_multi failed ({rc}): {L.dsm_last_error(self.h).decode()}", rc)
        return res

    def set_profiling(self, on: bool):
        lib().dsm_set_profiling(self.h, 1 if on else 0)

    def stats(self) -> Stats:
        st = Stats()
        lib().dsm_get_stats(self.h, C.byref(st))
        return st

    tuning = Context.tuning
    set_tuning = Context.set_tuning
    set_depth_cutoff = Context.set_depth_cutoff
    autotune = Context.autotune

    def close(self):
        if self.h.value:
            lib().dsm_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_request(contexts, freq_lists, outputs: bool = True):
    """Runs several contexts (Context or MultiSourceContext, one device)
    together (dsm_run_request); returns, per context, the list of
    (tsgt, rsgt, synn, llog) of its sources (None with outputs=False: the
    run only computes, for timing)."""
    L = lib()
    n = len(contexts)
    keep, results = [], []
    handles = (C.c_void_p * n)()
    ilists = (_ip * n)()
    ns = (C.c_int * n)()
    outs = (C.POINTER(Out) * n)()
    for k, (ctx, freqs) in enumerate(zip(contexts, freq_lists)):
        setups = ctx.setups if isinstance(ctx, MultiSourceContext) else [ctx.setup]
        fl = np.ascontiguousarray(np.asarray(freqs, dtype=np.int32))
        o = (Out * len(setups))()
        res = []
        for j, s in enumerate(setups if outputs else []):
            t, r, y, llog = alloc_outputs(s, len(fl))
            res.append((t, r, y, llog))
            o[j].tsgt = t.ctypes.data_as(_dp)
            o[j].rsgt = r.ctypes.data_as(_dp)
            o[j].synn = y.ctypes.data_as(_dp)
            o[j].llog = llog.ctypes.data_as(_ip)
        keep += [fl, o]
        handles[k] = ctx.h.value
        ilists[k] = _ptr(fl, _ip)
        ns[k] = len(fl)
        outs[k] = C.cast(o, C.POINTER(Out)) if outputs else C.POINTER(Out)()
        results.append(res if outputs else None)
    rcs = np.zeros(n, np.int32)
    rc = L.dsm_run_request(handles, n, ilists, ns, outs, _ptr(rcs, _ip))
    if rc:
        nz = np.nonzero(rcs)[0]
        if len(nz) == 0:
            raise DsmError(f"dsm_run_request failed ({rc}): {L.dsm_strerror(rc).decode()}", rc)
        bad = int(nz[0])
        raise DsmError(f"dsm_run_request failed ({rc}) in context {bad}: "
                       f"{L.dsm_last_error(contexts[bad].h).decode()}", rc)
    return results


def cat_np1(tlen: float, fmax: int, sampling_hz: float, start: float, end: float):
    """(np1, samplingHz, iwin_start, iwin_end) of a time window (dsm_cat_np1)."""
    n1, s0, s1 = C.c_int(), C.c_int(), C.c_int()
    shz = C.c_double()
    rc = lib().dsm_cat_np1(tlen, fmax, sampling_hz, start, end, C.byref(n1), C.byref(shz), C.byref(s0),
                           C.byref(s1))
    if rc:
        raise DsmError(f"dsm_cat_np1 failed ({rc}): {lib().dsm_cat_last_error(None).decode()}")
    return n1.value, shz.value, s0.value, s1.value


def fp64_peak(device: int = 0, mma: bool = False) -> float:
    """Measured FP64 throughput of the device (TFLOP/s): fused multiply-adds,
    or tensor-core products with mma=True."""
    v = C.c_double()
    rc = (lib().dsm_fp64_mma_peak if mma else lib().dsm_fp64_peak)(device, C.byref(v))
    if rc:
        raise DsmError(f"dsm_fp64_peak failed ({rc}): {lib().dsm_cat_last_error(None).decode()}")
    return v.value


def cat_h3h4_coef(ang, compo: str = "Z", mt=None):
    """Combination matrices of rsgt2h3freq ([point][6][10]) and
    tsgt2h4freq ([point][6][20], None without mt) for points with the 12
    angle factors ang [point][12] (dsm_cat_h3h4_coef; host only)."""
    a = np.ascontiguousarray(ang, np.float64).reshape(-1, 12)
    n = a.shape[0]
    c3 = np.zeros((n, 6, 10), np.float64)
    c4 = None if mt is None else np.zeros((n, 6, 20), np.float64)
    m = None if mt is None else np.ascontiguousarray(mt, np.float64)
    rc = lib().dsm_cat_h3h4_coef(n, _ptr(a, _dp), compo.encode(), None if m is None else _ptr(m, _dp),
                                 C.c_void_p(c3.ctypes.data), None if c4 is None else C.c_void_p(c4.ctypes.data))
    if rc:
        raise DsmError(f"dsm_cat_h3h4_coef failed ({rc}): {lib().dsm_cat_last_error(None).decode()}", rc)
    return c3, c4


class Catalogue:
    """Catalogue consumer (dsm_cat_*): record sets of one receiver radius in,
    windowed time series at arbitrary distances out."""

    FIELDS = ("num", "theta_n", "theta_min", "theta_delta", "fmin", "fmax", "np1", "tlen", "omegai",
              "ipdistance", "c_red_reci", "iwin_start", "iwin_end")

    def __init__(self, params: dict, device: int = 0):
        self.p = dict(params)
        cp = CatParams(**{k: self.p[k] for k in self.FIELDS}, device=device)
        h = C.c_void_p()
        rc = lib().dsm_cat_create(C.byref(cp), C.byref(h))
        if rc:
            raise DsmError(f"dsm_cat_create failed ({rc}): {lib().dsm_cat_last_error(None).decode()}")
        self.h = h
        self._keep = []
        self.nwin = self.p["iwin_end"] - self.p["iwin_start"] + 1

    def _check(self, rc, what):
        if rc:
            raise DsmError(f"{what} failed ({rc}): {lib().dsm_cat_last_error(self.h).decode()}")

    def add(self, rec, dst=None, scale=None):
        """rec: numpy [nf][theta_n][ncomp] complex64/complex128 (host), or a
        torch CUDA tensor of that shape (kept alive until clear())."""
        dp = None if dst is None else np.ascontiguousarray(dst, np.int32)
        sp = None if scale is None else np.ascontiguousarray(scale, np.float64)
        on_dev = 0
        if hasattr(rec, "data_ptr"):
            assert rec.is_cuda and rec.is_contiguous()
            ptr, eb, nc, on_dev = rec.data_ptr(), rec.element_size(), rec.shape[-1], 1
        else:
            rec = np.ascontiguousarray(rec)
            assert rec.dtype in (np.complex64, np.complex128)
            ptr, eb, nc = rec.ctypes.data, rec.itemsize, rec.shape[-1]
        self._keep.append(rec)
        rc = lib().dsm_cat_add(self.h, C.c_void_p(ptr), eb, nc,
                               None if dp is None else _ptr(dp, _ip),
                               None if sp is None else _ptr(sp, _dp), on_dev)
        self._check(rc, "dsm_cat_add")

    def clear(self):
        self._check(lib().dsm_cat_clear(self.h), "dsm_cat_clear")
        self._keep = []

    def series(self, distances, coef=None, out=None):
        """Time series [npoint][nout][nwin] (numpy, or written into the torch
        CUDA tensor ``out``)."""
        d = np.ascontiguousarray(distances, np.float64)
        cf = None if coef is None else np.ascontiguousarray(coef, np.float64)
        nout = self.p["num"] if cf is None else cf.shape[1]
        if out is None:
            res = np.zeros((d.size, nout, self.nwin), np.float64)
            optr, on_dev = res.ctypes.data, 0
        else:
            assert out.is_cuda and out.is_contiguous() and out.numel() == d.size * nout * self.nwin
            res, optr, on_dev = out, out.data_ptr(), 1
        rc = lib().dsm_cat_series(self.h, d.size, _ptr(d, _dp), nout,
                                  None if cf is None else _ptr(cf, _dp), C.c_void_p(optr), on_dev)
        self._check(rc, "dsm_cat_series")
        return res

    def spectra(self, distances, coef=None):
        """Combined spectra [npoint][nout][fmax-fmin+1] (complex128) before the
        transform (dsm_cat_spectra)."""
        d = np.ascontiguousarray(distances, np.float64)
        cf = None if coef is None else np.ascontiguousarray(coef, np.float64)
        nout = self.p["num"] if cf is None else cf.shape[1]
        nf = self.p["fmax"] - self.p["fmin"] + 1
        res = np.zeros((d.size, nout, nf), np.complex128)
        rc = lib().dsm_cat_spectra(self.h, d.size, _ptr(d, _dp), nout,
                                   None if cf is None else _ptr(cf, _dp), C.c_void_p(res.ctypes.data), 0)
        self._check(rc, "dsm_cat_spectra")
        return res

    def transform(self, spectra):
        """vectorFFT_double of spectra [nseries][fmax-fmin+1] (complex128):
        windowed time series [nseries][nwin] (dsm_cat_transform)."""
        x = np.ascontiguousarray(spectra, np.complex128)
        x2 = x.reshape(-1, x.shape[-1])
        res = np.zeros((x2.shape[0], self.nwin), np.float64)
        rc = lib().dsm_cat_transform(self.h, x2.shape[0], C.c_void_p(x2.ctypes.data), 0,
                                     C.c_void_p(res.ctypes.data), 0)
        self._check(rc, "dsm_cat_transform")
        return res.reshape(x.shape[:-1] + (self.nwin,))

    def set_kernel_params(self, types: int, nfilter: int, fclp, fchp, npoles: int, sampling_hz: float,
                          nt1, nt2, coeff, jacobian=None):
        """Filters, integration windows and the reference's coeff(0:nfilter,
        1:nktype, 1:nr, window) / jacobianFuji(1:nr, fmin:fmax) arrays
        (numpy, Fortran order: coeff of shape [nwin][nr][nktype][nfilter+1]
        C-ordered, jacobian [nf][nr]) for dsm_cat_kernels."""
        nfl = nfilter + 1
        self._kp = dict(
            fclp=np.ascontiguousarray(fclp, np.float64), fchp=np.ascontiguousarray(fchp, np.float64),
            nt1=np.ascontiguousarray(nt1, np.int32), nt2=np.ascontiguousarray(nt2, np.int32),
            coeff=np.ascontiguousarray(coeff, np.float64),
            jac=None if jacobian is None else np.ascontiguousarray(jacobian, np.complex128))
        k = self._kp
        assert k["coeff"].ndim == 4 and k["coeff"].shape[0] == self.nwin and k["coeff"].shape[3] == nfl
        kp = CatKernelParams(types=types, nfilter=nfilter, fclp=_ptr(k["fclp"], _dp), fchp=_ptr(k["fchp"], _dp),
                             npoles=npoles, sampling_hz=sampling_hz, nt1=_ptr(k["nt1"], _ip),
                             nt2=_ptr(k["nt2"], _ip), nr=k["coeff"].shape[1], nktype=k["coeff"].shape[2],
                             coeff=_ptr(k["coeff"], _dp),
                             jacobian=None if k["jac"] is None else C.c_void_p(k["jac"].ctypes.data))
        self._check(lib().dsm_cat_set_kernel_params(self.h, C.byref(kp)), "dsm_cat_set_kernel_params")
        self._ker_shape = (nfl, k["coeff"].shape[2] + 1)
        self._ker_ns = (1 if types & KER_VP else 0) + (2 if types & KER_VS else 0)

    def kernels(self, ir, h3, h4, filtered: bool = False):
        """tmpker [point][nfilter+1][nktype+1] of points with radius indices
        ir and spectra h3, h4 [point][6][nf] (numpy complex128, or torch CUDA
        tensors), plus the filtered series [point][series][nfilter+1][nwin]
        when filtered is set (dsm_cat_kernels)."""
        irr = np.ascontiguousarray(ir, np.int32)
        n = irr.size
        if hasattr(h3, "data_ptr"):
            assert h3.is_cuda and h4.is_cuda and h3.is_contiguous() and h4.is_contiguous()
            p3, p4, on_dev = h3.data_ptr(), h4.data_ptr(), 1
        else:
            h3 = np.ascontiguousarray(h3, np.complex128)
            h4 = np.ascontiguousarray(h4, np.complex128)
            p3, p4, on_dev = h3.ctypes.data, h4.ctypes.data, 0
        ker = np.zeros((n,) + self._ker_shape, np.float64)
        filt = np.zeros((n, self._ker_ns, self._ker_shape[0], self.nwin), np.float64) if filtered else None
        rc = lib().dsm_cat_kernels(self.h, n, _ptr(irr, _ip), C.c_void_p(p3), C.c_void_p(p4), on_dev,
                                   C.c_void_p(ker.ctypes.data),
                                   None if filt is None else C.c_void_p(filt.ctypes.data), 0)
        self._check(rc, "dsm_cat_kernels")
        return (ker, filt) if filtered else ker

    def filter(self, series):
        """The filters set by set_kernel_params applied to window series
        [..., nwin] (numpy): [..., nfilter+1, nwin] (dsm_cat_filter)."""
        x = np.ascontiguousarray(series, np.float64)
        x2 = x.reshape(-1, self.nwin)
        nfl = self._ker_shape[0]
        res = np.zeros((x2.shape[0], nfl, self.nwin), np.float64)
        rc = lib().dsm_cat_filter(self.h, x2.shape[0], C.c_void_p(x2.ctypes.data), C.c_void_p(res.ctypes.data), 0)
        self._check(rc, "dsm_cat_filter")
        return res.reshape(x.shape[:-1] + (nfl, self.nwin))

    def set_profiling(self, on: bool):
        self._check(lib().dsm_cat_set_profiling(self.h, int(on)), "dsm_cat_set_profiling")

    def set_batch_bytes(self, nbytes: int):
        self._check(lib().dsm_cat_set_batch_bytes(self.h, nbytes), "dsm_cat_set_batch_bytes")

    def stats(self) -> Stats:
        st = Stats()
        self._check(lib().dsm_cat_get_stats(self.h, C.byref(st)), "dsm_cat_get_stats")
        return st

    def close(self):
        if self.h:
            lib().dsm_cat_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
