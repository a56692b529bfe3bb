"""ctypes bindings of the C ABI in include/specsim3d_gpu.h.

The shared library is built in-tree at specsim3d_b200/lib/libspecsim3d_gpu.so
(``make -C specsim3d_b200/csrc``).  There is no CPU fallback: loading fails
loudly when the library is missing, and every call that needs a GPU reports
the CUDA error through SpecsimError.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libspecsim3d_gpu.so")

SS3D_OK, SS3D_EINVAL, SS3D_ECUDA, SS3D_ENOMEM, SS3D_ETOOLARGE, SS3D_ENODATA = range(6)
FP64, FP32 = 0, 1
OUT_F32, OUT_F64 = 0, 1

# every symbol declared in include/specsim3d_gpu.h
EXPORTS = (
    "ss3d_setrot", "ss3d_covariance", "ss3d_grid_size",
    "ss3d_spectrum_create", "ss3d_spectrum_free", "ss3d_spectrum_info", "ss3d_spectrum_bytes", "ss3d_spectrum_amp",
    "ss3d_realize", "ss3d_debug_states", "ss3d_debug_coefficients", "ss3d_row_state",
    "ss3d_vario", "ss3d_condition", "ss3d_fft3d",
    "ss3d_set_stream", "ss3d_last_error", "ss3d_version", "ss3d_profile", "ss3d_profile_read", "ss3d_autotune", "ss3d_set_variant",
    "ss3d_preload_kernels",
    "ss3d_realize_workspace_bytes", "ss3d_release_workspace", "ss3d_trim_pool",
    "ss3d_batch_create", "ss3d_batch_run", "ss3d_batch_autotune", "ss3d_batch_info", "ss3d_batch_time",
    "ss3d_batch_schedule", "ss3d_batch_set_schedule", "ss3d_batch_split", "ss3d_batch_set_split", "ss3d_batch_free",
    "ss3d_server_create", "ss3d_server_submit", "ss3d_server_wait", "ss3d_server_stats", "ss3d_server_clock",
    "ss3d_server_free",
)


class SpecsimError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"specsim3d_gpu error {code}: {msg}")
        self.code = code


class Struct(ctypes.Structure):
    """ss3d_struct: one nested variogram structure (f90:95-100)."""
    _fields_ = [("itype", ctypes.c_int), ("sill", ctypes.c_double), ("ahmax", ctypes.c_double),
                ("ahmin", ctypes.c_double), ("avert", ctypes.c_double), ("azimuth", ctypes.c_double),
                ("dip", ctypes.c_double), ("plunge", ctypes.c_double)]


class SpecStats(ctypes.Structure):
    _fields_ = [("np", ctypes.c_int * 3), ("c0", ctypes.c_double), ("maximag", ctypes.c_double),
                ("maxreal", ctypes.c_double), ("spos", ctypes.c_double), ("sneg", ctypes.c_double)]


class BatchJob(ctypes.Structure):
    """ss3d_batch_job: realizations r_first.. of one spectrum into a device array."""
    _fields_ = [("sp", ctypes.c_void_p), ("iseed", ctypes.c_int), ("igauss", ctypes.c_int),
                ("r_first", ctypes.c_int64), ("nreal", ctypes.c_int), ("out", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("max_bypass", ctypes.c_int), ("max_cond", ctypes.c_int),
                ("hbm_budget", ctypes.c_int64),
                ("cache_budget", ctypes.c_int64), ("retain_bytes", ctypes.c_int64),
                ("dry_run_ns_per_cell", ctypes.c_double), ("premap_bytes", ctypes.c_int64)]


class Request(ctypes.Structure):
    """ss3d_request (serving form)."""
    _fields_ = [("st", ctypes.c_void_p), ("nst", ctypes.c_int), ("nugget", ctypes.c_double),
                ("d", ctypes.c_double * 3), ("n", ctypes.c_int * 3), ("ipad", ctypes.c_int),
                ("iseed", ctypes.c_int), ("igauss", ctypes.c_int), ("r_first", ctypes.c_int64),
                ("nreal", ctypes.c_int), ("precision", ctypes.c_int), ("out", ctypes.c_void_p),
                ("out_dtype", ctypes.c_int), ("t_arrival", ctypes.c_double), ("cp", ctypes.c_void_p),
                ("rows", ctypes.c_void_p), ("nrows", ctypes.c_int), ("nvar", ctypes.c_int),
                ("xmin", ctypes.c_double * 3)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("cache_hit", ctypes.c_int), ("t_arrival", ctypes.c_double),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
                ("footprint", ctypes.c_int64)]


class ServeStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "submitted", "completed", "failed", "cache_hits", "cache_misses", "evictions", "cells", "peak_bytes",
        "peak_running", "running", "queued", "cached_spectra", "cache_bytes", "charged_bytes", "budget_bytes")]


class CondParams(ctypes.Structure):
    _fields_ = [("ixc", ctypes.c_int), ("iyc", ctypes.c_int), ("izc", ctypes.c_int), ("ivc", ctypes.c_int),
                ("iwc", ctypes.c_int), ("tmin", ctypes.c_double), ("tmax", ctypes.c_double),
                ("itrans", ctypes.c_int), ("skmean", ctypes.c_double), ("zmin", ctypes.c_double),
                ("zmax", ctypes.c_double), ("ltail", ctypes.c_int), ("ltpar", ctypes.c_double),
                ("utail", ctypes.c_int), ("utpar", ctypes.c_double), ("radius", ctypes.c_double * 3),
                ("angles", ctypes.c_double * 3), ("ndmax", ctypes.c_int)]


class CondStats(ctypes.Structure):
    _fields_ = [("nd", ctypes.c_int), ("nmerged", ctypes.c_int), ("nout", ctypes.c_int),
                ("nsb", ctypes.c_int * 3), ("nsum", ctypes.c_int64), ("nfail", ctypes.c_int),
                ("nnone", ctypes.c_int), ("nexact", ctypes.c_int), ("data_mean", ctypes.c_double),
                ("data_var", ctypes.c_double)]


_lib = None


def lib():
    """Load (once) and return the CUDA library; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C specsim3d_b200/csrc` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    P, I, D, I64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64
    pI, pD = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    sig = {
        "ss3d_setrot": (I, [ctypes.POINTER(Struct), pD, pD]),
        "ss3d_covariance": (I, [ctypes.POINTER(Struct), I, D, D, D, D, pD]),
        "ss3d_grid_size": (I, [ctypes.POINTER(Struct), I, pD, pI, I, pI]),
        "ss3d_spectrum_create": (I, [ctypes.POINTER(Struct), I, D, pD, pI, I, ctypes.POINTER(P),
                                     ctypes.POINTER(SpecStats)]),
        "ss3d_spectrum_free": (None, [P]),
        "ss3d_spectrum_info": (I, [P, pI, pI, ctypes.POINTER(SpecStats)]),
        "ss3d_spectrum_bytes": (I64, [P]),
        "ss3d_spectrum_amp": (I, [P, P]),
        "ss3d_realize": (I, [P, I, I64, I, I, I, P, I, P]),
        "ss3d_debug_states": (I, [P, I, I64, I, P]),
        "ss3d_debug_coefficients": (I, [P, I, I64, I, I, P]),
        "ss3d_vario": (I, [P, pI, I, I, pI, pI, pI, pI, P, P]),
        "ss3d_condition": (I, [P, pI, I, pD, pD, ctypes.POINTER(Struct), I, D, ctypes.POINTER(CondParams), P, I, I,
                               I, ctypes.POINTER(CondStats), P, P, P, P, P, P, P]),
        "ss3d_fft3d": (I, [P, I, I, I, I]),
        "ss3d_set_stream": (I, [P]),
        "ss3d_last_error": (ctypes.c_char_p, []),
        "ss3d_version": (ctypes.c_char_p, []),
        "ss3d_profile": (I, [I]),
        "ss3d_profile_read": (I, [P, P, P]),
        "ss3d_autotune": (I, [P, I, I, I, P]),
        "ss3d_set_variant": (I, [I, I, I, I]),
        "ss3d_preload_kernels": (I, []),
        "ss3d_realize_workspace_bytes": (I64, [P, I, I, I]),
        "ss3d_release_workspace": (I, []),
        "ss3d_trim_pool": (I, []),
        "ss3d_row_state": (I, [P, I, I, I64, I, I, P]),
        "ss3d_batch_create": (I, [P, I, P]),
        "ss3d_batch_run": (I, [P]),
        "ss3d_batch_autotune": (I, [P]),
        "ss3d_batch_info": (I, [P, P, P, P, P]),
        "ss3d_batch_time": (I, [P, P]),
        "ss3d_batch_schedule": (I, [P, P, P, P, P]),
        "ss3d_batch_set_schedule": (I, [P, I, I, I, I, I]),
        "ss3d_batch_split": (I, [P, P]),
        "ss3d_batch_set_split": (I, [P, I]),
        "ss3d_batch_free": (None, [P]),
        "ss3d_server_create": (I, [P, P]),
        "ss3d_server_submit": (I, [P, P, P]),
        "ss3d_server_wait": (I, [P, I64, P]),
        "ss3d_server_stats": (I, [P, P]),
        "ss3d_server_clock": (D, [P]),
        "ss3d_server_free": (None, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != SS3D_OK:
        raise SpecsimError(rc, lib().ss3d_last_error().decode())
    return rc


def structs_array(structs):
    """structs: iterable of (itype, sill, ahmax, ahmin, avert, azimuth, dip, plunge)."""
    structs = list(structs)
    arr = (Struct * len(structs))()
    for a, s in zip(arr, structs):
        a.itype = int(s[0])
        a.sill, a.ahmax, a.ahmin, a.avert, a.azimuth, a.dip, a.plunge = (float(v) for v in s[1:8])
    return arr


def dptr(a):
    return ctypes.cast(a, ctypes.POINTER(ctypes.c_double)) if not isinstance(a, np.ndarray) else \
        a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
