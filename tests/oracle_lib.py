"""ctypes access to the CPU oracle (oracle/_build/liboracle.so) for the tests.

The oracle is the checker: a C restatement of src/specsim3d.f90 that the
tests run beside the CUDA library on the same inputs.  It is never part of
the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
EXE = os.path.join(ORACLE_DIR, "_build", "specsim3d_oracle")


class OraStruct(ctypes.Structure):
    _fields_ = [("itype", ctypes.c_int), ("sill", ctypes.c_double), ("ahmax", ctypes.c_double),
                ("ahmin", ctypes.c_double), ("avert", ctypes.c_double), ("az", ctypes.c_double),
                ("dip", ctypes.c_double), ("plg", ctypes.c_double), ("rot", ctypes.c_double * 9),
                ("axes", ctypes.c_double * 9)]


class OraSpecStats(ctypes.Structure):
    _fields_ = [("c0", ctypes.c_double), ("maximag", ctypes.c_double), ("maxreal", ctypes.c_double),
                ("spos", ctypes.c_double), ("sneg", ctypes.c_double)]


class OraCondParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("ixc", "iyc", "izc", "ivc", "iwc", "itrans", "ltail", "utail", "ndmax")] + \
               [(k, ctypes.c_double) for k in ("tmin", "tmax", "skmean", "zlo", "zhi", "ltpar", "utpar", "rmax", "rmed",
                                               "rvert", "sa1", "sa2", "sa3")]


class OraCondStats(ctypes.Structure):
    _fields_ = [("nd", ctypes.c_int), ("nmerged", ctypes.c_int), ("nout", ctypes.c_int), ("nsb", ctypes.c_int * 3),
                ("nsum", ctypes.c_int64), ("nfail", ctypes.c_int), ("nnone", ctypes.c_int), ("nexact", ctypes.c_int)]


_L = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        _L = ctypes.CDLL(LIB)
        _L.ora_urand.restype = ctypes.c_double
        _L.ora_rng_state.restype = ctypes.c_int64
        _L.ora_covariance.restype = ctypes.c_double
        _L.ora_npair_count.restype = ctypes.c_int64
        _L.ora_vario_lag.restype = ctypes.c_double
        _L.ora_gauinv.restype = ctypes.c_double
        _L.ora_gcum.restype = ctypes.c_double
        _L.ora_backtr.restype = ctypes.c_double
        _L.ora_covariance.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 4
        _L.ora_gauinv.argtypes = [ctypes.c_double]
        _L.ora_gcum.argtypes = [ctypes.c_double]
    return _L


def structs(sts):
    arr = (OraStruct * len(sts))()
    for a, s in zip(arr, sts):
        a.itype = int(s[0])
        a.sill, a.ahmax, a.ahmin, a.avert, a.az, a.dip, a.plg = (float(v) for v in s[1:8])
        lib().ora_setrot(ctypes.byref(a))
    return arr


def _i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return (ctypes.c_double * 3)(*[float(x) for x in v])


def grid(sts, d, n, ipad):
    arr = structs(sts)
    np_ = (ctypes.c_int * 3)()
    rc = lib().ora_periodic_grid(arr, len(arr), _d3(d), _i3(n), int(ipad), np_)
    return tuple(np_), rc


def spectrum(sts, nugget, d, np3):
    """amp (npz, npy, npx) and stats dict."""
    arr = structs(sts)
    amp = np.zeros((np3[2], np3[1], np3[0]))
    st = OraSpecStats()
    lib().ora_spectrum(arr, len(arr), ctypes.c_double(nugget), _d3(d), _i3(np3),
                       ctypes.c_void_p(amp.ctypes.data), ctypes.byref(st))
    return amp, dict(c0=st.c0, maximag=st.maximag, maxreal=st.maxreal, spos=st.spos, sneg=st.sneg)


def realize(amp, np3, n, iseed, nreal, igauss):
    """res (nreal, nz, ny, nx) float64 and zstats (nreal, 3)."""
    res = np.zeros((nreal, n[2], n[1], n[0]))
    zs = np.zeros((nreal, 3))
    lib().ora_realize(ctypes.c_void_p(amp.ctypes.data), _i3(np3), _i3(n), int(iseed), int(nreal), int(igauss),
                      ctypes.c_void_p(res.ctypes.data), ctypes.c_void_p(zs.ctypes.data))
    return res, zs


def realize_range(amp, np3, n, iseed, r_first, nreal, igauss):
    """Realizations r_first..r_first+nreal-1 (0-based) of the serial run of seed
    iseed: the earlier fills are drawn and discarded, as the serial stream does."""
    res = np.zeros((nreal, n[2], n[1], n[0]))
    zs = np.zeros((nreal, 3))
    rc = lib().ora_realize_range(ctypes.c_void_p(amp.ctypes.data), _i3(np3), _i3(n), int(iseed), int(r_first),
                                 int(nreal), int(igauss), ctypes.c_void_p(res.ctypes.data),
                                 ctypes.c_void_p(zs.ctypes.data))
    assert rc == 0
    return res, zs


def fill_states(np3, iseed, nreal, igauss):
    """First-draw states (nreal, npz, npy, npx) of the sequential stream (0 = no draw)."""
    lib().ora_rng_seed(ctypes.c_int(iseed))
    out = np.zeros((nreal, np3[2], np3[1], np3[0]), dtype=np.int64)
    for r in range(nreal):
        lib().ora_fill_states(_i3(np3), int(igauss), ctypes.c_void_p(out[r].ctypes.data))
    return out


def coefficients(amp, np3, iseed, r, igauss):
    """Full-spectrum coefficients of realization r (0-based), complex (npz, npy, npx)."""
    lib().ora_rng_seed(ctypes.c_int(iseed))
    c = np.zeros((np3[2], np3[1], np3[0], 2))
    for _ in range(r + 1):
        lib().ora_fill_coefficients(ctypes.c_void_p(amp.ctypes.data), _i3(np3), int(igauss),
                                    ctypes.c_void_p(c.ctypes.data))
    return c[..., 0] + 1j * c[..., 1]


def vario(res, dirs):
    """gam (nreal, ndir, nlagmax) of res (nreal, nz, ny, nx)."""
    nreal, nz, ny, nx = res.shape
    res = np.ascontiguousarray(res, dtype=np.float64)
    ndir = len(dirs)
    nlagmax = max(d[3] for d in dirs)
    cols = [(ctypes.c_int * ndir)(*[int(d[k]) for d in dirs]) for k in range(4)]
    gam = np.zeros((nreal, ndir, nlagmax))
    lib().ora_vario_all(ctypes.c_void_p(res.ctypes.data), _i3((nx, ny, nz)), nreal, ndir, *cols,
                        ctypes.c_void_p(gam.ctypes.data))
    return gam


def npair_count(n, lag):
    return lib().ora_npair_count(*[int(v) for v in n], *[int(v) for v in lag])


def condition(res, xmin, d, sts, nugget, params, rows):
    """In-place conditioning of res (nreal, nz, ny, nx) float64; returns stats dict and extras."""
    nreal, nz, ny, nx = res.shape
    cp = OraCondParams()
    for k, v in params.items():
        setattr(cp, k, v)
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    nrows, nvar = rows.shape
    arr = structs(sts)
    cs = OraCondStats()
    outs = {k: np.zeros(max(nrows, 1)) for k in ("vrt", "gtt", "dxs", "dys", "dzs", "dval", "dg")}
    rc = lib().ora_condition(ctypes.c_void_p(res.ctypes.data), _i3((nx, ny, nz)), nreal, _d3(xmin), _d3(d), arr,
                             len(arr), ctypes.c_double(nugget), ctypes.byref(cp), ctypes.c_void_p(rows.ctypes.data),
                             nrows, nvar, ctypes.byref(cs),
                             *[ctypes.c_void_p(outs[k].ctypes.data) for k in
                               ("vrt", "gtt", "dxs", "dys", "dzs", "dval", "dg")])
    st = dict(rc=rc, nd=cs.nd, nmerged=cs.nmerged, nout=cs.nout, nsb=tuple(cs.nsb), nsum=cs.nsum, nfail=cs.nfail,
              nnone=cs.nnone, nexact=cs.nexact)
    return st, {k: v[:cs.nd] for k, v in outs.items()}
