"""specsim3d_b200 -- B200-native SPECSIM3D spectral simulation path.

Python face of the C ABI (include/specsim3d_gpu.h), mirroring the stages of
the reference program src/specsim3d.f90:

    Model / grid_size      setrot, covariance, ipad rule     f90:107-188, 1234-1253
    Spectrum               covariance grid + FFT + sqrt      f90:1256-1292
    Spectrum.realize       Hermitian synthesis + inverse FFT f90:1302-1345
    vario                  experimental variograms           f90:394-480
    condition              kriging of the residual           f90:700-1081
    Batch                  many grids per CUDA-graph launch  (batched form)
    Server                 request loop, spectra cache       (serving form)

Arrays follow the Fortran layout res(nx,ny,nz,nreal), i.e. numpy shape
(nreal, nz, ny, nx).  Outputs can be numpy arrays (host) or torch CUDA tensors
(device); the library detects which.  All compute runs on the GPU; there is no
CPU fallback.
"""
import ctypes

import numpy as np

from . import _lib as L
from ._lib import FP32, FP64, OUT_F32, OUT_F64, SpecsimError

__all__ = ["Spectrum", "Batch", "Server", "row_state", "shard", "grid_size", "covariance", "setrot", "vario", "condition", "FP32", "FP64",
           "SpecsimError", "set_stream"]


def _np3(v, dtype):
    return np.ascontiguousarray(np.asarray(v, dtype=dtype).reshape(3))


def setrot(struct):
    """rot, axes (3x3 each) of one structure tuple (itype, sill, ahmax, ahmin, avert, az, dip, plunge)."""
    rot = np.zeros(9)
    axes = np.zeros(9)
    L.check(L.lib().ss3d_setrot(L.structs_array([struct]), L.dptr(rot), L.dptr(axes)))
    return rot.reshape(3, 3), axes.reshape(3, 3)


def covariance(structs, nugget, dx, dy, dz):
    arr = L.structs_array(structs)
    c = ctypes.c_double()
    L.check(L.lib().ss3d_covariance(arr, len(arr), float(nugget), float(dx), float(dy), float(dz), ctypes.byref(c)))
    return c.value


def grid_size(structs, d, n, ipad):
    """Periodic grid (npx, npy, npz) of the ipad rule (f90:1234-1253)."""
    arr = L.structs_array(structs)
    np_ = np.zeros(3, dtype=np.int32)
    L.check(L.lib().ss3d_grid_size(arr, len(arr), L.dptr(_np3(d, np.float64)), L.iptr(_np3(n, np.int32)),
                                   int(ipad), L.iptr(np_)))
    return tuple(int(v) for v in np_)


def set_stream(stream):
    """Issue later calls on a torch.cuda.Stream (or raw cudaStream_t int); None = default stream."""
    h = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
    L.check(L.lib().ss3d_set_stream(ctypes.c_void_p(h)))


NSTAGE = 5
STAGES = ("rowstates", "synthesis+first_pass", "middle_pass", "x_c2r_crop", "stats")


def profile(enable=True):
    """Switch per-stage CUDA-event timing of the realization path on/off (resets counters)."""
    L.check(L.lib().ss3d_profile(1 if enable else 0))


def profile_read():
    """{stage: (ms, launches)} accumulated since profile(True), and the total launch count."""
    ms = np.zeros(NSTAGE)
    ln = np.zeros(NSTAGE, dtype=np.int64)
    tot = ctypes.c_int64()
    L.check(L.lib().ss3d_profile_read(ctypes.c_void_p(ms.ctypes.data), ctypes.c_void_p(ln.ctypes.data),
                                      ctypes.byref(tot)))
    return {name: (float(ms[q]), int(ln[q])) for q, name in enumerate(STAGES)}, int(tot.value)


def preload_kernels():
    """Load every kernel of the library on the current device now (CUDA loads
    a kernel on its first launch, and a load may synchronise the device)."""
    L.check(L.lib().ss3d_preload_kernels())


def autotune(spectrum, igauss=1, precision=FP32, nreal=2):
    """Pick the fastest tile variant of each realization kernel for this grid (kept for the process)."""
    ch = np.zeros(3, dtype=np.int32)
    L.check(L.lib().ss3d_autotune(spectrum.handle, int(igauss), int(precision), int(nreal),
                                  ctypes.c_void_p(ch.ctypes.data)))
    return {"middle_pass": int(ch[0]), "synthesis_pass": int(ch[1]), "row_pass": int(ch[2])}


def row_state(np3, igauss, iseed, r, j, k):
    """Park-Miller state right after the first draw of row (j, k) of realization r
    (0-based) on periodic grid np3, by host jump-ahead (no GPU)."""
    st = ctypes.c_uint32()
    L.check(L.lib().ss3d_row_state(L.iptr(_np3(np3, np.int32)), int(igauss), int(iseed), int(r), int(j), int(k),
                                   ctypes.byref(st)))
    return int(st.value)


def shard(rank, world, nreal_per_rank):
    """Realizations of one rank when realizations are split over processes or
    GPUs: (r_first, nreal) = (rank * nreal_per_rank, nreal_per_rank).  Every
    rank draws from the same seed's stream by jump-ahead, so the union of the
    shards equals one run of world * nreal_per_rank realizations."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return rank * int(nreal_per_rank), int(nreal_per_rank)


def _out_ptr(out):
    """(pointer, dtype code, nbytes) of a numpy array or a torch tensor."""
    if isinstance(out, np.ndarray):
        if not out.flags.c_contiguous:
            raise ValueError("output array must be C-contiguous")
        code = {np.dtype(np.float32): OUT_F32, np.dtype(np.float64): OUT_F64}[out.dtype]
        return ctypes.c_void_p(out.ctypes.data), code
    # torch tensor
    import torch
    if not out.is_contiguous():
        raise ValueError("output tensor must be contiguous")
    code = {torch.float32: OUT_F32, torch.float64: OUT_F64}[out.dtype]
    return ctypes.c_void_p(out.data_ptr()), code


class Spectrum:
    """Device-resident amplitude spectrum of one model on one grid (f90:1256-1292)."""

    def __init__(self, structs, nugget, d, n, ipad):
        self.structs = [tuple(s) for s in structs]
        self.nugget = float(nugget)
        self.d = tuple(float(v) for v in d)
        self.n = tuple(int(v) for v in n)
        self.ipad = int(ipad)
        arr = L.structs_array(self.structs)
        h = ctypes.c_void_p()
        st = L.SpecStats()
        L.check(L.lib().ss3d_spectrum_create(arr, len(arr), self.nugget, L.dptr(_np3(self.d, np.float64)),
                                             L.iptr(_np3(self.n, np.int32)), self.ipad, ctypes.byref(h),
                                             ctypes.byref(st)))
        self._h = h
        self.np = tuple(st.np)
        self.stats = dict(c0=st.c0, maximag=st.maximag, maxreal=st.maxreal, spos=st.spos, sneg=st.sneg)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            L.lib().ss3d_spectrum_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nbytes(self):
        return int(L.lib().ss3d_spectrum_bytes(self._h))

    def amp(self):
        """FP64 amplitude on the half spectrum, shape (npz, npy, npx//2+1)."""
        npx, npy, npz = self.np
        h = npx // 2 + 1 if npx >= 2 else 1
        a = np.zeros((npz, npy, h))
        L.check(L.lib().ss3d_spectrum_amp(self._h, ctypes.c_void_p(a.ctypes.data)))
        return a

    def realize(self, iseed, nreal, igauss=0, precision=FP64, r_first=0, out=None, dtype=np.float64, zstats=False):
        """Realizations r_first..r_first+nreal-1 of seed iseed (f90:1302-1345).

        Returns an array of shape (nreal, nz, ny, nx) (``out`` if given: numpy
        host array or torch CUDA tensor of float32/float64), and with
        zstats=True also the (nreal, 3) mean / variance / max|Im| table."""
        nx, ny, nz = self.n
        if out is None:
            out = np.empty((nreal, nz, ny, nx), dtype=dtype)
        ptr, code = _out_ptr(out)
        zs = np.zeros((max(nreal, 1), 3)) if zstats else None
        L.check(L.lib().ss3d_realize(self._h, int(iseed), int(r_first), int(nreal), int(igauss), int(precision), ptr,
                                     code, ctypes.c_void_p(zs.ctypes.data) if zs is not None else None))
        return (out, zs[:nreal]) if zstats else out

    def debug_states(self, iseed, r, igauss):
        npx, npy, npz = self.np
        h = npx // 2 + 1 if npx >= 2 else 1
        s = np.zeros((npz, npy, h), dtype=np.uint32)
        L.check(L.lib().ss3d_debug_states(self._h, int(iseed), int(r), int(igauss), ctypes.c_void_p(s.ctypes.data)))
        return s

    def debug_coefficients(self, iseed, r, igauss, precision=FP64):
        npx, npy, npz = self.np
        h = npx // 2 + 1 if npx >= 2 else 1
        c = np.zeros((npz, npy, h, 2))
        L.check(L.lib().ss3d_debug_coefficients(self._h, int(iseed), int(r), int(igauss), int(precision),
                                                ctypes.c_void_p(c.ctypes.data)))
        return c[..., 0] + 1j * c[..., 1]


class Batch:
    """Many realizations of many grids in one CUDA-graph launch (FP32).

    jobs: iterable of (spectrum, iseed, igauss, r_first, nreal, out), ``out`` a
    contiguous float32 torch CUDA tensor of nreal * nz * ny * nx elements.
    Each run writes every job's realizations; each equals
    ``spectrum.realize(iseed, nreal, igauss, FP32, r_first, dtype=float32)``
    bit for bit."""

    CHAINS, PERSISTENT = 0, 1

    def __init__(self, jobs, autotune=False):
        jobs = list(jobs)
        arr = (L.BatchJob * len(jobs))()
        self._keep = []
        for a, (sp, iseed, igauss, r_first, nreal, out) in zip(arr, jobs):
            nx, ny, nz = sp.n
            if out.numel() != int(nreal) * nx * ny * nz:
                raise ValueError("output tensor has the wrong size")
            ptr, code = _out_ptr(out)
            if code != OUT_F32 or not out.is_cuda:
                raise ValueError("batch outputs must be float32 CUDA tensors")
            a.sp = sp.handle.value
            a.iseed, a.igauss, a.r_first, a.nreal, a.out = int(iseed), int(igauss), int(r_first), int(nreal), ptr.value
            self._keep.append((sp, out))
        h = ctypes.c_void_p()
        L.check(L.lib().ss3d_batch_create(arr, len(jobs), ctypes.byref(h)))
        self._h = h
        if autotune:
            self.autotune()

    def run(self):
        L.check(L.lib().ss3d_batch_run(self._h))

    def autotune(self):
        L.check(L.lib().ss3d_batch_autotune(self._h))

    def info(self):
        cells = ctypes.c_int64()
        grid = (ctypes.c_int * 3)()
        items = (ctypes.c_int * 3)()
        kern = ctypes.c_int()
        L.check(L.lib().ss3d_batch_info(self._h, ctypes.byref(cells), grid, items, ctypes.byref(kern)))
        return {"cells": int(cells.value), "grid": list(grid), "items": list(items), "kernels": int(kern.value)}

    def time(self):
        """One run timed outside the graph: [synthesis, middle, rows, whole] ms."""
        ms = (ctypes.c_float * 4)()
        L.check(L.lib().ss3d_batch_time(self._h, ms))
        return [float(v) for v in ms]

    def schedule(self):
        sched = ctypes.c_int()
        etv, mode, cps = ((ctypes.c_int * 3)() for _ in range(3))
        L.check(L.lib().ss3d_batch_schedule(self._h, ctypes.byref(sched), etv, mode, cps))
        split = ctypes.c_int()
        L.check(L.lib().ss3d_batch_split(self._h, ctypes.byref(split)))
        return {"schedule": "persistent" if sched.value == 1 else "chains",
                "elements_per_thread": [16 if v == 0 else 8 for v in etv], "mode": list(mode),
                "ctas_per_sm": list(cps), "split": int(split.value)}

    def set_schedule(self, sched, pass_=0, elements_per_thread=8, mode=2, ctas_per_sm=0):
        L.check(L.lib().ss3d_batch_set_schedule(self._h, int(sched), int(pass_),
                                                0 if elements_per_thread == 16 else 1, int(mode), int(ctas_per_sm)))

    def set_split(self, split):
        """Chains schedule: run each job's realizations as `split` staggered sub-chains."""
        L.check(L.lib().ss3d_batch_set_split(self._h, int(split)))

    def close(self):
        if self._h:
            L.lib().ss3d_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vario(res, dirs):
    """Experimental variograms (f90:394-480).

    res: float64 array (nreal, nz, ny, nx) (numpy or torch CUDA tensor).
    dirs: list of (sx, sy, sz, nlag).  Returns gam of shape (nreal, ndir, nlagmax)
    and the pair counts (ndir, nlagmax)."""
    nreal, nz, ny, nx = res.shape
    dirs = [tuple(int(v) for v in d) for d in dirs]
    ndir = len(dirs)
    nlagmax = max(d[3] for d in dirs)
    sx, sy, sz, nl = (np.ascontiguousarray(np.array([d[k] for d in dirs], dtype=np.int32)) for k in range(4))
    gam = np.zeros((nreal, ndir, nlagmax))
    npairs = np.zeros((ndir, nlagmax), dtype=np.int64)
    ptr, code = _out_ptr(res)
    if code != OUT_F64:
        raise ValueError("vario needs float64 fields")
    n = np.array([nx, ny, nz], dtype=np.int32)
    L.check(L.lib().ss3d_vario(ptr, L.iptr(n), nreal, ndir, L.iptr(sx), L.iptr(sy), L.iptr(sz), L.iptr(nl),
                               ctypes.c_void_p(gam.ctypes.data), ctypes.c_void_p(npairs.ctypes.data)))
    return gam, npairs


def fft3d(a, isign):
    """Unscaled 3D FFT in place (fft3d, f90:254-304) of a complex128 array of
    shape (nz, ny, nx) (numpy, or a torch CUDA tensor); isign -1 forward, +1
    inverse.  Every axis a power of two."""
    nz, ny, nx = a.shape
    if isinstance(a, np.ndarray):
        if a.dtype != np.complex128 or not a.flags.c_contiguous:
            raise ValueError("fft3d needs a C-contiguous complex128 array")
        ptr = ctypes.c_void_p(a.ctypes.data)
    else:
        import torch
        if a.dtype != torch.complex128 or not a.is_contiguous():
            raise ValueError("fft3d needs a contiguous complex128 tensor")
        ptr = ctypes.c_void_p(a.data_ptr())
    L.check(L.lib().ss3d_fft3d(ptr, int(nx), int(ny), int(nz), int(isign)))
    return a


def condition(res, xmin, d, structs, nugget, params, rows, precision=FP64):
    """Conditioning by kriging of the residual, in place on res (f90:700-1081).

    params: dict with the conditioning-block fields of ss3d_cond_params.
    rows: (nrows, nvar) float64 data rows.  Returns (stats dict, extras dict)."""
    nreal, nz, ny, nx = res.shape
    cp = L.CondParams()
    for k, v in params.items():
        if k in ("radius", "angles"):
            getattr(cp, k)[:] = [float(x) for x in v]
        else:
            setattr(cp, k, v)
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.float64))
    nrows, nvar = rows.shape
    outs = {k: np.zeros(max(nrows, 1)) for k in ("vrt", "gtt", "dxs", "dys", "dzs", "dval", "dg")}
    cs = L.CondStats()
    arr = L.structs_array(structs)
    ptr, code = _out_ptr(res)
    if code != OUT_F64:
        raise ValueError("condition needs float64 fields")
    n = np.array([nx, ny, nz], dtype=np.int32)
    L.check(L.lib().ss3d_condition(ptr, L.iptr(n), nreal, L.dptr(_np3(xmin, np.float64)),
                                   L.dptr(_np3(d, np.float64)), arr, len(arr), float(nugget), ctypes.byref(cp),
                                   ctypes.c_void_p(rows.ctypes.data), nrows, nvar, int(precision), ctypes.byref(cs),
                                   *[ctypes.c_void_p(outs[k].ctypes.data) for k in
                                     ("vrt", "gtt", "dxs", "dys", "dzs", "dval", "dg")]))
    stats = dict(nd=cs.nd, nmerged=cs.nmerged, nout=cs.nout, nsb=tuple(cs.nsb), nsum=cs.nsum, nfail=cs.nfail,
                 nnone=cs.nnone, nexact=cs.nexact, data_mean=cs.data_mean, data_var=cs.data_var)
    nd = cs.nd
    return stats, {k: v[:nd] for k, v in outs.items()}


def _cond_params(params):
    cp = L.CondParams()
    for k, v in params.items():
        if k in ("radius", "angles"):
            getattr(cp, k)[:] = [float(x) for x in v]
        else:
            setattr(cp, k, v)
    return cp


class Server:
    """Serving form: a request loop over the simulation path (ss3d_server_*).

    ``slots`` requests run on the GPU at once, each on its own stream; queued
    requests are admitted in arrival order as slots and HBM free up (budget
    ``hbm_budget`` bytes, 0 = 80 % of free memory); spectra of seen models stay
    resident (LRU, ``cache_budget`` bytes of idle spectra).  ``premap_bytes`` of
    device memory are mapped into the stream-ordered pool at creation, so that
    requests do not stall on page mapping.  ``dry_run_ns_per_cell`` > 0 replaces
    the GPU work by sleeps (scheduler tests without a GPU)."""

    def __init__(self, slots=4, hbm_budget=0, cache_budget=0, retain_bytes=0, max_bypass=0, max_cond=0,
                 dry_run_ns_per_cell=0.0, premap_bytes=0):
        cfg = L.ServerConfig(int(slots), int(max_bypass), int(max_cond), int(hbm_budget), int(cache_budget),
                             int(retain_bytes), float(dry_run_ns_per_cell), int(premap_bytes))
        h = ctypes.c_void_p()
        L.check(L.lib().ss3d_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, model, iseed, nreal, igauss=1, precision=FP32, r_first=0, out=None, t_arrival=-1.0, cond=None):
        """Queue one request; returns its ticket.

        model: dict(structs, nugget, d, n, ipad).  out: numpy array or torch
        tensor of shape (nreal, nz, ny, nx), float32 or float64 (float64 with
        cond); None only in a dry run.  cond: dict(params, rows, xmin) as for
        condition().  t_arrival: arrival on the server clock (< 0: now)."""
        arr = L.structs_array(model["structs"])
        q = L.Request()
        q.st = ctypes.cast(arr, ctypes.c_void_p)
        q.nst = len(arr)
        q.nugget = float(model["nugget"])
        q.d[:] = [float(v) for v in model["d"]]
        q.n[:] = [int(v) for v in model["n"]]
        q.ipad = int(model["ipad"])
        q.iseed, q.igauss, q.r_first, q.nreal, q.precision = int(iseed), int(igauss), int(r_first), int(nreal), int(precision)
        q.t_arrival = float(t_arrival)
        keep = [arr, out]
        if out is not None:
            ptr, code = _out_ptr(out)
            q.out, q.out_dtype = ptr.value, code
        else:
            q.out, q.out_dtype = None, (OUT_F64 if cond is not None else OUT_F32)
        if cond is not None:
            cp = _cond_params(cond["params"])
            rows = np.ascontiguousarray(np.asarray(cond["rows"], dtype=np.float64))
            q.cp = ctypes.cast(ctypes.pointer(cp), ctypes.c_void_p)
            q.rows = rows.ctypes.data
            q.nrows, q.nvar = rows.shape
            q.xmin[:] = [float(v) for v in cond["xmin"]]
            keep += [cp, rows]
        t = ctypes.c_int64()
        L.check(L.lib().ss3d_server_submit(self._h, ctypes.byref(q), ctypes.byref(t)))
        self._keep[t.value] = keep
        return t.value

    def wait(self, ticket):
        """Block until the request is done: dict(status, message, cache_hit, t_arrival, t_submit, t_admit,
        t_done, footprint)."""
        r = L.Result()
        rc = L.lib().ss3d_server_wait(self._h, int(ticket), ctypes.byref(r))
        msg = L.lib().ss3d_last_error().decode() if rc else ""
        self._keep.pop(int(ticket), None)
        return dict(status=rc, message=msg, cache_hit=bool(r.cache_hit), t_arrival=r.t_arrival, t_submit=r.t_submit,
                    t_admit=r.t_admit, t_done=r.t_done, footprint=int(r.footprint))

    def stats(self):
        st = L.ServeStats()
        L.check(L.lib().ss3d_server_stats(self._h, ctypes.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in L.ServeStats._fields_}

    def clock(self):
        return float(L.lib().ss3d_server_clock(self._h))

    def close(self):
        if self._h:
            L.lib().ss3d_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
