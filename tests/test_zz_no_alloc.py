"""The allocation-free realization entry point (ss3d_realize_noalloc).

It exists for callers that cannot call cudaMalloc when they need realizations:
an application whose device memory is already handed to its own pool, or a
latency-bound loop that cannot take the device-wide synchronisation of
cudaMalloc/cudaFree.  Its scratch is one fixed 64 MiB device array shared by
every call.  These tests call it through the C ABI and compare it with
ss3d_realize on two calls in a row.  Both run the same kernels on the same
inputs, so the results must be the same bits: a tolerance could hide a read of
the previous call's leftovers in the shared array.  They also check that an
oversized grid, host output and a misaligned device output are refused.  This
file is collected last so that a run stopping at the first failure has run
every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STRUCTS = [(1, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)]
N = (64, 64, 16)


def _noalloc(ss):
    from specsim3d_b200 import _lib
    f = _lib.lib().ss3d_realize_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int]
    return f


@pytest.mark.parametrize("precision", [1, 0])
@pytest.mark.parametrize("igauss", [0, 1])
def test_noalloc_matches_realize_twice(gpu, precision, igauss):
    import torch
    ss = gpu
    f = _noalloc(ss)
    sp = ss.Spectrum(STRUCTS, 0.0, (1.0, 1.0, 1.0), N, 1)
    calls = [(69069, 0, 2), (4711, 3, 1)]          # (seed, first realization, count), back to back
    for seed, r0, k in calls:
        ref = sp.realize(seed, k, igauss, precision, r_first=r0, dtype=np.float64)
        out = torch.full((k, N[2], N[1], N[0]), float("nan"), dtype=torch.float64, device="cuda")
        rc = f(sp.handle, seed, r0, k, igauss, precision, ctypes.c_void_p(out.data_ptr()), 1)
        assert rc == 0, ss._lib.lib().ss3d_last_error().decode()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.array_equal(got, ref), float(np.max(np.abs(got - ref)))
    sp.close()


def test_noalloc_rejects_oversized_grid(gpu):
    import torch
    ss = gpu
    f = _noalloc(ss)
    sp = ss.Spectrum(STRUCTS, 0.0, (1.0, 1.0, 1.0), (256, 256, 256), 0)   # periodic 256^3, nz = 256
    out = torch.empty((1, 256, 256, 256), dtype=torch.float32, device="cuda")
    rc = f(sp.handle, 1, 0, 1, 0, 1, ctypes.c_void_p(out.data_ptr()), 0)
    assert rc == ss._lib.SS3D_ETOOLARGE
    assert "bytes of scratch" in ss._lib.lib().ss3d_last_error().decode()
    sp.close()


def test_noalloc_rejects_host_output(gpu):
    ss = gpu
    f = _noalloc(ss)
    sp = ss.Spectrum(STRUCTS, 0.0, (1.0, 1.0, 1.0), N, 1)
    host = np.zeros((1, N[2], N[1], N[0]), dtype=np.float32)
    rc = f(sp.handle, 1, 0, 1, 0, 1, ctypes.c_void_p(host.ctypes.data), 0)
    assert rc == ss._lib.SS3D_EINVAL
    sp.close()


def test_noalloc_rejects_misaligned_output(gpu):
    """Rows of even length are stored as pairs: a device output that starts off
    a pair boundary is refused before any kernel runs."""
    import torch
    ss = gpu
    f = _noalloc(ss)
    sp = ss.Spectrum(STRUCTS, 0.0, (1.0, 1.0, 1.0), N, 1)
    flat = torch.zeros(N[0] * N[1] * N[2] + 1, dtype=torch.float32, device="cuda")
    rc = f(sp.handle, 1, 0, 1, 0, 1, ctypes.c_void_p(flat.data_ptr() + 4), 0)
    assert rc == ss._lib.SS3D_EINVAL
    assert "multiple of 8 bytes" in ss._lib.lib().ss3d_last_error().decode()
    torch.cuda.synchronize()
    assert float(flat.abs().sum().item()) == 0.0
    sp.close()
