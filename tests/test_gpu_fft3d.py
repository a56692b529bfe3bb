"""The full-grid transform export ss3d_fft3d against the oracle's restatement
of the reference's radix-2 fft3d (f90:208-304): unscaled, in place, isign -1
forward and +1 inverse, on random complex grids including axes of length 1.
The Stockham radix-8/4/2 transforms round differently from the radix-2 DIT:
agreement to 1e-12 of the largest magnitude; forward then inverse returns
N times the input."""
import ctypes

import numpy as np
import pytest

import oracle_lib as ora

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8, 8), (1, 16, 32), (4, 1, 64), (2, 8, 1), (1, 1, 2048), (32, 64, 16), (1, 1, 1)]


def _oracle_fft3d(a, isign):
    nz, ny, nx = a.shape
    b = np.ascontiguousarray(a).copy()
    ora.lib().ora_fft3d(ctypes.c_void_p(b.ctypes.data), nx, ny, nz, int(isign))
    return b


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("isign", [-1, 1])
def test_fft3d_matches_oracle(gpu, shape, isign):
    rng = np.random.default_rng(sum(shape) + isign)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    got = gpu.fft3d(a.copy(), isign)
    ref = _oracle_fft3d(a, isign)
    assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_fft3d_round_trip_and_device_input(gpu):
    import torch
    rng = np.random.default_rng(3)
    a = rng.normal(size=(16, 32, 64)) + 1j * rng.normal(size=(16, 32, 64))
    t = torch.from_numpy(a.copy()).cuda()
    gpu.fft3d(t, -1)
    gpu.fft3d(t, 1)
    back = t.cpu().numpy() / a.size
    assert np.max(np.abs(back - a)) <= 1e-12 * np.max(np.abs(a))


def test_fft3d_rejects_non_power_of_two(gpu):
    a = np.zeros((4, 4, 6), dtype=np.complex128)
    with pytest.raises(gpu.SpecsimError, match="powers of two"):
        gpu.fft3d(a, -1)
