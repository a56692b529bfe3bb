"""GPU experimental variograms against the oracle's vario_lag (f90:405-431).

Pair counts are exact integers (closed form of npair_count, f90:394-402).  The
FP64 sums are accumulated in a different order than the reference's serial
loop, so gamma is compared to a relative 1e-12.
"""
import numpy as np
import pytest

import oracle_lib as ora
import recipes

pytestmark = pytest.mark.gpu

DIRS = [(1, 1, 0, 9), (1, -1, 0, 9), (0, 0, 1, 6), (2, 0, 0, 8), (-1, 0, 0, 5), (0, -1, 0, 7), (1, 2, -1, 4),
        (0, 3, 2, 3), (-2, 1, 1, 5), (0, 0, 0, 2), (40, 0, 0, 2)]


@pytest.mark.parametrize("shape", [(3, 7, 13, 21), (2, 1, 17, 33), (1, 12, 1, 40), (2, 5, 6, 1), (1, 24, 24, 24)])
def test_vario_matches_oracle(gpu, shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.normal(size=shape)
    gam, npairs = gpu.vario(f, DIRS)
    ref = ora.vario(f, DIRS)
    assert np.allclose(gam, ref, rtol=1e-12, atol=1e-14)
    nreal, nz, ny, nx = shape
    for k, (sx, sy, sz, nl) in enumerate(DIRS):
        for l in range(1, nl + 1):
            assert npairs[k, l - 1] == ora.npair_count((nx, ny, nz), (l * sx, l * sy, l * sz))


def test_vario_device_input(gpu):
    import torch
    rng = np.random.default_rng(5)
    f = rng.normal(size=(2, 16, 20, 24))
    g_host, _ = gpu.vario(f, DIRS[:4])
    g_dev, _ = gpu.vario(torch.from_numpy(f).cuda(), DIRS[:4])
    assert np.array_equal(g_host, g_dev)


def test_vario_long_lags_and_strides(gpu):
    """Lags beyond one launch (chunks of 128) and large strides."""
    rng = np.random.default_rng(9)
    f = rng.normal(size=(1, 4, 6, 300))
    dirs = [(1, 0, 0, 299), (3, 0, 0, 99), (1, 1, 0, 5), (1, 0, 1, 3)]
    gam, _ = gpu.vario(f, dirs)
    assert np.allclose(gam, ora.vario(f, dirs), rtol=1e-12, atol=1e-14)


def test_vario_fortran_recipe(gpu):
    """Reference tests/test_vario_fortran.py: Yao case, 5 realizations, lags 1..40,
    program variogram vs numpy on the float32 .bin within 2e-6."""
    c = recipes.YAO
    sp = gpu.Spectrum(c["structs"], c["nugget"], c["d"], c["n"], 1)
    res = sp.realize(31791191, 5, 0, gpu.FP64)
    dirs = [(1, 1, 0, 40), (1, -1, 0, 40), (0, 0, 1, 40)]
    gam, npairs = gpu.vario(res, dirs)
    fx = res.astype(np.float32).astype(np.float64).transpose(0, 3, 2, 1)
    for k, (sx, sy, sz, nl) in enumerate(dirs):
        g, _ = recipes.vario_shift(fx, (sx, sy, sz), nl)
        m = g.shape[1]
        assert np.max(np.abs(g.mean(0) - gam[:, k, :m].mean(0))) <= 2e-6


def test_cfg1_pair_total(gpu):
    """64x64x16 grid, directions N45E, N45W, vertical, lags 1..30."""
    f = np.zeros((1, 16, 64, 64))
    _, npairs = gpu.vario(f, [(1, 1, 0, 30), (1, -1, 0, 30), (0, 0, 1, 30)])
    want = sum(ora.npair_count((64, 64, 16), (l * a, l * b, l * c)) for a, b, c in [(1, 1, 0), (1, -1, 0), (0, 0, 1)]
               for l in range(1, 31))
    assert int(npairs.sum()) == want
