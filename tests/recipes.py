"""Statistics recipes used by the golden pins (restated from the descriptions in
tests/golden/reference_pins.json) and small helpers shared by the tests."""
import numpy as np

RANGES = (20.0, 10.0, 5.0)
YAO = dict(n=(64, 64, 16), structs=[(1, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)], nugget=0.0, d=(1.0, 1.0, 1.0))


def vario_shift(f, step, kmax):
    """numpy all-pairs semivariogram of f (nreal, x, y, z) along k*step, k=1..kmax."""
    out, lags = [], []
    for k in range(1, kmax + 1):
        d = [k * s for s in step]
        if any(abs(di) >= n for di, n in zip(d, f.shape[1:])):
            break
        sa = [slice(None)] + [slice(max(0, -di), n - max(0, di)) for di, n in zip(d, f.shape[1:])]
        sb = [slice(None)] + [slice(max(0, di), n - max(0, -di)) for di, n in zip(d, f.shape[1:])]
        out.append(0.5 * np.mean((f[tuple(sa)] - f[tuple(sb)]) ** 2, axis=(1, 2, 3)))
        lags.append(k * np.linalg.norm(step))
    return np.array(out).T, np.array(lags)


def rho_sph(r):
    r = np.asarray(r, float)
    return np.where(r < 1, 1 - 1.5 * r + 0.5 * r ** 3, 0.0)


def scaling_rms(res_f32_first):
    """RMS recipe of the scaling benchmark on realization 1 given as float32 (nz, ny, nx)."""
    f = res_f32_first.astype(np.float64).transpose(2, 1, 0)[None]
    errs = []
    for step, a in [((1, 1, 0), RANGES[0]), ((1, -1, 0), RANGES[1]), ((0, 0, 1), RANGES[2])]:
        g, lag = vario_shift(f, step, int(a))
        errs.append(np.sqrt(np.mean((g[0] - (1 - rho_sph(lag / a))) ** 2)))
    return float(np.mean(errs))


def scaling_case(n):
    return dict(n=(n, n, n), structs=[(1, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)], nugget=0.0, d=(1.0, 1.0, 1.0),
                ipad=1, seed=99, nreal=1 if n >= 256 else 2)


def half_of_full(full, npx):
    """Restrict a full-spectrum array (..., npx) to the Hermitian half i <= npx/2."""
    h = npx // 2 + 1 if npx >= 2 else 1
    return full[..., :h]
