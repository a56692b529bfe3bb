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


# ---------------------------------------------------------------- conditional tables
# Restatement of the reference's seeded conditional runs (docs/make_figures.py
# cond_case 770-786, sk_reference 719-736, fig12_cond_validation 804-847,
# fig13_cond_nscore 850-885): the grid, model, seeds, data sites and cpar
# contents are those recorded in tests/golden/reference_pins.json "cases".
COND = dict(n=(64, 64, 16), structs=[(2, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)], nugget=0.0, d=(1.0, 1.0, 1.0),
            ipad=1)


def cond_params(itrans=0, zlim=(0.0, 100.0)):
    """The cpar of make_cond_par with the recipe's arguments (columns 1 2 3 4 0,
    trimming +-1e21, skmean 0, linear tails, radii 30/15/8, angles 45/0/0,
    ndmax 24), as the GPU binding names its fields."""
    return dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1.0e21, tmax=1.0e21, itrans=itrans, skmean=0.0,
                zmin=zlim[0], zmax=zlim[1], ltail=1, ltpar=0.0, utail=1, utpar=0.0, radius=(30.0, 15.0, 8.0),
                angles=(45.0, 0.0, 0.0), ndmax=24)


def oracle_cond_params(p):
    """The same parameters under the oracle binding's field names."""
    return dict(ixc=p["ixc"], iyc=p["iyc"], izc=p["izc"], ivc=p["ivc"], iwc=p["iwc"], tmin=p["tmin"], tmax=p["tmax"],
                itrans=p["itrans"], skmean=p["skmean"], zlo=p["zmin"], zhi=p["zmax"], ltail=p["ltail"],
                ltpar=p["ltpar"], utail=p["utail"], utpar=p["utpar"], rmax=p["radius"][0], rmed=p["radius"][1],
                rvert=p["radius"][2], sa1=p["angles"][0], sa2=p["angles"][1], sa3=p["angles"][2], ndmax=p["ndmax"])


def as_bin(res):
    """What the recipe reads back from a .bin file: float32 values as float64, (nreal, x, y, z)."""
    return res.astype(np.float32).astype(np.float64).transpose(0, 3, 2, 1)


def gslib_value(v):
    """A data value after the round trip through the recipe's data file ('%.8g')."""
    return float("%.8g" % v)


def cond_sites(truth_xyz, nd=150):
    """Data sites of cond_case: nd distinct nodes of default_rng(7), (x, y, z) C order."""
    rng = np.random.default_rng(7)
    idx = rng.choice(int(np.prod(COND["n"])), nd, replace=False)
    ijk = np.array(np.unravel_index(idx, COND["n"])).T
    return ijk


def cond_rows(ijk, val):
    return np.array([[float(i), float(j), float(k), gslib_value(v)] for (i, j, k), v in zip(ijk, val)])


def _corr(it, r):
    r = np.asarray(r, float)
    if it == 1:
        return np.where(r < 1, 1 - 1.5 * r + 0.5 * r ** 3, 0.0)
    return np.exp(-3 * r) if it == 2 else np.exp(-3 * r ** 2)


def exact_sk(xyz, val):
    """Simple kriging (mean 0) with all data at every node, in the recipe's
    covariance (azimuth rotation only) and with its ridge 1e-10: estimate and
    variance, shape (nx, ny, nz)."""
    it, sill, a1, a2, a3, az = COND["structs"][0][:6]
    c0 = COND["nugget"] + sum(s[1] for s in COND["structs"])
    azr = np.radians(az)
    u = np.array([np.sin(azr), np.cos(azr), 0.0])
    w = np.array([np.cos(azr), -np.sin(azr), 0.0])

    def cov(dv):
        h = np.sqrt((dv @ u / a1) ** 2 + (dv @ w / a2) ** 2 + (dv[..., 2] / a3) ** 2)
        return sill * _corr(it, h)

    K = cov(xyz[:, None, :] - xyz[None, :, :]) + COND["nugget"] * np.eye(len(xyz))
    grid = COND["n"]
    gx, gy, gz = np.meshgrid(*(np.arange(n, dtype=float) for n in grid), indexing="ij")
    P = np.c_[gx.ravel(), gy.ravel(), gz.ravel()]
    k = cov(xyz[None, :, :] - P[:, None, :])
    W = np.linalg.solve(K + 1e-10 * np.eye(len(xyz)), k.T).T
    return (W @ val).reshape(grid), (c0 - (W * k).sum(1)).reshape(grid)


def fig12_row(sims, est, var, xyz, val):
    """The SPECSIM3D row of fig12_conditional_validation.csv from realizations
    sims (nreal, x, y, z), at the printed precision."""
    n = len(sims)
    m = sims.mean(0)
    v = sims.var(0, ddof=1)
    se = np.sqrt(var / n)
    zs = (m - est) / np.maximum(se, 1e-9)
    free = var > 1e-6
    ii = xyz.astype(int)
    return dict(
        rms_mean_diff=round(float(np.sqrt(np.mean((m - est) ** 2))), 4),
        mc_error_mean=round(float(np.sqrt(np.mean(se ** 2))), 4),
        rms_var_diff=round(float(np.sqrt(np.mean((v - var) ** 2))), 4),
        mc_error_var=round(float(np.sqrt(np.mean(2 * var ** 2 / (n - 1)))), 4),
        var_slope=round(float(np.sum(v * var) / np.sum(var * var)), 4),
        std_of_standardized_mean_diff=round(float(np.std(zs[free])), 3),
        max_abs_data_error=float("%.2e" % float(np.abs(sims[:, ii[:, 0], ii[:, 1], ii[:, 2]] - val).max())))


def fig13_table(truth_ln, val, sims, ijk):
    """fig13_conditional_nscore.csv from the lognormal truth (x, y, z), the data
    values and the realizations (nreal, x, y, z), at the printed precision."""
    dmax = float(np.abs(sims[:, ijk[:, 0], ijk[:, 1], ijk[:, 2]] - val).max() / val.max())
    return {"max |realization - data| / max data at data nodes": float("%.2e" % dmax),
            "mean truth": round(float(truth_ln.mean()), 3), "mean data": round(float(val.mean()), 3),
            "mean realizations": round(float(sims.mean()), 3), "variance truth": round(float(truth_ln.var()), 3),
            "variance data": round(float(val.var()), 3), "variance realizations": round(float(sims.var()), 3)}


def conditional_tables(realize, condition, which=("fig12", "fig13")):
    """Run the reference's seeded conditional recipe through a backend:
    realize(seed, nreal) -> res (nreal, nz, ny, nx) float64 of the COND model;
    condition(res, params, rows) conditions res in place.  Returns the fig12
    row and the fig13 table as the reference prints them."""
    out = {}
    truth = as_bin(realize(2024, 1))[0]
    ijk = cond_sites(truth)
    xyz = ijk.astype(float)
    if "fig12" in which:
        val = truth[ijk[:, 0], ijk[:, 1], ijk[:, 2]]
        res = realize(777, 200)
        condition(res, cond_params(itrans=0), cond_rows(ijk, val))
        est, var = exact_sk(xyz, val)
        out["fig12"] = fig12_row(as_bin(res), est, var, xyz, val)
    if "fig13" in which:
        truth_ln = np.exp(1.0 + 0.8 * truth)
        val = truth_ln[ijk[:, 0], ijk[:, 1], ijk[:, 2]]
        zhi = float(val.max() * 2)
        res = realize(99, 50)
        condition(res, cond_params(itrans=1, zlim=(0.0, zhi)), cond_rows(ijk, val))
        out["fig13"] = fig13_table(truth_ln, val, as_bin(res), ijk)
    return out


# ---------------------------------------------------------------- anisotropy cases
# Restatement of docs/make_figures.py fig05_cases (459-495): 6 anisotropy cases x
# 3 models plus a nested model with nugget on a 64x64x16 grid, 20 realizations of
# seed 2024 each; the mean experimental semivariogram at up to 300 arbitrary
# integer lag vectors (one-lag directions of the --vario file, drawn from a
# fresh default_rng(12345)) against the model; the CSV values are the
# reference's es14.6 (vario_report f90:433-530).
FIG05_CASES = [
    ("A iso 15/15/15", 0.0, [(1.0, 15, 15, 15, 0, 0, 0)]),
    ("B 2:1 20/10/10", 0.0, [(1.0, 20, 10, 10, 30, 0, 0)]),
    ("C 4:1 20/5/5", 0.0, [(1.0, 20, 5, 5, 60, 0, 0)]),
    ("D layered 10/10/2", 0.0, [(1.0, 10, 10, 2, 0, 0, 0)]),
    ("E extreme 40/4/2", 0.0, [(1.0, 40, 4, 2, 135, 0, 0)]),
    ("F rotated 20/8/4 (az30 dip20 plg15)", 0.0, [(1.0, 20, 8, 4, 30, 20, 15)]),
]
FIG05_NESTED = ("G nested + nugget 0.1 (sph + exp)", 0.1, [(1, 0.5, 20, 10, 5, 45, 0, 0), (2, 0.4, 8, 8, 3, 0, 0, 0)])
FIG05_MODELS = (("spherical", 1), ("exponential", 2), ("gaussian", 3))


def fig05_lags():
    rng = np.random.default_rng(12345)
    cand = np.column_stack([rng.integers(-30, 31, 1500), rng.integers(-30, 31, 1500), rng.integers(-12, 13, 1500)])
    return cand[np.any(cand != 0, axis=1)]


def fig05_jobs():
    jobs = []
    for cname, nug, st in FIG05_CASES:
        for mname, it in FIG05_MODELS:
            jobs.append((cname, mname, nug, [(it,) + tuple(float(v) for v in s) for s in st]))
    jobs.append((FIG05_NESTED[0], "nested", FIG05_NESTED[1], [tuple(float(v) for v in s) for s in FIG05_NESTED[2]]))
    return jobs


def es14_6(v):
    return float("%.6e" % v)


def fig05_row(gam, lags, nugget, structs, covariance):
    """One row of fig05_cases.csv from gam (nreal, ndir) at the one-lag
    directions `lags` (np > 0 for all of them on this grid); covariance(structs,
    nugget, hx, hy, hz) is the model covariance of f90:153-178."""
    nreal = gam.shape[0]
    c0 = nugget + sum(s[1] for s in structs)
    gm = np.array([es14_6(sum(gam[r, d] for r in range(nreal)) / nreal) for d in range(gam.shape[1])])
    gsd = []
    for d in range(gam.shape[1]):
        mean = sum(gam[r, d] for r in range(nreal)) / nreal
        gsd.append(es14_6(np.sqrt(sum((gam[r, d] - mean) ** 2 for r in range(nreal)) / (nreal - 1))))
    gsd = np.array(gsd)
    gt = np.array([es14_6(c0 - covariance(structs, nugget, float(a), float(b), float(c))) for a, b, c in lags])
    se = gsd / np.sqrt(nreal)
    keep = (gt > 0.05 * c0) & (gt < 0.97 * c0)
    idx = np.flatnonzero(keep)[:300]
    rms = float(np.sqrt(np.mean((gm[idx] - gt[idx]) ** 2)))
    noise = float(np.sqrt(np.mean(se[idx] ** 2)))
    return dict(n_lags=len(idx), rms=round(rms, 4), mc_noise=round(noise, 4), rms_over_noise=round(rms / noise, 2),
                bias=round(float(np.mean(gm[idx] - gt[idx])), 4))
