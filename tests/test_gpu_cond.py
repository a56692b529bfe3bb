"""GPU conditioning (kriging of the residual) against the oracle's condition_field.

The neighbour search reproduces the reference's sets exactly (same FP64
expression order without FMA, same visit order and insertion rules), so the
search statistics must match exactly.  The FP64 kriging solve differs from the
reference only in the order of the Cholesky sums: conditioned values agree to
1e-9.  The FP32 form (FP32 factor and solve, one FP64-residual refinement)
agrees to 1e-5 of the field's standard deviation.
"""
import numpy as np
import pytest

import oracle_lib as ora

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=0, skmean=0.0, zlo=-5.0, zhi=5.0,
             ltail=1, ltpar=0.0, utail=1, utpar=0.0, rmax=100.0, rmed=100.0, rvert=100.0, sa1=0.0, sa2=0.0, sa3=0.0,
             ndmax=100)
    p.update(kw)
    return p


def _gpu_params(p):
    return dict(ixc=p["ixc"], iyc=p["iyc"], izc=p["izc"], ivc=p["ivc"], iwc=p["iwc"], tmin=p["tmin"], tmax=p["tmax"],
                itrans=p["itrans"], skmean=p["skmean"], zmin=p["zlo"], zmax=p["zhi"], ltail=p["ltail"],
                ltpar=p["ltpar"], utail=p["utail"], utpar=p["utpar"], radius=(p["rmax"], p["rmed"], p["rvert"]),
                angles=(p["sa1"], p["sa2"], p["sa3"]), ndmax=p["ndmax"])


def _run_both(gpu, sts, nug, n, xmin, d, p, rows, nreal, seed, precision):
    sp = gpu.Spectrum(sts, nug, d, n, 1)
    res = sp.realize(seed, nreal, 0, gpu.FP64)
    a = res.copy()
    b = res.copy()
    st_o, ex_o = ora.condition(a, xmin, d, sts, nug, p, rows)
    st_g, ex_g = gpu.condition(b, xmin, d, sts, nug, _gpu_params(p), rows, precision=precision)
    return a, b, st_o, st_g, ex_o, ex_g


def _check_stats(st_o, st_g):
    for k in ("nd", "nmerged", "nout", "nsb", "nsum", "nnone", "nexact", "nfail"):
        assert st_o[k] == st_g[k], (k, st_o[k], st_g[k])


def test_gaussian_all_data_in_neighbourhood(gpu):
    """Reference tests/test_conditional.py:test_gaussian setting (30x30x10, 40 data, radii 100, ndmax 100)."""
    rng = np.random.default_rng(3)
    n = (30, 30, 10)
    idx = rng.choice(n[0] * n[1] * n[2], 40, replace=False)
    i, j, k = np.unravel_index(idx, n)
    rows = np.c_[i, j, k, rng.normal(size=40)].astype(float)
    sts = [(1, 1.0, 12.0, 8.0, 6.0, 30.0, 0.0, 0.0)]
    p = _params()
    a, b, so, sg, eo, eg = _run_both(gpu, sts, 0.0, n, (0, 0, 0), (1, 1, 1), p, rows, 6, 12345, gpu.FP64)
    _check_stats(so, sg)
    assert np.max(np.abs(a - b)) <= 1e-9
    # data reproduced at their nodes
    assert np.max(np.abs(b[:, k, j, i] - rows[:, 3][:, None].T)) < 1e-9


def test_nscore_backtransform_2d(gpu):
    """Reference test_nscore setting: 64x64 2D, 200 lognormal data, itrans 1, linear tails."""
    rng = np.random.default_rng(5)
    idx = rng.choice(64 * 64, 200, replace=False)
    x, y = (idx % 64).astype(float), (idx // 64).astype(float)
    v = np.exp(rng.normal(1.0, 0.8, 200))
    rows = np.c_[x, y, v]
    sts = [(2, 1.0, 15.0, 15.0, 15.0, 0.0, 0.0, 0.0)]
    p = _params(ixc=1, iyc=2, izc=0, ivc=3, tmin=0.0, itrans=1, zlo=0.0, zhi=200.0, rmax=30.0, rmed=30.0,
                rvert=30.0, ndmax=16)
    a, b, so, sg, eo, eg = _run_both(gpu, sts, 0.0, (64, 64, 1), (0, 0, 0), (1, 1, 1), p, rows, 4, 777, gpu.FP64)
    _check_stats(so, sg)
    assert np.array_equal(eo["gtt"], eg["gtt"]) or np.max(np.abs(eo["gtt"] - eg["gtt"])) < 1e-14
    assert np.array_equal(eo["vrt"], eg["vrt"])
    assert np.max(np.abs(a - b) / np.maximum(1.0, np.abs(a))) <= 1e-9


@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (1, 1e-5)])
def test_conditional_config_small(gpu, precision, tol):
    """Configuration-4-like case: exponential 40/20/8 N60E, nugget 0.05, ndmax 24, skewed data through nscore."""
    rng = np.random.default_rng(99)
    n = (48, 40, 16)
    sts = [(2, 1.0, 40.0, 20.0, 8.0, 60.0, 0.0, 0.0)]
    sp = gpu.Spectrum(sts, 0.05, (1, 1, 1), n, 1)
    truth = sp.realize(4242, 1, 0, gpu.FP64)[0]
    pts = rng.uniform(0, np.array(n) - 1, size=(300, 3))
    ii = np.rint(pts).astype(int)
    val = np.exp(0.5 * truth[ii[:, 2], ii[:, 1], ii[:, 0]])
    rows = np.c_[pts, val]
    p = _params(tmin=0.0, itrans=1, zlo=0.0, zhi=2 * val.max(), rmax=40.0, rmed=20.0, rvert=8.0, sa1=60.0, ndmax=24)
    a, b, so, sg, eo, eg = _run_both(gpu, sts, 0.05, n, (0, 0, 0), (1, 1, 1), p, rows, 4, 4243, precision)
    _check_stats(so, sg)
    err = np.max(np.abs(a - b)) / max(1e-12, float(np.std(a)))
    assert err <= tol, err


@pytest.mark.parametrize("angles,radii,ndmax,n", [((30.0, 20.0, 10.0), (30.0, 15.0, 6.0), 16, (60, 50, 24)),
                                                  ((120.0, -35.0, 60.0), (25.0, 25.0, 5.0), 24, (40, 44, 30)),
                                                  ((75.0, 0.0, 0.0), (50.0, 10.0, 10.0), 8, (90, 30, 1)),
                                                  ((10.0, 60.0, -20.0), (12.0, 6.0, 3.0), 32, (32, 32, 32))])
def test_search_tilted_ellipsoids(gpu, angles, radii, ndmax, n):
    """Neighbour search with the search ellipsoid rotated out of the xy plane
    (dip and plunge), strongly anisotropic, in 2D and 3D: the neighbour counts,
    empty and exact-data nodes equal the oracle's and the fields agree to 1e-9
    (super blocks that can hold no datum inside the ellipsoid are never scanned;
    this is where a wrongly skipped block would show)."""
    rng = np.random.default_rng(sum(n) + ndmax)
    sts = [(1, 0.9, radii[0], radii[1], radii[2], angles[0], angles[1], angles[2])]
    nd = 250
    pts = np.stack([rng.uniform(0, n[a] - 1, nd) for a in range(3)], axis=1)
    if n[2] == 1:
        pts[:, 2] = 0.0
    rows = np.c_[pts, rng.normal(size=nd)]
    p = _params(rmax=radii[0], rmed=radii[1], rvert=radii[2], sa1=angles[0], sa2=angles[1], sa3=angles[2],
                ndmax=ndmax)
    a, b, so, sg, eo, eg = _run_both(gpu, sts, 0.1, n, (0, 0, 0), (1, 1, 1), p, rows, 3, 2468, gpu.FP64)
    _check_stats(so, sg)
    assert np.max(np.abs(a - b)) <= 1e-9


@pytest.mark.parametrize("maxdup,ties", [(2, False), (4, False), (1, True), (3, True)])
def test_merged_nodes_and_tied_values(gpu, maxdup, ties):
    """Data sharing nodes (groups of up to maxdup data on one node, merged by
    weighted average) and, with ties, repeated data values before the normal
    scores: the merged values, the normal-score table and every statistic
    equal the oracle's bit for bit, and the fields agree to 1e-9 (the sort of
    the merge and of the scores must order equal keys as the reference does
    wherever that order shows)."""
    rng = np.random.default_rng(17 * maxdup + ties)
    n = (40, 36, 12)
    nodes = rng.choice(n[0] * n[1] * n[2], 120, replace=False)
    i, j, k = np.unravel_index(nodes, (n[0], n[1], n[2]), order="F")
    reps = rng.integers(1, maxdup + 1, size=120)
    pts = np.repeat(np.c_[i, j, k].astype(float), reps, axis=0)
    pts += rng.uniform(-0.3, 0.3, size=pts.shape)           # snapped back to the same node
    vals = np.exp(rng.normal(size=len(pts)))
    if ties:
        vals = np.round(vals, 1)                             # repeated values
    wts = rng.uniform(0.5, 2.0, size=len(pts))
    rows = np.c_[pts, vals, wts]
    sts = [(2, 1.0, 15.0, 10.0, 5.0, 30.0, 0.0, 0.0)]
    p = _params(iwc=5, tmin=0.0, itrans=1, zlo=0.0, zhi=2 * float(vals.max()), rmax=20.0, rmed=15.0, rvert=6.0,
                sa1=30.0, ndmax=16)
    a, b, so, sg, eo, eg = _run_both(gpu, sts, 0.05, n, (0, 0, 0), (1, 1, 1), p, rows, 2, 1357, gpu.FP64)
    _check_stats(so, sg)
    if maxdup >= 2:
        assert so["nmerged"] > 0
    for key in ("dval", "vrt", "gtt", "dg"):
        assert np.array_equal(eo[key], eg[key]), key
    assert np.max(np.abs(a - b)) <= 1e-9


def test_condition_device_array(gpu):
    import torch
    rng = np.random.default_rng(8)
    n = (20, 16, 8)
    sts = [(1, 1.0, 10.0, 8.0, 4.0, 0.0, 0.0, 0.0)]
    rows = np.c_[rng.uniform(0, 19, 30), rng.uniform(0, 15, 30), rng.uniform(0, 7, 30), rng.normal(size=30)]
    sp = gpu.Spectrum(sts, 0.0, (1, 1, 1), n, 1)
    res = sp.realize(5, 3, 0, gpu.FP64)
    h = res.copy()
    gpu.condition(h, (0, 0, 0), (1, 1, 1), sts, 0.0, _gpu_params(_params(rmax=10, rmed=10, rvert=10, ndmax=12)), rows)
    t = torch.from_numpy(res.copy()).cuda()
    gpu.condition(t, (0, 0, 0), (1, 1, 1), sts, 0.0, _gpu_params(_params(rmax=10, rmed=10, rvert=10, ndmax=12)), rows)
    assert np.array_equal(t.cpu().numpy(), h)


def test_no_data_inside_grid(gpu):
    rows = np.array([[100.0, 100.0, 100.0, 1.0]])
    res = np.zeros((1, 4, 4, 4))
    with pytest.raises(gpu.SpecsimError, match="no conditioning data"):
        gpu.condition(res, (0, 0, 0), (1, 1, 1), [(1, 1.0, 5, 5, 5, 0, 0, 0)], 0.0, _gpu_params(_params()), rows)


@pytest.mark.parametrize("precision", [0, 1])
def test_conditional_tables_fig12_fig13_gpu(gpu, precision):
    """The reference's seeded conditional tables (fig12 SPECSIM3D row, fig13)
    through the CUDA path, to every printed digit: FP64 realizations, kriging
    in FP64 or in the precision form (FP32 solves + one FP64 refinement)."""
    import json
    import os
    import recipes
    pins = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))
    c = recipes.COND
    sp = gpu.Spectrum(c["structs"], c["nugget"], c["d"], c["n"], c["ipad"])

    def realize(seed, nreal):
        return sp.realize(seed, nreal, 0, gpu.FP64)

    def condition(res, p, rows):
        st, _ = gpu.condition(res, (0.0, 0.0, 0.0), c["d"], c["structs"], c["nugget"], p, rows, precision=precision)
        assert st["nd"] == len(rows)

    got = recipes.conditional_tables(realize, condition)
    sp.close()
    want12 = {k: v for k, v in pins["fig12"].items() if k not in ("code", "nreal", "seconds_per_realization")}
    assert got["fig12"] == want12
    assert got["fig13"] == pins["fig13"]


@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (1, 1e-5)])
def test_conditional_config_full_size(gpu, precision, tol):
    """The conditional configuration at full size against the oracle:
    128x128x64, exponential 40/20/8 N60E, nugget 0.05; truth = realization 1 of
    seed 4242 (igauss 0); 2,000 data at default_rng(99) uniform locations with
    values exp(0.5 z) of the truth; nscore + back transform (zmax = 2 max, linear
    tails); search = the ranges, ndmax 24; 16 realizations of seed 4243.  The
    search statistics (neighbours, exact data nodes, empty nodes, regularised
    systems) are equal; the fields agree to 1e-9 (FP64) or 1e-5 of their
    standard deviation (precision form).  On a lattice the integer distance
    ties of the insertion rule are common: this is where they would show."""
    n = (128, 128, 64)
    sts = [(2, 1.0, 40.0, 20.0, 8.0, 60.0, 0.0, 0.0)]
    sp = gpu.Spectrum(sts, 0.05, (1, 1, 1), n, 1)
    truth = sp.realize(4242, 1, 0, gpu.FP64)[0]
    rng = np.random.default_rng(99)
    pts = np.stack([rng.uniform(0, n[a] - 1, 2000) for a in range(3)], axis=1)
    ii = np.rint(pts).astype(int)
    val = np.exp(0.5 * truth[ii[:, 2], ii[:, 1], ii[:, 0]])
    rows = np.c_[pts, val]
    p = _params(itrans=1, zlo=0.0, zhi=2 * float(val.max()), rmax=40.0, rmed=20.0, rvert=8.0, sa1=60.0, ndmax=24)
    res = sp.realize(4243, 16, 0, gpu.FP64)
    sp.close()
    a = res.copy()
    b = res.copy()
    st_o, ex_o = ora.condition(a, (0, 0, 0), (1, 1, 1), sts, 0.05, p, rows)
    st_g, ex_g = gpu.condition(b, (0, 0, 0), (1, 1, 1), sts, 0.05, _gpu_params(p), rows, precision=precision)
    _check_stats(st_o, st_g)
    assert np.array_equal(ex_o["vrt"], ex_g["vrt"])
    err = np.max(np.abs(a - b)) / float(np.std(a))
    assert err <= tol, err
