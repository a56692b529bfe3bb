"""Serving form on the GPU: every request's result is the same alone and in
the mix.

Bar: bit for bit.  A request runs the library's own stages (spectrum build
on a cache miss, ss3d_realize, ss3d_condition) on its slot's stream; none of
them depends on what else runs (no cross-request reduction, deterministic
sums), so the mixed results must equal the same calls made one at a time.
"""
import numpy as np
import pytest

import specsim3d_b200 as ss
from specsim3d_b200 import workloads

pytestmark = pytest.mark.gpu


def _cond_for(model, ndata, seed):
    """Conditioning data as in the conditional recipe: uniform locations,
    skewed values exp(0.5 g); normal-score transform, search = the ranges."""
    rng = np.random.default_rng(seed)
    n = model["n"]
    xyz = np.stack([rng.uniform(0, n[a] - 1, ndata) for a in range(3)], axis=1)
    val = np.exp(0.5 * rng.standard_normal(ndata))
    rows = np.column_stack([xyz, val])
    st = model["structs"][0]
    params = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=1, skmean=0.0, zmin=0.0,
                  zmax=2.0 * float(val.max()), ltail=1, ltpar=0.0, utail=1, utpar=0.0,
                  radius=(st[2], st[3], st[4]), angles=(st[5], st[6], st[7]), ndmax=12)
    return dict(params=params, rows=rows, xmin=(0.0, 0.0, 0.0))


def _requests(count, seed=7):
    pool = workloads.model_pool(seed=seed, size=6, lo=16, hi=56)
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        m = pool[int(rng.integers(len(pool)))]
        cond = (q % 5 == 4)
        out.append(dict(model=m, iseed=int(rng.integers(1, 1 << 30)), nreal=int(rng.integers(1, 5)),
                        igauss=int(q % 2), precision=ss.FP64 if (cond or q % 3 == 0) else ss.FP32,
                        device=(q % 2 == 0),
                        cond=_cond_for(m, int(rng.integers(20, 80)), seed + q) if cond else None))
    return out


def _alloc(r):
    import torch
    nx, ny, nz = r["model"]["n"]
    shape = (r["nreal"], nz, ny, nx)
    f64 = r["cond"] is not None or r["precision"] == ss.FP64
    if r["device"]:
        return torch.full(shape, float("nan"), dtype=torch.float64 if f64 else torch.float32, device="cuda")
    return np.full(shape, np.nan, dtype=np.float64 if f64 else np.float32)


def _alone(r):
    m = r["model"]
    sp = ss.Spectrum(m["structs"], m["nugget"], m["d"], m["n"], m["ipad"])
    out = _alloc(r)
    sp.realize(r["iseed"], r["nreal"], r["igauss"], r["precision"], out=out)
    if r["cond"] is not None:
        c = r["cond"]
        ss.condition(out, c["xmin"], m["d"], m["structs"], m["nugget"], c["params"], c["rows"], r["precision"])
    sp.close()
    return _host(out)


def _host(out):
    if isinstance(out, np.ndarray):
        return out
    import torch
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _run_mix(reqs, **cfg):
    import threading
    import time
    import torch
    srv = ss.Server(**cfg)
    outs = [_alloc(r) for r in reqs]
    torch.cuda.synchronize()        # the NaN fills run on torch's stream, the requests on the slots' streams
    tickets = [None] * len(reqs)

    def feeder():
        for k, (r, o) in enumerate(zip(reqs, outs)):
            tickets[k] = srv.submit(r["model"], r["iseed"], r["nreal"], r["igauss"], r["precision"], out=o,
                                    cond=r["cond"])
            time.sleep(0.002 * (k % 3))

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    return [_host(o) for o in outs], res, st


def test_mix_equals_alone():
    reqs = _requests(24)
    got, res, st = _run_mix(reqs, slots=4)
    assert all(r["status"] == 0 for r in res), [r["message"] for r in res if r["status"]]
    assert st["peak_running"] >= 2
    assert st["cache_hits"] > 0
    for r, g in zip(reqs, got):
        ref = _alone(r)
        assert np.array_equal(g, ref), (r["model"]["n"], r["precision"], r["cond"] is not None)


def test_mix_equals_alone_under_tight_budget():
    """A budget that admits about one request at a time (the largest of these
    needs 27 MB with host output), and a cache smaller than one spectrum: admissions wait and
    spectra are rebuilt, results do not change."""
    reqs = _requests(10, seed=11)
    got, res, st = _run_mix(reqs, slots=3, hbm_budget=3 * (1 << 20) + (48 << 20), cache_budget=1,
                            retain_bytes=1 << 20)
    assert all(r["status"] == 0 for r in res), [r["message"] for r in res if r["status"]]
    assert st["peak_bytes"] <= st["budget_bytes"]
    assert st["evictions"] > 0
    for r, g in zip(reqs, got):
        assert np.array_equal(g, _alone(r))
