"""Scheduler of the serving form, run without a GPU (dry-run mode: the GPU
stages become sleeps proportional to the work; admission, the spectra cache and
the memory accounting are the production code paths).

Checks: the device bytes charged never exceed the budget; slots run requests
at the same time; repeated models hit the cache; a request that can never fit
fails with SS3D_ENOMEM instead of blocking the queue; a large request waiting
at the head is passed at most max_bypass times; a conditional request that
waits at the head only for a conditional slot does not hold back the
unconditional requests behind it.
"""
import numpy as np
import pytest

from specsim3d_b200 import _lib, workloads
import specsim3d_b200 as ss

GB = 1 << 30


def _server(**kw):
    kw.setdefault("slots", 4)
    kw.setdefault("retain_bytes", 1 << 20)
    kw.setdefault("dry_run_ns_per_cell", 0.02)
    return ss.Server(**kw)


def test_budget_cache_and_overlap():
    pool = workloads.model_pool(size=12, lo=16, hi=96)
    reqs = workloads.request_stream(rate=1000.0, count=120, pool_size=12, cond_frac=0.0, max_real=6)
    srv = _server(hbm_budget=2 * GB, cache_budget=GB // 2)
    tickets = [srv.submit(pool[q["model"]], q["iseed"], q["nreal"]) for q in reqs]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert all(r["status"] == 0 for r in res)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_bytes"] <= st["budget_bytes"]
    assert st["peak_running"] >= 2
    assert st["cache_hits"] > 0 and st["cache_hits"] + st["cache_misses"] == len(reqs)
    assert all(r["t_admit"] >= r["t_submit"] and r["t_done"] >= r["t_admit"] for r in res)


def test_tight_budget_serialises_without_deadlock():
    pool = workloads.model_pool(size=4, lo=48, hi=64)
    srv = _server(hbm_budget=120 << 20, cache_budget=0)
    tickets = [srv.submit(pool[k % 4], 11 + k, 2) for k in range(16)]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert all(r["status"] == 0 for r in res), [r["message"] for r in res if r["status"]]
    assert st["peak_bytes"] <= st["budget_bytes"]


def test_request_above_budget_fails_alone():
    big = dict(structs=[(1, 1.0, 50.0, 50.0, 50.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(256, 256, 256), ipad=1)
    small = dict(structs=[(1, 1.0, 5.0, 5.0, 5.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(16, 16, 16), ipad=1)
    srv = _server(hbm_budget=256 << 20)
    t_big = srv.submit(big, 1, 4)
    t_small = [srv.submit(small, 2 + k, 1) for k in range(3)]
    r_big = srv.wait(t_big)
    assert r_big["status"] == _lib.SS3D_ENOMEM and "budget" in r_big["message"]
    assert all(srv.wait(t)["status"] == 0 for t in t_small)
    srv.close()


def test_head_of_queue_is_not_starved():
    big = dict(structs=[(2, 1.0, 30.0, 30.0, 30.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(128, 128, 64), ipad=1)
    small = dict(structs=[(1, 1.0, 5.0, 5.0, 5.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(24, 24, 24), ipad=1)
    srv = _server(slots=2, hbm_budget=1 * GB, max_bypass=3, dry_run_ns_per_cell=1.0)
    # fill the budget with a first big request, then queue a second big one and many small ones
    t0 = srv.submit(big, 1, 16)
    t1 = srv.submit(big, 2, 16)
    ts = [srv.submit(small, 10 + k, 1) for k in range(20)]
    r1 = srv.wait(t1)
    rs = [srv.wait(t) for t in ts]
    srv.wait(t0)
    srv.close()
    passed = sum(1 for r in rs if r["t_admit"] < r1["t_admit"])
    assert r1["status"] == 0
    assert passed <= 3 + 1, passed      # max_bypass, plus one admitted before the head was queued behind memory


def test_invalid_requests_rejected_at_submit():
    srv = _server(hbm_budget=GB)
    good = dict(structs=[(1, 1.0, 5.0, 5.0, 5.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(16, 16, 16), ipad=1)
    with pytest.raises(_lib.SpecsimError):
        srv.submit(good, 1, 0)
    with pytest.raises(_lib.SpecsimError):
        srv.submit(good, 1, 1, igauss=3)
    bad = dict(good, n=(16, 0, 16))
    with pytest.raises(_lib.SpecsimError):
        srv.submit(bad, 1, 1)
    srv.close()


def test_idle_slots_give_back_work_space():
    """Slots keep their work spaces between requests; a large request that only
    fits once they give them back must still run."""
    med = dict(structs=[(1, 1.0, 10.0, 10.0, 10.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(96, 96, 96), ipad=1)
    big = dict(structs=[(1, 1.0, 20.0, 20.0, 20.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(200, 200, 200), ipad=1)
    probe = _server(slots=1, hbm_budget=64 * GB)
    fp_med = probe.wait(probe.submit(med, 1, 16))["footprint"]
    fp_big = probe.wait(probe.submit(big, 1, 16))["footprint"]
    probe.close()
    budget = fp_big + fp_med // 2
    srv = _server(slots=4, hbm_budget=budget, retain_bytes=budget, cache_budget=1)
    ts = [srv.submit(med, 10 + k, 16) for k in range(8)]
    tb = srv.submit(big, 3, 16)
    res = [srv.wait(t) for t in ts] + [srv.wait(tb)]
    st = srv.stats()
    srv.close()
    assert all(r["status"] == 0 for r in res), [r["message"] for r in res if r["status"]]
    assert st["peak_bytes"] <= st["budget_bytes"]


def test_head_waiting_for_a_conditional_slot_does_not_block():
    """max_cond 1: while one long conditional request runs, a second one waits
    at the head of the queue for the conditional slot.  The unconditional
    requests behind it take no such slot and must all be admitted while the
    first one runs, not only max_bypass of them."""
    big = dict(structs=[(2, 1.0, 30.0, 30.0, 30.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(128, 128, 64), ipad=1)
    small = dict(structs=[(1, 1.0, 5.0, 5.0, 5.0, 0.0, 0.0, 0.0)], nugget=0.0, d=(1, 1, 1), n=(16, 16, 16), ipad=1)
    params = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=0, skmean=0.0, zmin=0.0, zmax=1.0,
                  ltail=1, ltpar=0.0, utail=1, utpar=0.0, radius=(10.0, 10.0, 10.0), angles=(0.0, 0.0, 0.0), ndmax=8)
    cond = dict(params=params, rows=np.array([[1.0, 2.0, 3.0, 0.5], [5.0, 6.0, 7.0, -0.5]]), xmin=(0.0, 0.0, 0.0))
    srv = _server(slots=4, hbm_budget=4 * GB, max_bypass=2, max_cond=1, dry_run_ns_per_cell=2.0)
    t_a = srv.submit(big, 1, 16, cond=cond)
    t_b = srv.submit(big, 2, 16, cond=cond)
    ts = [srv.submit(small, 10 + k, 1) for k in range(12)]
    rs = [srv.wait(t) for t in ts]
    r_a = srv.wait(t_a)
    r_b = srv.wait(t_b)
    srv.close()
    assert r_a["status"] == 0 and r_b["status"] == 0 and all(r["status"] == 0 for r in rs)
    assert r_b["t_admit"] >= r_a["t_done"]                       # one conditional slot
    assert all(r["t_done"] <= r_a["t_done"] for r in rs), [round(r["t_admit"] - r_a["t_admit"], 4) for r in rs]
