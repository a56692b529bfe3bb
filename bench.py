#!/usr/bin/env python3
"""bench.py -- throughput of the SPECSIM3D spectral simulation path on B200.

Workload (the precision configuration, one GPU): unconditional 256x256x256 grid,
cell size 1, gaussian model sill 1.0 nugget 0.1 ranges 60/30/15 azimuth 30 dip 20
plunge 10, ipad 1 (periodic grid 512^3), igauss 1, seed 12345, 8 realizations per
GPU.  The FP64 spectrum is built once and stays resident; a step is one batch of
8 realizations synthesised, inverse-transformed and cropped into a device
float32 buffer in the FP32 precision form, issued as one CUDA-graph launch of
the batched form.  Next to it: the same step through the per-call entry point
in FP32 and in the plain FP64 form, the FP32-vs-FP64 error, an end-to-end run
through the C ABI into pinned host memory, and the mixed-grid batched workload
(1,024 realizations over 16 grid shapes in one graph launch).

Multi-GPU: one process per GPU (torchrun); rank g takes realizations
8g .. 8g+7 of the same stream (exact jump-ahead sharding, no collective in the
data path), time = max over ranks.

`--impl reference` times the reference algorithm on the host cores instead: the
CPU oracle (a C restatement of the Fortran, built with OpenMP), one realization
of the same workload per step, rank 0 only.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcells/s at 256³ FP32 vs plain FP64 (same GPU, stated err); serving p50/p99 ms"
WL = dict(n=(256, 256, 256), structs=[(3, 1.0, 60.0, 30.0, 15.0, 30.0, 20.0, 10.0)], nugget=0.1, d=(1.0, 1.0, 1.0),
          ipad=1, igauss=1, seed=12345, nreal=8)
WORKLOAD_NAME = ("unconditional 256^3 gaussian sill 1 nugget 0.1 ranges 60/30/15 az 30 dip 20 plunge 10, "
                 "ipad 1 (periodic 512^3), igauss 1, seed 12345, 8 realizations per GPU")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the mixed-grid batched workload")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving workload")
    ap.add_argument("--profile-case", nargs="?", const="realize", default=None,
                    choices=["realize", "cond", "vario", "spectrum"],
                    help="profiling case, no timing: realize (the bench grid, 1 realization, three FP32 calls), "
                         "cond (the conditional workload, one FP64 and one FP32 conditioning call), vario (one FP64 "
                         "256^3 realization, directions x, y, z, lags 1..100), spectrum (one 512^3 spectrum build)")
    ap.add_argument("--tile-variant", action="append", default=[], metavar="PASS=V",
                    help="realize profiling case: after the autotuner, run pass PASS (middle, synthesis, rows) of "
                         "the bench grid with FP32 tile variant V instead (may be repeated)")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers
def cells_per_real():
    n = WL["n"]
    return n[0] * n[1] * n[2]


def half_spectrum_size(np3):
    npx, npy, npz = np3
    return (npx // 2 + 1) * npy * npz


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = os.path.join("/tmp", f"ss3d_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.remove(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def oracle_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ora
    return ora


def cpu_reference_sample(k_steps, warmup, budget_s=None):
    """Oracle (C restatement, OpenMP) on the host cores: seconds per realization
    of the workload.  With budget_s the timed steps stop once that many seconds
    have passed (at least one step).  Returns (seconds per step, spectrum
    seconds, threads, steps timed)."""
    ora = oracle_lib()
    np3, rc = ora.grid(WL["structs"], WL["d"], WL["n"], WL["ipad"])
    t0 = time.perf_counter()
    amp, _ = ora.spectrum(WL["structs"], WL["nugget"], WL["d"], np3)
    t_spec = time.perf_counter() - t0
    for _ in range(warmup):
        ora.realize(amp, np3, WL["n"], WL["seed"], 1, WL["igauss"])
    times = []
    start = time.perf_counter()
    for _ in range(k_steps):
        t0 = time.perf_counter()
        ora.realize(amp, np3, WL["n"], WL["seed"], 1, WL["igauss"])
        times.append(time.perf_counter() - t0)
        if budget_s is not None and time.perf_counter() - start > budget_s:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return float(np.mean(times)), t_spec, cores, len(times)


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference algorithm on the host cores (the oracle: a C restatement of
    the Fortran path, OpenMP on every host thread; no Fortran compiler exists on
    these machines).  One step = one realization of the 256^3 workload (about
    4 s), so the timed steps are a bounded sample: they stop after 150 s, and
    at most 2 warm-up steps run.  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    k = max(1, args.steps)
    w = min(2, max(0, args.warmup))
    sec, t_spec, cores, done = cpu_reference_sample(k, w, budget_s=150.0)
    value = cells_per_real() / sec / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mcells/s", "n_gpus": args.gpus,
        "steps": done, "steps_requested": k, "warmup": w, "ms_per_step": round(sec * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "sample": f"1 realization per step, {done} steps timed (150 s cap), "
                   "spectrum excluded", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mcells/s", "cores": cores, "kind": "port",
                         "sample": "1 realization of the 256^3 workload per step (C restatement of the Fortran, "
                                   f"OpenMP, {cores} threads); spectrum build {t_spec:.2f} s not counted"},
        "e2e": {"value": round(value, 3), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- our arm
def _ev_ms(stream, fn, k, w):
    """Mean device time (ms) of fn over k calls after w warm-up calls (CUDA events)."""
    import torch
    for _ in range(w):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / k


def bench_mixed_grids(ss, stream, seed=777):
    """Batched form on the mixed-grid workload: 1,024 realizations over 16 grid
    shapes in one graph launch, against the per-call FP32 and FP64 paths on the
    same jobs, with the FP32-vs-FP64 error."""
    import torch
    from specsim3d_b200 import workloads
    specs = workloads.mixed_grids(seed=seed)
    jobs, sps = [], []
    for c in specs:
        sp = ss.Spectrum(c["structs"], c["nugget"], c["d"], c["n"], c["ipad"])
        nx, ny, nz = c["n"]
        out = torch.empty((c["nreal"], nz, ny, nx), dtype=torch.float32, device="cuda")
        jobs.append((sp, c["iseed"], c["igauss"], 0, c["nreal"], out))
    cells = sum(j[4] * int(np.prod(j[0].n)) for j in jobs)
    b = ss.Batch(jobs, autotune=True)
    ms_b = _ev_ms(stream, b.run, 5, 2)
    def per_call(prec, outs):
        def f():
            for (sp, iseed, ig, r0, nr, _), o in zip(jobs, outs):
                sp.realize(iseed, nr, ig, prec, out=o)
        return f
    ms_32 = _ev_ms(stream, per_call(ss.FP32, [j[5] for j in jobs]), 3, 1)
    err_max, err_rms_num, err_den = 0.0, 0.0, 0
    ms_64 = 0.0
    for (sp, iseed, ig, r0, nr, o) in jobs:          # FP64 per job (memory bounded), error on the way
        o64 = torch.empty(o.shape, dtype=torch.float64, device="cuda")
        ms_64 += _ev_ms(stream, lambda: sp.realize(iseed, nr, ig, ss.FP64, out=o64), 2, 1)
        b_out = o.double()
        d = (b_out - o64).abs_() / np.sqrt(sp.stats["c0"])
        err_max = max(err_max, float(d.amax().item()))
        err_rms_num += float(d.pow_(2).sum().item())
        err_den += d.numel()
        del o64, b_out, d
    b.run()
    info, sched = b.info(), b.schedule()
    b.close()
    for sp in [j[0] for j in jobs]:
        sp.close()
    return {
        "workload": "1,024 unconditional realizations over 16 grid shapes, nx/ny/nz log-uniform 32..256 (every 4th "
                    "shape 2D), model cycling sph/exp/gauss, ranges U(5, 0.4 extent), azimuth U(0,180), dip "
                    "U(-30,30), nugget U(0,0.3), ipad 1, igauss 1, seed 777",
        "cells": cells, "graph_ms": round(ms_b, 3), "value": round(cells / (ms_b * 1e-3) / 1e6, 1),
        "unit": "Mcells/s", "per_call_fp32": round(cells / (ms_32 * 1e-3) / 1e6, 1),
        "per_call_fp64": round(cells / (ms_64 * 1e-3) / 1e6, 1), "batched_fp32_over_fp64": round(ms_64 / ms_b, 3),
        "error_vs_fp64": {"max_abs_over_sqrt_c0": err_max, "rms_over_sqrt_c0": float(np.sqrt(err_rms_num / err_den))},
        "schedule": sched["schedule"], "kernels_per_launch": info["kernels"],
    }


def _serving_cond(model, ndata, seed):
    """Conditioning data of a serving request: ndata points at uniform-random
    locations with skewed values exp(0.5 g), g standard normal (the conditional
    recipe's value transform, without its truth field); normal-score transform,
    linear tails, search ellipsoid = the model's ranges and angles, ndmax 24."""
    rng = np.random.default_rng(seed)
    n = model["n"]
    xyz = np.stack([rng.uniform(0, n[a] - 1, ndata) for a in range(3)], axis=1)
    val = np.exp(0.5 * rng.standard_normal(ndata))
    st = model["structs"][0]
    params = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=1, skmean=0.0, zmin=0.0,
                  zmax=2.0 * float(val.max()), ltail=1, ltpar=0.0, utail=1, utpar=0.0,
                  radius=(st[2], st[3], st[4]), angles=(st[5], st[6], st[7]), ndmax=24)
    return dict(params=params, rows=np.column_stack([xyz, val]), xmin=(0.0, 0.0, 0.0))


SERVING_RATES = (50.0, 100.0, 200.0, 500.0, 1000.0, 2000.0)


def _pcts(lat_ms):
    if len(lat_ms) == 0:
        return {"n": 0}
    a = np.asarray(lat_ms)
    return {"n": int(a.size), "p50_ms": round(float(np.percentile(a, 50)), 3),
            "p99_ms": round(float(np.percentile(a, 99)), 3)}


def bench_serving(ss, rates=SERVING_RATES, count=4000, slots=8, budget=64 << 30, premap=40 << 30,
                  arena_bytes=40 << 30):
    """Serving form on the stated configuration: a Poisson request stream of
    `count` requests (seed 2024) at each rate over a pool of 64 models (seed
    2025): grids log-uniform 32..256 per axis, nreal 1..16, 20 % conditional
    with 200..2000 data, precision form throughout (FP32 synthesis and
    transforms; conditional fields are float64 and their kriging solves FP32
    with one FP64 residual refinement).  Open loop: a feeder submits each
    request at its arrival time; latency = completion - arrival, reported for
    all requests and per class (unconditional / conditional).  Beside it the
    plain path, one request at a time with no spectra cache: its service times
    are measured, and its latency at each rate is the FIFO single-server
    recursion on those times.

    Outputs: the 4,000 requests' fields would take about 200 GB, so each
    request writes into a slice of one preallocated device arena taken in
    arrival order as a ring (`arena_bytes`).  Two requests share bytes only when
    about a thousand requests lie between them in the queue, while the
    admission order keeps running requests within slots + max_bypass queue
    positions of each other; the bench does not read the fields."""
    import threading
    import torch
    from specsim3d_b200 import workloads
    pool = workloads.model_pool()
    out = {"workload": f"{count} requests per rate, Poisson arrivals (seed 2024), pool of 64 models (seed 2025), "
                       "grids log-uniform 32..256 per axis, nreal U{1..16}, 20 % conditional (200..2000 points); "
                       "unmeasured closed-loop and open-loop passes first; outputs in a ring arena",
           "slots": slots, "hbm_budget_gb": budget / 2 ** 30, "premap_gb": premap / 2 ** 30,
           "arena_gb": arena_bytes / 2 ** 30, "rates": {}}
    base_reqs = workloads.request_stream(1.0, count=count)
    arena = torch.empty(arena_bytes, dtype=torch.uint8, device="cuda")
    outs, off = [], 0
    for q in base_reqs:
        m = pool[q["model"]]
        nx, ny, nz = m["n"]
        dt = torch.float64 if q["ndata"] else torch.float32
        nb = q["nreal"] * nx * ny * nz * (8 if q["ndata"] else 4)
        if off + nb > arena_bytes:
            off = 0
        outs.append(arena[off:off + nb].view(dt).view(q["nreal"], nz, ny, nx))
        off = (off + nb + 255) // 256 * 256
    conds = [_serving_cond(pool[q["model"]], q["ndata"], 5000 + k) if q["ndata"] else None
             for k, q in enumerate(base_reqs)]
    cells_of = [q["nreal"] * int(np.prod(pool[q["model"]]["n"])) for q in base_reqs]
    is_cond = np.array([q["ndata"] > 0 for q in base_reqs])
    prec = ss.FP32
    # warm-up (not measured): a closed-loop pass over the first requests maps
    # the device memory the slots and spectra use; every measured rate then
    # starts from an empty spectra cache on a new server
    srv = ss.Server(slots=slots, hbm_budget=budget, premap_bytes=premap)
    nw = min(count, 1000)
    ts = [srv.submit(pool[q["model"]], q["iseed"], q["nreal"], 1, prec, out=outs[k], cond=conds[k])
          for k, q in enumerate(base_reqs[:nw])]
    for t in ts:
        srv.wait(t)
    srv.close()

    def open_loop(rate):
        import gc
        reqs = workloads.request_stream(rate, count=count)
        srv = ss.Server(slots=slots, hbm_budget=budget, premap_bytes=premap)
        tickets = [None] * count
        lag = np.zeros(count)   # submission time - scheduled arrival (the harness's own delay)
        # no garbage collection of the harness while it feeds requests: a
        # collection pause would delay submissions and count as latency
        gc.collect()
        gc.freeze()
        gc.disable()
        t_start = srv.clock() + 0.05

        def feeder():
            for k, q in enumerate(reqs):
                t_arr = t_start + q["t_arrival"]
                dt = t_arr - srv.clock()
                if dt > 0:
                    time.sleep(dt)
                tickets[k] = srv.submit(pool[q["model"]], q["iseed"], q["nreal"], 1, prec, out=outs[k],
                                        t_arrival=t_arr, cond=conds[k])
                lag[k] = srv.clock() - t_arr

        th = threading.Thread(target=feeder)
        th.start()
        res = []
        for k in range(count):
            while tickets[k] is None:
                time.sleep(0.0005)
            res.append(srv.wait(tickets[k]))
        th.join()
        gc.enable()
        gc.unfreeze()
        st = srv.stats()
        srv.close()
        return res, st, t_start, lag

    # one unmeasured open-loop pass at the highest rate maps the pages of an
    # open-loop run's peak footprint before any timing
    def pool_reserved_gb():
        # reserved bytes of the device's stream-ordered pool (high-water mark
        # and current): growth while requests run maps new pages under all of them
        try:
            from cuda.bindings import runtime as rt
            dev = torch.cuda.current_device()
            _, pool_h = rt.cudaDeviceGetDefaultMemPool(dev)
            _, hi = rt.cudaMemPoolGetAttribute(pool_h, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemHigh)
            _, cur = rt.cudaMemPoolGetAttribute(pool_h, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
            return round(int(hi) / 2 ** 30, 2), round(int(cur) / 2 ** 30, 2)
        except Exception:
            return None, None

    open_loop(max(rates))
    torch.cuda.synchronize()
    for rate in rates:
        pool_before = pool_reserved_gb()
        res, st, t_start, lag = open_loop(rate)
        pool_after = pool_reserved_gb()
        ok = np.array([r["status"] == 0 for r in res])
        lat = np.array([r["t_done"] - r["t_arrival"] for r in res]) * 1e3
        span = max(r["t_done"] for r in res) - t_start
        cells = sum(c for c, r in zip(cells_of, res) if r["status"] == 0)
        out["rates"][str(int(rate))] = {
            **_pcts(lat[ok]), "mcells_s": round(cells / span / 1e6, 1), "completed": int(ok.sum()),
            "failed": int((~ok).sum()), "unconditional": _pcts(lat[ok & ~is_cond]),
            "conditional": _pcts(lat[ok & is_cond]), "cache_hits": st["cache_hits"],
            "cache_misses": st["cache_misses"], "peak_running": st["peak_running"],
            "peak_gb": round(st["peak_bytes"] / 2 ** 30, 2),
            "submit_lag_ms": {"p99": round(1e3 * float(np.percentile(lag, 99)), 3),
                              "max": round(1e3 * float(lag.max()), 3)},
            "pool_reserved_gb": {"high_before": pool_before[0], "high_after": pool_after[0],
                                 "current_after": pool_after[1]}}
    # plain path: one request at a time, no cache
    svc = []
    for k, q in enumerate(base_reqs):
        m = pool[q["model"]]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o = outs[k]
        sp = ss.Spectrum(m["structs"], m["nugget"], m["d"], m["n"], m["ipad"])
        sp.realize(q["iseed"], q["nreal"], 1, prec, out=o)
        if conds[k] is not None:
            c = conds[k]
            ss.condition(o, c["xmin"], m["d"], m["structs"], m["nugget"], c["params"], c["rows"], prec)
        sp.close()
        torch.cuda.synchronize()
        svc.append(time.perf_counter() - t0)
    svc = np.array(svc)
    tot_cells = sum(cells_of)
    plain = {"mcells_s": round(tot_cells / svc.sum() / 1e6, 1), "mean_service_ms": round(1e3 * float(svc.mean()), 3),
             "service_share_conditional": round(float(svc[is_cond].sum() / svc.sum()), 3), "rates": {}}
    for rate in rates:
        reqs = workloads.request_stream(rate, count=count)
        done, lat = 0.0, []
        for q, sv in zip(reqs, svc):
            done = max(done, q["t_arrival"]) + sv
            lat.append(done - q["t_arrival"])
        lat = np.array(lat) * 1e3
        plain["rates"][str(int(rate))] = {**_pcts(lat), "unconditional": _pcts(lat[~is_cond]),
                                         "conditional": _pcts(lat[is_cond])}
    out["one_at_a_time"] = plain
    del outs, arena
    return out


def bench_conditional(ss, stream, cpu=True):
    """Conditional configuration: 128x128x64, exponential sill 1 nugget 0.05
    ranges 40/20/8 azimuth 60; truth = realization of seed 4242 (igauss 0); 2,000
    data at uniform-random locations (seed 99) with values exp(0.5 z) of the
    truth, normal-score transform and back transform (zmax = 2 max, linear
    tails); search = the ranges, ndmax 24; 16 realizations of seed 4243.  FP64
    kriging against FP32 solves with one FP64-residual refinement: time per call
    (realizations excluded) and the difference of the conditioned fields
    relative to their standard deviation."""
    import torch
    n = (128, 128, 64)
    structs = [(2, 1.0, 40.0, 20.0, 8.0, 60.0, 0.0, 0.0)]
    sp = ss.Spectrum(structs, 0.05, (1.0, 1.0, 1.0), n, 1)
    truth = sp.realize(4242, 1, 0, ss.FP64)[0]
    rng = np.random.default_rng(99)
    xyz = np.stack([rng.uniform(0, n[a] - 1, 2000) for a in range(3)], axis=1)
    ix = np.rint(xyz).astype(int)
    val = np.exp(0.5 * truth[ix[:, 2], ix[:, 1], ix[:, 0]])
    rows = np.column_stack([xyz, val])
    params = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=1, skmean=0.0, zmin=0.0,
                  zmax=2.0 * float(val.max()), ltail=1, ltpar=0.0, utail=1, utpar=0.0, radius=(40.0, 20.0, 8.0),
                  angles=(60.0, 0.0, 0.0), ndmax=24)
    fields = {}
    times = {}
    for name, prec in (("fp64", ss.FP64), ("fp32", ss.FP32)):
        f = torch.empty((16, n[2], n[1], n[0]), dtype=torch.float64, device="cuda")
        ts = []
        for rep in range(3):
            sp.realize(4243, 16, 0, ss.FP64, out=f)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st, _ = ss.condition(f, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), structs, 0.05, params, rows, prec)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        times[name] = min(ts)
        fields[name] = f
    d = (fields["fp32"] - fields["fp64"]).abs_()
    sd = float(fields["fp64"].std().item())
    M = n[0] * n[1] * n[2]
    out = {"workload": "128x128x64, exponential 40/20/8 az 60, nugget 0.05, 2,000 data (seed 99) from the seed-4242 "
                       "truth through exp(0.5 z), nscore + backtr, ndmax 24, 16 realizations (seed 4243)",
           "fp64_ms": round(times["fp64"] * 1e3, 3), "fp32_ms": round(times["fp32"] * 1e3, 3),
           "mcells_s_fp32": round(M * 16 / times["fp32"] / 1e6, 1),
           "neighbours_total": st["nsum"], "regularised_systems": st["nfail"],
           "fp32_vs_fp64": {"max_abs_over_sd": float(d.amax().item()) / sd,
                            "rms_over_sd": float(d.pow_(2).mean().sqrt().item()) / sd, "target": 1e-5}}
    if cpu:
        # the same conditioning through the oracle (C restatement of the Fortran,
        # OpenMP) on the host cores, on the same unconditioned fields
        ora = oracle_lib()
        host = sp.realize(4243, 16, 0, ss.FP64)
        op = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=1, skmean=0.0, zlo=0.0,
                  zhi=params["zmax"], ltail=1, ltpar=0.0, utail=1, utpar=0.0, rmax=40.0, rmed=20.0, rvert=8.0,
                  sa1=60.0, sa2=0.0, sa3=0.0, ndmax=24)
        t0 = time.perf_counter()
        ost, _ = ora.condition(host, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), structs, 0.05, op, rows)
        tc = time.perf_counter() - t0
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        out["cpu_baseline"] = {"ms": round(tc * 1e3, 1), "mcells_s": round(M * 16 / tc / 1e6, 1), "cores": cores,
                               "kind": "port", "neighbours_total": ost["nsum"],
                               "sample": "one conditioning call of the same workload (C restatement of the Fortran, "
                                         f"OpenMP {cores} threads)",
                               "gpu_fp64_speedup": round(tc / times["fp64"], 1)}
    sp.close()
    return out


def bench_vario(ss, sp, nreal, seed, igauss, cpu=True):
    """--vario on the precision configuration: directions (1,0,0), (0,1,0),
    (0,0,1), lags 1..100, FP64 sums over all node pairs of the FP64
    realizations; exact pair counts."""
    import torch
    n = sp.n
    f = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float64, device="cuda")
    sp.realize(seed, nreal, igauss, ss.FP64, out=f)
    dirs = [(1, 0, 0, 100), (0, 1, 0, 100), (0, 0, 1, 100)]
    ts = []
    for rep in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gam, npairs = ss.vario(f, dirs)
        ts.append(time.perf_counter() - t0)
    pairs = int(npairs.sum()) * nreal
    t = min(ts)
    # the sample variogram against the model, gamma(h) = C(0) - C(h), ensemble mean over the realizations
    c0 = ss.covariance(WL["structs"], WL["nugget"], 0.0, 0.0, 0.0)
    rms = []
    for di, (sx, sy, sz, nl) in enumerate(dirs):
        model = np.array([c0 - ss.covariance(WL["structs"], WL["nugget"], l * sx, l * sy, l * sz) for l in range(1, nl + 1)])
        rms.append(float(np.sqrt(np.mean((gam[:, di, :nl].mean(axis=0) - model) ** 2)) / c0))
    out = {"workload": "256^3, 8 FP64 realizations, directions x, y, z, lags 1..100", "ms": round(t * 1e3, 3),
           "pairs": pairs, "gpairs_s": round(pairs / t / 1e9, 2), "fp64_gflop_s": round(3 * pairs / t / 1e9, 1),
           "pair_count_check": int(npairs[0, 0]) == (n[0] - 1) * n[1] * n[2],
           "sample_vs_model_rms_over_sill": [round(x, 4) for x in rms]}
    if cpu:
        # the oracle's all-pairs loops (f90:405-431, OpenMP over directions and
        # lags) on one of the realizations, on the host cores
        ora = oracle_lib()
        h = f[:1].cpu().numpy()
        t0 = time.perf_counter()
        ora.vario(h, dirs)
        tc = time.perf_counter() - t0
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        out["cpu_baseline"] = {"ms_per_realization": round(tc * 1e3, 1), "gpairs_s": round(pairs / nreal / tc / 1e9, 3),
                               "cores": cores, "kind": "port",
                               "sample": f"1 realization of the same workload (C restatement, OpenMP {cores} threads)",
                               "gpu_speedup": round(tc * nreal / t, 1)}
    return out


def bench_cfg1(ss, stream, k=200, cpu=True):
    """Plain method, small: 64x64x16, spherical 20/10/5 N45E, ipad 1, igauss 0,
    seed 69069, FP64 throughout; one realization per call into device memory
    (spectrum built once), and the oracle's spectrum + realization on the host."""
    import torch
    n = (64, 64, 16)
    st = [(1, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sp = ss.Spectrum(st, 0.0, (1.0, 1.0, 1.0), n, 1)
    t_spec = time.perf_counter() - t0
    o = torch.empty((1, n[2], n[1], n[0]), dtype=torch.float64, device="cuda")
    ms = _ev_ms(stream, lambda: sp.realize(69069, 1, 0, ss.FP64, out=o), k, 10)
    M = n[0] * n[1] * n[2]
    out = {"workload": "64x64x16 spherical 20/10/5 az 45, ipad 1 (periodic 128x128x32), igauss 0, seed 69069, FP64",
           "ms_per_realization": round(ms, 4), "mcells_s": round(M / (ms * 1e-3) / 1e6, 1),
           "spectrum_ms_wall": round(t_spec * 1e3, 3)}
    if cpu:
        ora = oracle_lib()
        np3, _ = ora.grid(st, (1.0, 1.0, 1.0), n, 1)
        t0 = time.perf_counter()
        amp, _ = ora.spectrum(st, 0.0, (1.0, 1.0, 1.0), np3)
        t1 = time.perf_counter()
        reps = 5
        for _ in range(reps):
            ora.realize(amp, np3, n, 69069, 1, 0)
        t2 = time.perf_counter()
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        out["cpu_baseline"] = {"ms_per_realization": round((t2 - t1) / reps * 1e3, 2),
                               "spectrum_ms": round((t1 - t0) * 1e3, 2), "cores": cores, "kind": "port"}
    sp.close()
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    import specsim3d_b200 as ss

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    ss.set_stream(stream)
    n = WL["n"]
    nreal = WL["nreal"]
    M = cells_per_real()
    r_first, _ = ss.shard(rank, world, nreal)
    sp = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
    c0 = sp.stats["c0"]
    out32 = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float32, device=dev)
    out64 = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float64, device=dev)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    def timed(fn, k, w, nvtx=None):
        """k steps of fn after w warm-up steps; barrier + synchronize on both
        sides; ms per step (max over ranks) and library launches in the region."""
        for _ in range(w):
            fn()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        _, l0 = ss.profile_read()
        if nvtx:
            torch.cuda.nvtx.range_push(nvtx)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        if nvtx:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        _, l1 = ss.profile_read()
        barrier()
        ms = e0.elapsed_time(e1) / k
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, l1 - l0

    # tile variants of the per-call kernels and the batch schedule, picked by
    # the autotuners (untimed, once per process)
    tuned = {"fp32": ss.autotune(sp, WL["igauss"], ss.FP32, nreal), "fp64": ss.autotune(sp, WL["igauss"], ss.FP64, nreal)}
    batch = ss.Batch([(sp, WL["seed"], WL["igauss"], r_first, nreal, out32)], autotune=True)
    k, w = max(1, args.steps), max(3, args.warmup)
    # headline: the batched form (one CUDA-graph launch per step of 8 realizations)
    clk = ClockSampler(local)
    clk.start()
    ms32, launches = timed(batch.run, k, w, nvtx="timed_fp32")
    clocks = clk.stop()
    ms32_call, _ = timed(lambda: sp.realize(WL["seed"], nreal, WL["igauss"], ss.FP32, r_first=r_first, out=out32),
                         max(1, k // 4), 3)
    ms64, _ = timed(lambda: sp.realize(WL["seed"], nreal, WL["igauss"], ss.FP64, r_first=r_first, out=out64),
                    max(1, k // 4), 3)
    # per-kernel durations for the roofline: a separate per-call pass with stage
    # events (stages then run back to back instead of overlapping)
    ss.profile(True)
    kprof = max(1, min(k, 10))
    for _ in range(kprof):
        sp.realize(WL["seed"], nreal, WL["igauss"], ss.FP32, r_first=r_first, out=out32)
    torch.cuda.synchronize()
    stages, _ = ss.profile_read()
    ss.profile(False)
    # precision-form error against the FP64 path on the same realizations
    batch.run()
    sp.realize(WL["seed"], nreal, WL["igauss"], ss.FP64, r_first=r_first, out=out64)
    torch.cuda.synchronize()
    diff = (out32.double() - out64).abs_()
    err_max = float(diff.amax().item()) / np.sqrt(c0)
    err_rms = float(diff.pow_(2).mean().sqrt().item()) / np.sqrt(c0)
    del diff
    batch_sched = batch.schedule()
    batch.close()
    # end to end through the C ABI: spectrum build + realizations into pinned host memory
    host = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float32).pin_memory()
    hn = host.numpy()
    ke = max(1, min(k, 5))
    ts, parts = [], []
    for s in range(ke + 1):
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        spe = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
        t1 = time.perf_counter()
        spe.realize(WL["seed"], nreal, WL["igauss"], ss.FP32, r_first=r_first, out=hn)
        t2 = time.perf_counter()
        spe.close()
        t3 = time.perf_counter()
        if s > 0:
            ts.append(t3 - t0)
            parts.append((t1 - t0, t2 - t1, t3 - t2))
    e2e_s = float(np.mean(ts))
    e2e_parts = np.mean(np.array(parts), axis=0) * 1e3
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    # roofline of the dominant kernel: synthesis fused with the first (z) inverse
    # pass; algorithmic bytes per launch = FP32 amplitude read once + the pruned
    # complex z-pass output of every realization
    np3 = sp.np
    nh = half_spectrum_size(np3)
    rho_z = n[2] / np3[2]
    bytes_gen = nh * 4 + nh * 8 * rho_z * nreal
    st_ms, st_launch = stages["synthesis+first_pass"]
    per_launch_ms = st_ms / max(1, st_launch)
    achieved = bytes_gen / (per_launch_ms * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = tr.get("k_colgen_fp32_256cubed_8real_per_launch_bytes")
    except Exception:
        pass
    # whole-step roofline (all kernels of the realization path, FP32 form):
    # amplitude once, z-pass output, y-pass read + pruned write, x-pass read, float output
    rho_y = n[1] / np3[1]
    b_step = nh * 4 + nreal * (nh * 8 * (rho_z + rho_z + rho_z * rho_y + rho_z * rho_y) + 4 * M)
    b_blue = nh * (4 + 8 * (1 + rho_z + 2 * rho_z * rho_y)) + 4 * M
    value = M * nreal * world / (ms32 * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mcells/s", "n_gpus": world, "steps": k, "warmup": w,
        "ms_per_step": round(ms32, 4), "realizations_per_s": round(nreal * world / (ms32 * 1e-3), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "global_batch": nreal * world,
                   "precision": "FP32 synthesis and FFTs on the FP64 spectrum",
                   "form": "batched: one CUDA-graph launch of 8 realizations per step",
                   "parallelism": f"realizations sharded over {world} GPU(s)",
                   "l2": "inputs larger than L2 (FP32 amplitude 269 MB, complex work 2.2 GB)",
                   "tile_variants": tuned, "batch_schedule": batch_sched},
        "per_call_fp32": {"value": round(M * nreal * world / (ms32_call * 1e-3) / 1e6, 1), "unit": "Mcells/s",
                          "ms_per_step": round(ms32_call, 4)},
        "fp64": {"value": round(M * nreal * world / (ms64 * 1e-3) / 1e6, 1), "unit": "Mcells/s",
                 "ms_per_step": round(ms64, 4)},
        "fp32_over_fp64": round(ms64 / ms32, 3),
        "error_vs_fp64": {"max_abs_over_sqrt_c0": err_max, "rms_over_sqrt_c0": err_rms, "target": 1e-5},
        "clocks": clocks,
        "e2e": {"value": round(M * nreal * world / e2e_s / 1e6, 1), "unit": "Mcells/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(M * nreal * 4),
                "includes": "spectrum build + realizations + D2H into pinned host memory (ss3d_realize)",
                "ms_spectrum_realize_free": [round(float(x), 3) for x in e2e_parts]},
        "gpu_launches": int(launches),
        "stages_ms_per_step_serialized": {kk: round(v[0] / kprof, 4) for kk, v in stages.items()},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "kernel": "k_colgen<float,9> (synthesis + z inverse pass), per launch of 8 realizations",
                     "note": "instruction-issue bound (see profiles/), so the HBM fraction is low",
                     "peak_source": "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks
                     else "of fallback 6650"},
        "roofline_step": {"algorithmic_bytes_per_step": int(b_step),
                          "achieved_gbs": round(b_step / (ms32 * 1e-3) / 1e9, 1),
                          "frac": round(b_step / (ms32 * 1e-3) / 1e9 / peak, 4),
                          "note": "bytes the fused path must move: amplitude once per step, no coefficient grid"},
        # the per-realization figure of the design blueprint, for a pruned Hermitian
        # one-pass-per-axis inverse with the coefficients read by the z pass:
        # B = N_h [s_a + s_c (1 + rz + 2 rz ry)] + 4 M, FP32 s_a = 4, s_c = 8
        "roofline_blueprint": {"bytes_per_realization": int(b_blue),
                               "achieved_gbs": round(b_blue * nreal / (ms32 * 1e-3) / 1e9, 1),
                               "frac": round(b_blue * nreal / (ms32 * 1e-3) / 1e9 / peak, 4),
                               "mcells_s_at_60pct": round(0.6 * peak * 1e9 / b_blue * M / 1e6, 1)},
    }
    if world == 1 and not args.no_batch:
        line["mixed_grids"] = bench_mixed_grids(ss, stream)
    if world == 1 and not args.no_serving:
        line["serving"] = bench_serving(ss)
    if world == 1 and not args.no_batch:
        cpu = not args.no_cpu_baseline
        line["conditional"] = bench_conditional(ss, stream, cpu=cpu)
        line["vario"] = bench_vario(ss, sp, nreal, WL["seed"], WL["igauss"], cpu=cpu)
        line["cfg1"] = bench_cfg1(ss, stream, cpu=cpu)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sec, t_spec, cores, _ = cpu_reference_sample(1, 0)
            line["cpu_baseline"] = {"value": round(M / sec / 1e6, 3), "unit": "Mcells/s", "cores": cores,
                                    "kind": "port",
                                    "sample": "1 realization of the same workload on the host (C restatement of the "
                                              f"Fortran, OpenMP {cores} threads), spectrum ({t_spec:.1f} s) excluded"}
        except Exception as ex:
            line["cpu_baseline"] = {"value": None, "unit": "Mcells/s", "cores": 0, "kind": "port",
                                    "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sp.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_profile_case(kind="realize", variants=()):
    """Small cases for ncu.  realize: the bench grid with one realization per
    call (about 1.5 GB on the device), tile variants autotuned as in the bench,
    then three FP32 calls into a device buffer inside the NVTX range "profile".
    cond: the conditional workload (128x128x64, 2,000 data, 16 realizations,
    about 0.2 GB), one FP64 then one FP32 conditioning call.  vario: one FP64
    realization of the bench grid (134 MB) and its variograms along x, y, z,
    lags 1..100.  spectrum: one spectrum build of the bench model (512^3
    periodic grid, about 3 GB of temporaries).  variants: (pass, variant)
    pairs set after the autotuner in the realize case (the other tile variants
    of a pass give the same bits; this profiles one of them)."""
    import torch
    import specsim3d_b200 as ss
    n = WL["n"]
    if kind == "cond":
        nc = (128, 128, 64)
        structs = [(2, 1.0, 40.0, 20.0, 8.0, 60.0, 0.0, 0.0)]
        sp = ss.Spectrum(structs, 0.05, (1.0, 1.0, 1.0), nc, 1)
        truth = sp.realize(4242, 1, 0, ss.FP64)[0]
        rng = np.random.default_rng(99)
        xyz = np.stack([rng.uniform(0, nc[a] - 1, 2000) for a in range(3)], axis=1)
        ix = np.rint(xyz).astype(int)
        val = np.exp(0.5 * truth[ix[:, 2], ix[:, 1], ix[:, 0]])
        params = dict(ixc=1, iyc=2, izc=3, ivc=4, iwc=0, tmin=-1e21, tmax=1e21, itrans=1, skmean=0.0, zmin=0.0,
                      zmax=2.0 * float(val.max()), ltail=1, ltpar=0.0, utail=1, utpar=0.0, radius=(40.0, 20.0, 8.0),
                      angles=(60.0, 0.0, 0.0), ndmax=24)
        f = torch.empty((16, nc[2], nc[1], nc[0]), dtype=torch.float64, device="cuda")
        for prec in (ss.FP64, ss.FP32):
            sp.realize(4243, 16, 0, ss.FP64, out=f)
            ss.condition(f, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), structs, 0.05, params, np.column_stack([xyz, val]), prec)
        torch.cuda.synchronize()
        sp.close()
        return 0
    if kind == "spectrum":
        sp = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
        torch.cuda.synchronize()
        sp.close()
        return 0
    if kind == "vario":
        sp = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
        f = torch.empty((1, n[2], n[1], n[0]), dtype=torch.float64, device="cuda")
        sp.realize(WL["seed"], 1, WL["igauss"], ss.FP64, out=f)
        ss.vario(f, [(1, 0, 0, 100), (0, 1, 0, 100), (0, 0, 1, 100)])
        torch.cuda.synchronize()
        sp.close()
        return 0
    sp = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
    ss.autotune(sp, WL["igauss"], ss.FP32, 1)
    from specsim3d_b200 import _lib
    kinds = {"middle": 0, "synthesis": 1, "rows": 2}
    for pas, v in variants:
        # the log2 length a pass's variant is registered under: middle / synthesis
        # passes of npy / npz points, the row pass of npx / 2
        lg = {0: int(sp.np[1]).bit_length() - 1, 1: int(sp.np[2]).bit_length() - 1,
              2: int(sp.np[0]).bit_length() - 2}[kinds[pas]]
        if _lib.lib().ss3d_set_variant(kinds[pas], ss.FP32, lg, int(v)) != 0:
            raise SystemExit(f"invalid tile variant {pas}={v}")
    out = torch.empty((1, n[2], n[1], n[0]), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("profile")
    for _ in range(3):
        sp.realize(WL["seed"], 1, WL["igauss"], ss.FP32, out=out)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    sp.close()
    return 0


def main():
    args = parse()
    if args.profile_case:
        pairs = []
        for tv in args.tile_variant:
            pas, _, v = tv.partition("=")
            if pas not in ("middle", "synthesis", "rows") or not v.isdigit():
                raise SystemExit(f"--tile-variant wants PASS=V with PASS middle, synthesis or rows, got {tv!r}")
            pairs.append((pas, int(v)))
        return run_profile_case(args.profile_case, pairs)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
