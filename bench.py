#!/usr/bin/env python3
"""bench.py -- throughput of the SPECSIM3D spectral simulation path on B200.

Workload (the precision configuration, one GPU): unconditional 256x256x256 grid,
cell size 1, gaussian model sill 1.0 nugget 0.1 ranges 60/30/15 azimuth 30 dip 20
plunge 10, ipad 1 (periodic grid 512^3), igauss 1, seed 12345, 8 realizations per
GPU.  The FP64 spectrum is built once and stays resident; a step is one batch of
8 realizations synthesised, inverse-transformed and cropped into a device
float32 buffer in the FP32 precision form.  The same step in the plain FP64
form, the FP32-vs-FP64 error and an end-to-end run through the C ABI into pinned
host memory are reported next to it.

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
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers
def cells_per_real():
    n = WL["n"]
    return n[0] * n[1] * n[2]


def half_spectrum_size(np3):
    npx, npy, npz = np3
    return (npx // 2 + 1) * npy * npz


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

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
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
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


def cpu_reference_sample(k_steps, warmup):
    """Oracle (C restatement, OpenMP) on the host cores: seconds per realization of the workload."""
    ora = oracle_lib()
    np3, rc = ora.grid(WL["structs"], WL["d"], WL["n"], WL["ipad"])
    t0 = time.perf_counter()
    amp, _ = ora.spectrum(WL["structs"], WL["nugget"], WL["d"], np3)
    t_spec = time.perf_counter() - t0
    times = []
    for s in range(warmup + k_steps):
        t0 = time.perf_counter()
        ora.realize(amp, np3, WL["n"], WL["seed"], 1, WL["igauss"])
        if s >= warmup:
            times.append(time.perf_counter() - t0)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return float(np.mean(times)), t_spec, cores


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    k = max(1, args.steps)
    w = max(0, args.warmup)
    sec, t_spec, cores = cpu_reference_sample(k, w)
    value = cells_per_real() / sec / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mcells/s", "n_gpus": args.gpus,
        "steps": k, "warmup": w, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "sample": "1 realization per step, spectrum excluded",
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mcells/s", "cores": cores, "kind": "port",
                         "sample": "1 realization of the 256^3 workload per step (C restatement of the Fortran, "
                                   f"OpenMP, {cores} threads); spectrum build {t_spec:.2f} s not counted"},
        "e2e": {"value": round(value, 3), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- our arm
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
    ss.set_stream(stream)
    n = WL["n"]
    nreal = WL["nreal"]
    M = cells_per_real()
    r_first = rank * nreal
    sp = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
    c0 = sp.stats["c0"]
    out32 = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float32, device=dev)
    out64 = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float64, device=dev)

    def step(prec, out):
        sp.realize(WL["seed"], nreal, WL["igauss"], prec, r_first=r_first, out=out)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    def timed(prec, out, k, w, prof=False):
        for _ in range(w):
            step(prec, out)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if prof:
            ss.profile(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        _, l0 = ss.profile_read()
        e0.record(stream)
        for _ in range(k):
            step(prec, out)
        e1.record(stream)
        torch.cuda.synchronize()
        stages, l1 = ss.profile_read()
        if prof:
            ss.profile(False)
        barrier()
        ms = e0.elapsed_time(e1) / k
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, stages, l1 - l0

    # tile variants picked by the autotuner for this grid (untimed, once per process)
    tuned = {"fp32": ss.autotune(sp, WL["igauss"], ss.FP32, nreal), "fp64": ss.autotune(sp, WL["igauss"], ss.FP64, nreal)}
    k, w = max(1, args.steps), max(3, args.warmup)
    clk = ClockSampler(local)
    clk.start()
    ms32, _, launches = timed(ss.FP32, out32, k, w)
    clocks = clk.stop()
    ms64, _, _ = timed(ss.FP64, out64, max(1, k // 2), 3)
    # per-kernel durations for the roofline: a separate pass with stage events
    # (stages then run back to back instead of overlapped across realizations)
    _, stages, _ = timed(ss.FP32, out32, max(1, k // 2), 1, prof=True)
    kprof = max(1, k // 2)
    # precision-form error against the FP64 path on the same realizations
    step(ss.FP64, out64)
    step(ss.FP32, out32)
    torch.cuda.synchronize()
    diff = (out32.double() - out64).abs_()
    err_max = float(diff.amax().item()) / np.sqrt(c0)
    err_rms = float(diff.pow_(2).mean().sqrt().item()) / np.sqrt(c0)
    del diff
    # end to end through the C ABI: spectrum build + realizations into pinned host memory
    host = torch.empty((nreal, n[2], n[1], n[0]), dtype=torch.float32).pin_memory()
    hn = host.numpy()
    ke = max(1, min(k, 5))
    ts = []
    for s in range(ke + 1):
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        spe = ss.Spectrum(WL["structs"], WL["nugget"], WL["d"], n, WL["ipad"])
        spe.realize(WL["seed"], nreal, WL["igauss"], ss.FP32, r_first=r_first, out=hn)
        spe.close()
        t1 = time.perf_counter()
        if s > 0:
            ts.append(t1 - t0)
    e2e_s = float(np.mean(ts))
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    # roofline of the dominant kernel: synthesis fused with the first (z) inverse pass
    np3 = sp.np
    nh = half_spectrum_size(np3)
    rho_z = n[2] / np3[2]
    bytes_gen = nh * (4 + 8 * rho_z) * nreal           # amp read (float) + pruned complex write, per launch
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
        traffic = tr.get("k_colgen_float_9_per_launch_bytes")
    except Exception:
        pass
    # whole-step roofline (all kernels of the realization path)
    rho_y = n[1] / np3[1]
    b_real = nh * (4 + 8 * (1 + rho_z + 2 * rho_z * rho_y)) + 4 * M   # per realization, FP32 form
    value = M * nreal * world / (ms32 * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mcells/s", "n_gpus": world, "steps": k, "warmup": w,
        "ms_per_step": round(ms32, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "global_batch": nreal * world, "precision": "FP32 synthesis and FFTs "
                   "on the FP64 spectrum", "parallelism": f"realizations sharded over {world} GPU(s)",
                   "l2": "inputs larger than L2 (FP32 amplitude 269 MB, complex work 2.2 GB)",
                   "tile_variants": tuned},
        "fp64": {"value": round(M * nreal * world / (ms64 * 1e-3) / 1e6, 1), "unit": "Mcells/s",
                 "ms_per_step": round(ms64, 4)},
        "fp32_over_fp64": round(ms64 / ms32, 3),
        "error_vs_fp64": {"max_abs_over_sqrt_c0": err_max, "rms_over_sqrt_c0": err_rms, "target": 1e-5},
        "clocks": clocks,
        "e2e": {"value": round(M * nreal * world / e2e_s / 1e6, 1), "unit": "Mcells/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(M * nreal * 4),
                "includes": "spectrum build + realizations + D2H into pinned host memory"},
        "gpu_launches": int(launches),
        "stages_ms_per_step_serialized": {kk: round(v[0] / kprof, 4) for kk, v in stages.items()},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "kernel": "k_colgen<float,9> (synthesis + z inverse pass)",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650"},
        "roofline_step": {"algorithmic_bytes_per_realization": int(b_real),
                          "achieved_gbs": round(b_real * nreal / (ms32 * 1e-3) / 1e9, 1),
                          "frac": round(b_real * nreal / (ms32 * 1e-3) / 1e9 / peak, 4)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sec, t_spec, cores = cpu_reference_sample(1, 0)
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


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
