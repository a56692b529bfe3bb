"""Seeded synthetic workloads of the batched and serving forms.

The reference benchmarks one grid per run; these generators draw the mixed
workloads the batched and serving forms are measured on.  Every draw comes
from numpy's PCG64 generator with the stated seed, so a workload is fully
determined by its arguments.

Variogram structures are tuples (itype, sill, ahmax, ahmin, avert, azimuth,
dip, plunge) with itype 1 spherical, 2 exponential, 3 gaussian (the model
codes of src/specsim3d.f90:95-139).
"""
import math

import numpy as np


def _log_uniform_int(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def random_model(rng, n, itype):
    """One structure: ranges U(5, 0.4 x extent) drawn per axis (x, y, z) and
    sorted so that ahmax >= ahmin >= avert (an extent below 12.5 gives range
    5), azimuth U(0, 180), dip U(-30, 30), plunge 0, sill 1, nugget U(0, 0.3)."""
    ranges = sorted((rng.uniform(5.0, max(5.0, 0.4 * e)) for e in n), reverse=True)
    azimuth = rng.uniform(0.0, 180.0)
    dip = rng.uniform(-30.0, 30.0)
    nugget = rng.uniform(0.0, 0.3)
    return [(itype, 1.0, ranges[0], ranges[1], ranges[2], azimuth, dip, 0.0)], nugget


def mixed_grids(seed=777, nshapes=16, total_real=1024, lo=32, hi=256, two_d_mod=8):
    """Batched workload: total_real unconditional realizations over nshapes grid
    shapes.  Shape s: nx, ny, nz = round(exp(U(ln lo, ln hi))) each, then
    nz = 1 when s = two_d_mod - 1 (mod two_d_mod); model family s mod 3
    (spherical, exponential, gaussian) drawn by random_model; ipad 1, igauss 1,
    iseed = seed + s.  Realizations are split evenly over the shapes.  Returns
    a list of dicts (n, structs, nugget, d, ipad, igauss, iseed, nreal)."""
    rng = np.random.default_rng(seed)
    per = total_real // nshapes
    jobs = []
    for s in range(nshapes):
        n = [_log_uniform_int(rng, lo, hi) for _ in range(3)]
        if two_d_mod and s % two_d_mod == two_d_mod - 1:
            n[2] = 1
        structs, nugget = random_model(rng, n, 1 + s % 3)
        nreal = per + (1 if s < total_real - per * nshapes else 0)
        jobs.append(dict(n=tuple(n), structs=structs, nugget=nugget, d=(1.0, 1.0, 1.0), ipad=1, igauss=1,
                         iseed=seed + s, nreal=nreal))
    return jobs


def model_pool(seed=2025, size=64, lo=32, hi=256):
    """Serving model pool: size (grid, model) entries drawn like mixed_grids
    (per-axis log-uniform grids, no 2D shapes)."""
    rng = np.random.default_rng(seed)
    pool = []
    for m in range(size):
        n = [_log_uniform_int(rng, lo, hi) for _ in range(3)]
        structs, nugget = random_model(rng, n, 1 + m % 3)
        pool.append(dict(n=tuple(n), structs=structs, nugget=nugget, d=(1.0, 1.0, 1.0), ipad=1))
    return pool


def request_stream(rate, count=4000, seed=2024, pool_size=64, cond_frac=0.2, max_real=16):
    """Serving request stream: Poisson arrivals at `rate` requests/s.  The draws
    do not depend on the rate (inter-arrival times are unit exponentials divided
    by the rate), so every rate replays the same requests: a pool model
    (uniform), nreal uniform in 1..max_real, a seed, and with probability
    cond_frac a conditional request carrying 200..2000 data points.  Returns a
    list of dicts (t_arrival, model, nreal, iseed, ndata)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0, size=count)) / float(rate)
    reqs = []
    for q in range(count):
        cond = rng.uniform() < cond_frac
        reqs.append(dict(t_arrival=float(t[q]), model=int(rng.integers(pool_size)),
                         nreal=int(rng.integers(1, max_real + 1)), iseed=int(rng.integers(1, 2 ** 31 - 1)),
                         ndata=int(rng.integers(200, 2001)) if cond else 0))
    return reqs
