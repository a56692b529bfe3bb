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
    """One structure with ranges uniform in [5, 0.4 x extent] per axis (the two
    horizontal draws sorted into ahmax >= ahmin), azimuth uniform in [0, 180),
    dip uniform in [-30, 30] (0 for 2D grids), nugget uniform in [0, 0.3] and
    sill 1 - nugget, so that the total sill is 1."""
    nx, ny, nz = n
    a1 = rng.uniform(5.0, max(5.0, 0.4 * nx))
    a2 = rng.uniform(5.0, max(5.0, 0.4 * ny))
    ahmax, ahmin = max(a1, a2), min(a1, a2)
    avert = rng.uniform(5.0, max(5.0, 0.4 * nz)) if nz > 1 else 5.0
    azimuth = rng.uniform(0.0, 180.0)
    dip = rng.uniform(-30.0, 30.0) if nz > 1 else 0.0
    nugget = rng.uniform(0.0, 0.3)
    return [(itype, 1.0 - nugget, ahmax, ahmin, avert, azimuth, dip, 0.0)], nugget


def mixed_grids(seed=777, nshapes=16, total_real=1024, lo=32, hi=256, two_d_every=4):
    """Batched workload: total_real unconditional realizations over nshapes grid
    shapes; nx, ny, nz log-uniform in [lo, hi], every two_d_every-th shape 2D
    (nz = 1); model family cycling spherical / exponential / gaussian; ipad 1,
    igauss 1; job s seeded seed + 1000 s.  Returns a list of dicts (n, structs,
    nugget, d, ipad, igauss, iseed, nreal); realizations split evenly."""
    rng = np.random.default_rng(seed)
    per = total_real // nshapes
    jobs = []
    for s in range(nshapes):
        nx = _log_uniform_int(rng, lo, hi)
        ny = _log_uniform_int(rng, lo, hi)
        nz = 1 if (two_d_every and s % two_d_every == two_d_every - 1) else _log_uniform_int(rng, lo, hi)
        structs, nugget = random_model(rng, (nx, ny, nz), 1 + s % 3)
        nreal = per + (1 if s < total_real - per * nshapes else 0)
        jobs.append(dict(n=(nx, ny, nz), structs=structs, nugget=nugget, d=(1.0, 1.0, 1.0), ipad=1, igauss=1,
                         iseed=seed + 1000 * s, nreal=nreal))
    return jobs


def model_pool(seed=2024, size=64, lo=32, hi=256):
    """Serving model pool: size (grid, model) entries, cubic grids with edge
    log-uniform in [lo, hi], models drawn as in mixed_grids."""
    rng = np.random.default_rng(seed)
    pool = []
    for m in range(size):
        n = _log_uniform_int(rng, lo, hi)
        structs, nugget = random_model(rng, (n, n, n), 1 + m % 3)
        pool.append(dict(n=(n, n, n), structs=structs, nugget=nugget, d=(1.0, 1.0, 1.0), ipad=1))
    return pool


def request_stream(rate, count=4000, seed=2024, pool_size=64, cond_frac=0.2, max_real=16):
    """Serving request stream: Poisson arrivals at `rate` requests/s, a pool
    model per request (uniform), nreal uniform in 1..max_real, conditional with
    probability cond_frac and then carrying 200..2000 data points.  Returns a
    list of dicts (t_arrival, model, nreal, iseed, ndata)."""
    rng = np.random.default_rng([seed, int(rate)])
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    reqs = []
    for q in range(count):
        cond = rng.uniform() < cond_frac
        reqs.append(dict(t_arrival=float(t[q]), model=int(rng.integers(pool_size)),
                         nreal=int(rng.integers(1, max_real + 1)), iseed=int(rng.integers(1, 2 ** 31 - 1)),
                         ndata=int(rng.integers(200, 2001)) if cond else 0))
    return reqs
