"""Batched form: many grids in one CUDA-graph launch.

Bar: every job's realizations equal the per-call FP32 path (ss3d_realize,
SS3D_FP32, float output) bit for bit under both schedules -- the batch runs
the same tile bodies with the same Park-Miller row states -- and so sit within
the FP32 precision bar (1e-5 * sqrt(C0)) of the oracle, which one job also
checks directly.
"""
import numpy as np
import pytest

import oracle_lib as ora
from specsim3d_b200 import workloads

pytestmark = pytest.mark.gpu


def _specs_small():
    base = workloads.mixed_grids(seed=5, nshapes=6, total_real=12, lo=16, hi=48)
    extra = [
        dict(n=(64, 64, 16), structs=[(1, 1.0, 20.0, 10.0, 5.0, 45.0, 0.0, 0.0)], nugget=0.0, d=(1.0, 1.0, 1.0),
             ipad=1, igauss=0, iseed=69069, nreal=3),
        dict(n=(30, 20, 9), structs=[(2, 0.7, 12.0, 6.0, 3.0, 30.0, 10.0, 5.0)], nugget=0.3, d=(1.0, 1.5, 0.5),
             ipad=1, igauss=1, iseed=31, nreal=2),
        dict(n=(33, 17, 1), structs=[(3, 1.0, 8.0, 4.0, 4.0, 120.0, 0.0, 0.0)], nugget=0.1, d=(1.0, 1.0, 1.0),
             ipad=1, igauss=0, iseed=7, nreal=2),
    ]
    return base + extra


def _build(gpu, specs, r_first=0):
    import torch
    jobs = []
    for c in specs:
        sp = gpu.Spectrum(c["structs"], c["nugget"], c["d"], c["n"], c["ipad"])
        nx, ny, nz = c["n"]
        out = torch.full((c["nreal"], nz, ny, nx), float("nan"), dtype=torch.float32, device="cuda")
        jobs.append((sp, c["iseed"], c["igauss"], r_first, c["nreal"], out))
    return jobs


def _check_against_per_call(gpu, jobs):
    import torch
    torch.cuda.synchronize()
    for sp, iseed, igauss, r_first, nreal, out in jobs:
        ref = sp.realize(iseed, nreal, igauss, gpu.FP32, r_first=r_first, dtype=np.float32)
        got = out.cpu().numpy()
        assert np.array_equal(got, ref), (sp.n, sp.np, float(np.nanmax(np.abs(got - ref))))


def _clear(jobs):
    for j in jobs:
        j[5].fill_(float("nan"))


@pytest.mark.parametrize("sched", ["chains", "persistent"])
def test_batch_equals_per_call(gpu, sched):
    jobs = _build(gpu, _specs_small())
    b = gpu.Batch(jobs)
    if sched == "persistent":
        for p in range(3):
            b.set_schedule(gpu.Batch.PERSISTENT, p, elements_per_thread=8, mode=p, ctas_per_sm=0)
    assert b.schedule()["schedule"] == sched
    b.run()
    _check_against_per_call(gpu, jobs)
    info = b.info()
    assert info["cells"] == sum(j[4] * int(np.prod(j[0].n)) for j in jobs)
    assert info["kernels"] >= 3
    # a second run of the same graph rewrites the same values
    _clear(jobs)
    b.run()
    _check_against_per_call(gpu, jobs)
    b.close()


@pytest.mark.parametrize("split", [2, 3, 8])
def test_batch_split_sub_chains(gpu, split):
    """Realizations of each job split into staggered sub-chains: same bits as
    one chain per job (and as the per-call path)."""
    jobs = _build(gpu, _specs_small())
    b = gpu.Batch(jobs)
    b.set_split(split)
    assert b.schedule()["split"] == split and b.schedule()["schedule"] == "chains"
    b.run()
    _check_against_per_call(gpu, jobs)
    _clear(jobs)
    b.run()
    _check_against_per_call(gpu, jobs)
    b.close()


def test_batch_persistent_variants_identical(gpu):
    jobs = _build(gpu, _specs_small()[:5])
    b = gpu.Batch(jobs)
    for et in (16, 8):
        for mode in (0, 1, 2):
            for p in range(3):
                b.set_schedule(gpu.Batch.PERSISTENT, p, elements_per_thread=et, mode=mode, ctas_per_sm=1)
            _clear(jobs)
            b.run()
            _check_against_per_call(gpu, jobs)
    b.close()


def test_batch_offsets_shared_spectrum_and_oracle(gpu):
    import torch
    c = dict(n=(40, 36, 20), structs=[(1, 1.0, 15.0, 9.0, 6.0, 60.0, 15.0, 5.0)], nugget=0.05, d=(1.0, 1.0, 1.0),
             ipad=1)
    sp = gpu.Spectrum(c["structs"], c["nugget"], c["d"], c["n"], c["ipad"])
    nx, ny, nz = c["n"]
    outs = [torch.empty((k, nz, ny, nx), dtype=torch.float32, device="cuda") for k in (2, 3, 1)]
    jobs = [(sp, 4242, 1, 0, 2, outs[0]), (sp, 4242, 1, 2, 3, outs[1]), (sp, 99, 0, 5, 1, outs[2])]
    b = gpu.Batch(jobs)
    b.run()
    _check_against_per_call(gpu, jobs)
    # realizations r_first.. of one seed split over two jobs equal one call of all five
    full = sp.realize(4242, 5, 1, gpu.FP32, dtype=np.float32)
    assert np.array_equal(np.concatenate([outs[0].cpu().numpy(), outs[1].cpu().numpy()]), full)
    # and the FP32 precision bar against the oracle
    amp_o, st = ora.spectrum(c["structs"], c["nugget"], c["d"], sp.np)
    res_o, _ = ora.realize(amp_o, sp.np, c["n"], 4242, 5, 1)
    err = np.max(np.abs(full.astype(np.float64) - res_o)) / np.sqrt(st["c0"])
    assert err <= 1e-5, err
    b.close()


def test_batch_autotune_keeps_results(gpu):
    jobs = _build(gpu, _specs_small()[:4])
    b = gpu.Batch(jobs, autotune=True)
    _clear(jobs)
    b.run()
    _check_against_per_call(gpu, jobs)
    ms = b.time()
    assert ms[3] > 0
    b.close()


def test_batch_rejects_bad_jobs(gpu):
    import torch
    from specsim3d_b200 import _lib
    # a 1D grid runs under the chains schedule but not the persistent one
    sp = gpu.Spectrum([(1, 1.0, 4.0, 4.0, 4.0, 0.0, 0.0, 0.0)], 0.0, (1.0, 1.0, 1.0), (40, 1, 1), 1)
    out = torch.empty((2, 1, 1, 40), dtype=torch.float32, device="cuda")
    b = gpu.Batch([(sp, 1, 0, 0, 2, out)])
    b.run()
    _check_against_per_call(gpu, [(sp, 1, 0, 0, 2, out)])
    with pytest.raises(_lib.SpecsimError):
        b.set_schedule(gpu.Batch.PERSISTENT)
    b.close()
    sp2 = gpu.Spectrum([(1, 1.0, 6.0, 6.0, 6.0, 0.0, 0.0, 0.0)], 0.0, (1.0, 1.0, 1.0), (20, 20, 20), 1)
    with pytest.raises(ValueError):
        gpu.Batch([(sp2, 1, 0, 0, 2, torch.empty(10, dtype=torch.float32, device="cuda"))])
    with pytest.raises(_lib.SpecsimError):
        gpu.Batch([(sp2, 1, 3, 0, 1, torch.empty((1, 20, 20, 20), dtype=torch.float32, device="cuda"))])
