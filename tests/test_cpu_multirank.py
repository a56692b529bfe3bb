"""The multi-process split of realizations, on CPU with two gloo ranks.

Each rank takes its shard of realizations (specsim3d_b200.shard, the split
bench.py uses under torchrun) and computes the Park-Miller row states its GPU
kernels would start from (host jump-ahead, ss3d_row_state); rank 0 gathers
them and checks them against the oracle's serial stream (f90:1302-1334) for
the whole run, and the step time is reduced as the maximum over ranks.  Bar:
bit-exact.
"""
import os
import socket

import numpy as np
import pytest

WORLD = 2
PER_RANK = 2
NP3 = (16, 8, 6)
ISEED = 4711


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, igauss, out_path):
    import torch
    import torch.distributed as dist
    import specsim3d_b200 as ss
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        r_first, nreal = ss.shard(rank, WORLD, PER_RANK)
        states = np.zeros((nreal, NP3[2], NP3[1]), dtype=np.int64)
        for r in range(nreal):
            for k in range(NP3[2]):
                for j in range(NP3[1]):
                    states[r, k, j] = ss.row_state(NP3, igauss, ISEED, r_first + r, j, k)
        gathered = [None] * WORLD
        dist.all_gather_object(gathered, (r_first, states))
        t = torch.tensor([0.5 + rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            full = np.concatenate([s for _, s in sorted(gathered, key=lambda x: x[0])])
            np.save(out_path, full)
            np.save(out_path + ".max.npy", t.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("igauss", [0, 1])
def test_two_rank_shards_reproduce_serial_stream(tmp_path, igauss):
    import torch.multiprocessing as mp
    import oracle_lib as ora
    out = str(tmp_path / f"states_{igauss}.npy")
    mp.spawn(_rank_main, args=(_free_port(), igauss, out), nprocs=WORLD, join=True)
    got = np.load(out)
    assert float(np.load(out + ".max.npy")[0]) == 1.5
    full = ora.fill_states((NP3[0], NP3[1], NP3[2]), ISEED, WORLD * PER_RANK, igauss)   # (r, k, j, i)
    npz, npy = NP3[2], NP3[1]
    checked = 0
    for r in range(WORLD * PER_RANK):
        for k in range(npz):
            for j in range(npy):
                kp, jp = (-k) % npz, (-j) % npy
                if (k, j) <= (kp, jp):            # rows that draw: i = 0 is their first representative
                    assert got[r, k, j] == full[r, k, j, 0], (r, k, j)
                    checked += 1
    assert checked > 0
