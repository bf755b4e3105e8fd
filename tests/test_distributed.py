"""Multi-rank row sharding on CPU (gloo, world size 2): the partition covers
every row once with balanced cost, the signal broadcast and the shard gather
reassemble exactly the single-process result, and each shard follows the
reference's reused-O1 semantics (rows computed per shard equal the same rows
of the full transform). The per-rank transform is the float64 oracle here;
the GPU path of the same class is covered by test_gpu_parity's shard test."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from fcwt_b200.distributed import row_costs, row_partition


def test_partition_covers_rows_and_balances():
    rng = np.random.default_rng(0)
    for fn, world in [(3000, 8), (7, 4), (3, 8), (0, 2), (1, 1)]:
        costs = rng.uniform(1, 3, fn)
        blocks = row_partition(costs, world)
        assert len(blocks) == world
        assert blocks[0][0] == 0 and blocks[-1][1] == fn
        for (b0, e0), (b1, e1) in zip(blocks, blocks[1:]):
            assert e0 == b1 and b0 <= e0
        if fn >= 8 * world:
            loads = [costs[b:e].sum() for b, e in blocks]
            assert max(loads) - min(loads) <= 2 * costs.max() + 1e-9


def test_row_costs_follow_windows():
    from oracle.oracle import LINFREQS, Restatement

    sc = Restatement().scales(LINFREQS, 1000, 1.0, 101.0, 300)
    c = row_costs(100000, sc)
    assert c.shape == (300,) and np.all(c > 0)
    # low-frequency rows (last rows of a LINFREQS grid) have narrower windows
    assert c[-1] < c[0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, fn, result_path):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from fcwt_b200.distributed import ShardedCWT
        from oracle.oracle import LOGSCALES, Restatement

        o = Restatement()
        sc = o.scales(LOGSCALES, 1000, 2.0, 300.0, fn)

        def compute(x, rb, re_):
            full = o.cwt_fp64(x.numpy(), sc, 0.5, 2, True, rows=list(range(rb, re_)))
            return torch.from_numpy(full.astype(np.complex64))

        sh = ShardedCWT(n, sc, fb=0.5, threads=2, compute=compute)
        x = torch.zeros(n, dtype=torch.float32)
        if rank == 0:
            x = torch.from_numpy(np.random.default_rng(1).standard_normal(n).astype(np.float32))
        sh.broadcast_signal(x, src=0)
        local = sh(x)
        full = sh.gather(local, dst=0)
        if rank == 0:
            np.save(result_path, full.numpy())
            np.save(result_path + ".x.npy", x.numpy())
            np.save(result_path + ".blocks.npy", np.array(sh.blocks))
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_gather_matches_single_process(tmp_path):
    import torch.multiprocessing as mp

    from oracle.oracle import LOGSCALES, Restatement

    n, fn = 3000, 37
    res = str(tmp_path / "full.npy")
    mp.start_processes(_worker, args=(2, _free_port(), n, fn, res), nprocs=2, join=True, start_method="spawn")
    full = np.load(res)
    x = np.load(res + ".x.npy")
    blocks = np.load(res + ".blocks.npy")
    assert blocks[0][1] == blocks[1][0] and blocks[1][1] == fn and 0 < blocks[0][1] < fn
    o = Restatement()
    sc = o.scales(LOGSCALES, 1000, 2.0, 300.0, fn)
    ref = o.cwt_fp64(x, sc, 0.5, 2, True).astype(np.complex64)
    # σ = 0.5: rows past the split carry bins written by rows of the other shard
    assert np.array_equal(full, ref)
