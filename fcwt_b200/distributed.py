"""Multi-GPU CWT by scale-row sharding, one process per GPU.

The rows of a CWT are independent once the (tiny) input signal is known, so
each rank computes a contiguous block of rows on its own GPU; there is no
collective in the data path. The signal is broadcast once from `src`
(torch.distributed, NCCL on GPUs), and the sharded output can optionally be
gathered to one rank. The reference has no distributed layer; this is the
scale-out of its transform (FCWT::cwt, src/fcwt/fcwt.cpp:447-529): every shard
keeps the reference's reused-O1 semantics because each shard's plan still
walks all rows (fcwt_plan_create with a row range).

Rows are balanced by estimated cost: each row costs its output write
(n samples) plus its inverse transform, which grows with the row's bin window
(N log2 of the window).
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from . import api


def row_costs(n: int, scales, fb: float = 2.0, threads: int = 1, exact_support: bool = False) -> np.ndarray:
    """Relative cost of each row: output samples plus N*log2(window) for the
    row's transform (host-only; uses the planner's bin windows)."""
    sc = np.ascontiguousarray(scales, np.float32)
    _, lo, hi = api.row_truncation(n, sc, threads=threads, exact_support=exact_support, fb=fb)
    N = 1 << int(np.ceil(np.log2(max(n, 1)))) if n > 1 else 1
    win = np.maximum(hi - (lo // 1024) * 1024, 1).astype(np.float64)
    return n + 0.25 * N * np.log2(np.maximum(win, 2.0))


def row_partition(costs, world: int) -> list[tuple[int, int]]:
    """Contiguous [begin, end) row blocks, one per rank, with near-equal total
    cost (greedy prefix split). Blocks may be empty when rows < ranks."""
    c = np.asarray(costs, np.float64)
    fn = c.size
    if world <= 0:
        raise ValueError("world must be >= 1")
    if fn == 0:
        return [(0, 0)] * world
    csum = np.concatenate([[0.0], np.cumsum(c)])
    total = csum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(csum, target, side="left"))
        if b > 0 and abs(csum[b - 1] - target) <= abs(csum[min(b, fn)] - target):
            b -= 1  # the prefix boundary nearest to the target
        b = min(max(b, bounds[-1]), fn)
        bounds.append(b)
    bounds.append(fn)
    return [(bounds[i], bounds[i + 1]) for i in range(world)]


class ShardedCWT:
    """Row-sharded CWT over a torch.distributed process group.

    Each rank builds a plan for its row block on its current CUDA device;
    ``__call__`` returns the local block [rows_local, n] (device tensor);
    ``gather`` assembles the full [fn, n] output on `dst` (host or device).
    ``compute`` replaces the GPU transform (used by CPU tests of the
    plumbing); by default the rank's fcwt_b200 plan runs the block.
    """

    def __init__(self, n: int, scales, fb: float = 2.0, threads: int = 1, norm: bool = True,
                 group=None, balance: bool = True,
                 compute: Optional[Callable] = None, device: Optional[int] = None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.n = int(n)
        self.scales = np.ascontiguousarray(scales, np.float32)
        self.fn = self.scales.size
        self.fb = float(fb)
        self.threads = int(threads)
        self.norm = bool(norm)
        costs = row_costs(self.n, self.scales, self.fb, self.threads) if balance else np.ones(self.fn)
        self.blocks = row_partition(costs, self.world)
        self.rows = self.blocks[self.rank]
        self.compute = compute
        self.plan = None
        if compute is None:
            import torch

            self.device = torch.cuda.current_device() if device is None else device
            self.plan = api.Plan(self.n, self.scales, fb=self.fb, threads=self.threads, norm=self.norm,
                                 rows=self.rows, device=self.device)

    def broadcast_signal(self, x, src: int = 0):
        """Send rank src's signal to every rank (in place on `x`, a torch tensor
        of length n on the rank's communication device)."""
        self.dist.broadcast(x, src=src, group=self.group)
        return x

    def __call__(self, x):
        import torch

        rb, re_ = self.rows
        if self.compute is not None:
            return self.compute(x, rb, re_)
        out = torch.empty((re_ - rb, self.n), dtype=torch.complex64, device=x.device)
        if re_ > rb:
            self.plan.execute(x, out)
        return out

    def gather(self, local, dst: int = 0):
        """Full [fn, n] output on rank dst (None elsewhere). Each rank's block
        travels point to point straight into its rows of the destination
        tensor: no padding to the largest block and no second copy on dst.
        Complex blocks travel as float32 pairs (backends without complex
        support)."""
        import torch

        if self.rank != dst:
            if local.shape[0]:
                self.dist.send(torch.view_as_real(local.contiguous()), dst=dst, group=self.group)
            return None
        full = torch.empty((self.fn, self.n), dtype=torch.complex64, device=local.device)
        fr = torch.view_as_real(full)
        reqs = []
        for r, (b, e) in enumerate(self.blocks):
            if e == b:
                continue
            if r == self.rank:
                fr[b:e].copy_(torch.view_as_real(local))
            else:
                reqs.append(self.dist.irecv(fr[b:e], src=r, group=self.group))
        for q in reqs:
            q.wait()
        return full

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None
