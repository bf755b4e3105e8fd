"""GPU tests of the batched multichannel path: many signals of different
lengths and scale grids in one plan (one persistent row-engine launch),
checked against the single-signal transform of each channel and the float64
oracle; CUDA-graph replay equals direct execution and follows new inputs."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import LINFREQS, LOGSCALES, rel_l2

pytestmark = pytest.mark.gpu


def _channels(oracle, seed, lengths, fs=30000):
    rng = np.random.default_rng(seed)
    xs, scs = [], []
    for n in lengths:
        xs.append(rng.standard_normal(n).astype(np.float32))
        fn = int(rng.integers(16, 64))
        scs.append(oracle.scales(LOGSCALES, fs, 1.0, 5000.0, fn))
    return xs, scs


def test_batched_equals_per_channel_transform(fcwt, oracle):
    import torch

    # direct (N < 1024), fused (N <= 8192) and two-phase rows in one launch
    lengths = [700, 5000, 20000, 65536, 33000, 1024, 120000]
    xs, scs = _channels(oracle, 1, lengths)
    bp = fcwt.BatchPlan(lengths, scs, fb=6.0, threads=8)
    ins = [torch.from_numpy(x).cuda() for x in xs]
    outs = bp.outputs_like()
    bp.execute(ins, outs)
    torch.cuda.synchronize()
    for x, sc, o in zip(xs, scs, outs):
        single = np.zeros((sc.size, x.size), np.complex64)
        fcwt.FCWT(fcwt.Morlet(6.0), 8, False, True).cwt(x, sc, single)
        assert np.array_equal(o.cpu().numpy(), single)
    # float64 oracle on two channels
    for k in (0, 4):
        assert rel_l2(outs[k].cpu().numpy(), oracle.cwt_fp64(xs[k], scs[k], 6.0, 8, True)) < 1e-5
    bp.close()


def test_batched_host_buffers(fcwt, oracle):
    lengths = [3000, 17000]
    xs, scs = _channels(oracle, 2, lengths, fs=1000)
    bp = fcwt.BatchPlan(lengths, scs, fb=2.0, threads=1, norm=False)
    outs = [np.zeros((sc.size, x.size), np.complex64) for x, sc in zip(xs, scs)]
    bp.execute(xs, outs)
    for x, sc, o in zip(xs, scs, outs):
        assert rel_l2(o, oracle.cwt_fp64(x, sc, 2.0, 1, False)) < 1e-5
    bp.close()


def test_graph_replay(fcwt, oracle):
    import torch

    lengths = [40000, 9000, 300, 70000]
    xs, scs = _channels(oracle, 3, lengths)
    bp = fcwt.BatchPlan(lengths, scs, fb=6.0, threads=1)
    ins = [torch.from_numpy(x).cuda() for x in xs]
    ref = bp.outputs_like()
    bp.execute(ins, ref)
    outs = bp.outputs_like()
    bp.execute(ins, outs, graph=True)   # capture + launch
    torch.cuda.synchronize()
    for a, b in zip(outs, ref):
        assert torch.equal(a, b)
    # new data in the same buffers: the replayed graph reads it
    for t in ins:
        t.mul_(-0.5)
    bp.execute(ins, outs, graph=True)   # replay
    torch.cuda.synchronize()
    for a, b in zip(outs, ref):
        assert torch.allclose(a, -0.5 * b, rtol=1e-5, atol=1e-6)
    fcwt.synchronize()
    bp.close()


def test_graph_first_execution_of_a_larger_plan(fcwt, oracle):
    """A graph captured for a plan with more rows than any earlier execution
    of the process: every per-execution buffer is sized before the capture
    starts (nothing may allocate while the stream is capturing)."""
    import torch

    rng = np.random.default_rng(9)
    lengths = [3000, 2500, 4000, 3500]
    grids = [oracle.scales(LOGSCALES, 30000, 1.0, 5000.0, 2500) for _ in lengths]
    xs = [torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda() for n in lengths]
    bp = fcwt.BatchPlan(lengths, grids, fb=6.0, threads=1)
    outs = bp.outputs_like()
    bp.execute(xs, outs, graph=True)
    torch.cuda.synchronize()
    ref = bp.outputs_like()
    bp.execute(xs, ref)
    torch.cuda.synchronize()
    for a, b in zip(outs, ref):
        assert torch.equal(a, b)
    bp.close()
