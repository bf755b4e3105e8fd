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


def test_back_to_back_executions_into_different_buffers(fcwt, oracle):
    """Consecutive executions enqueue their forward jobs and per-output tensor
    maps from host staging without waiting on the device: each must keep its
    own buffers (complex64 and BF16 outputs, no synchronisation in between)."""
    import torch

    lengths = [40000, 9000, 70000, 25000, 131072]
    xs, scs = _channels(oracle, 4, lengths)
    bp = fcwt.BatchPlan(lengths, scs, fb=6.0, threads=1)
    sets = []
    for k in range(6):
        ins = [torch.from_numpy(x * (1.0 + k)).cuda() for x in xs]
        outs = bp.outputs_like()
        o16 = [torch.empty((fn, n, 2), dtype=torch.bfloat16, device="cuda") for fn, n in zip(bp.fns, bp.ns)]
        sets.append((k, ins, outs, o16))
    torch.cuda.synchronize()
    for k, ins, outs, o16 in sets:
        bp.execute(ins, outs)
        bp.execute(ins, o16, out_type=fcwt.FCWT_OUT_BF16)
    torch.cuda.synchronize()
    base = bp.outputs_like()
    bp.execute([torch.from_numpy(x).cuda() for x in xs], base)
    torch.cuda.synchronize()
    for k, ins, outs, o16 in sets:
        for a, b, h in zip(outs, base, o16):
            assert rel_l2(a.cpu().numpy(), (1.0 + k) * b.cpu().numpy()) < 1e-5
            h64 = torch.complex(h[..., 0].double(), h[..., 1].double())
            assert rel_l2(h64.cpu().numpy(), a.cpu().numpy()) < 3e-3
    for c in (0, 4):
        assert rel_l2(base[c].cpu().numpy(), oracle.cwt_fp64(xs[c], scs[c], 6.0, 1, True)) < 1e-5
    bp.close()


def test_output_without_tensor_map(fcwt, oracle):
    """An output whose base is only 8-byte aligned cannot be a TMA target: its
    rows take the plain store path while the other outputs keep theirs."""
    import torch

    lengths = [30000, 50000, 30000]
    xs, scs = _channels(oracle, 5, lengths)
    bp = fcwt.BatchPlan(lengths, scs, fb=6.0, threads=1)
    ins = [torch.from_numpy(x).cuda() for x in xs]
    ref = bp.outputs_like()
    bp.execute(ins, ref)
    fn1, n1 = bp.fns[1], bp.ns[1]
    raw = torch.full((fn1 * n1 + 1,), float("nan"), dtype=torch.complex64, device="cuda")
    odd = raw[1:].view(fn1, n1)
    assert odd.data_ptr() % 16 == 8
    outs = [torch.empty_like(ref[0]), odd, torch.empty_like(ref[2])]
    bp.execute(ins, outs)
    torch.cuda.synchronize()
    for a, b in zip(outs, ref):
        assert torch.equal(a, b)
    bp.close()


def test_context_destroyed_before_its_plans(fcwt, oracle):
    """Destroying a context first (any order is possible when a garbage
    collector finalises both) releases its plans' device resources and leaves
    their handles valid: executing one reports an error, destroying it is safe."""
    import ctypes

    import torch

    from fcwt_b200 import _lib

    lengths = [30000, 9000]
    xs, scs = _channels(oracle, 6, lengths)
    lib = _lib.load()
    ctx = _lib.Context(0)
    nsig = len(lengths)
    h = ctypes.c_void_p()
    _lib.call("fcwt_plan_create_batched", ctx.handle, nsig, (ctypes.c_int * nsig)(*lengths), 0, ctypes.c_float(6.0),
              (ctypes.c_void_p * nsig)(*[sc.ctypes.data for sc in scs]),
              (ctypes.c_int * nsig)(*[sc.size for sc in scs]), 1, _lib.FCWT_NORM, ctypes.byref(h))
    ins = [torch.from_numpy(x).cuda() for x in xs]
    outs = [torch.empty((sc.size, n), dtype=torch.complex64, device="cuda") for sc, n in zip(scs, lengths)]
    in_arr = (ctypes.c_void_p * nsig)(*[t.data_ptr() for t in ins])
    out_arr = (ctypes.c_void_p * nsig)(*[t.data_ptr() for t in outs])
    torch.cuda.synchronize()
    _lib.call("fcwt_plan_execute_batched", h, in_arr, out_arr, fcwt.FCWT_OUT_C64)
    _lib.call("fcwt_synchronize", ctx.handle)
    assert rel_l2(outs[1].cpu().numpy(), oracle.cwt_fp64(xs[1], scs[1], 6.0, 1, True)) < 1e-5
    ctx.close()
    rc = lib.fcwt_plan_execute_batched(h, in_arr, out_arr, fcwt.FCWT_OUT_C64)
    assert rc == _lib.FCWT_ERR_INVALID and b"context" in lib.fcwt_last_error()
    assert lib.fcwt_plan_destroy(h) == 0
