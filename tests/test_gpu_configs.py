"""GPU parity of the batched, long-signal and differentiable forms at their
full workload shapes (the same generators bench.py times), on sampled rows
and channels against the float64 oracle:

  - 384 real channels of 20k-200k samples at 30 kHz, Morlet sigma 6, per-channel
    LOGSCALES grids of 64-256 rows, one batched plan replayed from a CUDA graph:
    rel-L2 <= 1e-5 (complex64);
  - complex 2^20 signal, 1024 LOGSCALES rows 10 Hz-80 kHz at 200 kHz, sigma 4:
    complex64 <= 1e-5 and BF16 output <= 3e-3;
  - differentiable 64 x 16384 x 128 (learnable sigma and centre frequencies,
    loss MSE(|W|^2, target)): forward <= 1e-5 and gradients <= 1e-4 against
    float64 torch autograd of the same operator.

Reference path all forms must equal: FCWT::cwt, src/fcwt/fcwt.cpp:447-529."""
from __future__ import annotations

import numpy as np
import pytest

import bench
from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def test_batched_384_channels_vs_fp64(fcwt, oracle):
    import torch

    xs_np, ns, fns = bench.batched_workload()
    assert len(ns) == 384 and min(ns) >= 20000 and max(ns) <= 200000
    morl = fcwt.Morlet(6.0)
    grids = [fcwt.Scales(morl, fcwt.FCWT_LOGSCALES, 30000, 1.0, 5000.0, k).scales for k in fns]
    xs = [torch.from_numpy(x).cuda() for x in xs_np]
    outs = [torch.full((k, n), float("nan"), dtype=torch.complex64, device="cuda") for k, n in zip(fns, ns)]
    bp = fcwt.BatchPlan(ns, grids, fb=6.0, threads=1, norm=True)
    bp.execute(xs, outs, graph=True)
    bp.execute(xs, outs, graph=True)  # replay of the captured graph
    torch.cuda.synchronize()
    chans = bench._batched_check_channels(ns)
    assert any(ns[c] % 2 == 1 for c in chans)
    for c in chans:
        rows = sorted({0, fns[c] // 2, fns[c] - 1})
        got = outs[c][torch.tensor(rows, device="cuda")].cpu().numpy()
        assert np.isfinite(got).all()
        ref = oracle.cwt_fp64(xs_np[c], grids[c], 6.0, 1, True, rows=rows)
        assert rel_l2(got, ref) < 1e-5, (c, ns[c], fns[c])
    # every output element written: no NaN left anywhere
    for o in outs:
        assert not torch.isnan(torch.view_as_real(o)).any()
    bp.close()


def test_long_complex_2e20_x_1024_bf16_vs_fp64(fcwt, oracle):
    import torch

    x = bench.long_workload()
    n, F = x.size, 1024
    sc = fcwt.Scales(fcwt.Morlet(4.0), fcwt.FCWT_LOGSCALES, 200000, 10.0, 80000.0, F)
    plan = fcwt.Plan(n, sc, fb=4.0, threads=1, norm=True, complex_input=True)
    xd = torch.from_numpy(x).cuda()
    sel = np.arange(0, F, 64).tolist() + [F - 1]
    ref = oracle.cwt_fp64(x, sc.scales, 4.0, 1, True, rows=sel)
    tsel = torch.tensor(sel, device="cuda")
    out64 = torch.empty((F, n), dtype=torch.complex64, device="cuda")
    plan.execute(xd, out64)
    r64 = out64[tsel].cpu().numpy()
    del out64
    assert rel_l2(r64, ref) < 1e-5
    out16 = torch.empty((F, n, 2), dtype=torch.bfloat16, device="cuda")
    plan.execute(xd, out16, out_type=fcwt.FCWT_OUT_BF16)
    r16 = torch.complex(out16[tsel, :, 0].double(), out16[tsel, :, 1].double()).cpu().numpy()
    assert rel_l2(r16, ref) < 3e-3
    plan.close()


def test_grad_64_x_16384_x_128_vs_fp64():
    import torch

    from fcwt_b200.autograd import LearnableMorletCWT
    from oracle.grad_ref import power_mse, ref_forward

    xs, freqs, target_np = bench.grad_workload()
    assert xs.shape == (64, 16384) and freqs.size == 128
    x = torch.from_numpy(xs).cuda().requires_grad_(True)
    layer = LearnableMorletCWT(freqs, 1000.0, sigma=2.0)
    target = torch.from_numpy(target_np).cuda()
    y = layer(x)
    loss = power_mse(y, target)
    loss.backward()

    xr = torch.from_numpy(xs).cuda().double().requires_grad_(True)
    sr = torch.tensor(2.0, dtype=torch.float64, device="cuda", requires_grad=True)
    fr = torch.tensor(freqs, dtype=torch.float64, device="cuda", requires_grad=True)
    yr = ref_forward(xr, sr, fr, 1000.0, True)
    Lr = power_mse(yr, target.double())
    Lr.backward()

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    assert rel(y.detach().to(torch.complex128), yr.detach()) < 1e-5
    assert rel(x.grad.double(), xr.grad) < 1e-4
    assert abs(float(layer.sigma.grad) - float(sr.grad)) <= 1e-4 * abs(float(sr.grad))
    gf = layer.freqs.grad.cuda()
    assert float(torch.max(torch.abs(gf - fr.grad)) / torch.max(torch.abs(fr.grad))) < 1e-4
