"""GPU tests of the differentiable Morlet CWT: forward against a float64
torch.fft restatement of the same operator, gradients (signal, sigma, centre
frequencies) against float64 torch autograd of that restatement and against
float64 central finite differences. Tolerance 1e-4 (relative)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.grad_ref import ref_forward

pytestmark = pytest.mark.gpu


def loss_fn(y, target):
    return ((y.abs() ** 2 - target) ** 2).mean()


@pytest.mark.parametrize("n,F,norm", [(1500, 5, True), (5000, 7, False), (20000, 9, True)])
def test_forward_and_gradients(n, F, norm):
    import torch

    from fcwt_b200.autograd import morlet_cwt

    rng = np.random.default_rng(n)
    B, fs = 2, 1000.0
    t = np.arange(n) / fs
    x0 = np.stack([np.sin(2 * np.pi * (10 + 30 * t) * t) + 0.1 * rng.standard_normal(n) for _ in range(B)])
    f0 = np.geomspace(5.0, 150.0, F)
    sig0 = 2.0
    target = torch.from_numpy(rng.uniform(0, 0.05, (B, F, n)))
    if not norm:
        target = target * (1 << int(math.ceil(math.log2(n)))) ** 2

    # ours
    x = torch.tensor(x0, dtype=torch.float32, device="cuda", requires_grad=True)
    sigma = torch.tensor(sig0, dtype=torch.float64, requires_grad=True)
    freqs = torch.tensor(f0, dtype=torch.float64, requires_grad=True)
    y = morlet_cwt(x, sigma, freqs, fs, norm)
    L = loss_fn(y.to(torch.complex128).cpu(), target)
    L.backward()

    # float64 reference
    xr = torch.tensor(x0.astype(np.float32).astype(np.float64), requires_grad=True)
    sr = torch.tensor(sig0, dtype=torch.float64, requires_grad=True)
    fr = torch.tensor(f0, dtype=torch.float64, requires_grad=True)
    yr = ref_forward(xr, sr, fr, fs, norm)
    Lr = loss_fn(yr, target)
    Lr.backward()

    yd = y.detach().cpu().to(torch.complex128)
    assert float(torch.linalg.vector_norm(yd - yr.detach()) / torch.linalg.vector_norm(yr.detach())) < 1e-5
    gx, gxr = x.grad.cpu().double(), xr.grad
    assert float(torch.linalg.vector_norm(gx - gxr) / torch.linalg.vector_norm(gxr)) < 1e-4
    assert abs(float(sigma.grad) - float(sr.grad)) <= 1e-4 * abs(float(sr.grad)) + 1e-12
    gf, gfr = freqs.grad, fr.grad
    assert float(torch.max(torch.abs(gf - gfr)) / torch.max(torch.abs(gfr))) < 1e-4

    # central finite differences of the float64 operator
    def L_at(sv, fv):
        with torch.no_grad():
            return float(loss_fn(ref_forward(xr.detach(), torch.tensor(sv, dtype=torch.float64),
                                             torch.tensor(fv, dtype=torch.float64), fs, norm), target))
    h = 1e-6
    fd_sig = (L_at(sig0 + h, f0) - L_at(sig0 - h, f0)) / (2 * h)
    assert abs(float(sigma.grad) - fd_sig) <= 1e-4 * abs(fd_sig) + 1e-10
    # dL/dx along random unit directions v: <dL/dx, v> against central differences
    # of the float64 operator, L(x + h v) - L(x - h v) over 2h
    rngd = np.random.default_rng(n + 1)
    for _ in range(3):
        v = torch.from_numpy(rngd.standard_normal((B, n)))
        v /= torch.linalg.vector_norm(v)
        hx = 1e-4 * float(torch.linalg.vector_norm(xr.detach()))
        with torch.no_grad():
            Lp = float(loss_fn(ref_forward(xr.detach() + hx * v, torch.tensor(sig0, dtype=torch.float64),
                                           torch.tensor(f0, dtype=torch.float64), fs, norm), target))
            Lm = float(loss_fn(ref_forward(xr.detach() - hx * v, torch.tensor(sig0, dtype=torch.float64),
                                           torch.tensor(f0, dtype=torch.float64), fs, norm), target))
        fd_x = (Lp - Lm) / (2 * hx)
        got_x = float((gx * v).sum())
        scale_x = float(torch.linalg.vector_norm(gxr))
        assert abs(got_x - fd_x) <= 1e-4 * max(abs(fd_x), 1e-3 * scale_x), (got_x, fd_x)
    k = F // 2
    fp, fm = f0.copy(), f0.copy()
    hf = 1e-6 * f0[k]
    fp[k] += hf
    fm[k] -= hf
    fd_f = (L_at(sig0, fp) - L_at(sig0, fm)) / (2 * hf)
    assert abs(float(gf[k]) - fd_f) <= 1e-4 * max(abs(fd_f), float(torch.max(torch.abs(gfr)))) + 1e-12


def test_learnable_module_trains():
    import torch

    from fcwt_b200.autograd import LearnableMorletCWT

    n, fs = 4096, 1000.0
    t = np.arange(n) / fs
    x = torch.tensor(np.sin(2 * np.pi * 40 * t), dtype=torch.float32, device="cuda").reshape(1, n)
    layer = LearnableMorletCWT([30.0, 55.0], fs, sigma=2.0)
    y = layer(x)
    e0 = float((y.detach().abs() ** 2).mean())
    (-(y.abs() ** 2).mean()).backward()
    # moving the centre frequencies toward 40 Hz increases the energy
    assert float(layer.freqs.grad[0]) < 0 < float(layer.freqs.grad[1])
    assert e0 > 0 and layer.sigma.grad is not None and torch.isfinite(layer.sigma.grad)


@pytest.mark.parametrize("n,F,norm", [(1500, 5, True), (20000, 9, True), (5000, 7, False)])
def test_power_layer_forward_and_gradients(n, F, norm):
    """morlet_power_cwt: |y|^2 from the power epilogue and its gradients
    (recomputed y, dL/dy = 2 y dL/dP into the adjoint) against float64 torch
    autograd of |ref_forward|^2 and central differences in sigma."""
    import torch

    from fcwt_b200.autograd import morlet_power_cwt

    rng = np.random.default_rng(n + 7)
    B, fs = 2, 1000.0
    t = np.arange(n) / fs
    x0 = np.stack([np.sin(2 * np.pi * (10 + 30 * t) * t) + 0.1 * rng.standard_normal(n) for _ in range(B)])
    f0 = np.geomspace(5.0, 150.0, F)
    sig0 = 2.0
    target = torch.from_numpy(rng.uniform(0, 0.05, (B, F, n)))
    if not norm:
        target = target * (1 << int(math.ceil(math.log2(n)))) ** 2

    x = torch.tensor(x0, dtype=torch.float32, device="cuda", requires_grad=True)
    sigma = torch.tensor(sig0, dtype=torch.float64, requires_grad=True)
    freqs = torch.tensor(f0, dtype=torch.float64, requires_grad=True)
    P = morlet_power_cwt(x, sigma, freqs, fs, norm)
    assert P.dtype == torch.float32 and P.shape == (B, F, n)
    L = ((P.double().cpu() - target) ** 2).mean()
    L.backward()

    xr = torch.tensor(x0.astype(np.float32).astype(np.float64), requires_grad=True)
    sr = torch.tensor(sig0, dtype=torch.float64, requires_grad=True)
    fr = torch.tensor(f0, dtype=torch.float64, requires_grad=True)
    Pr = ref_forward(xr, sr, fr, fs, norm).abs() ** 2
    Lr = ((Pr - target) ** 2).mean()
    Lr.backward()

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    assert rel(P.detach().cpu().double(), Pr.detach()) < 2e-5
    assert rel(x.grad.cpu().double(), xr.grad) < 1e-4
    assert abs(float(sigma.grad) - float(sr.grad)) <= 1e-4 * abs(float(sr.grad)) + 1e-12
    assert float(torch.max(torch.abs(freqs.grad - fr.grad)) / torch.max(torch.abs(fr.grad))) < 1e-4

    def L_at(sv):
        with torch.no_grad():
            p = ref_forward(xr.detach(), torch.tensor(sv, dtype=torch.float64), fr.detach(), fs, norm).abs() ** 2
            return float(((p - target) ** 2).mean())
    h = 1e-6
    fd = (L_at(sig0 + h) - L_at(sig0 - h)) / (2 * h)
    assert abs(float(sigma.grad) - fd) <= 1e-4 * abs(fd) + 1e-10


def test_power_layer_module():
    import torch

    from fcwt_b200.autograd import LearnableMorletCWT

    n, fs = 4096, 1000.0
    t = np.arange(n) / fs
    x = torch.tensor(np.sin(2 * np.pi * 40 * t), dtype=torch.float32, device="cuda").reshape(1, n)
    lp = LearnableMorletCWT([30.0, 55.0], fs, sigma=2.0, power=True)
    lc = LearnableMorletCWT([30.0, 55.0], fs, sigma=2.0)
    P = lp(x)
    y = lc(x)
    assert torch.allclose(P.detach(), y.detach().abs() ** 2, rtol=1e-5, atol=1e-7 * float(P.detach().max()))
    (-P.mean()).backward()
    assert float(lp.freqs.grad[0]) < 0 < float(lp.freqs.grad[1])
