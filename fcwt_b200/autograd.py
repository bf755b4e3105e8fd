"""Differentiable Morlet CWT for PyTorch.

The reference's daughter wavelet is a lookup mother[(int)(scale/2 * q)]
(src/fcwt/fcwt.cpp:225-240): piecewise constant in the scale, so it has no
useful gradient with respect to frequency. This operator uses the continuous
Morlet instead,

    y[b, i, t] = c * IFFT_N( FFT_N(x_b) * g_i )[t],   t < n,
    g_i(q) = A * exp(-u^2 / 2),   u = 2*pi*sigma*(fs/f_i * q/N - 1),

(A the reference's mother-table amplitude, c = 1/N when normalising, bins
q < N/2 only), evaluated by the same GPU row engine (FCWT_CONTINUOUS), and
differentiates it with hand-written adjoint kernels
(fcwt_morlet_cwt_backward): gradients with respect to the signal, sigma and
every centre frequency. Spectra are recomputed in the backward pass.

`morlet_power_cwt` is the same operator followed by |y|^2, written by the row
kernels' power epilogue (float32, half the bytes of the complex output). Its
backward recomputes y and passes dL/dy = 2 y dL/dP to the same adjoint.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .api import BatchPlan


_PLAN_CACHE: "OrderedDict" = None
_PLAN_CACHE_SIZE = 4


def _plan_for(dev: int, n: int, B: int, sig: float, scales: np.ndarray, norm: bool) -> BatchPlan:
    """Batched continuous-Morlet plan, reused while the shape, bandwidth and
    frequency grid stay the same (evaluation loops, frozen parameters); a
    training step that moves sigma or the frequencies builds a new one."""
    global _PLAN_CACHE
    from collections import OrderedDict

    if _PLAN_CACHE is None:
        _PLAN_CACHE = OrderedDict()
    key = (dev, n, B, float(np.float32(sig)), scales.tobytes(), bool(norm))
    plan = _PLAN_CACHE.get(key)
    if plan is not None:
        _PLAN_CACHE.move_to_end(key)
        return plan
    plan = BatchPlan([n] * B, [scales] * B, fb=sig, norm=norm, device=dev, continuous=True)
    _PLAN_CACHE[key] = plan
    while len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
        _, old = _PLAN_CACHE.popitem(last=False)
        old.close()
    return plan


def _forward(ctx, x, sigma, freqs, fs: float, norm: bool, out_type: int):
    """Runs the transform of x [batch, n] into a new [batch, fn, n] tensor of
    out_type (complex64 or float32 |y|^2) and keeps what the backward needs."""
    if x.dim() != 2 or x.dtype != torch.float32 or not x.is_cuda:
        raise TypeError("x must be a CUDA float32 tensor [batch, n]")
    x = x.contiguous()
    B, n = x.shape
    sig = float(sigma.detach().cpu())
    f = freqs.detach().double().cpu().numpy()
    if np.any(f <= 0) or sig <= 0:
        raise ValueError("sigma and frequencies must be positive")
    scales = (float(fs) / f).astype(np.float32)
    dev = x.device.index or 0
    plan = _plan_for(dev, n, B, sig, scales, norm)
    dtype = torch.complex64 if out_type == _lib.FCWT_OUT_C64 else torch.float32
    y = torch.empty((B, f.size, n), dtype=dtype, device=x.device)
    plan.execute([x[b] for b in range(B)], [y[b] for b in range(B)], out_type=out_type)
    ctx.save_for_backward(x)
    ctx.sig, ctx.f, ctx.fs, ctx.norm, ctx.scales = sig, f, float(fs), bool(norm), scales
    ctx.sigma_like, ctx.freqs_like = sigma, freqs
    return y


def _adjoint(ctx, x, G):
    """(dL/dx, dL/dsigma, dL/dfreqs) for dL/dy = G (complex64 [batch, fn, n])."""
    B, n = x.shape
    F = ctx.f.size
    grad_x = torch.empty_like(x)
    gfb = ctypes.c_double(0.0)
    gf = np.zeros(F, np.float64)
    freqs32 = ctx.f.astype(np.float32)
    c = _lib.context(x.device.index or 0)
    c.set_stream(torch.cuda.current_stream(x.device).cuda_stream)
    try:
        _lib.call("fcwt_morlet_cwt_backward", c.handle, ctypes.c_void_p(x.data_ptr()), n, B,
                  ctypes.c_float(ctx.sig), ctypes.c_void_p(freqs32.ctypes.data), F, ctypes.c_float(ctx.fs),
                  _lib.FCWT_NORM if ctx.norm else 0, ctypes.c_void_p(G.data_ptr()),
                  ctypes.c_void_p(grad_x.data_ptr()), ctypes.byref(gfb), ctypes.c_void_p(gf.ctypes.data))
    finally:
        c.set_stream(None)
    gs = torch.tensor(gfb.value, dtype=ctx.sigma_like.dtype, device=ctx.sigma_like.device).reshape(
        ctx.sigma_like.shape)
    gfr = torch.from_numpy(gf).to(dtype=ctx.freqs_like.dtype, device=ctx.freqs_like.device)
    return grad_x, gs, gfr


class MorletCWTFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, sigma, freqs, fs: float, norm: bool = True):
        return _forward(ctx, x, sigma, freqs, fs, norm, _lib.FCWT_OUT_C64)

    @staticmethod
    def backward(ctx, grad_y):
        (x,) = ctx.saved_tensors
        grad_x, gs, gfr = _adjoint(ctx, x, grad_y.contiguous().to(torch.complex64))
        return grad_x, gs, gfr, None, None


class MorletPowerFunction(torch.autograd.Function):
    """P = |y|^2 of the continuous-Morlet transform (float32 [batch, fn, n])."""

    @staticmethod
    def forward(ctx, x, sigma, freqs, fs: float, norm: bool = True):
        return _forward(ctx, x, sigma, freqs, fs, norm, _lib.FCWT_OUT_POWER)

    @staticmethod
    def backward(ctx, grad_p):
        (x,) = ctx.saved_tensors
        B, n = x.shape
        plan = _plan_for(x.device.index or 0, n, B, ctx.sig, ctx.scales, ctx.norm)
        y = torch.empty((B, ctx.f.size, n), dtype=torch.complex64, device=x.device)
        plan.execute([x[b] for b in range(B)], [y[b] for b in range(B)])
        # dL/dy of L(|y|^2) in torch's convention for complex inputs: 2 y dL/dP
        yr = torch.view_as_real(y)
        yr.mul_((2.0 * grad_p.to(torch.float32)).unsqueeze(-1))
        grad_x, gs, gfr = _adjoint(ctx, x, y)
        return grad_x, gs, gfr, None, None


def morlet_cwt(x, sigma, freqs, fs: float, norm: bool = True):
    """y[b, i, t] for signals x [batch, n] (CUDA float32), a scalar tensor
    sigma and centre frequencies freqs [fn] (Hz) at sample rate fs."""
    return MorletCWTFunction.apply(x, sigma, freqs, fs, norm)


def morlet_power_cwt(x, sigma, freqs, fs: float, norm: bool = True):
    """|y[b, i, t]|^2 (float32) of morlet_cwt, from the row kernels' power
    epilogue; differentiable in x, sigma and freqs."""
    return MorletPowerFunction.apply(x, sigma, freqs, fs, norm)


class LearnableMorletCWT(torch.nn.Module):
    """CWT layer with a learnable Morlet bandwidth and centre frequencies;
    power=True returns the scalogram |y|^2 (float32) instead of y."""

    def __init__(self, freqs, fs: float, sigma: float = 2.0, norm: bool = True, power: bool = False):
        super().__init__()
        self.sigma = torch.nn.Parameter(torch.tensor(float(sigma), dtype=torch.float64))
        self.freqs = torch.nn.Parameter(torch.as_tensor(freqs, dtype=torch.float64).clone())
        self.fs = float(fs)
        self.norm = norm
        self.power = power

    def forward(self, x):
        f = morlet_power_cwt if self.power else morlet_cwt
        return f(x, self.sigma, self.freqs, self.fs, self.norm)
