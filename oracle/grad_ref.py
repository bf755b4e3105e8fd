"""Float64 torch.fft restatement of the differentiable Morlet CWT. TEST
INFRASTRUCTURE ONLY: the yardstick of the differentiable form's forward
values and gradients (tests/ and bench.py's parity check import it; the
product never does).

Operator (the continuous-Morlet form of the reference's daughter product,
src/fcwt/fcwt.cpp:197-275, followed by the inverse FFT and normalisation of
fcwt.cpp:418-445):

    y[b, i, t] = c * IFFT_N( FFT_N(x_b) * g_i )[t],   t < n,
    g_i(q) = A * exp(-u^2 / 2),   u = 2*pi*sigma*(fs/f_i * q/N - 1),  q < N/2,

with A the mother table's amplitude sqrt(2 pi) * IPI4 (src/fcwt/fcwt.h:59-61)
and c = 1/N when normalising. Gradients come from torch autograd in float64.
"""
from __future__ import annotations

import math

AMP = math.sqrt(2 * math.pi) * 0.75112554446


def ref_forward(x, sigma, freqs, fs, norm=True):
    """x [B, n] float64 tensor, sigma scalar tensor, freqs [F] tensor (Hz)."""
    import torch

    B, n = x.shape
    N = 1 << int(math.ceil(math.log2(n))) if n > 1 else 1
    X = torch.fft.fft(x, n=N)
    q = torch.arange(N // 2, dtype=torch.float64, device=x.device)
    s = fs / freqs
    u = 2 * math.pi * sigma * (s[:, None] * q[None, :] / N - 1)
    g = AMP * torch.exp(-0.5 * u * u)
    Z = torch.zeros((B, freqs.numel(), N), dtype=torch.complex128, device=x.device)
    Z[..., : N // 2] = X[:, None, : N // 2] * g[None]
    y = torch.fft.ifft(Z)
    if not norm:
        y = y * N
    return y[..., :n]


def power_mse(y, target):
    """The scalogram loss of the differentiable workload: MSE(|y|^2, target)."""
    return ((y.real ** 2 + y.imag ** 2 - target) ** 2).mean()
