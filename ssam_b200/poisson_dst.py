"""Exact discrete Poisson solutions for training the warm-start network.

The 7-point operator A u = (6 u - sum of the 6 neighbours) / h^2 with zero
Dirichlet values outside the n^3 interior is diagonalised by the type-I
discrete sine transform along each axis: mode sin(pi k i / (n+1)) has the
eigenvalue (2 - 2 cos(pi k / (n+1))) / h^2 per axis.  So A^-1 f =
DST^-1 (DST(f) / lambda), with DST-I computed from an FFT of the odd
extension [0, x, 0, -reverse(x)] of length 2(n+1).  Used only to generate
training targets (f, A^-1 f); the solver itself never calls it.
"""
from __future__ import annotations

import math


def _dst1(x, dim: int):
    import torch
    n = x.shape[dim]
    zero = torch.zeros_like(x.narrow(dim, 0, 1))
    ext = torch.cat([zero, x, zero, -torch.flip(x, [dim])], dim)
    # rfft(ext)_k = -2i sum_j x_j sin(pi j k / (n+1)), k = 1..n
    return -torch.fft.rfft(ext, dim=dim).imag.narrow(dim, 1, n)


def solve(f):
    """u = A^-1 f for f of shape (nb, n, n, n), float64, on f's device."""
    import torch
    n = f.shape[-1]
    assert f.shape[-3:] == (n, n, n)
    h = 1.0 / (n + 1)
    k = torch.arange(1, n + 1, dtype=torch.float64, device=f.device)
    lam1 = (2.0 - 2.0 * torch.cos(math.pi * k / (n + 1))) / (h * h)
    lam = lam1[:, None, None] + lam1[None, :, None] + lam1[None, None, :]
    t = f
    for d in (1, 2, 3):
        t = _dst1(t, d)
    # the transform above (twice the DST-I sum) applied twice is 2 (n+1)
    # times the identity per axis
    t = t / lam
    for d in (1, 2, 3):
        t = _dst1(t, d)
    return t / (2.0 * (n + 1)) ** 3


def random_spectrum_rhs(nb: int, n: int, seed: int, device="cuda"):
    """Right-hand sides with random sine-mode spectra: coefficient N(0,1) *
    |k|^-alpha * exp(-|k|^2 / (2 kc^2)) per mode, alpha ~ U[0, 2] and kc
    log-uniform in [4, 32] per sample, unit RMS.  These are the inputs the
    network meets inside defect correction: residuals after smoothing sweeps
    have lost their high-frequency part (the cut-off kc) and carry whatever
    smooth error the previous correction left (the power law), unlike the
    localised Gaussian bumps of the benchmark's right-hand sides."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    k = torch.arange(1, n + 1, dtype=torch.float64, device=device)
    kk2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    out = torch.empty((nb, n, n, n), dtype=torch.float64, device=device)
    for b in range(nb):
        u2 = torch.rand(2, generator=g, dtype=torch.float64, device=device).tolist()
        alpha = 2.0 * u2[0]
        kc = 4.0 * 8.0 ** u2[1]
        coef = torch.randn((n, n, n), generator=g, dtype=torch.float64, device=device)
        coef = coef * kk2 ** (-alpha / 2) * torch.exp(-kk2 / (2 * kc * kc))
        t = coef[None]
        for d in (1, 2, 3):
            t = _dst1(t, d)
        t = t[0]
        out[b] = t / t.pow(2).mean().sqrt()
    return out
