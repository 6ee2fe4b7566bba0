"""Seeded synthetic inputs of the benchmark configurations (numpy)."""
from __future__ import annotations

import numpy as np


def gaussian_rhs(nb: int, n: int, seed: int) -> np.ndarray:
    """Poisson right-hand sides, shape (nb, n, n, n), float64: each a sum of
    K ~ U{1..8} Gaussian bumps with centres U[0,1]^3, sigma U[0.03, 0.15] and
    amplitude N(0,1), sampled at the interior points (i+1)h, h = 1/(n+1)."""
    g = np.random.Generator(np.random.PCG64(seed))
    h = 1.0 / (n + 1)
    x = (np.arange(n) + 1) * h
    out = np.zeros((nb, n, n, n))
    for b in range(nb):
        for _ in range(int(g.integers(1, 9))):
            c = g.random(3)
            s = g.uniform(0.03, 0.15)
            a = g.normal()
            gz = np.exp(-(x - c[2]) ** 2 / (2 * s * s))
            gy = np.exp(-(x - c[1]) ** 2 / (2 * s * s))
            gx = np.exp(-(x - c[0]) ** 2 / (2 * s * s))
            out[b] += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return out


def gaussian_rhs_torch(nb: int, n: int, seed: int, device="cuda"):
    """gaussian_rhs with the same parameter draws, evaluated by torch on
    `device` (float64): the training and benchmark sets are generated where
    they are used."""
    import torch
    g = np.random.Generator(np.random.PCG64(seed))
    h = 1.0 / (n + 1)
    x = (torch.arange(n, dtype=torch.float64, device=device) + 1) * h
    out = torch.zeros((nb, n, n, n), dtype=torch.float64, device=device)
    for b in range(nb):
        for _ in range(int(g.integers(1, 9))):
            c = g.random(3)
            s = g.uniform(0.03, 0.15)
            a = g.normal()
            gz = torch.exp(-(x - c[2]) ** 2 / (2 * s * s))
            gy = torch.exp(-(x - c[1]) ** 2 / (2 * s * s))
            gx = torch.exp(-(x - c[0]) ** 2 / (2 * s * s))
            out[b] += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return out
