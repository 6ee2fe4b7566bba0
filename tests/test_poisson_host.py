"""Host-side pieces of the learned Poisson arm: the device RHS generator
matches the numpy one, and the sine-transform solve that makes the training
targets gives the exact discrete solution (checked by the FP64 oracle)."""
import numpy as np
import pytest
import torch

import oracle
from ssam_b200 import poisson_dst
from ssam_b200.workloads import gaussian_rhs, gaussian_rhs_torch


@pytest.mark.parametrize("nb,n,seed", [(1, 8, 0), (3, 17, 5), (2, 32, 100000)])
def test_torch_rhs_matches_numpy(nb, n, seed):
    np.testing.assert_allclose(gaussian_rhs_torch(nb, n, seed, "cpu").numpy(),
                               gaussian_rhs(nb, n, seed), rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("n", [5, 16, 31])
def test_sine_transform_solve_is_exact(n):
    f = gaussian_rhs(2, n, n)
    u = poisson_dst.solve(torch.from_numpy(f)).numpy()
    _, rel = oracle.residual7(f, u)
    assert rel.max() < 1e-12, rel


def test_sine_transform_solve_matches_converged_jacobi():
    n = 10
    f = gaussian_rhs(1, n, 2)
    u = poisson_dst.solve(torch.from_numpy(f)).numpy()
    uj = oracle.jacobi7(f, np.zeros_like(f), 3000)
    np.testing.assert_allclose(uj, u, rtol=0, atol=1e-10 * np.abs(u).max())


def test_random_spectrum_rhs_is_unit_rms_and_seeded():
    a = poisson_dst.random_spectrum_rhs(2, 12, 4, "cpu")
    b = poisson_dst.random_spectrum_rhs(2, 12, 4, "cpu")
    assert torch.equal(a, b)
    np.testing.assert_allclose(a.pow(2).mean(dim=(1, 2, 3)).numpy(), 1.0, rtol=1e-12)
    u = poisson_dst.solve(a).numpy()
    _, rel = oracle.residual7(a.numpy(), u)
    assert rel.max() < 1e-12
