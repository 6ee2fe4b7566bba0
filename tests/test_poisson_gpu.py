"""The Poisson path: Jacobi sweeps (the 3D TMA stencil kernel with a
right-hand side) and the FP64 residual against the FP64 oracle, and the
defect-correction solve reaching its tolerance as checked by the oracle."""
import numpy as np
import pytest
import torch

import oracle
from ssam_b200.workloads import gaussian_rhs
import ssam_b200 as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,rel", [(torch.float64, 1e-12), (torch.float32, 1e-5),
                                       (torch.bfloat16, 2.0**-8)])
@pytest.mark.parametrize("n,nb,sweeps", [(16, 3, 1), (16, 3, 2), (24, 2, 5), (17, 1, 3)])
def test_jacobi_sweeps_vs_oracle(cuda, dtype, rel, n, nb, sweeps):
    f = gaussian_rhs(nb, n, n * 10 + sweeps)
    u0 = np.random.Generator(np.random.PCG64(n)).standard_normal(f.shape) * 1e-3
    ft = torch.from_numpy(f).to(dtype).to(cuda)
    ut = torch.from_numpy(u0).to(dtype).to(cuda)
    got = S.poisson_jacobi(ft, ut, sweeps).double().cpu().numpy()
    # the oracle sees the same rounded inputs
    want = oracle.jacobi7(ft.double().cpu().numpy(), ut.double().cpu().numpy(), sweeps)
    h2 = 1.0 / (n + 1) ** 2
    scale = np.abs(want) + h2 * np.abs(f).max() / 6 + np.abs(u0).max()
    err = np.abs(got - want) / scale
    assert err.max() <= rel * sweeps, err.max()


def test_residual_vs_oracle(cuda):
    f = gaussian_rhs(3, 20, 1)
    u = np.random.Generator(np.random.PCG64(2)).standard_normal(f.shape) * 1e-4
    rel = S.poisson_residual(torch.from_numpy(f).to(cuda), torch.from_numpy(u).to(cuda))
    _, want = oracle.residual7(f, u)
    np.testing.assert_allclose(rel, want, rtol=1e-12)


@pytest.mark.parametrize("sweep_dtype", ["f32", "bf16"])
def test_defect_correction_reaches_tolerance(cuda, sweep_dtype):
    n, nb = 24, 2
    f = gaussian_rhs(nb, n, 7)
    ft = torch.from_numpy(f).to(cuda)
    u = torch.zeros_like(ft)
    st = S.poisson_solve(ft, u, tol=1e-5, sweep_dtype=sweep_dtype, sweeps_per_correction=200,
                         max_sweeps=20000)
    assert st["converged"] == 1, st
    assert st["rel_residual"] <= 1e-5
    _, rel = oracle.residual7(f, u.cpu().numpy())
    assert rel.max() <= 1.0001e-5, rel


def test_learned_solve_with_untrained_network_falls_back_and_converges(cuda):
    """A random network's corrections do not lower the residual: the solve
    rejects them, turns the network off and still reaches the tolerance."""
    n, nb = 32, 2
    f = gaussian_rhs(nb, n, 8)
    ft = torch.from_numpy(f).to(cuda)
    net = S.WarmStartCNN(n, nb, seed=3)
    u = torch.zeros_like(ft)
    st = S.poisson_solve(ft, u, tol=1e-5, sweep_dtype="bf16", sweeps_per_correction=300,
                         max_sweeps=40000, cnn=net)
    assert st["converged"] == 1, st
    _, rel = oracle.residual7(f, u.cpu().numpy())
    assert rel.max() <= 1.0001e-5, rel


def test_learned_solve_rejects_bad_arguments(cuda):
    n = 32
    ft = torch.from_numpy(gaussian_rhs(2, n, 1)).to(cuda)
    for net in (S.WarmStartCNN(64, 2, seed=0), S.WarmStartCNN(n, 1, seed=0)):
        with pytest.raises(S.SsamError):  # built for another n / fewer right-hand sides
            S.poisson_solve(ft, torch.zeros_like(ft), cnn=net)
        net.close()


def test_trained_network_beats_the_plain_method(cuda):
    """The committed network (trained on the GPU by the library's own kernels
    on plain-solver pairs) against plain FP32 Jacobi defect correction on
    right-hand sides it never saw: both reach 1e-5 (FP64-checked by the
    oracle), the learned arm with a tenth of the sweeps and in under a third
    of the time."""
    import os
    import time
    from ssam_b200.workloads import gaussian_rhs_torch
    n, nb = 128, 8
    f = gaussian_rhs_torch(nb, n, 31, cuda)
    net = S.WarmStartCNN(n, nb)
    net.load(os.path.join(os.path.dirname(S.__file__), "data", "poisson_cnn_n128.bin"))
    arms = {"plain": dict(sweep_dtype="f32", sweeps_per_correction=2000, omega=1.0),
            "learned": dict(sweep_dtype="bf16", sweeps_per_correction=250, omega=0.8,
                            cnn_smoothing=2, cnn=net)}
    out = {}
    for name, kw in arms.items():
        u = torch.zeros_like(f)
        S.poisson_solve(f, u, tol=1e-5, max_sweeps=100000, **kw)  # warm-up
        u.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = S.poisson_solve(f, u, tol=1e-5, max_sweeps=100000, **kw)
        torch.cuda.synchronize()
        out[name] = (time.perf_counter() - t0, st)
        assert st["converged"] == 1, (name, st)
        _, rel = oracle.residual7(f.cpu().numpy(), u.cpu().numpy())
        assert rel.max() <= 1.0001e-5, (name, rel)
    (tp, sp), (tl, sl) = out["plain"], out["learned"]
    assert sl["cnn_corrections"] >= 3 and sl["fell_back"] == 0, sl
    assert sl["sweeps"] * 10 <= sp["sweeps"], (sl, sp)
    assert tl * 3 <= tp, (tl, tp)
    net.close()
