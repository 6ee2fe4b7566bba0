"""The warm-start CNN's tensor-core kernels against PyTorch CPU float64
(the oracle for the learned component; no reference code exists for it)."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

import ssam_b200 as S

pytestmark = pytest.mark.gpu

TAPS = [(kz, ky, kx) for kz in range(3) for ky in range(3) for kx in range(3)]


def to_torch_weight(w):
    """(16, 27, cin) tap-major -> torch (16, cin, 3, 3, 3)."""
    co, _, ci = w.shape
    out = torch.zeros(co, ci, 3, 3, 3, dtype=torch.float64)
    for t, (kz, ky, kx) in enumerate(TAPS):
        out[:, :, kz, ky, kx] = w[:, t, :].double()
    return out


def ref_conv(xs, w, dil):
    """float64 CPU conv3d of channels-last inputs (concatenated)."""
    x = torch.cat([a.double() for a in xs], dim=-1).permute(0, 4, 1, 2, 3)
    y = F.conv3d(x, to_torch_weight(w), padding=dil, dilation=dil)
    return y.permute(0, 2, 3, 4, 1)


@pytest.mark.parametrize("nsrc", [1, 2])
@pytest.mark.parametrize("n,dil", [(32, 1), (16, 1), (32, 2), (64, 4)])
def test_conv3d_forward_vs_torch_cpu(cuda, nsrc, n, dil):
    g = torch.Generator().manual_seed(n * 10 + dil + nsrc)
    nb = 2
    xs = [torch.randn(nb, n, n, n, 16, generator=g).to(torch.bfloat16) for _ in range(nsrc)]
    w = (torch.randn(16, 27, 16 * nsrc, generator=g) * 0.1).to(torch.bfloat16)
    out = S.cnn_conv3d(xs[0].to(cuda), w.to(cuda), xs[1].to(cuda) if nsrc == 2 else None,
                       dilation=dil, scale=0.5)
    S.device_status()
    got = out.double().cpu()
    want = 0.5 * ref_conv(xs, w, dil)
    mag = 0.5 * ref_conv([a.abs() for a in xs], w.abs(), dil)
    # a second source is a second pass that adds the first pass's BF16
    # result: one more BF16 rounding, of the second source's part
    part = 0.5 * ref_conv(xs[1:], w[:, :, 16:], dil).abs() if nsrc == 2 else 0.0
    err = (got - want).abs() - (2.0**-8 * (want.abs() + part) + 1e-5 * mag)
    assert err.max().item() <= 0, f"max excess {err.max().item()}"


@pytest.mark.parametrize("nsrc", [1, 2])
@pytest.mark.parametrize("n,dil", [(128, 1), (64, 2), (32, 8), (8, 8)])
def test_conv3d_forward_planes_at_network_sizes(cuda, nsrc, n, dil):
    """The level sizes and dilations the network runs (n = 128 at the top,
    dilation 8 at the bottom, dilations >= n where every off-centre tap is
    outside the grid), checked on a few output planes."""
    g = torch.Generator().manual_seed(n + 100 * dil + nsrc)
    xs = [torch.randn(1, n, n, n, 16, generator=g).to(torch.bfloat16) for _ in range(nsrc)]
    w = (torch.randn(16, 27, 16 * nsrc, generator=g) * 0.1).to(torch.bfloat16)
    out = S.cnn_conv3d(xs[0].to(cuda), w.to(cuda), xs[1].to(cuda) if nsrc == 2 else None,
                       dilation=dil, scale=1.0).double().cpu()
    x = torch.cat([a.double() for a in xs], dim=-1).permute(0, 4, 1, 2, 3)
    xp = F.pad(x, (dil,) * 6)
    wt = to_torch_weight(w)
    for z in sorted({0, 1, n // 2, n - 1}):
        sl = xp[:, :, z:z + 2 * dil + 1]
        want = F.conv3d(sl, wt, dilation=dil)[0, :, 0].permute(1, 2, 0)
        mag = F.conv3d(sl.abs(), wt.abs(), dilation=dil)[0, :, 0].permute(1, 2, 0)
        part = 0.0
        if nsrc == 2:  # the second pass's extra BF16 rounding of source 1's part
            part = F.conv3d(sl[:, 16:], wt[:, 16:], dilation=dil)[0, :, 0].permute(1, 2, 0).abs()
        err = (out[0, z] - want).abs() - (2.0**-8 * (want.abs() + part) + 1e-5 * mag)
        assert err.max().item() <= 0, f"plane {z}: max excess {err.max().item()}"


def test_conv3d_gather_kernel_vs_torch_cpu(cuda):
    """The register-gather kernel (used where the TMA kernel's plan does not
    fit) on the same check, forced by SSAM_CONV_GATHER=1 in a child process."""
    import os
    import subprocess
    import sys
    code = (
        "import torch, torch.nn.functional as F, ssam_b200 as S\n"
        "g = torch.Generator().manual_seed(5)\n"
        "x = torch.randn(2, 16, 16, 16, 16, generator=g).to(torch.bfloat16)\n"
        "w = (torch.randn(16, 27, 16, generator=g) * 0.1).to(torch.bfloat16)\n"
        "out = S.cnn_conv3d(x.cuda(), w.cuda(), None, dilation=2, scale=1.0).double().cpu()\n"
        "wt = torch.zeros(16, 16, 3, 3, 3, dtype=torch.float64)\n"
        "for t in range(27): wt[:, :, t // 9, (t // 3) % 3, t % 3] = w[:, t, :].double()\n"
        "want = F.conv3d(x.double().permute(0, 4, 1, 2, 3), wt, padding=2, dilation=2)"
        ".permute(0, 2, 3, 4, 1)\n"
        "mag = F.conv3d(x.double().abs().permute(0, 4, 1, 2, 3), wt.abs(), padding=2,"
        " dilation=2).permute(0, 2, 3, 4, 1)\n"
        "err = (out - want).abs() - (2.0**-8 * want.abs() + 1e-5 * mag)\n"
        "assert err.max().item() <= 0, err.max().item()\n"
        "print('ok')\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, SSAM_CONV_GATHER="1", PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("nsrc", [1, 2])
@pytest.mark.parametrize("n,dil", [(16, 1), (32, 1), (32, 2)])
def test_conv3d_weight_grad_vs_torch_autograd(cuda, nsrc, n, dil):
    g = torch.Generator().manual_seed(n + dil * 7 + nsrc)
    nb = 2
    xs = [torch.randn(nb, n, n, n, 16, generator=g).to(torch.bfloat16) for _ in range(nsrc)]
    go = torch.randn(nb, n, n, n, 16, generator=g).to(torch.bfloat16)
    dw = S.cnn_conv3d_wgrad(xs[0].to(cuda), go.to(cuda), xs[1].to(cuda) if nsrc == 2 else None,
                            dilation=dil).double().cpu()
    # float64 autograd on CPU
    x = torch.cat([a.double() for a in xs], dim=-1).permute(0, 4, 1, 2, 3)
    wt = torch.zeros(16, 16 * nsrc, 3, 3, 3, dtype=torch.float64, requires_grad=True)
    y = F.conv3d(x, wt, padding=dil, dilation=dil)
    y.backward(go.double().permute(0, 4, 1, 2, 3))
    want = torch.stack([wt.grad[:, :, kz, ky, kx] for kz, ky, kx in TAPS], dim=1)
    xa = torch.cat([a.double().abs() for a in xs], dim=-1).permute(0, 4, 1, 2, 3)
    wa = torch.zeros_like(wt, requires_grad=True)
    F.conv3d(xa, wa, padding=dil, dilation=dil).backward(go.double().abs().permute(0, 4, 1, 2, 3))
    mag = torch.stack([wa.grad[:, :, kz, ky, kx] for kz, ky, kx in TAPS], dim=1)
    err = (dw - want).abs() - 1e-4 * mag
    assert err.max().item() <= 0, f"max excess {err.max().item()}"


# ---- the whole network: forward and gradient against a float64 CPU mirror --

LAYERS = [  # (level, nsrc, dilation) in parameter order
    (0, 1, 1), (0, 1, 1), (1, 1, 1), (1, 1, 1), (2, 1, 1), (2, 1, 2), (2, 1, 4), (2, 1, 8),
    (1, 2, 1), (1, 1, 1), (0, 2, 1), (0, 1, 1)]
OUT_SCALE = 0.03


def mirror_loss(params, f, target=None):
    """The network in float64 torch (channels-first); returns (u0, loss)."""
    ws, off = [], 0
    for lvl, nsrc, dil in LAYERS:
        cnt = 16 * 27 * 16 * nsrc
        ws.append(to_torch_weight(params[off:off + cnt].view(16, 27, 16 * nsrc)))
        off += cnt
    wh = params[off:off + 16]
    nb, n = f.shape[0], f.shape[1]
    rms = f.pow(2).mean(dim=(1, 2, 3)).sqrt()
    x = torch.zeros(nb, 16, n, n, n, dtype=torch.float64)
    x[:, 0] = f / rms.view(-1, 1, 1, 1)

    def conv(i, *xs):
        return F.conv3d(torch.cat(xs, 1), ws[i], padding=LAYERS[i][2], dilation=LAYERS[i][2])

    a1 = conv(0, x)
    s1 = conv(1, a1)
    p1 = F.avg_pool3d(s1, 2)
    a2 = conv(2, p1)
    s2 = conv(3, a2)
    p2 = F.avg_pool3d(s2, 2)
    b = conv(7, conv(6, conv(5, conv(4, p2))))
    u2 = F.interpolate(b, scale_factor=2, mode="nearest")
    d2 = conv(9, conv(8, u2, s2))
    u1 = F.interpolate(d2, scale_factor=2, mode="nearest")
    d1 = conv(11, conv(10, u1, s1))
    y = (d1 * wh.view(1, 16, 1, 1, 1)).sum(1)
    scale = (rms * OUT_SCALE).view(-1, 1, 1, 1)
    u0 = y * scale
    loss = None
    if target is not None:
        t = target / scale
        # mean over right-hand sides of the relative squared error
        loss = (((y - t) ** 2).sum(dim=(1, 2, 3)) / (t ** 2).sum(dim=(1, 2, 3))).mean()
    return u0, loss


def test_cnn_forward_and_gradient_vs_float64_mirror(cuda):
    from ssam_b200.workloads import gaussian_rhs
    n, nb = 32, 2
    net = S.WarmStartCNN(n, nb, seed=3)
    f = torch.from_numpy(gaussian_rhs(nb, n, 11))
    target = torch.from_numpy(gaussian_rhs(nb, n, 12)) * 0.01
    w, _ = net.params()
    # the mirror uses the BF16-rounded conv weights the GPU multiplies with
    pw = torch.from_numpy(w).double()
    nconv = net.num_params - 16
    pw[:nconv] = pw[:nconv].to(torch.bfloat16).double()
    pw.requires_grad_(True)
    u_ref, loss_ref = mirror_loss(pw, f, target)
    loss_ref.backward()
    u_gpu = net.forward(f.to(cuda)).cpu()
    rel_u = ((u_gpu - u_ref.detach()).norm() / u_ref.detach().norm()).item()
    assert rel_u < 3e-2, rel_u
    loss = net.gradient(f.to(cuda), target.to(cuda))
    assert abs(loss - loss_ref.item()) <= 3e-2 * loss_ref.item()
    _, g = net.params()
    g_ref = pw.grad.numpy()
    off = 0
    for i, (_, nsrc, _) in enumerate(LAYERS + [(0, 0, 0)]):
        cnt = 16 * 27 * 16 * nsrc if i < len(LAYERS) else 16
        a, b = g[off:off + cnt], g_ref[off:off + cnt]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 5e-2, f"layer {i}: relative gradient error {rel:.3e}"
        off += cnt
    net.close()


def test_cnn_training_reduces_loss_and_roundtrips(cuda, tmp_path):
    from ssam_b200.workloads import gaussian_rhs
    n, nb = 32, 4
    net = S.WarmStartCNN(n, nb, seed=5)
    f = torch.from_numpy(gaussian_rhs(nb, n, 21)).to(cuda)
    u = torch.zeros_like(f)
    S.poisson_solve(f, u, tol=1e-6, sweeps_per_correction=500, max_sweeps=50000)
    first = net.gradient(f, u)
    for _ in range(80):
        net.gradient(f, u)
        net.adam_step(5e-4)
    last = net.gradient(f, u)
    assert last < 0.7 * first, (first, last)
    p = str(tmp_path / "net.bin")
    net.save(p)
    u1 = net.forward(f).clone()
    other = S.WarmStartCNN(n, nb, seed=99)
    other.load(p)
    assert torch.equal(other.forward(f), u1)
    net.close()
    other.close()


@pytest.mark.parametrize("epi", [1, 2])
@pytest.mark.parametrize("issuers", [1, 2, 3, 4])
@pytest.mark.parametrize("ctas", [1, 2])
@pytest.mark.parametrize("nsrc", [1, 2])
@pytest.mark.parametrize("n", [128, 64, 32, 16])
def test_zstack_kernel_equals_27_mma_kernel(cuda, monkeypatch, epi, issuers, ctas, nsrc, n):
    """Dilation 1 runs the kernel that stacks the three z taps of an input
    plane on the MMA's N side (9 MMAs of N = 48 per plane and tile), with one
    or two CTAs a SM (SSAM_CONV_TWO_CTA=1: work items of fewer rows, 256 TMEM
    columns each); every output still sums its taps in the 27-MMA kernel's
    order, so all of them give the same bits (SSAM_CONV_RING27=1 selects the
    27-MMA kernel); likewise with 1 to 4 MMA-issuing warps a CTA
    (SSAM_CONV_ISSUERS) and one or two groups of epilogue warps
    (SSAM_CONV_EPI; two are compiled with 2-4 issuers)."""
    monkeypatch.setenv("SSAM_CONV_TWO_CTA", "1" if ctas == 2 else "0")
    monkeypatch.setenv("SSAM_CONV_ISSUERS", str(issuers))
    monkeypatch.setenv("SSAM_CONV_EPI", str(epi))
    g = torch.Generator().manual_seed(7 * n + nsrc)
    nb = 2 if n <= 64 else 1
    xs = [torch.randn(nb, n, n, n, 16, generator=g).to(torch.bfloat16).to(cuda)
          for _ in range(nsrc)]
    w = (torch.randn(16, 27, 16 * nsrc, generator=g) * 0.1).to(torch.bfloat16).to(cuda)
    args = (xs[0], w, xs[1] if nsrc == 2 else None)
    got = S.cnn_conv3d(*args, dilation=1, scale=0.75)
    monkeypatch.setenv("SSAM_CONV_RING27", "1")
    want = S.cnn_conv3d(*args, dilation=1, scale=0.75)
    S.device_status()
    assert torch.equal(got, want)

