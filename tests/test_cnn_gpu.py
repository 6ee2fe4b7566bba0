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
    err = (got - want).abs() - (2.0**-8 * want.abs() + 1e-5 * mag)
    assert err.max().item() <= 0, f"max excess {err.max().item()}"


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
