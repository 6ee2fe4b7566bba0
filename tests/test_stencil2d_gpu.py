"""Parity of the sm_100a 2D stencil / convolution kernels with the oracle.

Like the reference's own Test() drivers (stencil2D_9pt.cu:175-182,
conv2D.cu:149-159) each case runs the GPU path and the CPU golden on the same
input and compares them -- here on seeded inputs and with a pass/fail bound:

* integer inputs and integer coefficients (the reference's star tables and
  conv weights) make every partial sum exact, so FP32 and FP64 must agree
  BIT FOR BIT whatever the summation order;
* real coefficients: |gpu - oracle| <= rel * sum|w||x| per cell with
  rel = 1e-5 (FP32) and 1e-12 (FP64);
* BF16 / F16 storage: compared with the FP64 oracle on the same rounded
  input; the bound is one rounding of the stored result plus FP32
  accumulation, |err| <= 2^-8 (BF16) or 2^-11 (F16) times max(|out|, scale).
"""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_cases import (assert_rel_close, golden, magnitude2d, normalised, rng,
                        stable_seed, star_matrix, table2d, uniform)

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64}
REL = {np.float32: 1e-5, np.float64: 1e-12}


def dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ---------------------------------------------------------- known answers --

@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("r", range(1, 7))
def test_star_tables_bit_exact(cuda, tag, r):
    """The reference's 5..25-pt star tables on 0..255 integer input."""
    g = golden()
    t = table2d(f"star{r}")
    out = S.stencil2d(dev(g[f"int_in_{tag}"], cuda), S.star_coeffs_from_matrix(t), r, S.STAR)
    np.testing.assert_array_equal(host(out), g[f"star{r}_out_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("f", ["2", "3", "4", "5", "6", "7", "11", "21", "3x5", "4x2", "1x7"])
def test_conv_integer_weights_bit_exact(cuda, tag, f):
    """conv2D.cu's rand()%21-10 weights on an integer image: exact sums."""
    g = golden()
    out = S.conv2d(dev(g[f"int_in_{tag}"], cuda), g[f"conv{f}_w_{tag}"])
    np.testing.assert_array_equal(host(out), g[f"conv{f}_out_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("name", ["box64", "box81", "box121"])
def test_box_tables_vs_golden(cuda, tag, name):
    g = golden()
    dt = DT[tag]
    t = table2d(name)
    src = g[f"uni_in_{tag}"]
    out = S.stencil2d(dev(src, cuda), t.ravel(), len(t) // 2, S.BOX)
    assert_rel_close(host(out), g[f"{name}_out_{tag}"], magnitude2d(src, t), REL[dt], name)


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("name,steps", [("tmp5", 5), ("tmp9", 3)])
def test_temporal_tables_vs_golden(cuda, tag, name, steps):
    """stencil2d_temp_5pt/9pt: ITERATIVE_COUNT steps, zero-padded golden."""
    g = golden()
    dt = DT[tag]
    t = table2d(name)
    r = len(t) // 2
    src = g[f"tmp_in_{tag}"]
    out = S.stencil2d(dev(src, cuda), S.star_coeffs_from_matrix(t), r, S.STAR, steps=steps)
    assert_rel_close(host(out), g[f"{name}_out_{tag}"], magnitude2d(src, t, steps=steps),
                     REL[dt] * steps, name)


# ------------------------------------------------- seeded random families --

SHAPES = [(1, 1), (1, 7), (7, 1), (3, 200), (17, 33), (64, 64), (131, 257), (300, 1000)]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind,r", [("star", 1), ("star", 3), ("star", 6), ("box", 1),
                                    ("box", 2), ("box", 3), ("box", 5)])
@pytest.mark.parametrize("bnd", ["zero", "copy", "clamp"])
def test_stencil_family_vs_oracle(cuda, dt, shape, kind, r, bnd):
    seed = stable_seed(shape, kind, r, bnd, dt.__name__)
    src = uniform(shape, -1, 1, dt, seed)
    f = 2 * r + 1
    if kind == "star":
        c = normalised((4 * r + 1,), seed + 1)
        m = star_matrix(c, r)
        out = S.stencil2d(dev(src, cuda), c, r, S.STAR, boundary=bnd)
    else:
        m = normalised((f, f), seed + 1)
        out = S.stencil2d(dev(src, cuda), m.ravel(), r, S.BOX, boundary=bnd)
    want = oracle.conv2d(src, m.astype(dt), bnd)
    assert_rel_close(host(out), want, magnitude2d(src, m, bnd), REL[dt], f"{kind}{r}/{bnd}")


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("f", [1, 2, 3, 8, 9, 13, 15, 19, 21, 24, 28])
def test_conv_sizes_vs_oracle(cuda, dt, f):
    src = uniform((97, 211), -1, 1, dt, f)
    w = normalised((f, f), f + 100)
    out = S.conv2d(dev(src, cuda), w)
    assert_rel_close(host(out), oracle.conv2d(src, w.astype(dt)), magnitude2d(src, w),
                     REL[dt], f"conv{f}")


@pytest.mark.parametrize("fh,fw", [(1, 3), (3, 1), (2, 5), (5, 2), (6, 3), (7, 12), (28, 1)])
def test_conv_non_square_vs_oracle(cuda, fh, fw):
    src = uniform((45, 77), -1, 1, np.float32, fh * 31 + fw)
    w = rng(fh * 7 + fw).uniform(-1, 1, size=(fh, fw))
    out = S.conv2d(dev(src, cuda), w)
    assert_rel_close(host(out), oracle.conv2d(src, w.astype(np.float32)), magnitude2d(src, w),
                     1e-5, f"conv{fh}x{fw}")


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("kind,r", [("star", 1), ("box", 1), ("star", 2), ("box", 2), ("box", 3)])
@pytest.mark.parametrize("steps", [2, 3, 4, 5, 8, 16])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_multistep_vs_oracle(cuda, dt, kind, r, steps, bnd):
    """Temporal blocking (steps fused in registers) and launch chaining."""
    shape = (150, 333)
    seed = stable_seed(kind, r, steps, bnd)
    src = uniform(shape, 0, 1, dt, seed)
    f = 2 * r + 1
    if kind == "star":
        c = normalised((4 * r + 1,), seed + 1)
        m = star_matrix(c, r)
        out = S.stencil2d(dev(src, cuda), c, r, S.STAR, steps=steps, boundary=bnd)
    else:
        m = normalised((f, f), seed + 1)
        out = S.stencil2d(dev(src, cuda), m.ravel(), r, S.BOX, steps=steps, boundary=bnd)
    want = oracle.conv2d(src, m.astype(dt), bnd, steps=steps)
    assert_rel_close(host(out), want, magnitude2d(src, m, bnd, steps), REL[dt] * steps,
                     f"{kind}{r}x{steps}/{bnd}")


def test_pitched_and_unaligned_grids(cuda):
    """pitch > width (conv2D's cudaMalloc3D rows) and a base that is not
    16-byte aligned: both must give the dense result."""
    h, w, pitch = 61, 100, 131
    base = uniform((h, pitch), -1, 1, np.float32, 77)
    m = normalised((5, 5), 78)
    want = oracle.conv2d(np.ascontiguousarray(base[:, :w]), m.astype(np.float32))
    scale = magnitude2d(np.ascontiguousarray(base[:, :w]), m)
    t = dev(base, cuda)
    out = S.stencil2d(t[:, :w], m.ravel(), 2, S.BOX)
    assert_rel_close(host(out)[:, :w], want, scale, 1e-5, "pitched")
    # unaligned: a view starting one element in
    flat = dev(uniform((h * w + 1,), -1, 1, np.float32, 79), cuda)
    view = flat[1:].view(h, w)
    srcu = view.cpu().numpy()
    out = S.stencil2d(view, m.ravel(), 2, S.BOX)
    assert_rel_close(host(out), oracle.conv2d(srcu, m.astype(np.float32)),
                     magnitude2d(srcu, m), 1e-5, "unaligned")


# ------------------------------------------------------- 16-bit storage --

@pytest.mark.parametrize("tdt,rel", [(torch.bfloat16, 2.0**-8), (torch.float16, 2.0**-11)])
@pytest.mark.parametrize("kind,r,steps", [("star", 1, 1), ("box", 2, 1), ("box", 5, 1),
                                          ("star", 1, 4), ("box", 1, 8)])
def test_half_storage_vs_fp64_oracle(cuda, tdt, rel, kind, r, steps):
    shape = (123, 517)
    seed = stable_seed(kind, r, steps)
    src32 = uniform(shape, 0, 1, np.float32, seed)
    t = torch.from_numpy(src32).to(tdt)
    src64 = t.double().numpy()
    f = 2 * r + 1
    if kind == "star":
        c = normalised((4 * r + 1,), seed + 1)
        m = star_matrix(c, r)
    else:
        m = normalised((f, f), seed + 1)
        c = m.ravel()
    out = S.stencil2d(t.to(cuda), c, r, S.STAR if kind == "star" else S.BOX, steps=steps,
                      boundary="copy")
    got = host(out.double())
    want = oracle.conv2d(src64, m, "copy", steps=steps)
    scale = np.maximum(np.abs(want), magnitude2d(src64, m, "copy", steps))
    # one storage rounding per step, plus FP32 accumulation
    assert_rel_close(got, want, scale, rel * steps + 1e-5, f"{tdt}/{kind}{r}x{steps}")


# ------------------------------------------------- full benchmark sizes --

def test_config1_5pt_4096_copy_boundary(cuda):
    """5-pt, c=n=s=w=e=0.2, 4096^2 uniform[0,1), boundary copied, 1 step,
    checked against the reference golden on every cell."""
    n = 4096
    src = uniform((n, n), 0, 1, np.float32, 4096)
    c = [0.2] * 5
    out = host(S.stencil2d(dev(src, cuda), c, 1, S.STAR, boundary="copy"))
    m = star_matrix(c, 1)
    want = oracle.conv2d(src, m.astype(np.float32), "copy")
    assert_rel_close(out, want, magnitude2d(src, m, "copy"), 1e-5, "config1")


def _slab_check(out, src, m, rows, dt, what):
    """Compare sampled rows of a full-size result with the oracle run on the
    row slab around them (rows far from the slab edge are exact stand-ins)."""
    r = m.shape[0] // 2
    for y in rows:
        lo, hi = max(0, y - r), min(src.shape[0], y + r + 1)
        slab = np.ascontiguousarray(src[lo:hi])
        want = oracle.conv2d(slab, m.astype(dt))[y - lo]
        scale = magnitude2d(slab, m)[y - lo]
        assert_rel_close(out[y], want, scale, REL[dt], f"{what} row {y}")


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("r", [1, 2, 3, 4, 5])
def test_config2_box_8192_sampled_rows(cuda, dt, r):
    n = 8192
    src = uniform((n, n), -1, 1, dt, 8192 + r)
    f = 2 * r + 1
    m = normalised((f, f), r)
    out = host(S.stencil2d(dev(src, cuda), m.ravel(), r, S.BOX))
    rows = [0, 1, r, n // 2, n - 2, n - 1] + list(rng(r).integers(0, n, 4))
    _slab_check(out, src, m, rows, dt, f"box{r}")


def test_config2_linearity_8192(cuda):
    """S(a x + b y) = a S(x) + b S(y) on the whole 8192^2 grid (FP64)."""
    n = 8192
    x = torch.rand(n, n, dtype=torch.float64, device=cuda) * 2 - 1
    y = torch.rand(n, n, dtype=torch.float64, device=cuda) * 2 - 1
    m = normalised((7, 7), 1).ravel()
    sx = S.stencil2d(x, m, 3, S.BOX)
    sy = S.stencil2d(y, m, 3, S.BOX)
    sxy = S.stencil2d(0.25 * x + 1.5 * y, m, 3, S.BOX)
    err = (sxy - (0.25 * sx + 1.5 * sy)).abs().max().item()
    assert err < 1e-12


def test_config2_conv21_8192_sampled_rows(cuda):
    n = 8192
    src = uniform((n, n), -1, 1, np.float32, 21)
    w = normalised((21, 21), 21)
    out = host(S.conv2d(dev(src, cuda), w))
    _slab_check(out, src, w, [0, 9, 10, 4000, n - 11, n - 1], np.float32, "conv21")


@pytest.mark.parametrize("dt,r", [("f32", 1), ("f32", 2), ("f32", 3), ("f64", 1)])
def test_config2_sixteen_steps_8192_vs_oracle_rows(cuda, dt, r):
    """Config 2's 16-step run at its full size (8192^2, uniform[-1,1), box
    coefficients normalised to 1, zero padding), in the launch chain the
    autotuner picks for it (temporal blocking included), against the oracle
    on row slabs carrying 16r rows of halo on each side: rows that far from
    a slab cut see exactly the whole grid's values."""
    n, steps = 8192, 16
    npdt = DT[dt]
    src = uniform((n, n), -1, 1, npdt, 16000 + r)
    m = normalised((2 * r + 1, 2 * r + 1), 160 + r)
    x = dev(src, cuda)
    S.autotune_clear()
    try:
        S.autotune_stencil2d(x, m.ravel(), r, S.BOX, steps=steps)
        out = host(S.stencil2d(x, m.ravel(), r, S.BOX, steps=steps))
        S.device_status()
    finally:
        S.autotune_clear()
    halo = r * steps
    for y in [0, 1, halo, n // 2, n - 2, n - 1] + list(rng(r).integers(0, n, 3)):
        lo, hi = max(0, y - halo), min(n, y + halo + 1)
        slab = np.ascontiguousarray(src[lo:hi])
        want = oracle.conv2d(slab, m.astype(npdt), "zero", steps=steps)[y - lo]
        scale = magnitude2d(slab, m, "zero", steps)[y - lo]
        assert_rel_close(out[y], want, scale, REL[npdt] * steps, f"{dt} box{r} row {y}")


def test_sixteen_steps_8192_invariants(cuda):
    """16 steps of a normalised box on a constant field stay constant in the
    interior and the copied ring stays untouched (size-independent checks)."""
    n = 8192
    x = torch.full((n, n), 0.75, dtype=torch.float32, device=cuda)
    x[0, :] = 3.0
    m = normalised((3, 3), 5).ravel()
    out = S.stencil2d(x, m, 1, S.BOX, steps=16, boundary="copy")
    torch.cuda.synchronize()
    assert torch.equal(out[0], x[0]) and torch.equal(out[:, 0], x[:, 0])
    interior = out[17:-1, 1:-1]
    assert (interior - 0.75).abs().max().item() < 1e-5
