"""Parity of the 3D kernels that fuse two time steps per launch (temporal
blocking, stencil3d_t2.cuh) with the oracle's chain of single steps.

The reference fuses ITERATIVE_COUNT steps inside its 3D z-march
(ssai-3dstencil/tmp3d7pt-v2.cu:124-170) and checks the result against its
gold applied IT times (checkError3D, common.hpp:84-127).  Here:

* integer inputs with integer coefficients make every partial sum exact, so
  each compiled two-step configuration must equal the oracle bit for bit, on
  grids that exercise partial tiles in x and y, ragged z chunks, grids
  smaller than one tile, the TMA-staged and the plain-load producer paths,
  and both boundary rules;
* real-valued inputs follow the bounds of test_stencil3d_gpu.py, with one
  rounding per step;
* at the benchmark size (512^3) the fused runs are checked against the
  oracle on z-slabs, including the BF16-storage 100-step run against the
  FP64 oracle (its max and RMS error are printed).

A configuration is pinned through a tune-cache file (``choice3d`` with
t = 2, ``depth3d``), the public way to fix a launch configuration.
"""
import numpy as np
import pytest
import torch

import ssam_b200 as S
from ssam_b200.build import instances_3d_t2
from ssam_cases import taps_j3d13pt, taps_j3d7pt, uniform
from test_stencil3d_gpu import cube_from_taps, magnitude, oracle_steps, poisson_cube

pytestmark = pytest.mark.gpu

DTC = {"f32": 0, "f64": 1, "bf16": 2}
TDT = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}


def log2(v):
    return v.bit_length() - 1


def pin_t2(tmp_path, dt, shape, r, dims, cfg):
    """Pin the two-step configuration `cfg` = (PY, NW, S, V) and depth 2 for
    the size class of `dims` = (nz, ny, nx)."""
    nz, ny, nx = dims
    py, nw, s, v = cfg
    p = tmp_path / "pin3d_t2.txt"
    p.write_text("# ssam_b200 autotune cache v1\n"
                 f"choice3d {DTC[dt]} {shape} {r} 0 {log2(nx)} {log2(ny)} {log2(nz)} "
                 f"{py} {nw} {s} 0 {v} 2\n"
                 f"depth3d {DTC[dt]} {shape} {r} {log2(nx)} {log2(ny)} {log2(nz)} 2\n")
    S.autotune_clear()
    S.autotune_load(str(p))


def t2_cases():
    return [(dt, shape, r, (py, nw, s, v)) for (dt, shape, r, py, nw, s, v, _)
            in instances_3d_t2()]


def case_id(c):
    dt, shape, r, (py, nw, s, v) = c
    return f"{dt}-{'p19' if shape else 'star'}{r}-{py}x{nw}x{s}-v{v}"


def integer_cube(shape, r, seed):
    """Small integer coefficients on the shape's taps (the rest zero)."""
    g = np.random.Generator(np.random.PCG64(seed))
    if shape == 1:
        cube = (poisson_cube() != 0) * g.integers(1, 3, (3, 3, 3))
        return cube.astype(np.float64), S.POISSON19
    offs = [(0, 0, 0)] + [o for d in range(1, r + 1) for o in
                          [(-d, 0, 0), (d, 0, 0), (0, -d, 0), (0, d, 0), (0, 0, -d), (0, 0, d)]]
    return cube_from_taps([(a, b, c, float(g.integers(1, 3))) for a, b, c in offs], r), S.STAR3D


def run_pinned(cuda, tmp_path, dt, shape, r, cfg, src, cube, sh, steps, bnd):
    t = torch.from_numpy(np.ascontiguousarray(src)).to(TDT[dt]).to(cuda)
    pin_t2(tmp_path, dt, shape, r, src.shape, cfg)
    try:
        before = S.lib().ssam_kernel_launches()
        out = S.stencil3d(t, cube, r, sh, steps=steps, boundary=bnd)
        S.device_status()
        launches = S.lib().ssam_kernel_launches() - before
        return out.double().cpu().numpy(), launches
    finally:
        S.autotune_clear()


INT_DIMS = [(1, 1, 1), (5, 6, 7), (7, 33, 130), (17, 20, 24), (9, 40, 296), (40, 75, 296),
            (21, 130, 64)]


def chain_rounded(src, cube, steps, bnd, dt):
    """The oracle's single steps in FP64, each result rounded to the storage
    type as a chain of single-step launches stores it."""
    cur = src
    for _ in range(steps):
        cur = oracle_steps(cur, cube, 1, bnd)
        cur = torch.from_numpy(cur).to(TDT[dt]).double().numpy()
    return cur


@pytest.mark.parametrize("dt,shape,r,cfg", t2_cases(), ids=[case_id(c) for c in t2_cases()])
@pytest.mark.parametrize("dims", INT_DIMS, ids=lambda d: "x".join(map(str, d)))
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_every_t2_configuration_integer_exact(cuda, tmp_path, dt, shape, r, cfg, dims, bnd):
    """Two fused steps of integer data (0..3) with integer coefficients (1 or
    2): every partial sum is an integer below 2^13, exact in FP32/FP64
    arithmetic, so the result must equal the oracle's chain of single steps
    bit for bit -- for BF16 storage with each step rounded to BF16, as the
    fused kernel rounds its level-1 values."""
    cube, sh = integer_cube(shape, r, 7 + r + 3 * shape)
    g = np.random.Generator(np.random.PCG64(1000 + dims[2] + 10 * r + shape))
    src = g.integers(0, 4, dims).astype(np.float64)
    got, launches = run_pinned(cuda, tmp_path, dt, shape, r, cfg, src, cube, sh, 2, bnd)
    assert launches == 1, "two steps must run as one fused launch"
    want = chain_rounded(src, cube, 2, bnd, dt)
    bad = np.abs(got - want)
    assert np.array_equal(got, want), (
        f"max |diff| {bad.max()} at {np.unravel_index(bad.argmax(), got.shape)}")


@pytest.mark.parametrize("dt,shape,r,cfg", t2_cases(), ids=[case_id(c) for c in t2_cases()])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_every_t2_configuration_real_vs_oracle(cuda, tmp_path, dt, shape, r, cfg, bnd):
    """Real-valued data: two fused steps plus one single step (3 steps) against
    the oracle, rel 1e-5 (FP32) / 1e-12 (FP64) per step of sum|c||x|, BF16
    storage against the FP64 oracle with one storage rounding per step."""
    dims = (33, 70, 264)
    if shape == 1:
        cube, sh = poisson_cube(), S.POISSON19
    else:
        cube = cube_from_taps(taps_j3d7pt() if r == 1 else taps_j3d13pt(), r)
        cube, sh = cube / np.abs(cube).sum(), S.STAR3D
    src32 = uniform(dims, -1, 1, np.float32, 55 + r + shape)
    src = torch.from_numpy(src32).to(TDT[dt]).double().numpy() if dt != "f64" else \
        src32.astype(np.float64)
    got, launches = run_pinned(cuda, tmp_path, dt, shape, r, cfg, src, cube, sh, 3, bnd)
    assert launches == 2
    if dt == "bf16":
        want = oracle_steps(src, cube, 3, bnd)
        scale = np.maximum(np.abs(want), magnitude(src, cube, 3, bnd))
        rel = 3 * 2.0**-8 + 1e-5
    else:
        want = oracle_steps(src, cube.astype(src.dtype), 3, bnd)
        scale = magnitude(src, cube, 3, bnd)
        rel = 3 * (1e-5 if dt == "f32" else 1e-12)
    err = np.abs(got - want) / np.maximum(scale, 1e-30)
    assert err.max() <= rel, f"max scaled error {err.max():.3e}"


@pytest.mark.parametrize("steps", [2, 3, 4, 7])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_depth_two_chain_vs_oracle(cuda, tmp_path, steps, bnd):
    """With depth 2 pinned (and the default two-step configuration) a
    multi-step run takes steps // 2 fused launches and a single step for an
    odd count."""
    src = uniform((24, 40, 68), 0, 1, np.float32, 300 + steps)
    cube = cube_from_taps(taps_j3d7pt(), 1)
    p = tmp_path / "d2.txt"
    p.write_text(f"depth3d 0 0 1 {log2(68)} {log2(40)} {log2(24)} 2\n")
    S.autotune_clear()
    S.autotune_load(str(p))
    try:
        t = torch.from_numpy(src).to(cuda)
        before = S.lib().ssam_kernel_launches()
        out = S.stencil3d(t, cube, 1, S.STAR3D, steps=steps, boundary=bnd)
        S.device_status()
        assert S.lib().ssam_kernel_launches() - before == steps // 2 + steps % 2
    finally:
        S.autotune_clear()
    want = oracle_steps(src, cube.astype(np.float32), steps, bnd)
    err = np.abs(out.cpu().numpy() - want) / np.maximum(magnitude(src, cube, steps, bnd), 1e-30)
    assert err.max() <= steps * 1e-5


def test_depth_one_when_pinned(cuda, tmp_path):
    """A depth3d line of 1 (also the default without one) keeps multi-step
    runs at one step a launch."""
    src = uniform((24, 40, 68), 0, 1, np.float32, 17)
    cube = cube_from_taps(taps_j3d7pt(), 1)
    p = tmp_path / "d1.txt"
    p.write_text(f"depth3d 0 0 1 {log2(68)} {log2(40)} {log2(24)} 1\n")
    S.autotune_clear()
    S.autotune_load(str(p))
    try:
        t = torch.from_numpy(src).to(cuda)
        before = S.lib().ssam_kernel_launches()
        out = S.stencil3d(t, cube, 1, S.STAR3D, steps=4, boundary="copy")
        S.device_status()
        assert S.lib().ssam_kernel_launches() - before == 4
    finally:
        S.autotune_clear()
    want = oracle_steps(src, cube.astype(np.float32), 4, "copy")
    err = np.abs(out.cpu().numpy() - want) / np.maximum(magnitude(src, cube, 4, "copy"), 1e-30)
    assert err.max() <= 4e-5


# --------------------------------------------------- full benchmark sizes --

def pin_depth(tmp_path, dt, shape, r, dims, depth):
    nz, ny, nx = dims
    p = tmp_path / "depth.txt"
    p.write_text(f"depth3d {DTC[dt]} {shape} {r} {log2(nx)} {log2(ny)} {log2(nz)} {depth}\n")
    S.autotune_clear()
    S.autotune_load(str(p))


def slab_check(x_np, out, cube, steps, planes, bnd, rel):
    """Compare planes of `out` (steps applied to the whole grid) with the
    oracle applied to z-slabs of `x_np` that carry R*steps planes of halo on
    each side.  Returns (max scaled error, max abs error, rms error)."""
    n = x_np.shape[0]
    r = cube.shape[0] // 2
    halo = r * steps
    worst = 0.0
    abs_max, sq, cnt = 0.0, 0.0, 0
    for z in planes:
        lo, hi = max(0, z - halo), min(n, z + halo + 1)
        slab = np.ascontiguousarray(x_np[lo:hi]).astype(np.float64)
        want = oracle_steps(slab, cube, steps, bnd)[z - lo]
        if (slab < 0).any() or (cube < 0).any():
            scale = np.maximum(np.abs(want), magnitude(slab, cube, steps, bnd)[z - lo])
        else:  # non-negative data and taps: the magnitude is the result itself
            scale = np.abs(want)
        got = out[z].astype(np.float64)
        # a slab cut inside the grid turns its end planes into boundary
        # planes; the planes checked lie at least `halo` inside the cut
        d = np.abs(got - want)
        worst = max(worst, float((d / np.maximum(scale, 1e-30)).max()))
        abs_max = max(abs_max, float(d.max()))
        sq += float((d ** 2).sum())
        cnt += d.size
    assert worst <= rel, f"max scaled error {worst:.3e} > {rel:.1e}"
    return worst, abs_max, (sq / cnt) ** 0.5


@pytest.mark.parametrize("kind", ["7pt", "13pt", "19pt"])
def test_512_fused_two_steps_vs_oracle_slabs(cuda, tmp_path, kind):
    """512^3 FP32, two steps in one fused launch (depth 2, the default
    two-step configuration), against the oracle on z-slabs at both faces and
    inside."""
    n = 512
    g = torch.Generator(device=cuda)
    g.manual_seed(11)
    x = torch.rand(n, n, n, device=cuda, generator=g)
    if kind == "19pt":
        cube, sh, r = poisson_cube(), S.POISSON19, 1
        cube = cube / np.abs(cube).sum()
    else:
        r = 1 if kind == "7pt" else 2
        cube = cube_from_taps(taps_j3d7pt() if r == 1 else taps_j3d13pt(), r)
        cube, sh = cube / np.abs(cube).sum(), S.STAR3D
    pin_depth(tmp_path, "f32", 1 if kind == "19pt" else 0, r, (n, n, n), 2)
    try:
        before = S.lib().ssam_kernel_launches()
        out = S.stencil3d(x, cube, r, sh, steps=2, boundary="copy")
        S.device_status()
        assert S.lib().ssam_kernel_launches() - before == 1
    finally:
        S.autotune_clear()
    slab_check(x.cpu().numpy(), out.cpu().numpy(), cube, 2, (0, 1, 2, 3, 255, 508, 510, 511),
               "copy", 2e-5)


def test_512_bf16_100_steps_vs_fp64_oracle(cuda, tmp_path):
    """The benchmark's BF16-storage run: 512^3 7-point, 100 steps in one CUDA
    graph -- 100 single-step launches (the default depth) and 50 fused
    two-step launches -- against the FP64 oracle on z-slabs; states the max
    and RMS error of each."""
    n, steps = 512, 100
    g = torch.Generator(device=cuda)
    g.manual_seed(5)
    x = torch.rand(n, n, n, device=cuda, generator=g).to(torch.bfloat16)
    cube = cube_from_taps(taps_j3d7pt(), 1)
    cube = cube / np.abs(cube).sum()
    outs = {}
    for depth in (1, 2):
        pin_depth(tmp_path, "bf16", 0, 1, (n, n, n), depth)
        try:
            out = S.stencil3d(x, cube, 1, S.STAR3D, steps=steps, boundary="copy")
            S.device_status()
        finally:
            S.autotune_clear()
        outs[depth] = out.double().cpu().numpy()
        del out
    xs = x.double().cpu().numpy()
    for depth, o in outs.items():
        # one storage rounding per step, each at most 2^-8 relative
        worst, amax, rms = slab_check(xs, o, cube, steps, (0, 40, 300), "copy",
                                      steps * 2.0**-8)
        print(f"bf16 512^3 100 steps, {depth} step(s) a launch, vs FP64 oracle: max abs "
              f"{amax:.3e}, rms {rms:.3e}, max scaled {worst:.3e}")
        assert amax <= 0.05 and rms <= 0.01


@pytest.mark.parametrize("kind", ["13pt", "19pt"])
def test_512_autotuned_single_step_vs_oracle_slabs(cuda, kind):
    """512^3 FP32, the configuration the autotuner picks for the benchmark
    (one step a launch) against the oracle on z-slabs at both faces and
    inside, one step and a 4-step chain."""
    n = 512
    g = torch.Generator(device=cuda)
    g.manual_seed(13)
    x = torch.rand(n, n, n, device=cuda, generator=g)
    if kind == "19pt":
        cube, sh, r = poisson_cube(), S.POISSON19, 1
        cube = cube / np.abs(cube).sum()
    else:
        cube, sh, r = cube_from_taps(taps_j3d13pt(), 2), S.STAR3D, 2
        cube = cube / np.abs(cube).sum()
    S.autotune_clear()
    try:
        S.autotune_stencil3d(x, cube, r, sh, boundary="copy")
        outs = {k: S.stencil3d(x, cube, r, sh, steps=k, boundary="copy").cpu().numpy()
                for k in (1, 4)}
        S.device_status()
    finally:
        S.autotune_clear()
    xs = x.cpu().numpy()
    for k, o in outs.items():
        slab_check(xs, o, cube, k, (0, 1, 2, 255, 509, 510, 511), "copy", 1e-5 * k)


def test_512_bf16_13pt_100_steps_vs_fp64_oracle(cuda):
    """The benchmark's BF16-storage 13-point run (512^3, 100 steps in one CUDA
    graph, the autotuned kernel) against the FP64 oracle on z-slabs; states
    the max and RMS error."""
    n, steps = 512, 100
    g = torch.Generator(device=cuda)
    g.manual_seed(17)
    x = torch.rand(n, n, n, device=cuda, generator=g).to(torch.bfloat16)
    cube = cube_from_taps(taps_j3d13pt(), 2)
    cube = cube / np.abs(cube).sum()
    S.autotune_clear()
    try:
        S.autotune_stencil3d(x, cube, 2, S.STAR3D, boundary="copy")
        o = S.stencil3d(x, cube, 2, S.STAR3D, steps=steps, boundary="copy")
        S.device_status()
    finally:
        S.autotune_clear()
    o = o.double().cpu().numpy()
    worst, amax, rms = slab_check(x.double().cpu().numpy(), o, cube, steps, (0, 300),
                                  "copy", steps * 2.0**-8)
    print(f"bf16 512^3 13-point 100 steps vs FP64 oracle: max abs {amax:.3e}, "
          f"rms {rms:.3e}, max scaled {worst:.3e}")
    assert amax <= 0.05 and rms <= 0.01
