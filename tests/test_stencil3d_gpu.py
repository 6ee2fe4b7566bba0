"""Parity of the sm_100a 3D stencils (7-pt, 13-pt, 19-pt) with the oracle.

The reference checks its 3D kernels with checkError3D (common.hpp:84-127):
RMS error over the band [IT*r, N - IT*r) against the CPU gold iterated IT
times, tolerance 1e-5.  Here every cell of that band must satisfy
|gpu - gold| <= rel * sum|c||x| (rel = 1e-5 FP32, 1e-12 FP64), and the RMS
criterion of the reference is checked as well.
"""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_cases import stable_seed, coefficients, golden, rng, taps_j3d13pt, taps_j3d7pt, uniform

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64}
REL = {np.float32: 1e-5, np.float64: 1e-12}


def cube_from_taps(taps, r):
    f = 2 * r + 1
    c = np.zeros((f, f, f))
    for dz, dy, dx, v in taps:
        c[dz + r, dy + r, dx + r] = float(v)
    return c


def poisson_cube():
    c = coefficients()["coeffs3d"]["poisson"]
    cube = np.zeros((3, 3, 3))
    for k, v in c.items():
        cube[int(k[0]), int(k[1]), int(k[2])] = v
    return cube


def cube_taps(cube):
    r = cube.shape[0] // 2
    return [(z - r, y - r, x - r, cube[z, y, x]) for z in range(cube.shape[0])
            for y in range(cube.shape[1]) for x in range(cube.shape[2]) if cube[z, y, x] != 0]


def oracle_steps(src, cube, steps, boundary):
    taps = cube_taps(cube)
    taps = [(a, b, c, src.dtype.type(v)) for a, b, c, v in taps]
    cur = src
    for _ in range(steps):
        cur = oracle.taps3d(cur, taps, boundary)
    return cur


def magnitude(src, cube, steps, boundary):
    return oracle_steps(np.abs(src).astype(np.float64), np.abs(cube), steps,
                        "zero" if boundary == "zero" else "copy")


def band_close(got, want, scale, lo, rel, what):
    n = [s for s in got.shape]
    sl = tuple(slice(lo, d - lo) for d in n)
    g, w, s = got[sl].astype(np.float64), want[sl].astype(np.float64), scale[sl]
    err = np.abs(g - w) / np.maximum(s, 1e-30)
    assert err.size == 0 or err.max() <= rel, f"{what}: max scaled error {err.max():.3e}"


def run(src, cube, shape, steps=1, boundary="copy", cuda=None):
    r = cube.shape[0] // 2
    t = torch.from_numpy(np.ascontiguousarray(src)).to(cuda)
    out = S.stencil3d(t, cube, r, shape, steps=steps, boundary=boundary)
    S.device_status()
    return out.cpu().numpy()


# ------------------------------------------------ reference golden vectors --

@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("gold", ["j3d7pt", "j3d13pt", "poisson"])
@pytest.mark.parametrize("it", [1, 2])
def test_reference_golds(cuda, tag, gold, it):
    g = golden()
    dt = DT[tag]
    src = g[f"cube16_in_{tag}"]
    if gold == "j3d7pt":
        cube, shape, r = cube_from_taps(taps_j3d7pt(), 1), S.STAR3D, 1
    elif gold == "j3d13pt":
        cube, shape, r = cube_from_taps(taps_j3d13pt(), 2), S.STAR3D, 2
    else:
        cube, shape, r = poisson_cube(), S.POISSON19, 1
    got = run(src, cube, shape, steps=it, cuda=cuda)
    want = g[f"{gold}_n16_it{it}_{tag}"]
    scale = magnitude(src, cube, it, "copy")
    band_close(got, want, scale, it * r, REL[dt], f"{gold} it{it}")
    rms, _ = oracle.rms_max_error(got, want, it * r, it * r)
    assert rms <= 1e-5  # the reference's TOLERANCE (common.hpp:31)


# ------------------------------------------------------- seeded families --

SHAPES = [(1, 1, 1), (5, 5, 5), (16, 16, 16), (17, 20, 24), (7, 33, 130), (40, 70, 260),
          (64, 64, 64), (9, 300, 17)]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", ["7pt", "13pt", "19pt"])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_family_vs_oracle(cuda, dt, shape, kind, bnd):
    seed = stable_seed(shape, kind, bnd, dt.__name__)
    src = uniform(shape, 0, 1, dt, seed)
    g = rng(seed + 1)
    if kind == "7pt":
        r, sh = 1, S.STAR3D
        cube = cube_from_taps([(a, b, c, g.random()) for a, b, c in
                               [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0),
                                (0, 0, -1), (0, 0, 1)]], 1)
    elif kind == "13pt":
        r, sh = 2, S.STAR3D
        offs = [(0, 0, 0)] + [o for d in (1, 2) for o in
                              [(-d, 0, 0), (d, 0, 0), (0, -d, 0), (0, d, 0), (0, 0, -d), (0, 0, d)]]
        cube = cube_from_taps([(a, b, c, g.random()) for a, b, c in offs], 2)
    else:
        r, sh = 1, S.POISSON19
        cube = poisson_cube() * (1 + 0.1 * g.random((3, 3, 3)))
        cube[0, 0, 0] = cube[0, 0, 2] = cube[0, 2, 0] = cube[0, 2, 2] = 0
        cube[2, 0, 0] = cube[2, 0, 2] = cube[2, 2, 0] = cube[2, 2, 2] = 0
    got = run(src, cube, sh, 1, bnd, cuda)
    want = oracle_steps(src, cube, 1, bnd)
    scale = magnitude(src, cube, 1, bnd)
    band_close(got, want, scale, 0, REL[dt], f"{kind}/{bnd}/{shape}")


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("steps", [2, 3, 7])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_multistep_vs_oracle(cuda, dt, steps, bnd):
    src = uniform((24, 40, 68), 0, 1, dt, steps)
    cube = cube_from_taps(taps_j3d7pt(), 1)
    got = run(src, cube, S.STAR3D, steps, bnd, cuda)
    want = oracle_steps(src, cube, steps, bnd)
    band_close(got, want, magnitude(src, cube, steps, bnd), 0, REL[dt] * steps, "multistep")


@pytest.mark.parametrize("tdt,rel", [(torch.bfloat16, 2.0**-8), (torch.float16, 2.0**-11)])
@pytest.mark.parametrize("kind", ["7pt", "13pt"])
def test_half_storage_vs_fp64_oracle(cuda, tdt, rel, kind):
    src32 = uniform((20, 36, 132), 0, 1, np.float32, 11)
    t = torch.from_numpy(src32).to(tdt)
    src64 = t.double().numpy()
    if kind == "7pt":
        cube, r = cube_from_taps(taps_j3d7pt(), 1), 1
    else:
        cube, r = cube_from_taps(taps_j3d13pt(), 2), 2
    cube = cube / np.abs(cube).sum()
    out = S.stencil3d(t.to(cuda), cube, r, S.STAR3D, steps=3, boundary="copy")
    got = out.double().cpu().numpy()
    want = oracle_steps(src64, cube, 3, "copy")
    scale = np.maximum(np.abs(want), magnitude(src64, cube, 3, "copy"))
    band_close(got, want, scale, 0, 3 * rel + 1e-5, f"{tdt}/{kind}")


# --------------------------------------------------- full benchmark sizes --

def test_512_graph_equals_chain_and_slabs(cuda):
    """512^3 FP32 7-pt, 100 steps through the library's captured CUDA graph
    must equal 100 plain single-step calls bit for bit, and one step must match
    the oracle on sampled z-slabs."""
    n = 512
    g = torch.Generator(device=cuda)
    g.manual_seed(3)
    x = torch.rand(n, n, n, device=cuda, generator=g)
    cube = cube_from_taps(taps_j3d7pt(), 1)
    cube = cube / cube.sum()
    one = S.stencil3d(x, cube, 1, S.STAR3D, boundary="copy")
    xs = x.cpu().numpy()
    o = one.cpu().numpy()
    for z in (0, 1, 255, 510, 511):
        lo, hi = max(0, z - 1), min(n, z + 2)
        slab = np.ascontiguousarray(xs[lo:hi])
        want = oracle_steps(slab, cube, 1, "copy")[z - lo]
        scale = magnitude(slab, cube, 1, "copy")[z - lo]
        if 0 < z < n - 1:  # slab edge planes are ring planes of the slab
            err = np.abs(o[z] - want) / np.maximum(scale, 1e-30)
            assert err.max() <= 1e-5, f"plane {z}"
        else:
            assert np.array_equal(o[z], xs[z])
    steps = 100
    graph_out = S.stencil3d(x, cube, 1, S.STAR3D, steps=steps, boundary="copy")
    graph_again = S.stencil3d(x, cube, 1, S.STAR3D, steps=steps, boundary="copy")
    cur = x
    for _ in range(steps):
        cur = S.stencil3d(cur, cube, 1, S.STAR3D, boundary="copy")
    S.device_status()
    assert torch.equal(graph_out, cur)
    assert torch.equal(graph_again, cur)


def test_512_linearity_13pt(cuda):
    n = 512
    x = torch.rand(n, n, n, device=cuda, dtype=torch.float64)
    y = torch.rand(n, n, n, device=cuda, dtype=torch.float64)
    cube = cube_from_taps(taps_j3d13pt(), 2)
    sx = S.stencil3d(x, cube, 2)
    sy = S.stencil3d(y, cube, 2)
    sxy = S.stencil3d(2.0 * x - 0.5 * y, cube, 2)
    assert (sxy - (2.0 * sx - 0.5 * sy)).abs().max().item() < 1e-11
