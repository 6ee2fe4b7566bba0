"""Every compiled 3D configuration (rows per warp PY, consumer warps NW,
ring slots S, the variant with each thread's own cells in a register ring
along z, and columns a thread V: 4, or 8 with each plane staged as two TMA
boxes) against the oracle, and the 3D autotuners.

A configuration is pinned for the grid's size class through a tune-cache
file (``choice3d`` lines, read by ssam_autotune_load), the public way to fix
a launch configuration; the bounds are those of test_stencil3d_gpu.py and
test_poisson_gpu.py.  Grids: a TMA-staged one (row bytes a multiple of 16,
partial column tiles in x and y, z chunks with a ragged end) and one whose
rows take the plain-load producer path.
"""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_b200.build import instances_3d, instances_3d_t2
from ssam_b200.workloads import gaussian_rhs
from ssam_cases import taps_j3d13pt, taps_j3d7pt, uniform
from test_stencil3d_gpu import band_close, cube_from_taps, magnitude, oracle_steps, poisson_cube

pytestmark = pytest.mark.gpu

DTC = {"f32": 0, "f64": 1, "bf16": 2, "f16": 3}
TDT = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}


def log2(v):
    return v.bit_length() - 1


def pin(tmp_path, dt, shape, r, rhs, nx, ny, nzb, cfg):
    py, nw, s, zreg, v = cfg
    p = tmp_path / "pin3d.txt"
    p.write_text("# ssam_b200 autotune cache v1\n"
                 f"choice3d {DTC[dt]} {shape} {r} {int(rhs)} {log2(nx)} {log2(ny)} {log2(nzb)} "
                 f"{py} {nw} {s} {int(zreg)} {v}\n")
    S.autotune_clear()
    S.autotune_load(str(p))


def stencil_cases():
    out = []
    for (dt, shape, r, py, nw, s, rhs, _, zreg, v) in instances_3d():
        if not rhs and dt in ("f32", "f64", "bf16"):
            out.append((dt, shape, r, (py, nw, s, zreg, v)))
    return out


def cube_for(shape, r):
    if shape == 1:
        return poisson_cube(), S.POISSON19
    cube = cube_from_taps(taps_j3d7pt() if r == 1 else taps_j3d13pt(), r)
    return cube / np.abs(cube).sum(), S.STAR3D


def case_id(c):
    dt, shape, r, (py, nw, s, zreg, v) = c
    return (f"{dt}-{'p19' if shape else 'star'}{r}-{py}x{nw}x{s}{'z' if zreg else ''}"
            f"{'-v8' if v == 8 else ''}")


def check_configuration(cuda, tmp_path, dt, shape, r, cfg, dims, bnd):
    nz, ny, nx = dims
    cube, sh = cube_for(shape, r)
    src32 = uniform(dims, -1, 1, np.float32, nx + 7 * r + shape)
    t = torch.from_numpy(src32).to(TDT[dt])
    src = t.numpy() if dt != "bf16" else t.double().numpy()
    pin(tmp_path, dt, shape, r, False, nx, ny, nz, cfg)
    try:
        out = S.stencil3d(t.to(cuda), cube, r, sh, boundary=bnd)
        S.device_status()
        got = out.double().cpu().numpy()
    finally:
        S.autotune_clear()
    if dt == "bf16":
        want = oracle_steps(src, cube, 1, bnd)
        scale = np.maximum(np.abs(want), magnitude(src, cube, 1, bnd))
        band_close(got, want, scale, 0, 2.0**-8 + 1e-5, f"bf16 {cfg}")
    else:
        want = oracle_steps(src, cube.astype(src.dtype), 1, bnd)
        rel = 1e-5 if dt == "f32" else 1e-12
        band_close(got, want, magnitude(src, cube, 1, bnd), 0, rel, f"{dt} {cfg}")


@pytest.mark.parametrize("dt,shape,r,cfg", stencil_cases(), ids=[case_id(c) for c in stencil_cases()])
@pytest.mark.parametrize("dims", [(40, 75, 296), (19, 33, 130)])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_every_3d_configuration_vs_oracle(cuda, tmp_path, dt, shape, r, cfg, dims, bnd):
    check_configuration(cuda, tmp_path, dt, shape, r, cfg, dims, bnd)


def wide_cases():
    return [c for c in stencil_cases() if c[3][4] == 8]


@pytest.mark.parametrize("dt,shape,r,cfg", wide_cases(), ids=[case_id(c) for c in wide_cases()])
@pytest.mark.parametrize("dims", [(6, 10, 44), (5, 7, 136)])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_8_column_tiles_on_narrow_grids(cuda, tmp_path, dt, shape, r, cfg, dims, bnd):
    """A 256-column tile on grids narrower than it: at 44 columns the second
    TMA box of every plane lies wholly outside the grid (filled with zeros)
    and the first is partial (a ragged last chunk of 4 columns); at 136 the
    second box holds 8 columns.  FP32 rows are 16-byte multiples at both
    widths (TMA); BF16 rows of 44 are not (plain-load producer)."""
    check_configuration(cuda, tmp_path, dt, shape, r, cfg, dims, bnd)


def sweep_cases():
    return [(dt, (py, nw, s, zreg, v))
            for (dt, shape, r, py, nw, s, rhs, _, zreg, v) in instances_3d() if rhs]


@pytest.mark.parametrize("dt,cfg", sweep_cases(),
                         ids=[f"{d}-{c[0]}x{c[1]}x{c[2]}{'z' if c[3] else ''}"
                              f"{'-v8' if c[4] == 8 else ''}" for d, c in sweep_cases()])
def test_every_jacobi_configuration_vs_oracle(cuda, tmp_path, dt, cfg):
    n, nb, sweeps = 24, 3, 2
    rel = {"f64": 1e-12, "f32": 1e-5, "bf16": 2.0**-8}[dt]
    f = gaussian_rhs(nb, n, 5)
    u0 = np.random.Generator(np.random.PCG64(3)).standard_normal(f.shape) * 1e-3
    ft = torch.from_numpy(f).to(TDT[dt]).to(cuda)
    ut = torch.from_numpy(u0).to(TDT[dt]).to(cuda)
    pin(tmp_path, dt, 0, 1, True, n, n, n * nb, cfg)
    try:
        got = S.poisson_jacobi(ft, ut, sweeps).double().cpu().numpy()
    finally:
        S.autotune_clear()
    want = oracle.jacobi7(ft.double().cpu().numpy(), ut.double().cpu().numpy(), sweeps)
    h2 = 1.0 / (n + 1) ** 2
    scale = np.abs(want) + h2 * np.abs(f).max() / 6 + np.abs(u0).max()
    assert (np.abs(got - want) / scale).max() <= rel * sweeps


@pytest.mark.parametrize("shape,r", [(0, 1), (0, 2), (1, 1)])
def test_autotune_stencil3d_then_parity(cuda, tmp_path, shape, r):
    dims = (48, 80, 256)
    cube, sh = cube_for(shape, r)
    src = uniform(dims, 0, 1, np.float32, 31 + r)
    t = torch.from_numpy(src).to(cuda)
    S.autotune_clear()
    try:
        rep = S.autotune_stencil3d(t, cube, r, sh, boundary="copy")
        # every single-step and every two-step configuration is timed
        assert rep["candidates"] == sum(1 for c in stencil_cases()
                                        if c[0] == "f32" and c[1] == shape and c[2] == r) + \
            sum(1 for c in instances_3d_t2() if c[:3] == ("f32", shape, r))
        assert rep["ms_per_step"] > 0 and rep["consumer_warps"] >= 1
        assert rep["fused_steps"] in (1, 2)
        got = S.stencil3d(t, cube, r, sh, steps=3, boundary="copy").cpu().numpy()
        S.device_status()
        # the choice survives a save / load round trip
        p = tmp_path / "tune3d.txt"
        S.autotune_save(str(p))
        assert "choice3d" in p.read_text()
        S.autotune_clear()
        S.autotune_load(str(p))
        again = S.stencil3d(t, cube, r, sh, steps=3, boundary="copy").cpu().numpy()
    finally:
        S.autotune_clear()
    want = oracle_steps(src, cube.astype(np.float32), 3, "copy")
    band_close(got, want, magnitude(src, cube, 3, "copy"), 0, 3e-5, "tuned")
    np.testing.assert_array_equal(again, got)


def test_autotune_jacobi3d_then_solve(cuda):
    S.autotune_clear()
    try:
        for dt in ("f32", "bf16"):
            rep = S.autotune_jacobi3d(32, 2, dt)
            assert rep["candidates"] >= 2 and rep["ms_per_step"] > 0
        f = torch.from_numpy(gaussian_rhs(2, 32, 9)).to(cuda)
        u = torch.zeros_like(f)
        st = S.poisson_solve(f, u, tol=1e-6, sweep_dtype="bf16", sweeps_per_correction=200,
                             max_sweeps=40000)
    finally:
        S.autotune_clear()
    assert st["converged"] == 1
    _, rel = oracle.residual7(f.cpu().numpy(), u.cpu().numpy())
    assert rel.max() <= 1.0001e-6


def test_autotune3d_rejects_bad_arguments(cuda):
    with pytest.raises(S.SsamError):
        S.autotune_jacobi3d(0, 1, "f32")
    t = torch.zeros((8, 8, 8), device=cuda)
    with pytest.raises(S.SsamError):
        S.autotune_stencil3d(t, np.ones((3, 3, 3)), 3, S.POISSON19)
