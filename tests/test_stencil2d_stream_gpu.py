"""Parity of the row-streaming 2D kernels (a warp walks SEG rows of its strip
with a register ring) with the oracle.

Each case forces one compiled streaming kernel -- P = SEG (32 or 128) -- for
the grid's size class through a tune-cache file (ssam_autotune_load, the
public way to pin a launch configuration), then compares with the oracle
under the bounds of test_stencil2d_gpu.py.  Grid widths are multiples of the
strip width V (the streaming kernel's requirement: every lane's 16-byte chunk
lies wholly inside or outside the grid) with heights that end in a partial
ring group and a partial segment; one unaligned width checks that the
launcher hands such grids to the windowed kernel.
"""

import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_cases import stable_seed, assert_rel_close, magnitude2d, normalised, star_matrix, uniform

pytestmark = pytest.mark.gpu

DTC = {np.float32: 0, np.float64: 1, "bf16": 2}
VDEF = {np.float32: 4, np.float64: 4, "bf16": 8}


def force(tmp_path, dt_key, r, star, w, h, seg, warps=4, v=None):
    """Pin (P = seg, warps, V) for this stencil and size class."""
    wb, hb = w.bit_length() - 1, h.bit_length() - 1  # floor(log2), as the cache keys
    line = (f"choice {DTC[dt_key]} {r} {r} {r} {r} {star} 1 {wb} {hb} {seg} {warps} "
            f"{v or VDEF[dt_key]}\n")
    p = tmp_path / "pin.txt"
    p.write_text("# ssam_b200 autotune cache v1\n" + line)
    S.autotune_clear()
    S.autotune_load(str(p))


def stencil(kind, r, seed):
    f = 2 * r + 1
    if kind == "star":
        c = normalised((4 * r + 1,), seed)
        return c, star_matrix(c, r), S.STAR, 1
    m = normalised((f, f), seed)
    return m.ravel(), m, S.BOX, 0


CASES = [("star", 1), ("star", 2), ("star", 3), ("star", 5), ("box", 1), ("box", 2),
         ("box", 3), ("box", 5)]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("kind,r", CASES)
@pytest.mark.parametrize("seg,v", [(32, None), (128, None)])
@pytest.mark.parametrize("bnd", ["zero", "copy", "clamp"])
def test_streaming_kernels_vs_oracle(cuda, tmp_path, dt, kind, r, seg, v, bnd):
    h, w = 301, 520  # 520 = 8 * 65: whole 16/32-byte chunks; 301 rows: ragged tail
    seed = stable_seed(kind, r, seg, bnd, dt.__name__)
    src = uniform((h, w), -1, 1, dt, seed)
    c, m, shape, star = stencil(kind, r, seed + 1)
    force(tmp_path, dt, r, star, w, h, seg, v=v)
    try:
        out = S.stencil2d(torch.from_numpy(src).to(cuda), c, r, shape, boundary=bnd)
        got = out.cpu().numpy()
    finally:
        S.autotune_clear()
    want = oracle.conv2d(src, m.astype(dt), bnd)
    rel = 1e-5 if dt == np.float32 else 1e-12
    assert_rel_close(got, want, magnitude2d(src, m, bnd), rel, f"{kind}{r}/seg{seg}/{bnd}")


@pytest.mark.parametrize("kind,r", [("star", 1), ("box", 2), ("box", 5)])
@pytest.mark.parametrize("seg", [32, 128])
def test_streaming_bf16_vs_fp64_oracle(cuda, tmp_path, kind, r, seg):
    h, w = 259, 1024
    src32 = uniform((h, w), 0, 1, np.float32, 11 * r + seg)
    t = torch.from_numpy(src32).to(torch.bfloat16)
    src64 = t.double().numpy()
    c, m, shape, star = stencil(kind, r, 5 + r)
    force(tmp_path, "bf16", r, star, w, h, seg)
    try:
        got = S.stencil2d(t.to(cuda), c, r, shape, boundary="copy").double().cpu().numpy()
    finally:
        S.autotune_clear()
    want = oracle.conv2d(src64, m, "copy")
    scale = np.maximum(np.abs(want), magnitude2d(src64, m, "copy"))
    assert_rel_close(got, want, scale, 2.0**-8 + 1e-5, f"bf16 {kind}{r}/seg{seg}")


@pytest.mark.parametrize("h,w", [(40, 515), (1, 64), (2, 8), (133, 4), (3, 64), (4, 8)])
def test_streaming_pin_on_unaligned_and_tiny_grids(cuda, tmp_path, h, w):
    """Widths that are not a multiple of V go to the windowed kernel; tiny
    grids (one row, one strip, one chunk) stream with most lanes outside."""
    src = uniform((h, w), -1, 1, np.float32, h * 1000 + w)
    for r in (1, 2):  # r = 2: heights up to 4 lie wholly in the ring COPY keeps
        c, m, shape, star = stencil("box", r, 3)
        force(tmp_path, np.float32, r, star, w, h, 32)
        try:
            for bnd in ("zero", "copy", "clamp"):
                got = S.stencil2d(torch.from_numpy(src).to(cuda), c, r, shape,
                                  boundary=bnd).cpu().numpy()
                want = oracle.conv2d(src, m.astype(np.float32), bnd)
                assert_rel_close(got, want, magnitude2d(src, m, bnd), 1e-5,
                                 f"r{r} {h}x{w}/{bnd}")
        finally:
            S.autotune_clear()


def test_streaming_rows_band(cuda, tmp_path):
    """The host-buffer entry point writes row bands (y_begin, y_end) of the
    grid; with a streaming kernel pinned, the result is the whole-grid one."""
    h, w = 20000, 256  # three bands of 8192 rows
    src = uniform((h, w), -1, 1, np.float32, 77)
    c, m, shape, star = stencil("box", 2, 9)
    force(tmp_path, np.float32, 2, star, w, h, 128)
    try:
        hs = torch.from_numpy(src).pin_memory()
        hd = torch.empty_like(hs).pin_memory()
        S.stencil2d_host(hs, hd, c, 2, shape, 1, "zero", cuda,
                         torch.cuda.current_stream(cuda))
        torch.cuda.synchronize()
        got = hd.numpy().copy()
    finally:
        S.autotune_clear()
    want = oracle.conv2d(src, m.astype(np.float32), "zero")
    assert_rel_close(got, want, magnitude2d(src, m, "zero"), 1e-5, "band")


@pytest.mark.parametrize("dt", ["f32", "f64", "bf16"])
@pytest.mark.parametrize("kind,r", [("star", 1), ("box", 2), ("star", 3), ("box", 3)])
@pytest.mark.parametrize("w", [517, 6, 1, 33])
@pytest.mark.parametrize("bnd", ["zero", "copy", "clamp"])
def test_streaming_pitched_rows_with_a_partial_last_chunk(cuda, tmp_path, dt, kind, r, w, bnd):
    """Rows 16-byte aligned (pitch a multiple of 32 elements) but widths that
    are not a multiple of V: the row's last chunk is partly inside the grid
    (loaded whole inside the row's pitch, its outside columns fixed by the
    boundary rule, stored per element)."""
    h = 77
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}[dt]
    pitch = -(-w // 32) * 32
    base = torch.empty(h, pitch, dtype=tdt, device=cuda)
    x32 = uniform((h, w), -1, 1, np.float32, w * 10 + r)
    src = base[:, :w]
    src.copy_(torch.from_numpy(x32).to(tdt))
    c, m, shape, star = stencil(kind, r, 3 + r)
    force(tmp_path, {"f32": np.float32, "f64": np.float64, "bf16": "bf16"}[dt], r, star, w, h, 32)
    dbase = torch.full((h, pitch), 7.0, dtype=tdt, device=cuda)
    dst = dbase[:, :w]
    try:
        S.stencil2d(src, c, r, shape, boundary=bnd, dst=dst)
        got = dst.double().cpu().numpy()
        pad = dbase[:, w:].double().cpu().numpy()
    finally:
        S.autotune_clear()
    assert (pad == 7.0).all(), "wrote outside the grid's width"
    ref_in = src.double().cpu().numpy()
    want = oracle.conv2d(ref_in, m, bnd)
    if dt == "bf16":
        scale = np.maximum(np.abs(want), magnitude2d(ref_in, m, bnd))
        assert_rel_close(got, want, scale, 2.0**-8 + 1e-5, f"{dt} {kind}{r} w{w} {bnd}")
    else:
        np_dt = np.float32 if dt == "f32" else np.float64
        want = oracle.conv2d(ref_in.astype(np_dt), m.astype(np_dt), bnd)
        rel = 1e-5 if dt == "f32" else 1e-12
        assert_rel_close(got, want, magnitude2d(ref_in, m, bnd), rel, f"{dt} {kind}{r} w{w} {bnd}")
