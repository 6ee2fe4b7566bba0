"""Parity of the row-loop 2D kernels (one output row at a time, filter rows in
a loop) with the oracle, for wide square filters.

Each case pins P = 1 (the row-loop kernel) for the grid's size class through
a tune-cache file and compares with the oracle under the bounds of
test_stencil2d_gpu.py; grids cover aligned and unaligned widths, pitched
rows, and heights shorter than the filter.
"""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_b200.build import rowloop_instances
from ssam_cases import assert_rel_close, magnitude2d, normalised, uniform

pytestmark = pytest.mark.gpu

DTC = {np.float32: 0, np.float64: 1}


def pin(tmp_path, dt, rl, rr, w, h, v, warps=4):
    line = (f"choice {DTC[dt]} {rl} {rr} {rl} {rr} 0 1 {w.bit_length() - 1} "
            f"{h.bit_length() - 1} 1 {warps} {v}\n")
    p = tmp_path / "pin_rowloop.txt"
    p.write_text("# ssam_b200 autotune cache v1\n" + line)
    S.autotune_clear()
    S.autotune_load(str(p))


CASES = sorted({(dt, rl, rr, v) for (dt, rl, rr, v) in rowloop_instances()
                if rl + rr + 1 in (7, 8, 11, 15, 21, 28)})


@pytest.mark.parametrize("dtn,rl,rr,v", CASES, ids=[f"{c[0]}-F{c[1]+c[2]+1}-v{c[3]}" for c in CASES])
@pytest.mark.parametrize("shape", [(97, 264), (40, 515), (9, 64)])
@pytest.mark.parametrize("bnd", ["zero", "copy", "clamp"])
def test_rowloop_vs_oracle(cuda, tmp_path, dtn, rl, rr, v, shape, bnd):
    dt = np.float32 if dtn == "f32" else np.float64
    f = rl + rr + 1
    h, w = shape
    src = uniform(shape, -1, 1, dt, f * 100 + w)
    m = normalised((f, f), f)
    pin(tmp_path, dt, rl, rr, w, h, v)
    try:
        out = S.conv2d(torch.from_numpy(src).to(cuda), m, boundary=bnd)
        got = out.cpu().numpy()
    finally:
        S.autotune_clear()
    want = oracle.conv2d(src, m.astype(dt), bnd)
    rel = 1e-5 if dt == np.float32 else 1e-12
    assert_rel_close(got, want, magnitude2d(src, m, bnd), rel, f"F{f} {shape} {bnd}")


def test_rowloop_pitched_grid_and_box_entry(cuda, tmp_path):
    """Pitched rows through ssam_stencil2d (box r = 5, V = 8): nothing past
    the width is written."""
    h, w, pitch = 70, 300, 320
    base = torch.full((h, pitch), 5.0, device=cuda)
    src = uniform((h, w), -1, 1, np.float32, 3)
    view = base[:, :w]
    view.copy_(torch.from_numpy(src))
    m = normalised((11, 11), 8)
    pin(tmp_path, np.float32, 5, 5, w, h, 8)
    dbase = torch.full((h, pitch), 9.0, device=cuda)
    try:
        S.stencil2d(view, m.ravel(), 5, S.BOX, boundary="copy", dst=dbase[:, :w])
        got = dbase[:, :w].cpu().numpy()
        assert bool((dbase[:, w:] == 9.0).all())
    finally:
        S.autotune_clear()
    want = oracle.conv2d(src, m.astype(np.float32), "copy")
    assert_rel_close(got, want, magnitude2d(src, m, "copy"), 1e-5, "box5 pitched")
