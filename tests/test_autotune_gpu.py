"""The autotuner times every compiled (P, V, warps, temporal depth) for a
stencil on the caller's grid, and the tuned choice still gives the oracle's
result."""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_cases import assert_rel_close, magnitude2d, normalised, star_matrix, uniform

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,r,steps", [("box", 1, 16), ("star", 1, 1), ("box", 5, 1),
                                          ("star", 2, 6)])
def test_autotune_then_parity(cuda, kind, r, steps, tmp_path):
    S.autotune_clear()
    src = uniform((600, 1000), 0, 1, np.float32, r * 100 + steps)
    t = torch.from_numpy(src).to(cuda)
    f = 2 * r + 1
    if kind == "star":
        c = normalised((4 * r + 1,), 7)
        m = star_matrix(c, r)
        shape = S.STAR
    else:
        m = normalised((f, f), 7)
        c = m.ravel()
        shape = S.BOX
    rep = S.autotune_stencil2d(t, c, r, shape, steps=steps, boundary="copy")
    assert rep["candidates"] >= 3
    assert rep["fused_steps"] >= 1 and rep["fused_steps"] <= max(1, steps)
    assert rep["columns_per_thread"] in (4, 8) and rep["warps_per_block"] in (2, 4, 8)
    assert rep["ms_per_step"] > 0
    out = S.stencil2d(t, c, r, shape, steps=steps, boundary="copy").cpu().numpy()
    want = oracle.conv2d(src, m.astype(np.float32), "copy", steps=steps)
    assert_rel_close(out, want, magnitude2d(src, m, "copy", steps), 1e-5 * steps, "tuned")
    # the saved choice reloads into an empty cache and gives the same result
    p = tmp_path / "tune.txt"
    S.autotune_save(str(p))
    S.autotune_clear()
    S.autotune_load(str(p))
    again = S.stencil2d(t, c, r, shape, steps=steps, boundary="copy").cpu().numpy()
    np.testing.assert_array_equal(again, out)
    S.autotune_clear()
