"""Parity of the row-streaming 2D kernels with T fused steps (levels of
register rings, one row of every step per iteration) with the oracle.

A case pins the fused kernel -- P = 64, depth T -- and the temporal depth
for the grid's size class through a tune-cache file, runs `steps` steps
(fused launches of T, the rest single steps) and compares with the oracle's
steps under the bounds of test_stencil2d_gpu.py's multi-step test.
"""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_b200.build import stream_t_instances
from ssam_cases import stable_seed, assert_rel_close, magnitude2d, normalised, star_matrix, uniform

pytestmark = pytest.mark.gpu

DTC = {"f32": 0, "f64": 1, "bf16": 2}
NPDT = {"f32": np.float32, "f64": np.float64}


def pin(tmp_path, dt, star, r, w, h, t, v, warps=4):
    wb, hb = w.bit_length() - 1, h.bit_length() - 1
    lines = [f"choice {DTC[dt]} {r} {r} {r} {r} {star} {t} {wb} {hb} 64 {warps} {v}",
             f"depth {DTC[dt]} {r} {r} {r} {r} {star} {wb} {hb} {t}"]
    p = tmp_path / "pin_t.txt"
    p.write_text("# ssam_b200 autotune cache v1\n" + "\n".join(lines) + "\n")
    S.autotune_clear()
    S.autotune_load(str(p))


CASES = sorted(set(stream_t_instances()))


@pytest.mark.parametrize("dt,star,r,seg,v,t", CASES,
                         ids=[f"{c[0]}-{'star' if c[1] else 'box'}{c[2]}-T{c[5]}" for c in CASES])
@pytest.mark.parametrize("shape", [(301, 520), (70, 64), (5, 8)])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_fused_streaming_vs_oracle(cuda, tmp_path, dt, star, r, seg, v, t, shape, bnd):
    h, w = shape
    steps = t + 1 if shape[0] == 70 else t  # one case adds a single step after the fused launch
    seed = stable_seed(dt, star, r, t, shape, bnd)
    src32 = uniform(shape, 0, 1, np.float32, seed)
    if star:
        c = normalised((4 * r + 1,), seed + 1)
        m = star_matrix(c, r)
    else:
        m = normalised((2 * r + 1, 2 * r + 1), seed + 1)
        c = m.ravel()
    if dt == "bf16":
        x = torch.from_numpy(src32).to(torch.bfloat16)
        ref_in = x.double().numpy()
    else:
        ref_in = src32.astype(NPDT[dt])
        x = torch.from_numpy(ref_in)
    pin(tmp_path, dt, star, r, w, h, t, v)
    try:
        out = S.stencil2d(x.to(cuda), c, r, S.STAR if star else S.BOX, steps=steps, boundary=bnd)
        got = out.double().cpu().numpy()
    finally:
        S.autotune_clear()
    if dt == "bf16":
        want = oracle.conv2d(ref_in, m, bnd, steps=steps)
        scale = np.maximum(np.abs(want), magnitude2d(ref_in, m, bnd, steps))
        assert_rel_close(got, want, scale, 2.0**-8 * steps + 1e-5, f"bf16 r{r} T{t} {bnd}")
    else:
        want = oracle.conv2d(ref_in, m.astype(NPDT[dt]), bnd, steps=steps)
        rel = (1e-5 if dt == "f32" else 1e-12) * steps
        assert_rel_close(got, want, magnitude2d(ref_in, m, bnd, steps), rel,
                         f"{dt} r{r} T{t} {bnd}")
