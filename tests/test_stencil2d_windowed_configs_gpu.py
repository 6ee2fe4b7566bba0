"""Every compiled windowed 2D kernel (ssam_b200/build.py: instances()) against
the oracle.

The autotuner times these configurations -- P rows a thread (4, 8, 16), V
columns a thread (4 or 8), T fused steps, star and box radii, the even and
wide correlation sizes -- and keeps the fastest per size class, so any of them
can be the one a caller gets.  Each case pins one configuration for the
grid's size class through a tune-cache file (``choice`` line, plus a
``depth`` line for T > 1: the public way to fix a launch configuration) and
compares one call of T steps with the oracle under the bounds of
test_stencil2d_gpu.py (rel 1e-5 FP32 / 1e-12 FP64 of sum|c||x| per step;
16-bit storage against the FP64 oracle with one storage rounding per step).
"""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_b200.build import instances
from ssam_cases import assert_rel_close, magnitude2d, normalised, stable_seed, star_matrix, uniform

pytestmark = pytest.mark.gpu

DTC = {"f32": 0, "f64": 1, "bf16": 2, "f16": 3}
TDT = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16,
       "f16": torch.float16}
H, W = 259, 264  # 264 columns: whole 16-byte rows in every type; ragged strips


def pin(tmp_path, dt, rl, rr, star, p, t, v):
    wb, hb = W.bit_length() - 1, H.bit_length() - 1
    lines = [f"choice {DTC[dt]} {rl} {rr} {rl} {rr} {star} {t} {wb} {hb} {p} 4 {v}"]
    if t > 1:
        lines.append(f"depth {DTC[dt]} {rl} {rr} {rl} {rr} {star} {wb} {hb} {t}")
    path = tmp_path / "pin2d.txt"
    path.write_text("# ssam_b200 autotune cache v1\n" + "\n".join(lines) + "\n")
    S.autotune_clear()
    S.autotune_load(str(path))


def case_id(c):
    dt, star, rl, rr, p, t, v = c
    return f"{dt}-{'star' if star else 'box'}{rl}.{rr}-P{p}-T{t}-V{v}"


@pytest.mark.parametrize("inst", instances(), ids=[case_id(c) for c in instances()])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_every_windowed_configuration_vs_oracle(cuda, tmp_path, inst, bnd):
    dt, star, rl, rr, p, t, v = inst
    f = rl + rr + 1
    seed = stable_seed(*inst, bnd)
    src32 = uniform((H, W), -1, 1, np.float32, seed)
    src_t = torch.from_numpy(src32).to(TDT[dt])
    src = src_t.double().numpy() if dt in ("bf16", "f16") else src_t.numpy()
    if star:
        c = normalised((4 * rl + 1,), seed + 1)
        m = star_matrix(c, rl)
    else:
        m = normalised((f, f), seed + 1)
    pin(tmp_path, dt, rl, rr, star, p, t, v)
    try:
        x = src_t.to(cuda)
        if rl == rr and 1 <= rl <= 10:
            out = S.stencil2d(x, c if star else m.ravel(), rl, S.STAR if star else S.BOX,
                              steps=t, boundary=bnd)
        else:  # 1x1, even-width and very wide correlations: one step (their only depth)
            assert t == 1
            out = S.conv2d(x, m, boundary=bnd)
        S.device_status()
        got = out.double().cpu().numpy()
    finally:
        S.autotune_clear()
    if dt in ("bf16", "f16"):
        want = oracle.conv2d(src, m, bnd, steps=t)
        scale = np.maximum(np.abs(want), magnitude2d(src, m, bnd, t))
        rel = t * (2.0**-8 if dt == "bf16" else 2.0**-11) + 1e-5
    else:
        want = oracle.conv2d(src, m.astype(src.dtype), bnd, steps=t)
        scale = magnitude2d(src, m, bnd, t)
        rel = t * (1e-5 if dt == "f32" else 1e-12)
    assert_rel_close(got, want, scale, rel, case_id(inst))
