"""Generate the committed golden fixtures for the SSAM stencil path.

Run where the reference tree is readable ($SSAM_REFERENCE_DIR, else a
directory named ``reference`` beside this checkout) and ``oracle/_ref`` is
built (``make -C oracle ref``):

    python tests/golden/make_golden.py

It writes two files next to itself:

* ``coefficients.json`` -- the reference's own coefficient tables, parsed from
  its sources: the ``DataType filter[..][..]`` matrices of the 2D tests
  (stencil2D_*pt.cu, stencil2d_temp_*pt.cu) and the ``_F...`` defines of the 3D
  programs (tmp3d7pt-v2.cu, tmp3d13pt.cu, tmpPoisson.cu);
* ``ssam_golden.npz`` -- seeded inputs and the outputs of the reference's own
  compiled CPU golds (``Convolution<T>``, ``v2::j3d7pt_gold``,
  ``j3d13pt_gold``, ``poisson_gold``) on them.

The GPU box never runs this script; tests read the two files.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

REF = oracle.reference_dir()

# 2D tables: name -> (file, which `DataType filter` block in the file)
TABLES_2D = {
    "star1": "ssai-2dstencil/stencil2D_5pt-v1.cu",
    "star2": "ssai-2dstencil/stencil2D_9pt.cu",
    "star3": "ssai-2dstencil/stencil2D_13pt.cu",
    "star4": "ssai-2dstencil/stencil2D_17pt.cu",
    "star5": "ssai-2dstencil/stencil2D_21pt.cu",
    "star6": "ssai-2dstencil/stencil2D_25pt.cu",
    "box64": "ssai-2dstencil/stencil2D_64pt.cu",
    "box81": "ssai-2dstencil/stencil2D_81pt.cu",
    "box121": "ssai-2dstencil/stencil2D_121pt.cu",
    "tmp5": "ssai-2dstencil/stencil2d_temp_5pt.cu",
    "tmp9": "ssai-2dstencil/stencil2d_temp_9pt.cu",
}
DEFINES_3D = {
    "j3d7pt": ("ssai-3dstencil/tmp3d7pt-v2.cu", r"_F3d7PT_(\d)(\d)(\d)"),
    "j3d13pt": ("ssai-3dstencil/tmp3d13pt.cu", r"_F3d13PT_(\d)(\d)(\d)"),
    "poisson": ("ssai-3dstencil/tmpPoisson.cu", r"_F(\d)(\d)(\d)"),
}
NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def _active_text(src: str) -> str:
    """Drop `#else ... #endif` branches of `#if 1` blocks (the reference keeps
    alternative tables behind `#if 1 / #else`)."""
    out, skip = [], []
    for line in src.splitlines():
        s = line.strip()
        if s.startswith("#if"):
            skip.append(False)
        elif s.startswith("#else") and skip:
            skip[-1] = True
            continue
        elif s.startswith("#endif") and skip:
            skip.pop()
            continue
        if not any(skip):
            out.append(line)
    return "\n".join(out)


def parse_filter_table(path: str) -> list[list[float]]:
    text = _active_text(open(path).read())
    m = re.search(r"DataType\s+filter\s*\[[^\]]*\]\s*\[[^\]]*\]\s*=\s*\{", text)
    if not m:
        raise ValueError(f"no filter table in {path}")
    depth, i = 1, m.end()
    while depth:
        depth += {"{": 1, "}": -1}.get(text[i], 0)
        i += 1
    body = re.sub(r"//[^\n]*", "", text[m.end():i - 1])
    rows = re.findall(r"\{([^{}]*)\}", body)
    table = [[float(v) for v in re.findall(NUM, r)] for r in rows]
    n = len(table)
    assert all(len(r) == n for r in table), path
    return table


def parse_defines_3d(path: str, pattern: str) -> dict[str, float]:
    text = _active_text(open(path).read())
    out = {}
    for m in re.finditer(r"#define\s+" + pattern + r"\s+\(\(T\)\s*(" + NUM + r")\s*\)", text):
        out[m.group(1) + m.group(2) + m.group(3)] = float(m.group(4))
    return out


def main() -> None:
    if not os.path.isdir(REF):
        raise SystemExit(f"reference tree not found at {REF}")
    if not oracle.have_ref():
        oracle.build(ref=True)
        oracle._ref = None
    assert oracle.have_ref(), "oracle/_ref did not build"

    coeffs = {"tables2d": {}, "coeffs3d": {}, "sources": {}}
    for name, rel in TABLES_2D.items():
        coeffs["tables2d"][name] = parse_filter_table(os.path.join(REF, rel))
        coeffs["sources"][name] = rel
    for name, (rel, pat) in DEFINES_3D.items():
        coeffs["coeffs3d"][name] = parse_defines_3d(os.path.join(REF, rel), pat)
        coeffs["sources"][name] = rel
    assert len(coeffs["coeffs3d"]["j3d7pt"]) == 7
    assert len(coeffs["coeffs3d"]["j3d13pt"]) == 13
    assert len(coeffs["coeffs3d"]["poisson"]) == 19
    with open(os.path.join(HERE, "coefficients.json"), "w") as f:
        json.dump(coeffs, f, indent=1)

    rng = np.random.Generator(np.random.PCG64(20191117))
    arrays: dict[str, np.ndarray] = {}
    H, W = 37, 53

    for dt, tag in ((np.float32, "f32"), (np.float64, "f64")):
        # Star stencils: integer inputs 0..255 as in the reference tests
        # (stencil2D_9pt.cu:112), the reference's integer tables.
        ints = rng.integers(0, 256, size=(H, W)).astype(dt)
        arrays[f"int_in_{tag}"] = ints
        for r in range(1, 7):
            t = np.array(coeffs["tables2d"][f"star{r}"], dt)
            arrays[f"star{r}_out_{tag}"] = oracle.ref_convolution(ints, t)
        # Box stencils: uniform[-1,1) inputs, the reference's real tables.
        uni = rng.uniform(-1.0, 1.0, size=(H, W)).astype(dt)
        arrays[f"uni_in_{tag}"] = uni
        for name in ("box64", "box81", "box121"):
            t = np.array(coeffs["tables2d"][name], dt)
            arrays[f"{name}_out_{tag}"] = oracle.ref_convolution(uni, t)
        # Conv: weights rand()%21-10 style (conv2D.cu:115-119), integer image.
        for f in (2, 3, 4, 5, 6, 7, 11, 21):
            wt = rng.integers(-10, 11, size=(f, f)).astype(dt)
            arrays[f"conv{f}_w_{tag}"] = wt
            arrays[f"conv{f}_out_{tag}"] = oracle.ref_convolution(ints, wt)
        for fh, fw in ((3, 5), (4, 2), (1, 7)):
            wt = rng.integers(-10, 11, size=(fh, fw)).astype(dt)
            arrays[f"conv{fh}x{fw}_w_{tag}"] = wt
            arrays[f"conv{fh}x{fw}_out_{tag}"] = oracle.ref_convolution(ints, wt)
        # Temporal runs: get_random()+0.02121 inputs (stencil2d_temp_5pt.cu:12),
        # ITERATIVE_COUNT applications of Convolution with copy-back
        # (stencil2d_temp_5pt.cu:183-186): 5 steps of tmp5, 3 of tmp9.
        tin = (rng.random(size=(H, W)) + 0.02121).astype(dt)
        arrays[f"tmp_in_{tag}"] = tin
        for name, steps in (("tmp5", 5), ("tmp9", 3)):
            t = np.array(coeffs["tables2d"][name], dt)
            cur = tin
            for _ in range(steps):
                cur = oracle.ref_convolution(cur, t)
            arrays[f"{name}_out_{tag}"] = cur

        # 3D golds, N=16: getRandom3DArray-style inputs (common.hpp:62-74),
        # one call and two iterations with copy-back (tmp3d7pt-v2.cu:312-317).
        for n in (16,):
            cube = (rng.random(size=(n, n, n)) + 0.02121).astype(dt)
            arrays[f"cube{n}_in_{tag}"] = cube
            for g in ("j3d7pt", "j3d13pt", "poisson"):
                one = oracle.ref_gold3d(g, cube)
                two = oracle.ref_gold3d(g, one)
                arrays[f"{g}_n{n}_it1_{tag}"] = one
                arrays[f"{g}_n{n}_it2_{tag}"] = two

    np.savez_compressed(os.path.join(HERE, "ssam_golden.npz"), **arrays)
    size = os.path.getsize(os.path.join(HERE, "ssam_golden.npz"))
    print(f"wrote {len(arrays)} arrays, {size/1024:.0f} KiB")


if __name__ == "__main__":
    main()
