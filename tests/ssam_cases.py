"""Shared test data: the reference's coefficient tables, seeded inputs of the
benchmark distributions, the golden fixtures, and the error measure used by
the parity tests."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN_DIR = os.path.join(HERE, "golden")

_coeffs = None
_golden = None


def coefficients() -> dict:
    global _coeffs
    if _coeffs is None:
        with open(os.path.join(GOLDEN_DIR, "coefficients.json")) as f:
            _coeffs = json.load(f)
    return _coeffs


def golden():
    global _golden
    if _golden is None:
        _golden = dict(np.load(os.path.join(GOLDEN_DIR, "ssam_golden.npz")))
    return _golden


def table2d(name: str, dtype=np.float64) -> np.ndarray:
    return np.array(coefficients()["tables2d"][name], dtype)


def star_matrix(coeffs, r: int) -> np.ndarray:
    """(2r+1)^2 matrix from the reference's argument order c, n, s, w, e..."""
    f = 2 * r + 1
    m = np.zeros((f, f))
    m[r, r] = coeffs[0]
    for k in range(1, r + 1):
        n, s, w, e = coeffs[1 + 4 * (k - 1): 5 + 4 * (k - 1)]
        m[r - k, r], m[r + k, r], m[r, r - k], m[r, r + k] = n, s, w, e
    return m


# 3D tap lists in the order the reference golds sum them -------------------

def taps_j3d7pt(dtype=np.float64):
    """v2::j3d7pt_gold (tmp3d7pt-v2.cu:285-292): _F3d7PT_<z><y><x>, offset = digit-1."""
    c = coefficients()["coeffs3d"]["j3d7pt"]
    order = ["011", "101", "111", "121", "110", "112", "211"]
    return [(int(k[0]) - 1, int(k[1]) - 1, int(k[2]) - 1, dtype(c[k])) for k in order]


def taps_j3d13pt(dtype=np.float64):
    """j3d13pt_gold (tmp3d13pt.cu:310-323): offset = digit-2."""
    c = coefficients()["coeffs3d"]["j3d13pt"]
    order = ["022", "122", "222", "322", "422", "212", "202", "232", "242",
             "220", "221", "223", "224"]
    return [(int(k[0]) - 2, int(k[1]) - 2, int(k[2]) - 2, dtype(c[k])) for k in order]


# seeded inputs -------------------------------------------------------------

def stable_seed(*parts) -> int:
    """A seed derived from the test's parameters that is the same in every
    process (Python's hash() of strings is randomised per process, which
    would make a failing case impossible to replay)."""
    import zlib
    return zlib.crc32(repr(parts).encode()) & 0x7FFFFFFF


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def uniform(shape, lo, hi, dtype, seed):
    return rng(seed).uniform(lo, hi, size=shape).astype(dtype)


def normalised(shape, seed):
    """Coefficients uniform[0,1) normalised to sum 1 (the box-family config)."""
    c = rng(seed).random(size=shape)
    return c / c.sum()


# error measure -------------------------------------------------------------

def magnitude2d(src: np.ndarray, filt: np.ndarray, boundary="zero", steps=1):
    """Per-cell scale of the summation, sum |w| |x|, iterated like the
    operator: the natural bound for the rounding error of any summation
    order.  Computed in float64 by the oracle."""
    import oracle
    return oracle.conv2d(np.abs(src).astype(np.float64), np.abs(filt).astype(np.float64),
                         boundary, steps)


def assert_rel_close(got, want, scale, rel, what=""):
    """|got - want| <= rel * max(scale, tiny) everywhere."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    scale = np.maximum(np.asarray(scale, np.float64), 1e-30)
    err = np.abs(got - want) / scale
    worst = np.unravel_index(np.argmax(err), err.shape) if err.size else ()
    assert err.size == 0 or err.max() <= rel, (
        f"{what}: max scaled error {err.max():.3e} > {rel:.1e} at {worst}: "
        f"got {got[worst]!r} want {want[worst]!r}")
