"""The oracle (CPU restatement of the reference golds) is pinned to the
reference before anything is compared with it:

* against the committed golden fixtures, which were produced by the
  reference's own compiled golds (tests/golden/make_golden.py) -- always;
* against the compiled reference golds in oracle/_ref directly, on fresh
  seeded inputs and edge shapes -- where oracle/_ref is built.

All comparisons here are bit-exact: same algorithm, same order, same types.
"""
import numpy as np
import pytest

import oracle
from ssam_b200.workloads import gaussian_rhs
from ssam_cases import stable_seed, golden, rng, table2d, taps_j3d13pt, taps_j3d7pt

DT = {"f32": np.float32, "f64": np.float64}


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("r", range(1, 7))
def test_star_tables_match_golden(tag, r):
    g = golden()
    src = g[f"int_in_{tag}"]
    out = oracle.conv2d(src, table2d(f"star{r}", DT[tag]))
    np.testing.assert_array_equal(out, g[f"star{r}_out_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("name", ["box64", "box81", "box121"])
def test_box_tables_match_golden(tag, name):
    g = golden()
    out = oracle.conv2d(g[f"uni_in_{tag}"], table2d(name, DT[tag]))
    np.testing.assert_array_equal(out, g[f"{name}_out_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("f", ["2", "3", "4", "5", "6", "7", "11", "21", "3x5", "4x2", "1x7"])
def test_conv_matches_golden(tag, f):
    g = golden()
    out = oracle.conv2d(g[f"int_in_{tag}"], g[f"conv{f}_w_{tag}"])
    np.testing.assert_array_equal(out, g[f"conv{f}_out_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("name,steps", [("tmp5", 5), ("tmp9", 3)])
def test_temporal_matches_golden(tag, name, steps):
    g = golden()
    out = oracle.conv2d(g[f"tmp_in_{tag}"], table2d(name, DT[tag]), steps=steps)
    np.testing.assert_array_equal(out, g[f"{name}_out_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("gold", ["j3d7pt", "j3d13pt", "poisson"])
def test_3d_golds_match_golden(tag, gold):
    g = golden()
    cube = g[f"cube16_in_{tag}"]
    dt = DT[tag]

    def one(x):
        if gold == "poisson":
            return oracle.poisson19(x, "gold")
        taps = taps_j3d7pt(dt) if gold == "j3d7pt" else taps_j3d13pt(dt)
        return oracle.taps3d(x, taps, "gold")

    it1 = one(cube)
    np.testing.assert_array_equal(it1, g[f"{gold}_n16_it1_{tag}"])
    np.testing.assert_array_equal(one(it1), g[f"{gold}_n16_it2_{tag}"])


def test_check_error3d_restatement():
    a = rng(3).random((6, 7, 8))
    b = a.copy()
    b[2, 3, 4] += 0.5
    rms, mx = oracle.rms_max_error(a, b, 1, 1)
    assert mx == pytest.approx(0.5)
    assert rms == pytest.approx(np.sqrt(0.25 / (4 * 5 * 6)))


# ---- direct comparison with the compiled reference (where it is built) ----

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("shape", [(1, 1), (1, 9), (9, 1), (2, 3), (17, 33), (64, 50)])
@pytest.mark.parametrize("fshape", [(3, 3), (5, 5), (2, 2), (4, 7), (11, 11)])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_conv_vs_compiled_reference(shape, fshape, dt):
    g = rng(stable_seed(shape, fshape))
    src = g.uniform(-1, 1, size=shape).astype(dt)
    filt = g.uniform(-1, 1, size=fshape).astype(dt)
    np.testing.assert_array_equal(oracle.conv2d(src, filt), oracle.ref_convolution(src, filt))


@needs_ref
@pytest.mark.parametrize("n", [8, 12, 20])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_3d_vs_compiled_reference(n, dt):
    cube = (rng(n).random((n, n, n)) + 0.02121).astype(dt)
    np.testing.assert_array_equal(oracle.taps3d(cube, taps_j3d7pt(dt), "gold"),
                                  oracle.ref_gold3d("j3d7pt", cube))
    np.testing.assert_array_equal(oracle.taps3d(cube, taps_j3d13pt(dt), "gold"),
                                  oracle.ref_gold3d("j3d13pt", cube))
    np.testing.assert_array_equal(oracle.poisson19(cube, "gold"),
                                  oracle.ref_gold3d("poisson", cube))


# ---- boundary conventions of the restatement ------------------------------

def test_copy_boundary_keeps_ring_and_matches_zero_pad_inside():
    src = rng(5).random((20, 24)).astype(np.float64)
    filt = rng(6).random((5, 5))
    z = oracle.conv2d(src, filt, "zero")
    c = oracle.conv2d(src, filt, "copy")
    np.testing.assert_array_equal(c[2:-2, 2:-2], z[2:-2, 2:-2])
    ring = np.ones_like(src, bool)
    ring[2:-2, 2:-2] = False
    np.testing.assert_array_equal(c[ring], src[ring])


def test_clamp_boundary_equals_edge_padded_zero_conv():
    src = rng(7).random((13, 11))
    filt = rng(8).random((3, 3))
    padded = np.pad(src, 1, mode="edge")
    want = oracle.conv2d(padded, filt, "zero")[1:-1, 1:-1]
    np.testing.assert_allclose(oracle.conv2d(src, filt, "clamp"), want, rtol=0, atol=1e-15)


# ---- Poisson restatement (no reference code exists: checked by identities) --

def test_poisson_residual_identity_and_jacobi_fixed_point():
    g = rng(11)
    u = g.standard_normal((2, 9, 9, 9))
    # r = 0 - A u  =>  f := A u makes u the exact discrete solution
    r, rel0 = oracle.residual7(np.zeros_like(u), u)
    # f = 0: the residual norm itself (the library's rule), not a division by 0
    np.testing.assert_allclose(rel0, np.sqrt((r.reshape(2, -1) ** 2).sum(axis=1)), rtol=1e-12)
    f = -r
    _, rel = oracle.residual7(f, u)
    assert rel.max() < 1e-13
    # the exact solution is a fixed point of the Jacobi sweep
    np.testing.assert_allclose(oracle.jacobi7(f, u, 3), u, rtol=0, atol=1e-12)


def test_poisson_jacobi_reduces_residual():
    f = gaussian_rhs(2, 12, 5)
    u = oracle.jacobi7(f, np.zeros_like(f), 400)
    _, rel = oracle.residual7(f, u)
    assert rel.max() < 0.5
