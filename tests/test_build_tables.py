"""The compiled-configuration tables of ssam_b200/build.py, checked on the
CPU: every 3D configuration fits one SM's shared memory and has the ring
depth its kernel needs, defaults are unique per group, and the 2D tables
cover what the entry points and the autotuner look up."""
from collections import Counter

import pytest

from ssam_b200.build import instances, instances_3d, instances_3d_t2, stream_instances

ES = {"f32": 4, "f64": 8, "bf16": 2, "f16": 2}
SMEM_PER_CTA = 227 * 1024


def smem_3d(dt, shape, r, py, nw, s, v=4):
    """Dynamic shared memory of a 3D CTA as the launcher requests it
    (Stencil3DCfg::SMEM): S slots of (32*V + 2*HX) x (NW*PY + 2*RYM) elements,
    staged as one box (or two halves when wider than 256 elements), each box
    rounded to 128 bytes; two mbarriers per slot, 128 bytes of alignment."""
    es = ES[dt]
    hx = 16 // es
    xw = 32 * v + 2 * hx
    nbox = 2 if xw > 256 else 1
    rym = 1 if shape == 1 else r
    yw = nw * py + 2 * rym
    slot = nbox * ((xw // nbox * yw * es + 127) // 128 * 128)
    return s * slot + 2 * s * 8 + 128


@pytest.mark.parametrize("inst", instances_3d(), ids=lambda c: "-".join(map(str, c)))
def test_3d_configuration_fits_and_has_its_ring(inst):
    dt, shape, r, py, nw, s, rhs, dflt, zreg, v = inst
    assert smem_3d(dt, shape, r, py, nw, s, v) <= SMEM_PER_CTA
    if v == 8:  # two TMA boxes of at most 256 elements, 16-byte rows
        bw = (32 * v + 2 * (16 // ES[dt])) // 2
        assert bw <= 256 and (bw * ES[dt]) % 16 == 0
    assert 32 * (nw + 1) <= 1024
    rh = 1 if shape == 1 else 0  # planes read for halos: z-RH .. z+RH
    need = r + rh + 2 if zreg else 2 * r + 2
    assert s >= need, f"ring of {s} slots, kernel needs {need}"
    if rhs:
        assert shape == 0 and r == 1  # the Jacobi sweep is the 7-point star


@pytest.mark.parametrize("inst", instances_3d(), ids=lambda c: "-".join(map(str, c)))
def test_3d_slot_layout(inst):
    """The shared-memory slot layout of Stencil3DCfg, restated: every box's
    TMA destination starts on a 128-byte boundary and its first column on a
    16-byte one (for any column tile), each lane's vector reads are aligned
    and inside the slot, the x-halo reads of lanes 0 and 31 stay inside their
    box's row, and lane L's first column is tile origin + L*V."""
    dt, shape, r, py, nw, s, rhs, dflt, zreg, v = inst
    es = ES[dt]
    hx = 16 // es
    tx = 32 * v
    nbox = 2 if tx + 2 * hx > 256 else 1
    bw = (tx + 2 * hx) // nbox
    rym = 1 if shape == 1 else r
    yw = nw * py + 2 * rym
    boxs = (bw * yw * es + 127) // 128 * 128 // es
    slot = nbox * boxs
    lpb = 32 // nbox
    assert bw <= 256 and (bw * es) % 16 == 0 and (boxs * es) % 128 == 0

    def col_off(lane):
        return (lane // lpb) * boxs + (hx if lane // lpb == 0 else 0) + (lane % lpb) * v

    for tile in range(3):
        for b in range(nbox):
            assert ((tile * tx - hx + b * bw) * es) % 16 == 0
    for lane in range(32):
        b = lane // lpb
        assert -hx + b * bw + col_off(lane) - b * boxs == lane * v
        for row in range(yw):
            a = row * bw + col_off(lane)
            assert 0 <= a and a + v <= slot
            if (v * es) % 16 == 0:
                assert (a * es) % 16 == 0
    for row in range(yw):
        for h in range(r):
            left = row * bw + col_off(0) - 1 - h
            right = row * bw + col_off(31) + v + h
            assert row * bw <= left < (row + 1) * bw
            assert (nbox - 1) * boxs + row * bw <= right < (nbox - 1) * boxs + (row + 1) * bw


def smem_3d_t2(dt, shape, r, py, nw, s, v):
    """Dynamic shared memory of a two-step 3D CTA (Stencil3DT2Cfg::SMEM): the
    input ring of the single-step layout plus D slots of the level-1 halo
    rows (2R rows of 32*V elements per consumer warp, rounded to 128 bytes),
    D = R + L + RH + 1 with L = RH = 1 for the 19-point operator, 0 for stars;
    plus a second 128 bytes of slack."""
    es = ES[dt]
    rh = 1 if shape == 1 else 0
    lag = max(0, rh + 1 - r)
    d = r + lag + rh + 1
    hb = (d * nw * 2 * r * 32 * v * es + 127) // 128 * 128
    return smem_3d(dt, shape, r, py, nw, s, v) + hb + 128


@pytest.mark.parametrize("inst", instances_3d_t2(), ids=lambda c: "-".join(map(str, c)))
def test_3d_two_step_configuration_limits(inst):
    """The static limits of stencil3d_t2.cuh hold for every compiled two-step
    configuration: it fits one SM's shared memory, one x-halo value a lane
    (2R columns x (PY + 2*EY) rows x 2 sides <= 32), 2R staged halo columns,
    PY >= R, a ring of 2R+2 slots, a tile taller than its 2R rows of overlap,
    and no more than 8 warps a CTA unless the registers allow it."""
    dt, shape, r, py, nw, s, v, dflt = inst
    es = ES[dt]
    ey = 1 if shape == 1 else 0
    assert smem_3d_t2(dt, shape, r, py, nw, s, v) <= SMEM_PER_CTA
    assert 2 * r * (py + 2 * ey) <= 32
    assert 2 * r <= 16 // es
    assert py >= r and s >= 2 * r + 2 and nw * py > 2 * r
    assert nw + 1 <= 9  # one CTA an SM: 168 registers a thread at 9 warps


def test_3d_two_step_groups():
    """One default per (dtype, shape, radius) group of two-step kernels, and
    every group has a single-step table beside it (odd step counts)."""
    groups = Counter((dt, shape, r) for (dt, shape, r, *_rest, dflt) in instances_3d_t2() if dflt)
    every = {(dt, shape, r) for (dt, shape, r, *_rest) in instances_3d_t2()}
    assert set(groups) == every and all(v == 1 for v in groups.values())
    single = {(dt, shape, r) for (dt, shape, r, _, _, _, rhs, _, _, _) in instances_3d() if not rhs}
    assert every <= single
    for dt in ("f32", "bf16"):
        for shape, r in ((0, 1), (0, 2), (1, 1)):
            assert (dt, shape, r) in every


def test_3d_groups_have_exactly_one_default():
    groups = Counter((dt, shape, r, rhs) for (dt, shape, r, _, _, _, rhs, dflt, _, _)
                     in instances_3d() if dflt)
    every = {(dt, shape, r, rhs) for (dt, shape, r, _, _, _, rhs, _, _, _) in instances_3d()}
    assert set(groups) == every and all(v == 1 for v in groups.values())


def test_3d_table_covers_the_entry_points():
    have = {(dt, shape, r, rhs) for (dt, shape, r, _, _, _, rhs, _, _, _) in instances_3d()}
    for dt in ("f32", "f64", "bf16", "f16"):
        for shape, r in ((0, 1), (0, 2), (1, 1)):
            assert (dt, shape, r, False) in have
    for dt in ("f32", "f64", "bf16"):  # Poisson sweep storage types
        assert (dt, 0, 1, True) in have


def test_2d_tables():
    win = set(instances())
    # the windowed fallback every streaming launcher hands unaligned grids to
    for (dt, star, r, seg, v) in stream_instances():
        assert seg >= 32 and (dt, star, r, r, 8, 1, v) in win
    # single-step kernels for every star r <= 6 and box r <= 5 in every type
    for dt in ("f32", "f64", "bf16", "f16"):
        for star, rmax in ((1, 6), (0, 5)):
            for r in range(1, rmax + 1):
                assert any(k[:4] == (dt, star, r, r) and k[5] == 1 for k in win)


def test_fused_streaming_kernels_have_windowed_fallbacks():
    """Grids the fused-step streaming launcher cannot take go to the windowed
    kernel of the same stencil and depth (P = 8)."""
    from ssam_b200.build import stream_t_instances
    win = set(instances())
    for (dt, star, r, seg, v, t) in stream_t_instances():
        assert seg >= 32 and t >= 2
        assert (dt, star, r, r, 8, t, v) in win
