"""Many uneven grids in one persistent launch (ssam_stencil2d_batched) give
the oracle's result on every grid, and the same bits as stepping each grid
with its own launches."""
import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_cases import stable_seed, assert_rel_close, magnitude2d, normalised, rng, star_matrix

pytestmark = pytest.mark.gpu


def _grids(n, lo, hi, seed, dt=np.float32):
    g = rng(seed)
    sides = np.exp(g.uniform(np.log(lo), np.log(hi), size=(n, 2))).astype(int)
    return [g.uniform(0, 1, size=(int(h), int(w))).astype(dt) for h, w in sides]


@pytest.mark.parametrize("kind,r", [("star", 1), ("box", 2), ("box", 1), ("star", 2),
                                    ("box", 3)])
@pytest.mark.parametrize("steps", [1, 3, 7, 50])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_batched_vs_oracle_and_per_grid(cuda, kind, r, steps, bnd):
    hosts = _grids(12, 9, 300, stable_seed(kind, r, steps))
    if kind == "star":
        c = normalised((4 * r + 1,), r)
        m = star_matrix(c, r)
        shape = S.STAR
    else:
        m = normalised((2 * r + 1, 2 * r + 1), r)
        c = m.ravel()
        shape = S.BOX
    srcs = [torch.from_numpy(h).to(cuda) for h in hosts]
    got = S.stencil2d_batched(srcs, c, r, shape, steps, bnd, persistent=True)
    ref = S.stencil2d_batched(srcs, c, r, shape, steps, bnd, persistent=False)
    S.device_status()
    for h, a, b in zip(hosts, got, ref):
        a = a.cpu().numpy()
        want = oracle.conv2d(h, m.astype(np.float32), bnd, steps=steps)
        assert_rel_close(a, want, magnitude2d(h, m, bnd, steps), 1e-5 * steps, f"{h.shape}")
        np.testing.assert_array_equal(a, b.cpu().numpy())


@pytest.mark.parametrize("tdt", [torch.float64, torch.bfloat16])
def test_batched_other_dtypes(cuda, tdt):
    hosts = _grids(6, 20, 200, 5)
    c = normalised((5,), 1)
    m = star_matrix(c, 1)
    srcs = [torch.from_numpy(h).to(tdt).to(cuda) for h in hosts]
    got = S.stencil2d_batched(srcs, c, 1, S.STAR, 9, "copy")
    for s_, a in zip(srcs, got):
        x = s_.double().cpu().numpy()
        want = oracle.conv2d(x, m, "copy", steps=9)
        rel = 1e-12 * 9 if tdt == torch.float64 else 2.0**-8 * 9
        scale = np.maximum(np.abs(want), magnitude2d(x, m, "copy", 9))
        assert_rel_close(a.double().cpu().numpy(), want, scale, rel, str(tdt))


@pytest.mark.parametrize("kind,layout", [("star1", "dense"), ("star1", "pitched"),
                                         ("box2", "pitched")])
def test_batched_256_uneven_grids_config4(cuda, kind, layout):
    """The benchmark batch: 256 grids, sides log-uniform in [64, 2048], the
    5-point star or the 5x5 box, 50 steps, COPY; the persistent launch
    equals the per-grid launches bit for bit, and every one of the 256 grids
    matches the oracle (rel 1e-5 per step of sum|c||x|).  Dense rows take the
    windowed phases, pitched rows (the bench's layout) the row-streaming
    ones."""
    g = rng(256)
    sides = np.exp(g.uniform(np.log(64), np.log(2048), size=(256, 2))).astype(int)
    hosts = [g.uniform(0, 1, size=(int(h), int(w))).astype(np.float32) for h, w in sides]
    if kind == "star1":
        r, shape, c = 1, S.STAR, [0.2] * 5
        m = star_matrix(c, 1)
    else:
        r, shape = 2, S.BOX
        m = normalised((5, 5), 257)
        c = list(m.ravel())
    srcs = [_pitched(h, cuda) if layout == "pitched" else torch.from_numpy(h).to(cuda)
            for h in hosts]
    got = S.stencil2d_batched(srcs, c, r, shape, 50, "copy", persistent=True)
    ref = S.stencil2d_batched(srcs, c, r, shape, 50, "copy", persistent=False)
    S.device_status()
    for a, b in zip(got, ref):
        assert torch.equal(a, b)
    mf = m.astype(np.float32)
    for i, (h0, out) in enumerate(zip(hosts, got)):
        want = oracle.conv2d(h0, mf, "copy", steps=50)
        assert_rel_close(out.cpu().numpy(), want, magnitude2d(h0, m, "copy", 50), 5e-4,
                         f"grid {i} ({h0.shape[0]} x {h0.shape[1]})")


def _pitched(host, cuda, tdt=torch.float32):
    """A grid whose rows start on 128-byte boundaries (pitch rounded up),
    the layout that lets the persistent launch stream rows."""
    h, w = host.shape
    es = torch.empty((), dtype=tdt).element_size()
    pitch = -(-w * es // 128) * 128 // es
    base = torch.zeros(h, pitch, dtype=tdt, device=cuda)
    view = base[:, :w]
    view.copy_(torch.from_numpy(host).to(tdt))
    return view


@pytest.mark.parametrize("kind,r", [("star", 1), ("box", 2), ("box", 1), ("star", 2),
                                    ("box", 3)])
@pytest.mark.parametrize("steps", [1, 2, 7])
@pytest.mark.parametrize("bnd", ["zero", "copy"])
def test_batched_pitched_grids_stream_rows(cuda, kind, r, steps, bnd):
    """Pitched rows: the persistent launch's single-step phases take the
    row-streaming warp tiles (widths need not be a multiple of the strip's
    chunk); results equal the oracle's and, bit for bit, the per-grid
    launches', and nothing beyond each grid's width is written."""
    hosts = _grids(14, 1, 260, stable_seed(kind, r, steps, bnd))
    if kind == "star":
        c = normalised((4 * r + 1,), r)
        m = star_matrix(c, r)
        shape = S.STAR
    else:
        m = normalised((2 * r + 1, 2 * r + 1), r)
        c = m.ravel()
        shape = S.BOX
    srcs = [_pitched(h, cuda) for h in hosts]
    dsts = [_pitched(np.full(h.shape, 0, np.float32), cuda) for h in hosts]
    for d in dsts:
        d._base.fill_(9.0)  # the pitch padding must keep this value
    got = S.stencil2d_batched(srcs, c, r, shape, steps, bnd, dsts=dsts, persistent=True)
    ref = S.stencil2d_batched(srcs, c, r, shape, steps, bnd, persistent=False)
    S.device_status()
    for h, a, b, d in zip(hosts, got, ref, dsts):
        pad = d._base[:, h.shape[1]:]
        assert bool((pad == 9.0).all()), "wrote past a grid's width"
        a = a.cpu().numpy()
        want = oracle.conv2d(h, m.astype(np.float32), bnd, steps=steps)
        assert_rel_close(a, want, magnitude2d(h, m, bnd, steps), 1e-5 * steps, f"{h.shape}")
        np.testing.assert_array_equal(a, b.cpu().numpy())


@pytest.mark.parametrize("tdt,rel", [(torch.float64, 1e-12), (torch.bfloat16, 2.0**-8)])
@pytest.mark.parametrize("bnd", ["copy", "clamp"])
def test_batched_pitched_other_dtypes_and_clamp(cuda, tdt, rel, bnd):
    steps = 1 if bnd == "clamp" else 5
    hosts = _grids(9, 3, 150, 17)
    c = normalised((5,), 1)
    m = star_matrix(c, 1)
    srcs = [_pitched(h, cuda, tdt) for h in hosts]
    got = S.stencil2d_batched(srcs, c, 1, S.STAR, steps, bnd)
    for s_, a in zip(srcs, got):
        x = s_.double().cpu().numpy()
        want = oracle.conv2d(x, m, bnd, steps=steps)
        scale = np.maximum(np.abs(want), magnitude2d(x, m, bnd, steps))
        assert_rel_close(a.double().cpu().numpy(), want, scale, rel * steps, f"{tdt} {bnd}")


def test_grid_barrier_that_gives_up_reports_a_timeout(cuda):
    """The bounded-wait error path on the GPU, in the allowed form: a test
    hook makes every grid barrier of the persistent launch wait for one CTA
    more than the launch has, with a 1 ms limit.  Every CTA gives up at the
    first barrier (no copy or MMA is in flight there), records code 4 and
    returns; ssam_device_status reports SSAM_ERR_TIMEOUT, and with the hook
    off the next call on the same device succeeds and matches the oracle."""
    lib = S.lib()
    hosts = _grids(6, 40, 200, 77)
    srcs = [torch.from_numpy(h).to(cuda) for h in hosts]
    coeffs = [0.2] * 5
    assert lib.ssam_debug_batched_barrier(1, 1_000_000) == S.OK
    try:
        S.stencil2d_batched(srcs, coeffs, 1, S.STAR, steps=6, boundary="copy")
        with pytest.raises(S.SsamError) as exc:
            S.device_status()
        assert exc.value.status == S.ERR_TIMEOUT
        assert "code 4" in str(exc.value)
    finally:
        assert lib.ssam_debug_batched_barrier(0, 0) == S.OK
    outs = S.stencil2d_batched(srcs, coeffs, 1, S.STAR, steps=6, boundary="copy")
    S.device_status()
    m = star_matrix(coeffs, 1).astype(np.float32)
    for h, o in zip(hosts, outs):
        want = oracle.conv2d(h, m, "copy", steps=6)
        assert np.abs(o.cpu().numpy() - want).max() <= 6e-5



@pytest.mark.parametrize("depth", ["4", "6", "8"])
@pytest.mark.parametrize("tdt,kind,r", [(torch.float32, "star", 1), (torch.float32, "box", 2),
                                        (torch.float32, "star", 3), (torch.float64, "box", 2),
                                        (torch.bfloat16, "star", 1), (torch.bfloat16, "box", 2)])
def test_batched_stream_depths(cuda, monkeypatch, depth, tdt, kind, r):
    """Every compiled depth of the persistent streaming kernel (rows in
    flight a warp; SSAM_BATCH_DEPTH pins one) gives the bits of a chain of
    single-step per-grid launches (a 16-bit grid is rounded to its storage
    type after every step there too).  COPY boundary, so that every phase is
    a single streamed step; 16-byte aligned rows."""
    monkeypatch.setenv("SSAM_BATCH_DEPTH", depth)
    hosts = _grids(10, 20, 400, stable_seed(str(tdt), kind, r))
    if kind == "star":
        c = normalised((4 * r + 1,), r)
        shape = S.STAR
    else:
        c = normalised((2 * r + 1, 2 * r + 1), r).ravel()
        shape = S.BOX
    srcs = []
    for h in hosts:  # rows pitched to whole 16-byte chunks of 8 columns
        pitch = -(-h.shape[1] // 8) * 8
        base = torch.zeros(h.shape[0], pitch, dtype=tdt, device=cuda)
        base[:, :h.shape[1]] = torch.from_numpy(h).to(tdt)
        srcs.append(base[:, :h.shape[1]])
    got = S.stencil2d_batched(srcs, c, r, shape, 5, "copy", persistent=True)
    ref = srcs
    for _ in range(5):
        ref = S.stencil2d_batched(ref, c, r, shape, 1, "copy", persistent=False)
    S.device_status()
    for a, b in zip(got, ref):
        assert torch.equal(a, b), f"depth {depth} {a.shape}"
