"""One large grid over several GPUs: slabs along the slowest axis with halo
exchange -- row slabs of a 2D grid, z-slabs of a 3D one.

Each rank owns a contiguous band of rows or planes (``shard.partition`` of
the leading axis).  A block of T fused steps of a stencil with reach r needs
r*T rows (planes) of each neighbour: the ranks swap those halo slices with
point-to-point sends (NCCL between GPUs over NVLink, gloo on the CPU), then
every rank runs the single-GPU kernel on its band plus halos and keeps its
own slices.  Slices within r*T of a cut are wrong after T steps only inside
the halo, which is discarded: under ZERO the cut reads zeros, under COPY the
cut's outer r slices stay fixed, and either way the damage travels r slices
a step.  The grid's own first and last slices are the first and last rank's
buffer edges, so the boundary rule there is the grid's.

The exchange is one message per neighbour and temporal block; the stencil
itself is the caller's `compute(ext, steps) -> ext'` (``stencil2d_compute``
or ``stencil3d_compute`` on the GPU).
"""
from __future__ import annotations

from dataclasses import dataclass

from . import shard


@dataclass
class Band:
    start: int  # first owned row
    stop: int   # one past the last owned row
    lo: int     # first row of the extended buffer (start - halo, or 0)
    hi: int     # one past its last row (stop + halo, or the grid height)


def band(height: int, rank: int, world: int, halo: int) -> Band:
    """Owned rows of `rank` and the rows its extended buffer covers."""
    p = shard.partition(height, rank, world)
    return Band(p.start, p.stop, max(0, p.start - halo), min(height, p.stop + halo))


def check_bands(height: int, world: int, halo: int) -> None:
    """Every rank must own at least `halo` slices (a neighbour's halo may
    only hold rows that the neighbour owns).  The test is on the smallest
    band of the partition -- the same on every rank -- so all ranks raise
    together instead of some entering the exchange and waiting for a peer
    that gave up."""
    if world > 1 and height // world < halo:
        raise ValueError(f"every rank must own at least radius * depth = {halo} slices; "
                         f"{height} slices over {world} ranks leave {height // world}")


def exchange(ext, b: Band, height: int, halo: int, rank: int, world: int):
    """Fill the halo rows of `ext` (rows b.lo .. b.hi of the grid, owned rows
    already current) from the neighbouring ranks."""
    import torch.distributed as dist
    ops = []
    own0, own1 = b.start - b.lo, b.stop - b.lo  # owned rows inside ext
    if rank > 0 and b.start > 0:
        n_up = b.start - b.lo
        ops.append(dist.P2POp(dist.isend, ext[own0:own0 + halo].contiguous(), rank - 1))
        ops.append(dist.P2POp(dist.irecv, ext[0:n_up], rank - 1))
    if rank < world - 1 and b.stop < height:
        n_dn = b.hi - b.stop
        ops.append(dist.P2POp(dist.isend, ext[own1 - halo:own1].contiguous(), rank + 1))
        ops.append(dist.P2POp(dist.irecv, ext[own1:own1 + n_dn], rank + 1))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return ext


def run(local_rows, height: int, radius: int, steps: int, depth: int, compute):
    """`steps` steps on a grid distributed along its leading axis:
    `local_rows` holds this rank's owned rows of a 2D grid or planes of a 3D
    one (shard.partition of `height`); blocks of up to `depth` fused steps,
    one halo exchange (radius * depth slices) before each.  Returns the
    owned slices after `steps` steps."""
    import torch
    r = shard.ranks()
    halo = radius * depth
    check_bands(height, r.world, halo)
    b = band(height, r.rank, r.world, halo)
    ext = torch.zeros((b.hi - b.lo,) + tuple(local_rows.shape[1:]), dtype=local_rows.dtype,
                      device=local_rows.device)
    own0 = b.start - b.lo
    ext[own0:own0 + (b.stop - b.start)] = local_rows
    done = 0
    while done < steps:
        t = min(depth, steps - done)
        if r.world > 1:
            exchange(ext, b, height, halo, r.rank, r.world)  # the full halo, even if t < depth
        out = compute(ext, t)
        ext[own0:own0 + (b.stop - b.start)] = out[own0:own0 + (b.stop - b.start)]
        done += t
    return ext[own0:own0 + (b.stop - b.start)].clone()


def stencil2d_compute(coeffs, radius: int, shape: int, boundary: str = "zero", stream=None):
    """The `compute` for `run` on the GPU: T fused steps of the library's 2D
    kernel on the extended band with the grid's boundary rule (ZERO or COPY)
    at the band's edges -- the grid's own edges for the first and last rank,
    discarded halo rows otherwise."""
    from . import stencil2d

    if boundary not in ("zero", "copy"):
        raise ValueError("slabs take the ZERO or COPY boundary (CLAMP is single-step only)")

    def compute(ext, t):
        return stencil2d(ext, coeffs, radius, shape, steps=t, boundary=boundary, stream=stream)
    return compute


def stencil3d_compute(cube, radius: int, shape: int, boundary: str = "zero", stream=None):
    """The `compute` for `run` on z-slabs of a 3D grid: T steps of the
    library's 3D kernels (``stencil3d``) on the extended band, ZERO or COPY."""
    from . import stencil3d

    if boundary not in ("zero", "copy"):
        raise ValueError("3D grids take the ZERO or COPY boundary")

    def compute(ext, t):
        return stencil3d(ext, cube, radius, shape, steps=t, boundary=boundary, stream=stream)
    return compute
