"""One large 2D grid over several GPUs: row slabs with halo exchange.

Each rank owns a contiguous band of rows (``shard.partition``).  A block of T
fused steps of a stencil with reach r needs r*T rows of each neighbour: the
ranks swap those halo rows with point-to-point sends (NCCL between GPUs over
NVLink, gloo on the CPU), then every rank runs the single-GPU kernel on its
band plus halos and keeps its own rows.  Rows beyond r*T of the band are
wrong after T steps only inside the halo, which is discarded; the grid's own
top and bottom edges are the first and last rank's buffer edges, so the ZERO
boundary there is the grid's boundary.

The exchange is one message per neighbour and temporal block; the stencil
itself is the caller's `compute(ext, steps) -> ext'` (``ssam_b200.stencil2d``
on the GPU).
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
    """`steps` steps on a grid distributed by rows: `local_rows` holds this
    rank's owned rows (shard.partition of `height`); blocks of up to `depth`
    fused steps, one halo exchange (radius * depth rows) before each.
    Returns the owned rows after `steps` steps."""
    import torch
    r = shard.ranks()
    halo = radius * depth
    b = band(height, r.rank, r.world, halo)
    if b.stop - b.start < halo and r.world > 1:
        raise ValueError("every rank must own at least radius * depth rows")
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


def stencil2d_compute(coeffs, radius: int, shape: int, stream=None):
    """The `compute` for `run` on the GPU: T fused steps of the library's 2D
    kernel on the extended band, zero padding at its edges (the grid's own
    edges for the first and last rank; discarded halo rows otherwise)."""
    from . import stencil2d

    def compute(ext, t):
        return stencil2d(ext, coeffs, radius, shape, steps=t, boundary="zero", stream=stream)
    return compute
