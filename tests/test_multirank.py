"""The multi-rank plumbing of the benchmark (ssam_b200/shard.py) with two
gloo ranks on the CPU: the process group forms over 127.0.0.1, the timing
reduction returns the slowest rank's time on every rank, work partitions
cover every unit once, and a rank that never joins makes the others fail
within the short group timeout instead of hanging."""
import os
import socket
import subprocess
import sys

import pytest

from ssam_b200 import shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
from ssam_b200 import shard
r = shard.init("gloo", timeout_s={timeout})
shard.barrier()
t = shard.max_over_ranks(0.5 + r.rank)
part = list(shard.partition(10, r.rank, r.world))
print(json.dumps({{"rank": r.rank, "world": r.world, "max": t, "part": part}}), flush=True)
shard.finish()
"""


def launch(world, port, timeout=20, only=None):
    procs = []
    for rank in range(world):
        if only is not None and rank not in only:
            continue
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen(
            [sys.executable, "-c", WORKER.format(root=ROOT, timeout=timeout)], env=env,
            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    return procs


def test_two_gloo_ranks_share_the_slowest_time_and_partition_the_units():
    import json
    procs = launch(2, free_port())
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    assert all(o["world"] == 2 and o["max"] == 1.5 for o in outs)
    units = sorted(u for o in outs for u in o["part"])
    assert units == list(range(10))


def test_a_missing_rank_fails_the_others_instead_of_hanging():
    procs = launch(2, free_port(), timeout=5, only={0})
    out, err = procs[0].communicate(timeout=180)
    assert procs[0].returncode != 0


@pytest.mark.parametrize("n,world", [(10, 3), (3, 4), (256, 8), (0, 2)])
def test_partition_is_balanced_and_complete(n, world):
    parts = [shard.partition(n, r, world) for r in range(world)]
    sizes = [len(p) for p in parts]
    assert sum(sizes) == n and max(sizes) - min(sizes) <= 1
    assert [u for p in parts for u in p] == list(range(n))


def test_single_rank_needs_no_group():
    r = shard.ranks()
    assert shard.max_over_ranks(3.25) == 3.25
    assert shard.weak_rate(100.0, 4, 2.0) == 200.0
    assert r.world >= 1


SLAB_WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import numpy as np, torch
import oracle
from ssam_b200 import shard, slab
r = shard.init("gloo", timeout_s=30)
H, W, radius, steps, depth, bnd = {H}, {W}, {radius}, {steps}, {depth}, {bnd!r}
g = np.random.Generator(np.random.PCG64(5))
grid = g.uniform(-1, 1, size=(H, W))
m = g.random((2 * radius + 1, 2 * radius + 1)); m /= m.sum()
mine = shard.partition(H, r.rank, r.world)
local = torch.from_numpy(grid[mine.start:mine.stop].copy())
# the oracle stands in for the GPU kernel on the extended band (test only)
compute = lambda ext, t: torch.from_numpy(oracle.conv2d(ext.numpy(), m, bnd, steps=t))
out = slab.run(local, H, radius, steps, depth, compute)
want = oracle.conv2d(grid, m, bnd, steps=steps)[mine.start:mine.stop]
print(json.dumps({{"rank": r.rank, "maxerr": float(np.abs(out.numpy() - want).max())}}),
      flush=True)
shard.finish()
"""

ZSLAB_WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import numpy as np, torch
import oracle
from ssam_b200 import shard, slab
r = shard.init("gloo", timeout_s=30)
NZ, radius, steps, depth, bnd, p19 = {NZ}, {radius}, {steps}, {depth}, {bnd!r}, {p19}
g = np.random.Generator(np.random.PCG64(9))
grid = g.uniform(0, 1, size=(NZ, 11, 13))
f = 2 * radius + 1
taps = [(dz, dy, dx, g.random()) for dz in range(-radius, radius + 1)
        for dy in range(-radius, radius + 1) for dx in range(-radius, radius + 1)
        if (abs(dz) + abs(dy) + abs(dx) <= 2 if p19 else (dz, dy, dx).count(0) >= 2)]
mine = shard.partition(NZ, r.rank, r.world)
local = torch.from_numpy(grid[mine.start:mine.stop].copy())
def steps3d(a, t):
    for _ in range(t):
        a = oracle.taps3d(a, taps, bnd)
    return a
# the oracle stands in for the GPU kernel on the extended band (test only)
compute = lambda ext, t: torch.from_numpy(steps3d(ext.numpy(), t))
out = slab.run(local, NZ, radius, steps, depth, compute)
want = steps3d(grid, steps)[mine.start:mine.stop]
print(json.dumps({{"rank": r.rank, "maxerr": float(np.abs(out.numpy() - want).max())}}),
      flush=True)
shard.finish()
"""

GUARD_WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import torch
from ssam_b200 import shard, slab
r = shard.init("gloo", timeout_s=20)
mine = shard.partition({H}, r.rank, r.world)
try:
    slab.run(torch.zeros(mine.stop - mine.start, 5), {H}, {radius}, 3, {depth},
             lambda ext, t: ext)
    print(json.dumps({{"rank": r.rank, "raised": False}}), flush=True)
except ValueError:
    print(json.dumps({{"rank": r.rank, "raised": True}}), flush=True)
shard.finish()
"""


def run_workers(world, code_of_rank, timeout=180):
    import json
    port = free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code_of_rank], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        o, err = p.communicate(timeout=timeout)
        assert p.returncode == 0, err
        out.append(json.loads(o.strip().splitlines()[-1]))
    return out


@pytest.mark.parametrize("world,H,radius,steps,depth,bnd",
                         [(2, 40, 1, 5, 2, "zero"), (3, 31, 2, 4, 4, "zero"),
                          (2, 12, 2, 3, 1, "zero"), (2, 40, 1, 5, 2, "copy"),
                          (3, 31, 2, 4, 4, "copy")])
def test_row_slabs_with_halo_exchange_match_the_whole_grid(world, H, radius, steps, depth, bnd):
    """Row slabs over gloo ranks, halos of radius * depth rows swapped before
    every temporal block: each rank's rows equal the same steps on the whole
    grid (bit for bit: the same arithmetic on the same values), under the
    ZERO and the COPY boundary."""
    code = SLAB_WORKER.format(root=ROOT, H=H, W=23, radius=radius, steps=steps, depth=depth,
                              bnd=bnd)
    for res in run_workers(world, code):
        assert res["maxerr"] == 0.0, res


@pytest.mark.parametrize("world,NZ,radius,steps,depth,bnd,p19",
                         [(2, 20, 1, 5, 2, "zero", False), (3, 25, 2, 4, 2, "copy", False),
                          (2, 18, 1, 4, 2, "copy", True), (3, 16, 1, 3, 1, "zero", True)])
def test_z_slabs_of_a_3d_grid_match_the_whole_grid(world, NZ, radius, steps, depth, bnd, p19):
    """z-slabs of one 3D grid (star r = 1, 2 and the 19-point pattern), halos
    of radius * depth planes swapped before every temporal block: each rank's
    planes equal the steps on the whole grid bit for bit, ZERO and COPY."""
    code = ZSLAB_WORKER.format(root=ROOT, NZ=NZ, radius=radius, steps=steps, depth=depth,
                               bnd=bnd, p19=p19)
    for res in run_workers(world, code):
        assert res["maxerr"] == 0.0, res


def test_too_thin_bands_fail_on_every_rank():
    """10 rows over 3 ranks give bands of 4, 3 and 3; a halo of 4 rows is
    thicker than the thinnest band, so every rank (the one owning 4 rows
    too) raises before any exchange instead of one of them waiting for
    peers that gave up."""
    code = GUARD_WORKER.format(root=ROOT, H=10, radius=2, depth=2)
    res = run_workers(3, code, timeout=60)
    assert all(r["raised"] for r in res), res
