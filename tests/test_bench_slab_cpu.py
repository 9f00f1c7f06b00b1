"""bench.py --slab on CPU ranks (gloo, world size 2): the levels each rank
takes of the jets state (slab_levels) tile the grid, and the halo planes the
slab transport moves (halo_exchange, the same call DistSlab makes) give each
rank the planes of its periodic neighbours in z.  No GPU: the arrays are CPU
tensors."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from ps3d_b200.slab import K_DOWN, K_UP, halo_exchange


def test_slab_levels_tile_the_grid():
    for nz in (16, 64, 128):
        for world in (1, 2, 4, 8):
            if nz % world:
                continue
            got = []
            for r in range(world):
                k0, nzl = bench.slab_levels(nz, world, r)
                assert nzl == nz // world
                got.extend(range(k0, k0 + nzl))
            assert got == list(range(nz))


def _worker(rank, world, port, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        nz, ny, nx = 8, 3, 4
        g = np.arange(nz * ny * nx, dtype=np.float64).reshape(nz, ny, nx)   # one global field
        k0, nzl = bench.slab_levels(nz, world, rank)
        mine = g[k0:k0 + nzl]
        plane = ny * nx
        # the state halos: the bottom interior plane goes down, the top one up (4 fields each)
        nd, nu = K_DOWN[0], K_UP[0]
        hs = torch.zeros(8 * plane, dtype=torch.float64)
        for f in range(nd):
            hs[f * plane:(f + 1) * plane] = torch.from_numpy(mine[0].ravel() + 1000.0 * f)
        for f in range(nu):
            hs[(nd + f) * plane:(nd + f + 1) * plane] = torch.from_numpy(mine[-1].ravel() + 1000.0 * f)
        hr = torch.full((8 * plane,), -1.0, dtype=torch.float64)
        halo_exchange(hs, hr, plane, 0, rank, world)
        below = g[(k0 - 1) % nz].ravel()
        above = g[(k0 + nzl) % nz].ravel()
        for f in range(nu):   # from below: its top plane
            assert np.array_equal(hr[f * plane:(f + 1) * plane].numpy(), below + 1000.0 * f)
        for f in range(nd):   # from above: its bottom plane
            assert np.array_equal(hr[(nu + f) * plane:(nu + f + 1) * plane].numpy(), above + 1000.0 * f)
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except Exception as e:   # reported to the parent
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world", [2])
def test_bench_slab_partition_and_halos_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29850 + world
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert all(v == "ok" for v in res.values()), res
