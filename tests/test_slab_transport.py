"""The z-slab transports over torch.distributed on CPU (gloo, world sizes 2
and 3): the halo planes reach the right neighbours and the two all-to-all
transposes turn level slabs into column slabs and back, with the buffer
layouts slab.cu packs and unpacks (xbuf [r][nzl][ccnt[r]] complex, colbuf
[src][nzl][ccnt[rank]])."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ps3d_b200.slab import K_DOWN, K_UP, columns_backward, columns_forward, halo_exchange


def _counts(ncols, n):
    b = [ncols * r // n for r in range(n + 1)]
    return [b[r + 1] - b[r] for r in range(n)], b[:-1]


def _worker(rank, world, port, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        plane = 6
        # halos: every plane carries (sender rank, which, position) so the receiver can tell
        for which in (0, 1):
            nd, nu = K_DOWN[which], K_UP[which]
            hs = torch.zeros(8 * plane, dtype=torch.float64)
            for t in range(nd + nu):
                hs[t * plane:(t + 1) * plane] = 1000 * rank + 100 * which + t
            hr = torch.full((8 * plane,), -1.0, dtype=torch.float64)
            halo_exchange(hs, hr, plane, which, rank, world)
            below, above = (rank - 1) % world, (rank + 1) % world
            for t in range(nu):   # from below: what it sent up (its positions nd .. nd+nu-1)
                assert torch.all(hr[t * plane:(t + 1) * plane] == 1000 * below + 100 * which + nd + t)
            for t in range(nd):   # from above: what it sent down (positions 0 .. nd-1)
                assert torch.all(hr[(nu + t) * plane:(nu + t + 1) * plane] == 1000 * above + 100 * which + t)
        # transposes: a global complex array G[nz][ncols]; rank r holds levels r*nzl ..
        nzl, ncols = 3, 17
        counts, cbeg = _counts(ncols, world)
        rng = np.random.default_rng(0)
        G = rng.standard_normal((nzl * world, ncols)) + 1j * rng.standard_normal((nzl * world, ncols))
        FS = G[rank * nzl:(rank + 1) * nzl]
        xb = np.concatenate([FS[:, cbeg[r]:cbeg[r] + counts[r]].ravel() for r in range(world)])
        x = torch.from_numpy(xb.view(np.float64).copy())
        col = torch.zeros(2 * nzl * world * counts[rank], dtype=torch.float64)
        columns_forward(x, col, counts, nzl, rank)
        got = col.numpy().view(np.complex128).reshape(nzl * world, counts[rank])
        assert np.array_equal(got, G[:, cbeg[rank]:cbeg[rank] + counts[rank]])
        x2 = torch.zeros_like(x)
        columns_backward(x2, col, counts, nzl, rank)
        assert torch.equal(x2, x)
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except Exception as e:   # report to the parent instead of hanging it
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_slab_transports_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + world
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res == {r: "ok" for r in range(world)}, res


def test_combine_diagnostics_matches_whole_grid():
    """The ranks' partial sums and maxima combine to the whole grid's
    diagnose values (global_sum / global_max, parallel_mpi.f90:37-67)."""
    import numpy as np
    from ps3d_b200.slab import combine_diagnostics
    rng = np.random.default_rng(4)
    nz, ny, nx, nr = 8, 4, 6, 4
    u, v, w, b = (rng.standard_normal((nz, ny, nx)) for _ in range(4))
    dsqr, n0 = 0.5, 2e-3

    def part(sl):
        ke = 0.5 * (u[sl] ** 2 + v[sl] ** 2 + dsqr * w[sl] ** 2).sum()
        pe = 0.5 * (b[sl] ** 2).sum() / n0 ** 2
        return ke, pe, np.sqrt(u[sl] ** 2 + v[sl] ** 2).max(), np.abs(w[sl]).max(), 0
    parts = [part(slice(r * nz // nr, (r + 1) * nz // nr)) for r in range(nr)]
    whole = part(slice(0, nz))
    ke, pe, um, wm, nf = combine_diagnostics(parts, nx * ny * nz)
    assert np.isclose(ke, whole[0] / (nx * ny * nz), rtol=1e-14)
    assert np.isclose(pe, whole[1] / (nx * ny * nz), rtol=1e-14)
    assert um == whole[2] and wm == whole[3] and nf == 0
    assert combine_diagnostics(parts[:1] + [(0.0, 0.0, 0.0, 0.0, 1)], 1)[4] == 1
