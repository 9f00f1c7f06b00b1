"""Sharding independent grids over ranks (world_size 2, gloo, CPU).

Each rank integrates its share of a small ensemble with the CPU oracle
(standing in for one GPU per rank) and the per-member diagnostics are
gathered; a member whose work raises fails alone, on the host."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from ps3d_b200.shard import UnitError, bin_pack, run_sharded


def test_bin_pack_balances_and_covers():
    costs = [8, 1, 1, 4, 4, 2, 2, 8, 1, 1]
    parts = bin_pack(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)


def _units():
    return [(16, 16, 8, 0.05), (32, 16, 8, 0.1), (16, 16, 8, 0.2), (32, 32, 8, 0.15), (16, 32, 8, -1.0)]


def _run(unit):
    from oracle.binding import Oracle
    from ps3d_b200 import configs as cf
    nx, ny, nz, amp = unit
    if amp < 0:
        raise ValueError("planted failure")
    p = cf.eddy_params(nx, ny, nz)
    o = Oracle(p)
    f = cf.eddy_fields(p, amp=amp)
    for n in ("u", "v", "w", "b"):
        o.field(n)[...] = f[n]
    o.integrate(3)
    st, ke, pe, um, wm = o.diagnose()
    return np.array([ke, pe, um, wm])


def _cost(u):
    return u[0] * u[1] * u[2]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        units = _units()
        res = run_sharded(units, [_cost(u) for u in units], _run, group=dist)
        q.put((rank, [r.tolist() if isinstance(r, np.ndarray) else repr(r) for r in res]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_match_one_process_and_isolate_failure():
    units = _units()
    ref = run_sharded(units, [_cost(u) for u in units], _run, group=None)
    assert isinstance(ref[4], UnitError)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        res = got[rank]
        for i in range(4):
            assert np.allclose(res[i], ref[i].tolist(), rtol=0, atol=0)
        assert "planted failure" in res[4]
