"""Sharding independent grids (ensemble members, balance requests) over ranks.

One process per GPU.  Units are independent, so there is no data-path
collective: units are bin-packed by cost (greedy longest-processing-time
first), every rank runs its own units, and the small per-unit results are
gathered on the host with one all_gather_object.  A unit whose work raises
does not stop the others: its slot in the gathered list carries the error,
and every rank still takes the same collective steps.
"""
import heapq
import traceback


def bin_pack(costs, nranks):
    """Greedy LPT assignment: list of unit indices per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(nranks)]
    heapq.heapify(heap)
    out = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for lst in out:
        lst.sort()
    return out


class UnitError:
    """Result slot of a unit whose work raised."""

    def __init__(self, rank, unit, message):
        self.rank, self.unit, self.message = rank, unit, message

    def __repr__(self):
        return f"UnitError(rank={self.rank}, unit={self.unit}, {self.message!r})"


def run_sharded(units, costs, run_fn, group=None):
    """Run run_fn(unit) for this rank's share of `units`; return the results
    of all units (in unit order) on every rank.  `group` is a
    torch.distributed module/process group or None (single process)."""
    if group is None:
        world, rank = 1, 0
    else:
        import torch.distributed as dist
        world, rank = dist.get_world_size(), dist.get_rank()
    mine = bin_pack(costs, world)[rank]
    local = {}
    for i in mine:
        try:
            local[i] = run_fn(units[i])
        except Exception as e:   # the unit fails alone
            local[i] = UnitError(rank, i, f"{type(e).__name__}: {e}\n{traceback.format_exc(limit=2)}")
    if group is None:
        gathered = [local]
    else:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    out = [None] * len(units)
    for part in gathered:
        for i, r in part.items():
            out[i] = r
    return out
