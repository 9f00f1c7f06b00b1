"""Serving loop for optimal-balance and ensemble requests over the C ABI
(ps3d_server_*).

`Server.submit` copies one request (grid parameters, opt-balance knobs, the
initial state in the halo layout) into the engine's queue;
`Server.submit_ensemble` queues an ensemble run (members of any sizes,
nsteps steps each, in batched launches); requests are
admitted in arrival order as slots and HBM free up and run concurrently on
their own CUDA streams.  `replay_poisson` drives a seeded Poisson arrival
process against a server and reports latency percentiles and throughput.
"""
import ctypes as C
import time

import numpy as np

from . import abi
from . import configs as cf
from .abi import OptBal, Params, dptr, halo_shape
from .model import PS3DError, load


def _lib():
    L = load()
    if not hasattr(L, "_srv_ready"):
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.ps3d_server_create.argtypes = [C.c_int, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]
        L.ps3d_server_destroy.argtypes = [vp]
        L.ps3d_server_submit.argtypes = [vp, C.POINTER(Params), C.POINTER(OptBal), dp, dp, dp, dp,
                                         C.POINTER(C.c_longlong)]
        L.ps3d_server_wait.argtypes = [vp, C.c_longlong, C.c_int, dp, dp, dp, dp, dp]
        pp = C.POINTER(dp)
        L.ps3d_server_submit_ensemble.argtypes = [vp, C.POINTER(Params), C.c_int, C.c_int, pp, pp, pp, pp,
                                                  C.POINTER(C.c_longlong)]
        L.ps3d_server_wait_ensemble.argtypes = [vp, C.c_longlong, C.c_int, pp, pp, pp, pp, dp]
        L.ps3d_server_cancel.argtypes = [vp, C.c_longlong]
        L.ps3d_server_stats.argtypes = [vp, dp]
        L.ps3d_server_footprint.restype = C.c_longlong
        L.ps3d_server_footprint.argtypes = [C.POINTER(Params)]
        L.ps3d_server_set_batching.argtypes = [vp, C.c_int, C.c_longlong]
        L.ps3d_server_context_stats.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L._srv_ready = True
    return L


class Result:
    __slots__ = ("status", "norm", "iters", "latency_ms", "queue_ms", "run_ms", "fields")

    def __init__(self, res, fields):
        self.status = int(res[0])
        self.norm, self.iters = float(res[1]), int(res[2])
        self.latency_ms, self.queue_ms, self.run_ms = float(res[3]), float(res[4]), float(res[5])
        self.fields = fields


class Server:
    def __init__(self, device=0, hbm_budget_bytes=0, max_active=4, max_batch=1):
        self.L = _lib()
        h = C.c_void_p()
        rc = self.L.ps3d_server_create(device, hbm_budget_bytes, max_active, C.byref(h))
        if rc:
            raise PS3DError(rc, "ps3d_server_create")
        self.h = h
        self._params = {}
        if max_batch > 1:
            self.set_batching(max_batch)

    def set_batching(self, max_batch, max_points=0):
        """Run up to max_batch queued same-parameter optimal balances as the
        instances of one batched context (shared launches), while their grid
        points together stay within max_points (0: the engine's default)."""
        rc = self.L.ps3d_server_set_batching(self.h, int(max_batch), int(max_points))
        if rc:
            raise PS3DError(rc, "ps3d_server_set_batching")

    def close(self):
        if getattr(self, "h", None):
            self.L.ps3d_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def footprint(p):
        return _lib().ps3d_server_footprint(C.byref(p))

    def submit(self, p, opt, fields):
        arrs = [np.ascontiguousarray(fields[n], dtype=np.float64) for n in ("u", "v", "w", "b")]
        t = C.c_longlong()
        rc = self.L.ps3d_server_submit(self.h, C.byref(p), C.byref(opt), *[dptr(a) for a in arrs], C.byref(t))
        if rc:
            raise PS3DError(rc, "ps3d_server_submit")
        self._params[t.value] = p.copy()
        return t.value

    def wait(self, ticket, timeout_ms=600000, want_fields=True):
        """Result of a request; raises PS3DError(PS3D_ERR_TIMEOUT) if not done in time."""
        p = self._params.get(ticket)
        out = [np.zeros(halo_shape(p)) for _ in range(4)] if (want_fields and p is not None) else [None] * 4
        res = (C.c_double * 6)()
        rc = self.L.ps3d_server_wait(self.h, ticket, timeout_ms, *[dptr(a) for a in out], res)
        if rc == abi.PS3D_ERR_TIMEOUT and res[3] == 0.0:
            raise PS3DError(rc, "ps3d_server_wait")
        self._params.pop(ticket, None)
        return Result(res, dict(zip(("u", "v", "w", "b"), out)) if out[0] is not None else None)

    def submit_ensemble(self, members, states, nsteps):
        """An ensemble run: members (Params list), states[m] = {u, v, w, b}
        in the halo layout, nsteps steps each.  Returns a ticket for
        wait_ensemble."""
        n = len(members)
        arr = (Params * n)(*members)
        keep = [[np.ascontiguousarray(st[f], dtype=np.float64) for f in ("u", "v", "w", "b")] for st in states]
        ptrs = [(C.POINTER(C.c_double) * n)(*[dptr(keep[m][f]) for m in range(n)]) for f in range(4)]
        t = C.c_longlong()
        rc = self.L.ps3d_server_submit_ensemble(self.h, arr, n, nsteps, *ptrs, C.byref(t))
        if rc:
            raise PS3DError(rc, "ps3d_server_submit_ensemble")
        self._params[t.value] = [m.copy() for m in members]
        return t.value

    def wait_ensemble(self, ticket, timeout_ms=600000):
        """Result of an ensemble run: fields = [{u, v, w, b} per member]."""
        members = self._params.get(ticket)
        if members is None:
            raise PS3DError(abi.PS3D_ERR_BADPARAM, "ps3d_server_wait_ensemble")
        n = len(members)
        outs = [{f: np.zeros(halo_shape(m)) for f in ("u", "v", "w", "b")} for m in members]
        ptrs = [(C.POINTER(C.c_double) * n)(*[dptr(outs[m][f]) for m in range(n)]) for f in ("u", "v", "w", "b")]
        res = (C.c_double * 6)()
        rc = self.L.ps3d_server_wait_ensemble(self.h, ticket, timeout_ms, *ptrs, res)
        if rc == abi.PS3D_ERR_TIMEOUT and res[3] == 0.0:
            raise PS3DError(rc, "ps3d_server_wait_ensemble")
        self._params.pop(ticket, None)
        return Result(res, outs)

    def cancel(self, ticket):
        rc = self.L.ps3d_server_cancel(self.h, ticket)
        if rc:
            raise PS3DError(rc, "ps3d_server_cancel")

    def stats(self):
        s = (C.c_double * 6)()
        self.L.ps3d_server_stats(self.h, s)
        c, r = C.c_longlong(), C.c_longlong()
        self.L.ps3d_server_context_stats(self.h, C.byref(c), C.byref(r))
        return {"active": int(s[0]), "queued": int(s[1]), "bytes": s[2], "peak_bytes": s[3],
                "peak_active": int(s[4]), "budget": s[5], "contexts_created": c.value, "contexts_reused": r.value}


# --------------------------------------------------------------------------
# the optimal-balance request workload
# --------------------------------------------------------------------------
SIZES = [(64, 64, 32), (64, 64, 64), (128, 128, 32), (128, 128, 64), (256, 256, 32), (256, 256, 64)]


def request(nx, ny, nz, precision=abi.PS3D_FP64, ramp_steps=100, iters=5):
    """One opt-balance request on the eddy initial state (for_config/eddy1.f90
    template): ramp of n_end = int(T/dt)+1 = ramp_steps steps, `iters`
    iterations, tolerance 0 so that all iterations run.  No harmonic friction,
    as in for_config/test_opt_balance.f90: the backward integration runs with
    dt < 0 and keeps harmonic friction on (diag_opt_balance.f90:190-192 only
    switches the biharmonic terms off), which would make it anti-diffusive."""
    p = cf.eddy_params(nx, ny, nz, precision=precision)
    p.Ah = p.Av = p.Kh = p.Kv = 0.0
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=0)
    opt = OptBal(period=(ramp_steps - 0.5) * p.dt, average=0.0, max_itts=iters, average_times=1,
                 tol=0.0, enable_time_ave=0, adopt=0)
    return p, opt, f


def poisson_schedule(n, rate_hz, seed=4, sizes=SIZES):
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, n)
    arrivals = np.cumsum(gaps) - gaps[0]
    picks = rng.integers(0, len(sizes), n)
    return [(float(arrivals[i]), sizes[picks[i]]) for i in range(n)]


def replay_poisson(server, schedule, precision=abi.PS3D_FP64, ramp_steps=100, iters=5, timeout_ms=3600000):
    """Submit requests at their arrival times; wait for all; latency stats."""
    cache = {}
    tickets = []
    t0 = time.perf_counter()
    for t_arr, size in schedule:
        key = size
        if key not in cache:
            cache[key] = request(*size, precision=precision, ramp_steps=ramp_steps, iters=iters)
        p, opt, f = cache[key]
        now = time.perf_counter() - t0
        if t_arr > now:
            time.sleep(t_arr - now)
        tickets.append(server.submit(p, opt, f))
    results = [server.wait(t, timeout_ms, want_fields=False) for t in tickets]
    wall = time.perf_counter() - t0
    lat = np.array([r.latency_ms for r in results])
    ok = [r for r in results if r.status == 0]
    steps = sum(2 * r.iters * ramp_steps for r in ok)
    pts = sum(2 * r.iters * ramp_steps * np.prod(s) for (_, s), r in zip(schedule, results) if r.status == 0)
    failed = {}
    for (_, size), r in zip(schedule, results):
        if r.status != 0:
            key = f"{size[0]}x{size[1]}x{size[2]}:{r.status}"
            failed[key] = failed.get(key, 0) + 1
    return {"requests": len(results), "ok": len(ok), "failed": failed, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "wall_s": wall,
            "throughput_req_s": len(ok) / wall, "grid_point_steps_s": float(pts / wall), "steps": steps}
