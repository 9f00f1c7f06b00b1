"""Benchmark of the ps3D time step on B200.

Workload: the jet-instability case, 256 x 256 x 128, rigid lid, AB3,
Laplacian viscosity (two opposing Gaussian jets in thermal-wind balance plus
seeded 1e-3 noise in b; synthetic, seeded).  A step is one call of the
reference's integrate (tendencies, friction, AB3, FFT pressure projection).

Reported: grid-point-steps/s of the mixed FP32/FP64 path (value) and of the
plain FP64 path, the relative L2 distance between the two after the run, the
roofline of the dominant kernel from CUDA events on the engine's stream, an
end-to-end figure through the public C ABI with host buffers, and the CPU
oracle restatement timed on this host's cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): every rank runs an independent replica on its own GPU
(weak scaling); value = all ranks' grid-point-steps over the slowest rank's
time.  With --slab, the N ranks instead share one grid in z-slabs
(ps3d_b200.slab.DistSlab over NCCL: all-to-all transposes to column slabs,
halo planes between neighbours; strong scaling): value = the grid's
grid-point-steps over the slowest rank's time.

`value` is the median of five windows of exactly K steps each, replayed as
CUDA graphs with per-kernel profiling off (what a user's ps3d_integrate
runs); the per-kernel breakdown and the roofline come from a separate pass
of K steps with an event pair around every launch.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NX, NY, NZ = 256, 256, 128
WORKLOAD = "jets 256x256x128 rigid lid AB3 Laplacian friction"


def set_grid(nx, ny, nz):
    global NX, NY, NZ, WORKLOAD
    NX, NY, NZ = nx, ny, nz
    WORKLOAD = f"jets {nx}x{ny}x{nz} rigid lid AB3 Laplacian friction"

# DRAM bytes per grid point per launch of the step kernel, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) at 256x256x64, where its
# traffic already streams far beyond L2, so it scales with the grid points;
# the ncu commands that produced these figures are kept with the profiles.
MEASURED_TRAFFIC_PER_POINT = {
    "fp64": {"step": 165.8},
    "mixed": {"step": 128.4},
    "mixed_refined": {"step": 128.4},   # the same step kernel
}

# algorithmic HBM bytes per grid point per launch.  The step kernel reads
# u,v,w,b, 2 AB history slots x 4 fields and the pending pressure (the
# previous projection's gradient is applied while loading), and writes 4
# tendencies + 4 state fields.  FP64: 32 + 64 + 8 + 32 + 32 = 168.  Mixed
# (u,v,b history FP32, w history FP64): 32 + 40 + 8 + 20 + 32 = 132.
# A warm mixed step (every step after the first) solves once, for the
# residual against the previous step's p: its forward transform reads u, v,
# w and p (32 B) and writes complex64 (4 B); its inverse reads the spectra
# (4 B) and reads and writes p (16 B).
# PS3D_MIXED_REFINED runs a full solve (24 B read, 4 B written; 4 + 8 B)
# and the residual one (36 B; 20 B) every step: 32 and 16 B on average.
BYTES_PER_POINT = {
    "fp64": {"step": 168, "fft_fwd": 32, "vsolve": 16, "fft_inv": 16, "correct": 56, "other": 16},
    "mixed": {"step": 132, "fft_fwd": 36, "vsolve": 8, "fft_inv": 20, "correct": 56, "other": 24},
    "mixed_refined": {"step": 132, "fft_fwd": 32, "vsolve": 8, "fft_inv": 16, "correct": 56, "other": 24},
}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def jets_state(p):
    from ps3d_b200 import configs as cf
    f = cf.jets_fields(p)
    return cf.add_noise(p, f, "b", rel=1e-3, seed=1)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x, pg, dev):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, dev):
    import torch
    if pg is not None:
        pg.barrier(device_ids=[dev])
    torch.cuda.synchronize(dev)


def time_path(precision, steps, warmup, dev, pg, windows=5):
    """Warm up, then time `windows` windows of exactly `steps` steps with CUDA
    events on the engine's stream (graph replay, no profiling; median), then
    one profiled pass of `steps` steps for the per-kernel breakdown."""
    import torch
    from ps3d_b200 import configs as cf
    from ps3d_b200.model import Model
    p = cf.jets_params(NX, NY, NZ, precision=precision)
    f = jets_state(p)
    m = Model(p, device=dev)
    m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
    clocks = ClockSampler(dev)
    clocks.start()
    t_s = time.perf_counter()
    m.run(warmup)
    while time.perf_counter() - t_s < 1.0:   # nvidia-smi needs time to start sampling
        m.run(3)
    m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
    m.run(warmup)
    for _ in range(3):   # windows of any length start at every phase of the graphs' 3-step cycle
        m.run(steps)
    stream = torch.cuda.ExternalStream(m.stream(), device=f"cuda:{dev}")
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(windows):
        barrier(pg, dev)
        ev0.record(stream)
        m.enqueue(steps)
        ev1.record(stream)
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
    barrier(pg, dev)
    ms = float(np.median(times))
    # per-kernel breakdown: eager launches, an event pair around each
    m.profile(True)
    m.enqueue(steps)
    kern = m.profile_read()
    m.profile(False)
    try:
        diag = list(m.diagnose())
    except Exception as e:   # non-finite state: reported, not hidden
        diag = str(e)
    state = m.download(tendencies=False)   # after warmup + (windows + 1) x `steps` steps
    t_s = time.perf_counter()
    while time.perf_counter() - t_s < 0.5:   # keep the GPU loaded while the sampler catches up
        m.run(3)
    clk = clocks.stop()
    clk["diagnose_after_timed"] = diag
    barrier(pg, dev)
    ms_max = max_over_ranks(ms, pg, dev)
    return m, p, ms, ms_max, kern, clk, state, m.describe(), times


def e2e_run(precision, steps, dev):
    """main.f90's loop through the public C ABI with host buffers: upload the
    state, `steps` x (ps3d_step + host rotation), diagnose every 10 steps,
    download the state and p.  All host<->device copies are inside the timed
    region.  p is not uploaded: every step recomputes it before anything
    reads it (the first step after an upload applies no pending correction,
    and the mixed path's first solve after an upload is cold), so only the
    prognostic fields u, v, w, b go up."""
    import torch
    from ps3d_b200 import configs as cf
    from ps3d_b200.model import Model
    p = cf.jets_params(NX, NY, NZ, precision=precision)
    f = jets_state(p)
    m = Model(p, device=dev)
    m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
    m.run(3)                      # warm the kernels
    names = ("u", "v", "w", "b", "p")
    host = {}
    for n in names:   # page-locked host arrays, as a host code would keep its state
        a = torch.empty(f["u"].shape, dtype=torch.float64, pin_memory=True).numpy()
        a[...] = f[n] if n in f else 0.0
        host[n] = a
    out = {n: torch.empty(f["u"].shape, dtype=torch.float64, pin_memory=True).numpy() for n in names}
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    m.upload(**{n: host[n] for n in ("u", "v", "w", "b")}, itt=0, tau=3, taum1=2, taum2=1)
    itt, tau, t1, t2 = 0, 3, 2, 1
    ndiag = 0
    for n in range(steps):
        m.integrate(itt, tau, t1, t2)
        if n % 10 == 0:
            m.diagnose()
            ndiag += 1
        tau, t1, t2 = tau % 3 + 1, t1 % 3 + 1, t2 % 3 + 1
        itt += 1
    m.download_into(out)
    t = time.perf_counter() - t0
    m.close()
    field_bytes = host["u"].nbytes
    h2d = 4 * field_bytes
    d2h = 5 * field_bytes + ndiag * 32
    return t, h2d / steps, d2h / steps, out


def cpu_baseline_run(steps, warmup_steps=1, budget_s=60.0):
    """The CPU oracle restatement on all host cores, bounded to ~budget_s."""
    from oracle.binding import Oracle, set_threads
    from ps3d_b200 import configs as cf
    cores = os.cpu_count() or 1
    set_threads(cores)
    p = cf.jets_params(NX, NY, NZ)
    f = jets_state(p)
    o = Oracle(p)
    for n in ("u", "v", "w", "b"):
        o.field(n)[...] = f[n]
    t0 = time.perf_counter()
    o.integrate(warmup_steps)
    t_one = (time.perf_counter() - t0) / max(warmup_steps, 1)
    n = int(max(1, min(steps, budget_s / max(t_one, 1e-6))))
    t0 = time.perf_counter()
    o.integrate(n)
    t = time.perf_counter() - t0
    return NX * NY * NZ * n / t, cores, n


ENS_SIZES = [(32, 32, 16), (64, 64, 32), (128, 64, 32), (128, 128, 64)]


def ensemble_run(dev, pg, world, n_members=256, steps=200, seed=3):
    """Batched ensemble: 256 eddies, sizes drawn by seed from ENS_SIZES,
    amplitudes U(0.05, 0.2) m/s, `steps` steps, all members in batched
    launches replayed as CUDA graphs, in mixed precision and in FP64.
    Compared with the same members stepped one at a time on the plain FP64
    path: every member measured, one context per size class, the member's
    state uploaded and 5 steps run untimed (graph capture), then `steps`
    steps replayed as CUDA graphs and timed with events.  With N ranks each
    rank runs its own ensemble (weak scaling)."""
    import torch
    from ps3d_b200 import abi
    from ps3d_b200 import configs as cf
    from ps3d_b200.ensemble import Ensemble
    from ps3d_b200.model import Model
    rng = np.random.default_rng(seed)
    picks = rng.integers(0, len(ENS_SIZES), n_members)
    amps = rng.uniform(0.05, 0.2, n_members)
    fields = {}
    for k in sorted(set(int(x) for x in picks)):
        p = cf.eddy_params(*ENS_SIZES[k])
        fields[k] = cf.add_noise(p, cf.eddy_fields(p, amp=1.0), "b", rel=1e-3, seed=0)
    pts = sum(int(np.prod(ENS_SIZES[k])) for k in picks)

    def batched(prec):
        members = [cf.eddy_params(*ENS_SIZES[k], precision=prec) for k in picks]
        ens = Ensemble(members, device=dev)
        for i, (k, a) in enumerate(zip(picks, amps)):
            f = fields[int(k)]
            ens.upload(i, f["u"] * a, f["v"] * a, f["w"] * a, f["b"] * a)
        ens.integrate(5)   # eager first steps, then the 3-step graph captured and replayed once
        info0 = ens.info()
        stream = torch.cuda.ExternalStream(info0["stream"], device=f"cuda:{dev}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(pg, dev)
        e0.record(stream)
        ens.enqueue(steps)
        e1.record(stream)
        e1.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), pg, dev)
        launches = ens.info()["launches"] - info0["launches"]
        ens.close()
        return ms, int(launches)

    ms_mx, l_mx = batched(abi.PS3D_MIXED)
    ms_64, l_64 = batched(abi.PS3D_FP64)
    # serial plain FP64, every member
    serial_ms = 0.0
    per_size_ms = {}
    for k in sorted(set(int(x) for x in picks)):
        p = cf.eddy_params(*ENS_SIZES[k])
        m = Model(p, device=dev)
        st = torch.cuda.ExternalStream(m.stream(), device=f"cuda:{dev}")
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f = fields[k]
        tot = 0.0
        for i in np.nonzero(picks == k)[0]:
            a = amps[i]
            m.upload(**{n: f[n] * a for n in ("u", "v", "w", "b")})
            m.run(5)   # eager first steps, then the 3-step graph captured and replayed once
            a0.record(st)
            m.enqueue(steps)
            a1.record(st)
            a1.synchronize()
            tot += a0.elapsed_time(a1)
        m.close()
        per_size_ms[f"{ENS_SIZES[k][0]}x{ENS_SIZES[k][1]}x{ENS_SIZES[k][2]}"] = tot
        serial_ms += tot
    serial_ms = max_over_ranks(serial_ms, pg, dev)
    return {"members": n_members, "steps": steps, "sizes": [list(s) for s in ENS_SIZES],
            "members_per_size": [int((picks == k).sum()) for k in range(len(ENS_SIZES))],
            "batched_mixed_value": world * pts * steps / (ms_mx * 1e-3), "batched_mixed_ms": ms_mx,
            "batched_mixed_launches": l_mx,
            "batched_fp64_value": world * pts * steps / (ms_64 * 1e-3), "batched_fp64_ms": ms_64,
            "batched_fp64_launches": l_64,
            "serial_fp64_value": world * pts * steps / (serial_ms * 1e-3), "serial_fp64_ms": serial_ms,
            "serial_fp64_ms_per_size": per_size_ms,
            "batched_mixed_over_serial_fp64": serial_ms / ms_mx,
            "batched_fp64_over_serial_fp64": serial_ms / ms_64,
            "batched_mixed_over_batched_fp64": ms_64 / ms_mx,
            "note": "all three arms measured over every member with CUDA graphs (captured in 5 untimed steps); the "
                    "serial arm steps one member at a time (one context per size, state uploaded per member)"}


def slab_levels(nz, world, rank):
    """The global levels rank `rank` of `world` owns in a z-slab run."""
    nzl = nz // world
    return rank * nzl, nzl


def slab_run(precision, steps, warmup, dev, pg, world, rank):
    """One grid over `world` ranks in z-slabs (DistSlab, NCCL): each rank
    uploads its levels of the jets state, runs `warmup` steps, then `steps`
    steps timed with CUDA events on its slab stream; max over ranks."""
    import torch
    from ps3d_b200 import configs as cf
    from ps3d_b200.slab import DistSlab
    p = cf.jets_params(NX, NY, NZ, precision=precision)
    f = jets_state(p)
    k0, nzl = slab_levels(NZ, world, rank)
    sl = slice(k0 + 2, k0 + 2 + nzl)
    d = DistSlab(p, dev)
    d.upload(*[np.ascontiguousarray(f[n][sl, 2:-2, 2:-2]) for n in ("u", "v", "w", "b")])
    d.step(warmup)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(pg, dev)
    e0.record(d.stream)
    d.step(steps)
    e1.record(d.stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), pg, dev)
    out = d.download()
    d.close()
    return ms, out


def fp64_gemm_peak(dev, n=8192, reps=5):
    """FP64 throughput denominator measured here: torch.matmul in float64
    (cuBLAS DGEMM) on n x n operands, best of `reps`, 2 n^3 flop each."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{dev}")
    b = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{dev}")
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(reps):
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def projection_run(dev, nx=256, ny=256, nz=64):
    """normal_mode_projection (diag_opt_balance.f90:288-310) on a rigid-lid
    eddy of the largest serving size: forward transform (4 plane FFTs + 4
    vertical-mode transforms), eigen projection, backward transform.  Median
    of 5 timed calls in each form of the vertical-mode transform: the dense
    FP64 product (4 nz^2 flop per complex column, against the FP64 GEMM
    throughput measured here by cuBLAS DGEMM) and the FFTs (the engine's
    choice; an HBM-bound pass: the column data read and written once,
    against the measured copy bandwidth)."""
    import torch
    from ps3d_b200 import configs as cf
    from ps3d_b200.model import Model
    p = cf.eddy_params(nx, ny, nz)
    f = cf.eddy_fields(p)
    ncol = (nx // 2 + 1) * ny

    def measure(form):
        old = os.environ.get("PS3D_VMODE_FORM")
        os.environ["PS3D_VMODE_FORM"] = form
        try:
            m = Model(p, device=dev)
        finally:
            if old is None:
                del os.environ["PS3D_VMODE_FORM"]
            else:
                os.environ["PS3D_VMODE_FORM"] = old
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
        m.normal_mode_projection()
        st = torch.cuda.ExternalStream(m.stream(), device=f"cuda:{dev}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t = []
        for _ in range(5):
            e0.record(st)
            m.normal_mode_projection()
            e1.record(st)
            e1.synchronize()
            t.append(e0.elapsed_time(e1))
        m.profile(True)
        m.normal_mode_projection()
        kern = m.profile_read()
        m.profile(False)
        m.close()
        ms_v, n_v = kern["vmode"]
        return t, kern, ms_v / max(n_v, 1), int(n_v)

    t_d, kern_d, per_d, n_d = measure("1")
    t_f, kern_f, per_f, n_f = measure("2")
    nbytes = 2 * 16 * ncol * nz            # per launch: the columns read and written once
    flop = 4.0 * nz * nz * ncol            # per launch of the dense product
    try:
        peak_fp64, peak_kind = fp64_gemm_peak(dev), "measured: cuBLAS FP64 GEMM 8192^3, best of 5"
    except Exception:
        peak_fp64, peak_kind = 40.0, "nominal B200 FP64"
    hbm, hbm_kind = peaks()
    dense = {"ms_median": float(np.median(t_d)), "ms_windows": t_d, "ms_per_launch": per_d, "launches": n_d,
             "flop_per_launch": flop, "achieved_tflops": flop / (per_d * 1e-3) / 1e12 if n_d else None,
             "peak_tflops": peak_fp64, "peak_kind": peak_kind,
             "frac": (flop / (per_d * 1e-3) / 1e12) / peak_fp64 if n_d else None}
    fft = {"ms_median": float(np.median(t_f)), "ms_windows": t_f, "ms_per_launch": per_f, "launches": n_f,
           "bytes_per_launch": nbytes, "achieved_gbs": nbytes / (per_f * 1e-3) / 1e9 if n_f else None,
           "peak_gbs": hbm, "peak_kind": hbm_kind,
           "frac": (nbytes / (per_f * 1e-3) / 1e9) / hbm if n_f else None}
    default = "fft"
    chosen = fft if default == "fft" else dense
    return {"grid": [nx, ny, nz], "ms_median": chosen["ms_median"], "vmode_form": default,
            "vmode_dense": dense, "vmode_fft": fft,
            "kernels_ms": {k: v[0] for k, v in (kern_f if default == "fft" else kern_d).items() if v[1]}}


def serve_run(dev, n_requests=40, rate_hz=50.0, max_active=8, max_batch=8):
    """Optimal-balance requests: Poisson arrivals at rate_hz (seed 4), sizes
    drawn from 64x64x32 .. 256x256x64, 5 iterations of 100-step ramps each,
    admitted by HBM footprint, FP64 and mixed; each request on its own
    context, and with up to max_batch queued same-size requests sharing the
    launches of one batched context."""
    from ps3d_b200 import abi
    from ps3d_b200.serve import Server, poisson_schedule, replay_poisson
    sched = poisson_schedule(n_requests, rate_hz, seed=4)
    out = {"requests": n_requests, "rate_hz": rate_hz, "max_active": max_active, "max_batch": max_batch,
           "request": "diag_opt_balance, 5 iterations x (100 back + 100 forward steps) + projections"}
    for name, prec, mb in (("fp64", abi.PS3D_FP64, 1), ("mixed", abi.PS3D_MIXED, 1),
                           ("fp64_batched", abi.PS3D_FP64, max_batch), ("mixed_batched", abi.PS3D_MIXED, max_batch)):
        srv = Server(device=dev, max_active=max_active, max_batch=mb)
        r = replay_poisson(srv, sched, precision=prec)
        r["peak_active"] = srv.stats()["peak_active"]
        srv.close()
        out[name] = r
    # small requests only (64x64x32), where a request alone leaves the GPU idle
    small = poisson_schedule(n_requests, rate_hz, seed=5, sizes=[(64, 64, 32)])
    out["small_64x64x32"] = {}
    for name, mb in (("mixed", 1), ("mixed_batched", max_batch)):
        srv = Server(device=dev, max_active=max_active, max_batch=mb)
        r = replay_poisson(srv, small, precision=abi.PS3D_MIXED)
        r["peak_active"] = srv.stats()["peak_active"]
        srv.close()
        out["small_64x64x32"][name] = r
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--case", default="both", choices=["both", "fp64", "mixed", "mixed_refined"],
                    help="which time-step paths to time (profiling runs use one)")
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--ensemble", type=int, default=1, help="also run the batched-ensemble workload")
    ap.add_argument("--serve", type=int, default=1, help="also run the serving workload")
    ap.add_argument("--projection", type=int, default=1, help="also time the normal-mode projection")
    ap.add_argument("--projection-grid", default="256x256x64",
                    help="grid of the projection timing, NXxNYxNZ (rigid-lid eddy)")
    ap.add_argument("--slab", action="store_true",
                    help="one grid over the N ranks in z-slabs (strong scaling) instead of N replicas")
    args = ap.parse_args()
    set_grid(args.nx, args.ny, args.nz)
    unit = "grid-point-steps/s"
    metric = f"grid-point-steps/s of the ps3D time step, {NX}x{NY}x{NZ} jets, mixed FP32/FP64 path (FP64 path beside)"

    if args.impl == "reference":
        # the CPU restatement on the host cores: rank 0 alone, no process group
        if int(os.environ.get("RANK", "0")) != 0:
            return
        steps = max(1, args.steps)
        val, cores, n = cpu_baseline_run(steps, warmup_steps=min(max(args.warmup, 1), 2), budget_s=150.0)
        sample = f"{n} full steps of {NX}x{NY}x{NZ} (after warm-up) on {cores} threads"
        line = {"impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": args.gpus,
                "steps": n, "warmup": args.warmup, "ms_per_step": NX * NY * NZ / val * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded jets + noise)",
                "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ},
                "cpu_baseline": {"value": val, "unit": unit, "cores": cores, "kind": "port", "sample": sample},
                "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "reference Fortran/MPI/P3DFFT path is not buildable here; oracle C++ restatement timed"}
        print(json.dumps(line), flush=True)
        return

    world, rank, local, pg = dist_setup()
    if args.slab:
        return slab_main(args, world, rank, local, pg, metric, unit)
    import torch
    from ps3d_b200 import build as b
    from ps3d_b200 import abi
    from ps3d_b200 import configs as cf
    b.build()
    torch.cuda.set_device(local)
    dev = local
    npts = NX * NY * NZ

    peak, peak_kind = peaks()

    def roof(kern, prec):
        out = {}
        for k, (ms, n) in kern.items():
            if n == 0:
                continue
            per = ms / n
            bpp = BYTES_PER_POINT[prec].get(k, 0)
            out[k] = {"launches": n, "ms_total": ms, "ms_per_launch": per,
                      "algorithmic_gb_per_launch": bpp * npts / 1e9,
                      "achieved_gbs": bpp * npts / (per * 1e-3) / 1e9 if bpp else None,
                      "frac_of_peak": (bpp * npts / (per * 1e-3) / 1e9) / peak if bpp else None}
        return out

    res = {}
    for case, prec, name in ((("both", "fp64"), abi.PS3D_FP64, "fp64"), (("both", "mixed"), abi.PS3D_MIXED, "mixed"),
                             (("both", "mixed_refined"), abi.PS3D_MIXED_REFINED, "mixed_refined")):
        if args.case not in case:
            continue
        m_, p_, ms_, msmax_, k_, clk_, st_, desc_, win_ = time_path(prec, args.steps, args.warmup, dev, pg)
        m_.close()
        res[name] = {"p": p_, "ms_max": msmax_, "kern": k_, "clk": clk_, "state": st_, "desc": desc_,
                     "value": world * npts * args.steps / (msmax_ * 1e-3), "windows_ms": win_,
                     "roof": roof(k_, name)}
    hname = "mixed" if "mixed" in res else "fp64" if "fp64" in res else "mixed_refined"
    head = res[hname]
    dom_name, dom_v = max(head["roof"].items(), key=lambda kv: kv[1]["ms_total"])
    # kernels per library call of each class: the split transforms (rows +
    # y-lines passes) launch two kernels per call, the cluster ones one
    split = "plane_impl=cluster" not in head["desc"]
    per_call = {"fft_fwd": 2 if split else 1, "fft_inv": 2 if split else 1}
    launches = sum(n * per_call.get(k, 1) for k, (_, n) in head["kern"].items())
    line = {"metric": metric, "value": head["value"], "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_max"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if hname == "fp64" else "f32+f64 (FP64 state/AB/tridiagonal)",
            "data": "synthetic (seeded jets + 1e-3 b noise)",
            "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "parallelism": f"replicas x{world}",
                       "path": hname, "kernel_config": head["desc"],
                       "l2": "inputs larger than L2 (state > 1 GB)" if npts >= 2 ** 23 else "small case"},
            "kernels": head["roof"],
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": dom_v["achieved_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": (dom_v["achieved_gbs"] or 0) / peak,
                         "traffic": (MEASURED_TRAFFIC_PER_POINT[hname].get(dom_name, 0) * npts or None),
                         "traffic_unit": "DRAM bytes per launch (ncu, scaled by grid points)",
                         "algorithmic_bytes": BYTES_PER_POINT[hname].get(dom_name, 0) * npts,
                         "peak_kind": peak_kind},
            "gpu_launches": int(launches), "clocks": head["clk"],
            "timing": {"value": "median of 5 windows of exactly `steps` steps, CUDA-graph replay, profiling off",
                       "windows_ms": head["windows_ms"],
                       "kernels": "separate pass of `steps` steps, eager launches with an event pair each",
                       "profiled_ms_per_step": sum(v[0] for v in head["kern"].values()) / args.steps}}
    if "fp64" in res:
        r64 = res["fp64"]
        line["fp64"] = {"value": r64["value"], "ms_per_step": r64["ms_max"] / args.steps, "kernels": r64["roof"],
                        "kernel_config": r64["desc"], "clocks": r64["clk"], "windows_ms": r64["windows_ms"]}
    def max_div(st, pp):
        u, v, w = st["u"], st["v"], st["w"]
        div = ((u[2:-2, 2:-2, 2:-2] - u[2:-2, 2:-2, 1:-3]) / pp.dx + (v[2:-2, 2:-2, 2:-2] - v[2:-2, 1:-3, 2:-2]) / pp.dy
               + (w[2:-2, 2:-2, 2:-2] - w[1:-3, 2:-2, 2:-2]) / pp.dz)
        return float(np.abs(div).max())

    if "fp64" in res:
        line["fp64"]["max_div"] = max_div(res["fp64"]["state"], res["fp64"]["p"])
    if "fp64" in res and "mixed" in res:
        s64, smx, pmx = res["fp64"]["state"], res["mixed"]["state"], res["mixed"]["p"]
        line["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
        line["rel_l2_mixed_vs_fp64"] = {n: cf.rel_l2(cf.interior(smx[n]), cf.interior(s64[n]))
                                        for n in ("u", "v", "w", "b", "p")}
        line["max_div_mixed"] = max_div(smx, pmx)
    if "mixed_refined" in res and hname != "mixed_refined":
        rr = res["mixed_refined"]
        line["mixed_refined"] = {"value": rr["value"], "ms_per_step": rr["ms_max"] / args.steps, "kernels": rr["roof"],
                                 "max_div": max_div(rr["state"], rr["p"]),
                                 "note": "PS3D_MIXED_REFINED: full FP32 solve + FP64-residual refinement every step"}
        if "fp64" in res:
            line["mixed_refined"]["rel_l2_vs_fp64"] = {
                n: cf.rel_l2(cf.interior(rr["state"][n]), cf.interior(res["fp64"]["state"][n]))
                for n in ("u", "v", "w", "b", "p")}
    if not args.no_e2e:
        eprec = {"fp64": abi.PS3D_FP64, "mixed": abi.PS3D_MIXED, "mixed_refined": abi.PS3D_MIXED_REFINED}[hname]
        t, h2d, d2h, _ = e2e_run(eprec, args.steps, dev)
        t = max_over_ranks(t, pg, dev)
        line["e2e"] = {"value": world * npts * args.steps / t, "unit": unit, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h,
                       "path": "public C ABI: upload, ps3d_step per step, diagnose every 10 steps, download"}
    if args.ensemble:
        line["ensemble"] = ensemble_run(dev, pg, world)
    if args.projection:
        pg_nx, pg_ny, pg_nz = (int(x) for x in args.projection_grid.split("x"))
        line["projection"] = projection_run(dev, pg_nx, pg_ny, pg_nz)
    if args.serve:
        line["serving"] = serve_run(dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        val, cores, n = cpu_baseline_run(3, warmup_steps=1, budget_s=30.0)
        line["cpu_baseline"] = {"value": val, "unit": unit, "cores": cores, "kind": "port",
                                "sample": f"{n} full steps of {NX}x{NY}x{NZ} after 1 warm-up step, CPU oracle"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def slab_main(args, world, rank, local, pg, metric, unit):
    """bench.py --slab: the mixed path's time step on one grid shared by the
    ranks in z-slabs (strong scaling), FP64 beside it."""
    import datetime
    import torch
    import torch.distributed as dist
    from ps3d_b200 import abi
    from ps3d_b200 import build as b
    b.build()
    torch.cuda.set_device(local)
    if pg is None:   # one rank: a process group of one for DistSlab's collectives
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29641")
        dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    if NZ % world or NZ // world < 2:
        raise SystemExit(f"--slab: nz={NZ} does not split into {world} slabs of >= 2 levels")
    npts = NX * NY * NZ
    res = {}
    for name, prec in (("mixed", abi.PS3D_MIXED), ("fp64", abi.PS3D_FP64)):
        ms, _ = slab_run(prec, args.steps, args.warmup, local, pg, world, rank)
        res[name] = ms
    ms = res["mixed"]
    line = {"metric": metric + " (one grid in z-slabs)", "value": npts * args.steps / (ms * 1e-3), "unit": unit,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32+f64 (FP64 state/AB/tridiagonal)", "data": "synthetic (seeded jets + 1e-3 b noise)",
            "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "parallelism": f"z-slabs x{world}",
                       "path": "mixed", "levels_per_rank": NZ // world,
                       "l2": "inputs larger than L2 (state > 1 GB)" if npts >= 2 ** 23 else "small case"},
            "fp64": {"value": npts * args.steps / (res["fp64"] * 1e-3), "ms_per_step": res["fp64"] / args.steps},
            "timing": "CUDA events on each rank's slab stream around exactly `steps` steps, max over ranks"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
