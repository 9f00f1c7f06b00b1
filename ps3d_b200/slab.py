"""One grid over several GPUs: z-slabs (ps3d_b200/csrc/slab.cu).

The reference runs one grid on MPI ranks decomposed inside P3DFFT
(my_fft.f90; pressure_solver.f90 on its pencils).  Here rank r of n owns the
global levels k0 = r*nzl .. k0+nzl-1 (nzl = nz/n); the stencils and the
per-level 2D transforms stay on the rank, the vertical solves run on column
slabs after an all-to-all transpose, and halo planes move between
neighbours in z.

* ``SlabGroup``: all ranks in one process (one GPU or several), transport by
  device copies inside the library (``ps3d_slab_group_step``).
* ``DistSlab``: one rank per process over ``torch.distributed`` (NCCL on
  GPUs): the library runs the phases on its stream, the collectives below
  move the exchange buffers, which are torch tensors bound to the slab.

Host arrays are interior-only, [nz][ny][nx] (x fastest); ``SlabGroup`` takes
and returns whole-grid arrays, ``DistSlab`` the rank's levels.
"""
import ctypes as C

import numpy as np

from .abi import PS3D_ERR_NONFINITE, PS3D_FORCE_NONE, PS3D_FP64, Forcing, Params
from .model import _check, load

FORCING_FIELDS = ("u_r", "v_r", "w_r", "b_r", "u_i", "v_i", "w_i", "b_i", "u_back", "b_back")

PHASE = {"tendency": 0, "pack_state": 1, "unpack_state": 2, "forward": 3, "vsolve": 4, "inverse": 5,
         "pack_p": 6, "unpack_p": 7, "end_step": 8}
# planes sent down (to the rank below) and up (to the rank above): state
# u, v, w, b; p two down, one up (the step kernel reads p one level above)
K_DOWN = (4, 2)
K_UP = (4, 1)


def _lib():
    L = load()
    if getattr(L, "_slab_argtypes", False):
        return L
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    L.ps3d_slab_create.argtypes = [C.POINTER(Params), C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
    L.ps3d_slab_destroy.argtypes = [vp]
    L.ps3d_slab_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                 C.POINTER(C.c_longlong), C.POINTER(vp), C.POINTER(C.c_int)]
    L.ps3d_slab_buffers.argtypes = [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_longlong)]
    L.ps3d_slab_bind.argtypes = [vp, vp, vp, vp, vp]
    L.ps3d_slab_upload.argtypes = [vp, dp, dp, dp, dp]
    L.ps3d_slab_download.argtypes = [vp, dp, dp, dp, dp, dp]
    L.ps3d_slab_phase.argtypes = [vp, C.c_int]
    L.ps3d_slab_sync.argtypes = [vp]
    L.ps3d_slab_group_step.argtypes = [C.POINTER(vp), C.c_int, C.c_int]
    L.ps3d_slab_set_forcing.argtypes = [vp, C.POINTER(Forcing)]
    L.ps3d_slab_diagnose.argtypes = [vp, dp, dp, dp, dp, C.POINTER(C.c_int)]
    L._slab_argtypes = True
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def combine_diagnostics(parts, npoints):
    """diagnose over the whole grid from the ranks' (ke_sum, pe_sum, umax,
    wmax, nonfinite): global sums divided by the grid's points, global maxima
    (global_sum / global_max, parallel_mpi.f90:37-67).  Returns (ke, pe,
    umax, wmax, nonfinite)."""
    ke = sum(q[0] for q in parts) / npoints
    pe = sum(q[1] for q in parts) / npoints
    return ke, pe, max(q[2] for q in parts), max(q[3] for q in parts), max(int(q[4]) for q in parts)


class Slab:
    """Rank ``rank`` of ``nranks`` of the grid described by ``params``."""

    def __init__(self, params: Params, nranks: int, rank: int, device: int = 0):
        self.L = _lib()
        self.params = params.copy()
        self.nranks, self.rank = nranks, rank
        h = C.c_void_p()
        _check(self.L.ps3d_slab_create(C.byref(self.params), nranks, rank, device, C.byref(h)), "ps3d_slab_create")
        self.h = h
        k0, nzl, col0, ncl, st, ps = C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong(), C.c_void_p(), C.c_int()
        _check(self.L.ps3d_slab_info(h, C.byref(k0), C.byref(nzl), C.byref(col0), C.byref(ncl), C.byref(st),
                                     C.byref(ps)), "ps3d_slab_info")
        self.k0, self.nzl, self.col0, self.ncl, self.stream = k0.value, nzl.value, col0.value, ncl.value, st.value
        self.passes = ps.value   # solve passes of the first step (step_passes: of the next one)
        self.mixed = self.params.precision != PS3D_FP64
        xb, cb, hb = C.c_size_t(), C.c_size_t(), C.c_size_t()
        counts = (C.c_longlong * nranks)()
        _check(self.L.ps3d_slab_buffers(h, C.byref(xb), C.byref(cb), C.byref(hb), counts), "ps3d_slab_buffers")
        self.xbytes, self.colbytes, self.hbytes = xb.value, cb.value, hb.value
        self.col_counts = [int(c) for c in counts]
        self.plane = self.params.nx * self.params.ny

    def step_passes(self):
        """Solve passes of the next step: 1 in FP64; in the mixed path 2 after
        create or upload (full solve and FP64-residual refinement), then 1
        (the residual solve against the previous step's pressure)."""
        ps = C.c_int()
        _check(self.L.ps3d_slab_info(self.h, None, None, None, None, None, C.byref(ps)), "ps3d_slab_info")
        return ps.value

    def bind(self, xbuf, colbuf, hsend, hrecv):
        """Use caller-owned device buffers (addresses) for the exchanges."""
        _check(self.L.ps3d_slab_bind(self.h, xbuf, colbuf, hsend, hrecv), "ps3d_slab_bind")

    def upload(self, u, v, w, b):
        """This rank's interior levels, each [nzl][ny][nx]."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, b)]
        for a in arrs:
            assert a.shape == (self.nzl, self.params.ny, self.params.nx), a.shape
        _check(self.L.ps3d_slab_upload(self.h, *[_dp(a) for a in arrs]), "ps3d_slab_upload")

    def download(self):
        shape = (self.nzl, self.params.ny, self.params.nx)
        out = {n: np.empty(shape) for n in ("u", "v", "w", "b", "p")}
        _check(self.L.ps3d_slab_download(self.h, *[_dp(out[n]) for n in ("u", "v", "w", "b", "p")]),
               "ps3d_slab_download")
        return out

    def set_forcing(self, kind=PS3D_FORCE_NONE, omega=0.0, **fields):
        """set_forcing on this rank's levels: kind (wavemaker and/or background
        flow), omega, and whole-grid interior fields [nz][ny][nx] named as
        Model.set_forcing names them (u_r .. b_i, u_back, b_back; absent =
        zero).  The rank keeps its levels and one level each side, periodic
        in z."""
        f = Forcing()
        f.kind = kind
        f.omega = omega
        nz = self.params.nz
        lev = [(self.k0 - 1 + q) % nz for q in range(self.nzl + 2)]
        keep = []
        for name in FORCING_FIELDS:
            a = fields.get(name)
            if a is None:
                continue
            a = np.asarray(a, dtype=np.float64)
            assert a.shape == (nz, self.params.ny, self.params.nx), (name, a.shape)
            loc = np.ascontiguousarray(a[lev])
            keep.append(loc)
            setattr(f, name, _dp(loc))
        _check(self.L.ps3d_slab_set_forcing(self.h, C.byref(f)), "ps3d_slab_set_forcing")

    def diagnose_partial(self):
        """This rank's (ke_sum, pe_sum, umax, wmax, nonfinite) over its levels."""
        ke, pe, um, wm, nf = C.c_double(), C.c_double(), C.c_double(), C.c_double(), C.c_int()
        _check(self.L.ps3d_slab_diagnose(self.h, C.byref(ke), C.byref(pe), C.byref(um), C.byref(wm), C.byref(nf)),
               "ps3d_slab_diagnose")
        return ke.value, pe.value, um.value, wm.value, nf.value

    def phase(self, name):
        _check(self.L.ps3d_slab_phase(self.h, PHASE[name]), "ps3d_slab_phase " + name)

    def sync(self):
        _check(self.L.ps3d_slab_sync(self.h), "ps3d_slab_sync")

    def close(self):
        if getattr(self, "h", None):
            self.L.ps3d_slab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SlabGroup:
    """All ranks of one grid in this process; ``devices[r]`` hosts rank r."""

    def __init__(self, params: Params, nranks: int, devices=None):
        devices = devices or [0] * nranks
        self.params = params.copy()
        self.ranks = [Slab(params, nranks, r, devices[r]) for r in range(nranks)]
        self.L = self.ranks[0].L

    def upload(self, u, v, w, b):
        """Whole-grid interior arrays [nz][ny][nx]."""
        for s in self.ranks:
            sl = slice(s.k0, s.k0 + s.nzl)
            s.upload(u[sl], v[sl], w[sl], b[sl])

    def set_forcing(self, kind=PS3D_FORCE_NONE, omega=0.0, **fields):
        """Whole-grid interior forcing fields [nz][ny][nx] (Slab.set_forcing)."""
        for s in self.ranks:
            s.set_forcing(kind, omega, **fields)

    def step(self, nsteps=1):
        arr = (C.c_void_p * len(self.ranks))(*[s.h.value for s in self.ranks])
        _check(self.L.ps3d_slab_group_step(arr, len(self.ranks), nsteps), "ps3d_slab_group_step")

    def diagnose(self):
        """(ke, pe, umax, wmax) of the whole grid; raises PS3DError
        (PS3D_ERR_NONFINITE) where a value is not finite, as Model.diagnose."""
        p = self.params
        ke, pe, um, wm, nf = combine_diagnostics([s.diagnose_partial() for s in self.ranks], p.nx * p.ny * p.nz)
        if nf:
            _check(PS3D_ERR_NONFINITE, "ps3d_slab_diagnose")
        return ke, pe, um, wm

    def download(self):
        parts = [s.download() for s in self.ranks]
        return {n: np.concatenate([p[n] for p in parts], axis=0) for n in parts[0]}

    def close(self):
        for s in self.ranks:
            s.close()


# ---------------------------------------------------------------------------
# transport over torch.distributed: the same on CUDA tensors (NCCL) and on
# CPU tensors (gloo); flat float64 tensors laid out as slab.cu documents
# ---------------------------------------------------------------------------
def halo_exchange(hsend, hrecv, plane, which, rank, nranks, group=None):
    """hsend = [planes for the rank below][planes for the rank above];
    hrecv = [what the rank below sent up][what the rank above sent down];
    z is periodic over the ranks.  which: 0 state, 1 p."""
    import torch.distributed as dist
    nd, nu = K_DOWN[which] * plane, K_UP[which] * plane
    down, up = hsend[:nd], hsend[nd:nd + nu]
    from_below, from_above = hrecv[:nu], hrecv[nu:nu + nd]
    if nranks == 1:
        from_below.copy_(up)
        from_above.copy_(down)
        return
    below, above = (rank - 1) % nranks, (rank + 1) % nranks
    # every rank posts its sends and receives in the same order, so with two
    # ranks (below == above) the pair matches up with up and down with down
    ops = [dist.P2POp(dist.isend, up, above, group), dist.P2POp(dist.isend, down, below, group),
           dist.P2POp(dist.irecv, from_below, below, group), dist.P2POp(dist.irecv, from_above, above, group)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()


def columns_forward(xbuf, colbuf, counts, nzl, rank, group=None):
    """xbuf [r][nzl][counts[r]] complex -> colbuf [src][nzl][counts[rank]]."""
    import torch.distributed as dist
    dist.all_to_all_single(colbuf, xbuf, output_split_sizes=[2 * nzl * counts[rank]] * len(counts),
                           input_split_sizes=[2 * nzl * c for c in counts], group=group)


def columns_backward(xbuf, colbuf, counts, nzl, rank, group=None):
    """colbuf [dst][nzl][counts[rank]] -> xbuf [src][nzl][counts[src]]."""
    import torch.distributed as dist
    dist.all_to_all_single(xbuf, colbuf, output_split_sizes=[2 * nzl * c for c in counts],
                           input_split_sizes=[2 * nzl * counts[rank]] * len(counts), group=group)


class DistSlab:
    """This process's rank of one grid over ``torch.distributed`` (NCCL):
    the exchange buffers are torch tensors bound to the slab, and the
    collectives run on the slab's stream, in order with its kernels."""

    def __init__(self, params: Params, device: int, group=None):
        import torch
        import torch.distributed as dist
        self.torch, self.group = torch, group
        self.rank, self.nranks = dist.get_rank(group), dist.get_world_size(group)
        self.slab = Slab(params, self.nranks, self.rank, device)
        dev = torch.device("cuda", device)
        f8 = torch.float64
        # spectra: complex double, or complex float in the mixed path
        fs = torch.float32 if self.slab.mixed else torch.float64
        esz = 4 if fs == torch.float32 else 8
        self.xbuf = torch.empty(self.slab.xbytes // esz, dtype=fs, device=dev)
        self.colbuf = torch.empty(self.slab.colbytes // esz, dtype=fs, device=dev)
        self.hsend = torch.empty(self.slab.hbytes // 8, dtype=f8, device=dev)
        self.hrecv = torch.empty(self.slab.hbytes // 8, dtype=f8, device=dev)
        torch.cuda.synchronize(dev)
        self.slab.bind(self.xbuf.data_ptr(), self.colbuf.data_ptr(), self.hsend.data_ptr(), self.hrecv.data_ptr())
        self.stream = torch.cuda.ExternalStream(self.slab.stream, device=dev)
        self.need_halo = True

    def upload(self, u, v, w, b):
        """This rank's interior levels [nzl][ny][nx]."""
        self.slab.upload(u, v, w, b)
        self.need_halo = True

    def set_forcing(self, kind=PS3D_FORCE_NONE, omega=0.0, **fields):
        """Whole-grid interior forcing fields [nz][ny][nx]; this rank keeps
        its levels and one level each side (Slab.set_forcing)."""
        self.slab.set_forcing(kind, omega, **fields)

    def _halo(self, which):
        s = self.slab
        s.phase("pack_state" if which == 0 else "pack_p")
        with self.torch.cuda.stream(self.stream):
            halo_exchange(self.hsend, self.hrecv, s.plane, which, self.rank, self.nranks, self.group)
        s.phase("unpack_state" if which == 0 else "unpack_p")

    def step(self, nsteps=1):
        s, counts, nzl = self.slab, self.slab.col_counts, self.slab.nzl
        for _ in range(nsteps):
            if self.need_halo:
                self._halo(0)
                self.need_halo = False
            npass = s.step_passes()
            s.phase("tendency")
            self._halo(0)
            for _ in range(npass):
                s.phase("forward")
                with self.torch.cuda.stream(self.stream):
                    columns_forward(self.xbuf, self.colbuf, counts, nzl, self.rank, self.group)
                s.phase("vsolve")
                with self.torch.cuda.stream(self.stream):
                    columns_backward(self.xbuf, self.colbuf, counts, nzl, self.rank, self.group)
                s.phase("inverse")
                self._halo(1)
            s.phase("end_step")

    def diagnose(self):
        """(ke, pe, umax, wmax) of the whole grid: every rank's partial sums
        and maxima reduced over the process group (sums, then maxima)."""
        import torch.distributed as dist
        torch = self.torch
        p = self.slab.params
        ke, pe, um, wm, nf = self.slab.diagnose_partial()
        dev = self.xbuf.device
        sums = torch.tensor([ke, pe], dtype=torch.float64, device=dev)
        maxs = torch.tensor([um, wm, float(nf)], dtype=torch.float64, device=dev)
        with torch.cuda.stream(self.stream):
            dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=self.group)
            dist.all_reduce(maxs, op=dist.ReduceOp.MAX, group=self.group)
        self.stream.synchronize()
        n = p.nx * p.ny * p.nz
        ke, pe, um, wm, nf = combine_diagnostics([(sums[0].item(), sums[1].item(), maxs[0].item(), maxs[1].item(),
                                                   int(maxs[2].item()))], n)
        if nf:
            _check(PS3D_ERR_NONFINITE, "ps3d_slab_diagnose")
        return ke, pe, um, wm

    def download(self):
        return self.slab.download()

    def close(self):
        self.slab.close()
