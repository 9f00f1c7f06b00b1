"""Host-side mirror of the ps3D interface over the CUDA engine's C ABI.

The reference drives its hot path through argument-less Fortran routines on
module state (for_src/main_module.f90).  `Model` keeps the same names and
meaning on a device-resident context:

    Model.integrate()                         integrate.f90:2-115 (one call)
    Model.run(n)                              main.f90:139-162 loop body, n times
    Model.pressure_solver()                   pressure_solver.f90:2-120
    Model.normal_mode_projection()            diag_opt_balance.f90:288-310
    Model.geostrophic_base_point()            diag_opt_balance.f90:263-285
    Model.exchange_geostrophic_base_point()   diag_opt_balance.f90:313-335
    Model.diag_balance_zero_order()           diag_balance.f90:109-132
    Model.diag_opt_balance(opt)               diag_opt_balance.f90:55-179
    Model.diagnose()                          diagnose.F90:2-61

Errors come back as `PS3DError` carrying the C status code; where the
reference aborts (halt_stop on NaN, parallel_mpi.f90:5-18) the engine
returns PS3D_ERR_NONFINITE instead.  There is no CPU fallback: without the
built library every call raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import Params, OptBal, Forcing, dptr, halo_shape

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libps3d_gpu.so")
_lib = None


class PS3DError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {status} ({strerror(status)})")


def load():
    """Load libps3d_gpu.so (build it first with ps3d_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA engine not built: {LIB_PATH} is missing (run python -m ps3d_b200.build)")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.ps3d_create.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]
    L.ps3d_destroy.argtypes = [vp]
    L.ps3d_upload_state.argtypes = [vp] + [dp] * 9 + [C.c_int] * 4
    L.ps3d_download_state.argtypes = [vp] + [dp] * 9 + [ip] * 4
    L.ps3d_step.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.ps3d_integrate.argtypes = [vp, C.c_int]
    L.ps3d_set_step_params.argtypes = [vp] + [C.c_double] * 6
    L.ps3d_pressure_solve.argtypes = [vp]
    L.ps3d_project_geostrophic.argtypes = [vp, C.c_int]
    L.ps3d_opt_balance.argtypes = [vp, C.POINTER(OptBal), dp, ip]
    L.ps3d_get_fields.argtypes = [vp, C.c_int, dp, dp, dp, dp]
    L.ps3d_diag_balance.argtypes = [vp, C.c_int, C.c_int]
    L.ps3d_write_restart.argtypes = [vp, C.c_char_p]
    L.ps3d_snapshot_begin.argtypes = [vp, dp, dp, dp, dp, dp]
    L.ps3d_snapshot_wait.argtypes = [vp]
    L.ps3d_read_restart.argtypes = [vp, C.c_char_p, dp]
    L.ps3d_diagnose.argtypes = [vp, dp, dp, dp, dp]
    L.ps3d_set_forcing.argtypes = [vp, C.POINTER(Forcing)]
    L.ps3d_get_stream.argtypes = [vp, C.POINTER(C.c_void_p)]
    L.ps3d_enqueue.argtypes = [vp, C.c_int]
    L.ps3d_profile.argtypes = [vp, C.c_int]
    L.ps3d_profile_read.argtypes = [vp, dp, C.POINTER(C.c_longlong)]
    L.ps3d_describe.argtypes = [vp, C.c_char_p, C.c_int]
    L.ps3d_strerror.restype = C.c_char_p
    L.ps3d_strerror.argtypes = [C.c_int]
    _lib = L
    return L


def strerror(status):
    try:
        return load().ps3d_strerror(status).decode()
    except Exception:
        return "unknown"


def _check(rc, what):
    if rc != 0:
        raise PS3DError(rc, what)


class Model:
    """One grid on one GPU, state resident in HBM."""

    FIELDS = ("u", "v", "w", "b")

    def __init__(self, params: Params, device: int = 0):
        self.L = load()
        self.params = params.copy()
        self.shape = halo_shape(self.params)
        h = C.c_void_p()
        _check(self.L.ps3d_create(C.byref(self.params), device, C.byref(h)), "ps3d_create")
        self.h = h
        self._forcing_keep = None

    def close(self):
        if getattr(self, "h", None):
            self.L.ps3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state transfer (host halo layout) ----------------------------------
    def upload(self, u=None, v=None, w=None, b=None, p=None, du=None, dv=None, dw=None, db=None,
               itt=0, tau=3, taum1=2, taum2=1):
        arrs = [u, v, w, b, p, du, dv, dw, db]
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        _check(self.L.ps3d_upload_state(self.h, *[dptr(a) for a in arrs], itt, tau, taum1, taum2),
               "ps3d_upload_state")

    def download(self, tendencies=True):
        out = {n: np.zeros(self.shape) for n in ("u", "v", "w", "b", "p")}
        if tendencies:
            for n in ("du", "dv", "dw", "db"):
                out[n] = np.zeros((3,) + self.shape)
        tl = [C.c_int() for _ in range(4)]
        _check(self.L.ps3d_download_state(self.h, *[dptr(out.get(n)) for n in
                                                    ("u", "v", "w", "b", "p", "du", "dv", "dw", "db")],
                                          *[C.byref(t) for t in tl]), "ps3d_download_state")
        out["itt"], out["tau"], out["taum1"], out["taum2"] = (t.value for t in tl)
        return out

    def download_into(self, out):
        """Like download(tendencies=False), into caller-owned C-contiguous
        float64 arrays out["u"], ..., out["p"] of the halo shape (e.g. pinned)."""
        for n in ("u", "v", "w", "b", "p"):
            a = out[n]
            if a.shape != self.shape or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"download_into: {n} must be C-contiguous float64 of shape {self.shape}")
        _check(self.L.ps3d_download_state(self.h, *[dptr(out[n]) for n in ("u", "v", "w", "b", "p")],
                                          None, None, None, None, None, None, None, None), "ps3d_download_state")
        return out

    def get_fields(self, which=abi.PS3D_FIELDS_STATE):
        out = [np.zeros(self.shape) for _ in range(4)]
        _check(self.L.ps3d_get_fields(self.h, which, *[dptr(a) for a in out]), "ps3d_get_fields")
        return dict(zip(self.FIELDS, out))

    # -- hot path -------------------------------------------------------------
    def integrate(self, itt, tau, taum1, taum2):
        """integrate.f90 once with the caller's time levels (no rotation)."""
        _check(self.L.ps3d_step(self.h, itt, tau, taum1, taum2), "ps3d_step")

    def run(self, nsteps):
        """nsteps of the main loop body: integrate, rotate, time += dt, itt += 1."""
        _check(self.L.ps3d_integrate(self.h, nsteps), "ps3d_integrate")

    def set_step_params(self, dt, Ro, Ahbi=0.0, Avbi=0.0, Khbi=0.0, Kvbi=0.0):
        _check(self.L.ps3d_set_step_params(self.h, dt, Ro, Ahbi, Avbi, Khbi, Kvbi), "ps3d_set_step_params")

    def pressure_solver(self):
        _check(self.L.ps3d_pressure_solve(self.h), "ps3d_pressure_solve")

    def project(self, mode):
        _check(self.L.ps3d_project_geostrophic(self.h, mode), "ps3d_project_geostrophic")

    def normal_mode_projection(self):
        self.project(abi.PS3D_PROJ_NORMAL_MODE)

    def geostrophic_base_point(self):
        self.project(abi.PS3D_PROJ_BASE_POINT)

    def exchange_geostrophic_base_point(self):
        self.project(abi.PS3D_PROJ_EXCHANGE)

    def diag_balance_zero_order(self):
        self.project(abi.PS3D_PROJ_ZERO_ORDER)
        return self.get_fields(abi.PS3D_FIELDS_ZERO)

    def snapshot_begin(self, out):
        """Queue an asynchronous snapshot of u, v, w, b, p into caller-owned
        C-contiguous float64 arrays of the halo shape (page-locked to overlap);
        keep them alive until snapshot_wait()."""
        for n in ("u", "v", "w", "b", "p"):
            a = out.get(n)
            if a is not None and (a.shape != self.shape or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]):
                raise ValueError(f"snapshot_begin: {n} must be C-contiguous float64 of shape {self.shape}")
        self._snap_keep = out
        _check(self.L.ps3d_snapshot_begin(self.h, *[dptr(out.get(n)) for n in ("u", "v", "w", "b", "p")]),
               "ps3d_snapshot_begin")

    def snapshot_wait(self):
        _check(self.L.ps3d_snapshot_wait(self.h), "ps3d_snapshot_wait")
        self._snap_keep = None

    def write_restart(self, path):
        """write_restart (restart.f90:2-22): the reference's one-rank restart file."""
        _check(self.L.ps3d_write_restart(self.h, os.fsencode(path)), "ps3d_write_restart")

    def read_restart(self, path):
        """read_restart (restart.f90:27-82); returns the file's time."""
        t = C.c_double()
        _check(self.L.ps3d_read_restart(self.h, os.fsencode(path), C.byref(t)), "ps3d_read_restart")
        return t.value

    def diag_balance(self, order=3, filter_width=-1):
        """Warn-et-al. balance to `order` (diag_balance.f90:89-362): returns
        [components of order 0, 1, ...], each {"u","v","w","b"} in halo
        layout; the balanced state is their sum.  filter_width >= 0 turns on
        enable_diag_balance_filter with that width."""
        _check(self.L.ps3d_diag_balance(self.h, order, filter_width), "ps3d_diag_balance")
        sets = (abi.PS3D_FIELDS_ZERO, abi.PS3D_FIELDS_FIRST, abi.PS3D_FIELDS_SECOND, abi.PS3D_FIELDS_THIRD)
        return [self.get_fields(sets[n]) for n in range(order + 1)]

    def diag_opt_balance(self, opt: OptBal):
        norm, iters = C.c_double(), C.c_int()
        _check(self.L.ps3d_opt_balance(self.h, C.byref(opt), C.byref(norm), C.byref(iters)), "ps3d_opt_balance")
        return norm.value, iters.value

    def diagnose(self):
        """(ke, pe, umax, wmax); raises PS3DError(PS3D_ERR_NONFINITE) on NaN/Inf."""
        ke, pe, um, wm = (C.c_double() for _ in range(4))
        _check(self.L.ps3d_diagnose(self.h, C.byref(ke), C.byref(pe), C.byref(um), C.byref(wm)), "ps3d_diagnose")
        return ke.value, pe.value, um.value, wm.value

    # -- engine extensions ------------------------------------------------------
    def stream(self):
        """cudaStream_t handle (int) the context launches on."""
        s = C.c_void_p()
        _check(self.L.ps3d_get_stream(self.h, C.byref(s)), "ps3d_get_stream")
        return s.value or 0

    def enqueue(self, nsteps):
        """Queue nsteps of the main loop body without waiting for them."""
        _check(self.L.ps3d_enqueue(self.h, nsteps), "ps3d_enqueue")

    def profile(self, enable=True):
        _check(self.L.ps3d_profile(self.h, int(enable)), "ps3d_profile")

    def describe(self):
        buf = C.create_string_buffer(512)
        _check(self.L.ps3d_describe(self.h, buf, 512), "ps3d_describe")
        return buf.value.decode()

    KERNELS = ("step", "fft_fwd", "vsolve", "fft_inv", "correct", "other", "vmode")

    def profile_read(self):
        """{kernel class: (device ms summed over launches, launches)} since ps3d_profile."""
        ms = (C.c_double * len(self.KERNELS))()
        n = (C.c_longlong * len(self.KERNELS))()
        _check(self.L.ps3d_profile_read(self.h, ms, n), "ps3d_profile_read")
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNELS)}

    def set_forcing(self, kind=abi.PS3D_FORCE_NONE, omega=0.0, fn=None, user=None, **fields):
        """set_forcing hook: kind bitmask, wavemaker fields u_r..b_i, background u_back, b_back."""
        f = Forcing()
        f.kind = kind
        f.omega = omega
        keep = []
        for name in ("u_r", "v_r", "w_r", "b_r", "u_i", "v_i", "w_i", "b_i", "u_back", "b_back"):
            a = fields.get(name)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(a)
                setattr(f, name, dptr(a))
        if fn is not None:
            cb = abi.FORCING_FN(fn)
            keep.append(cb)
            f.fn = cb
        f.user = user
        self._forcing_keep = (f, keep)
        _check(self.L.ps3d_set_forcing(self.h, C.byref(f)), "ps3d_set_forcing")
