"""ctypes binding of the CPU oracle — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, and only to check the CUDA engine's results against it.  The
library under test never does.
Field arrays are halo-padded (nz+4, ny+4, nx+4) float64 views (C order z,y,x,
which is the reference's Fortran column-major (x,y,z) layout).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from ps3d_b200.abi import Params, OptBal, Forcing, halo_shape

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "libps3d_oracle.so")
_lib = None

FIELD_IDS = {"u": 0, "v": 1, "w": 2, "b": 3, "p": 4,
             "du": 5, "dv": 8, "dw": 11, "db": 14,
             "u_bal": 20, "v_bal": 21, "w_bal": 22, "b_bal": 23,
             "u_base": 24, "v_base": 25, "w_base": 26, "b_base": 27,
             "u0": 28, "v0": 29, "w0": 30, "b0": 31,
             "u1": 32, "v1": 33, "w1": 34, "b1": 35, "u2": 36, "v2": 37, "w2": 38, "b2": 39,
             "u3": 40, "v3": 41, "w3": 42, "b3": 43}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.ps3d_oracle_create.restype = vp
        L.ps3d_oracle_create.argtypes = [C.POINTER(Params)]
        L.ps3d_oracle_destroy.argtypes = [vp]
        L.ps3d_oracle_field.restype = dp
        L.ps3d_oracle_field.argtypes = [vp, C.c_int]
        L.ps3d_oracle_field_size.restype = C.c_long
        L.ps3d_oracle_field_size.argtypes = [vp]
        L.ps3d_oracle_get_time.argtypes = [vp, ip, ip, ip, ip, dp]
        L.ps3d_oracle_set_time.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
        L.ps3d_oracle_set_step_params.argtypes = [vp] + [C.c_double] * 6
        L.ps3d_oracle_border_exchange.argtypes = [vp, dp]
        L.ps3d_oracle_step.argtypes = [vp]
        L.ps3d_oracle_integrate.argtypes = [vp, C.c_int]
        L.ps3d_oracle_pressure_solver.argtypes = [vp]
        L.ps3d_oracle_project.argtypes = [vp, C.c_int]
        L.ps3d_oracle_diag_balance.argtypes = [vp, C.c_int, C.c_int]
        L.ps3d_oracle_forward_transform.argtypes = [vp]
        L.ps3d_oracle_opt_balance.argtypes = [vp, C.POINTER(OptBal), dp, ip]
        L.ps3d_oracle_diagnose.restype = C.c_int
        L.ps3d_oracle_diagnose.argtypes = [vp, dp, dp, dp, dp]
        L.ps3d_oracle_set_forcing.argtypes = [vp, C.POINTER(Forcing)]
        L.ps3d_oracle_ksqr.restype = dp
        L.ps3d_oracle_ksqr.argtypes = [vp, C.POINTER(C.c_long)]
        L.ps3d_oracle_modes.restype = dp
        L.ps3d_oracle_modes.argtypes = [vp, C.c_int]
        L.ps3d_oracle_wavenumbers.restype = dp
        L.ps3d_oracle_wavenumbers.argtypes = [vp, C.c_int]
        L.ps3d_oracle_spectral.restype = dp
        L.ps3d_oracle_spectral.argtypes = [vp, C.c_int]
        L.ps3d_oracle_eigen.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, dp]
        L.ps3d_oracle_fft.argtypes = [dp, C.c_int, C.c_int]
        L.ps3d_oracle_fft_field.argtypes = [vp, dp, dp, C.c_int]
        L.ps3d_oracle_ifft_field.argtypes = [vp, dp, dp, C.c_int]
        L.ps3d_oracle_tridiag.argtypes = [dp, dp, dp, dp, dp, C.c_int]
        L.ps3d_oracle_ramp.restype = C.c_double
        L.ps3d_oracle_ramp.argtypes = [C.c_double]
        L.ps3d_oracle_threads.restype = C.c_int
        L.ps3d_oracle_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One model instance of the CPU restatement."""

    def __init__(self, params: Params):
        self.params = params.copy()
        self.L = lib()
        self.h = self.L.ps3d_oracle_create(C.byref(self.params))
        self.shape = halo_shape(self.params)
        self._forcing_keep = None

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.ps3d_oracle_destroy(self.h)
                self.h = None
        except Exception:
            pass

    # -- fields --------------------------------------------------------------
    def field(self, name, slot=None):
        fid = FIELD_IDS[name] + (0 if slot is None else slot - 1)
        ptr = self.L.ps3d_oracle_field(self.h, fid)
        n = int(np.prod(self.shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(self.shape)

    def tendency(self, name):
        """(3, nz+4, ny+4, nx+4) copy of a tendency with its 3 time levels."""
        return np.stack([self.field(name, s).copy() for s in (1, 2, 3)])

    def set_tendency(self, name, arr3):
        for s in (1, 2, 3):
            self.field(name, s)[...] = arr3[s - 1]

    def interior(self, name, slot=None):
        return self.field(name, slot)[2:-2, 2:-2, 2:-2]

    def exchange(self, a):
        assert a.flags["C_CONTIGUOUS"] and a.shape == self.shape
        self.L.ps3d_oracle_border_exchange(self.h, _d(a))

    # -- time levels -----------------------------------------------------------
    def get_time(self):
        itt, tau, t1, t2 = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        time = C.c_double()
        self.L.ps3d_oracle_get_time(self.h, C.byref(itt), C.byref(tau), C.byref(t1), C.byref(t2), C.byref(time))
        return itt.value, tau.value, t1.value, t2.value, time.value

    def set_time(self, itt=0, tau=3, taum1=2, taum2=1, time=0.0):
        self.L.ps3d_oracle_set_time(self.h, itt, tau, taum1, taum2, time)

    def set_step_params(self, dt, Ro, Ahbi=0.0, Avbi=0.0, Khbi=0.0, Kvbi=0.0):
        self.L.ps3d_oracle_set_step_params(self.h, dt, Ro, Ahbi, Avbi, Khbi, Kvbi)

    # -- hot path --------------------------------------------------------------
    def step(self):
        self.L.ps3d_oracle_step(self.h)

    def integrate(self, nsteps):
        self.L.ps3d_oracle_integrate(self.h, nsteps)

    def pressure_solver(self):
        self.L.ps3d_oracle_pressure_solver(self.h)

    def project(self, mode):
        self.L.ps3d_oracle_project(self.h, mode)

    def diag_balance(self, order, filter_width=-1):
        """Warn-et-al. balance to `order` (diag_balance.f90:89-362); components
        in fields u0..b0, u1..b1, u2..b2, u3..b3."""
        self.L.ps3d_oracle_diag_balance(self.h, order, filter_width)

    def forward_transform(self):
        """forward_transform of the state; read the result with spectral(1..4)."""
        self.L.ps3d_oracle_forward_transform(self.h)

    def opt_balance(self, opt: OptBal):
        norm, iters = C.c_double(), C.c_int()
        self.L.ps3d_oracle_opt_balance(self.h, C.byref(opt), C.byref(norm), C.byref(iters))
        return norm.value, iters.value

    def diagnose(self):
        ke, pe, um, wm = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        st = self.L.ps3d_oracle_diagnose(self.h, C.byref(ke), C.byref(pe), C.byref(um), C.byref(wm))
        return st, ke.value, pe.value, um.value, wm.value

    def set_forcing(self, forcing: Forcing, keep=None):
        self._forcing_keep = (forcing, keep)
        self.L.ps3d_oracle_set_forcing(self.h, C.byref(forcing))

    # -- tables / spectral -----------------------------------------------------
    def ksqr(self):
        n = C.c_long()
        ptr = self.L.ps3d_oracle_ksqr(self.h, C.byref(n))
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).copy()

    def modes(self, which):
        nz = self.params.nz
        ptr = self.L.ps3d_oracle_modes(self.h, which)
        return np.ctypeslib.as_array(ptr, shape=(nz * nz,)).reshape(nz, nz).T.copy()  # [k, mode]

    def wavenumbers(self, axis):
        n = [self.params.nx // 2 + 1, self.params.ny, self.params.nz][axis]
        ptr = self.L.ps3d_oracle_wavenumbers(self.h, axis)
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

    def spectral(self, which=0):
        p = self.params
        n = (p.nx // 2 + 1) * p.ny * p.nz
        ptr = self.L.ps3d_oracle_spectral(self.h, which)
        a = np.ctypeslib.as_array(ptr, shape=(2 * n,)).copy()
        return (a[0::2] + 1j * a[1::2]).reshape(p.nz, p.ny, p.nx // 2 + 1)

    def eigen(self, kx, ky, kz, s):
        out = np.zeros(17)
        self.L.ps3d_oracle_eigen(self.h, kx, ky, kz, s, _d(out))
        q = out[0:8:2] + 1j * out[1:8:2]
        pv = out[8:16:2] + 1j * out[9:16:2]
        return q, pv, out[16]

    def fft_field(self, interior, three_d):
        p = self.params
        QP = np.ascontiguousarray(interior, dtype=np.float64)
        n = (p.nx // 2 + 1) * p.ny * p.nz
        QS = np.zeros(2 * n)
        self.L.ps3d_oracle_fft_field(self.h, _d(QP), _d(QS), int(three_d))
        return (QS[0::2] + 1j * QS[1::2]).reshape(p.nz, p.ny, p.nx // 2 + 1)

    def ifft_field(self, spec, three_d):
        p = self.params
        QS = np.zeros(2 * spec.size)
        QS[0::2] = spec.real.ravel()
        QS[1::2] = spec.imag.ravel()
        QP = np.zeros((p.nz, p.ny, p.nx))
        self.L.ps3d_oracle_ifft_field(self.h, _d(QS), _d(QP), int(three_d))
        return QP


def fft(x, sign=-1):
    """Complex FFT of the oracle's own Stockham implementation."""
    x = np.asarray(x, dtype=np.complex128)
    buf = np.empty(2 * x.size)
    buf[0::2], buf[1::2] = x.real, x.imag
    lib().ps3d_oracle_fft(_d(buf), x.size, sign)
    return buf[0::2] + 1j * buf[1::2]


def tridiag(a, b, c, d):
    n = len(b)
    dd = np.empty(2 * n)
    dd[0::2], dd[1::2] = np.real(d), np.imag(d)
    x = np.empty(2 * n)
    a, b, c = (np.ascontiguousarray(t, dtype=np.float64) for t in (a, b, c))
    lib().ps3d_oracle_tridiag(_d(a), _d(b), _d(c), _d(dd), _d(x), n)
    return x[0::2] + 1j * x[1::2]


def ramp(theta):
    return lib().ps3d_oracle_ramp(theta)


def set_threads(n):
    return lib().ps3d_oracle_threads(n)
