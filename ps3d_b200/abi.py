"""ctypes mirrors of the structs declared in include/ps3d_gpu.h.

The layouts follow the C header field for field; the reference module
variables they carry are listed there (for_src/main_module.f90:16-57).
"""
import ctypes as C

PS3D_OK = 0
PS3D_ERR_CUDA = -1
PS3D_ERR_NONFINITE = -2
PS3D_ERR_TIMEOUT = -3
PS3D_ERR_OOM = -4
PS3D_ERR_BADPARAM = -5
PS3D_ERR_UNSUPPORTED = -6
PS3D_ERR_CANCELLED = -7
PS3D_ERR_TOOLARGE = -8

PS3D_FP64 = 0
PS3D_MIXED = 1
PS3D_MIXED_REFINED = 2

PS3D_FORCE_NONE = 0
PS3D_FORCE_WAVEMAKER = 1
PS3D_FORCE_BACKGROUND = 2
PS3D_FORCE_CALLBACK = 4

PS3D_PROJ_NORMAL_MODE = 0
PS3D_PROJ_BASE_POINT = 1
PS3D_PROJ_EXCHANGE = 2
PS3D_PROJ_ZERO_ORDER = 3

PS3D_FIELDS_STATE = 0
PS3D_FIELDS_BALANCED = 1
PS3D_FIELDS_BASE = 2
PS3D_FIELDS_ZERO = 3
PS3D_FIELDS_FIRST = 4
PS3D_FIELDS_SECOND = 5
PS3D_FIELDS_THIRD = 6


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dt", C.c_double), ("f0", C.c_double), ("N0", C.c_double),
        ("Ro", C.c_double), ("dsqr", C.c_double), ("eps_ab", C.c_double),
        ("Ah", C.c_double), ("Av", C.c_double), ("Kh", C.c_double), ("Kv", C.c_double),
        ("Ahbi", C.c_double), ("Avbi", C.c_double), ("Khbi", C.c_double), ("Kvbi", C.c_double),
        ("enable_nonlinear", C.c_int), ("enable_vertical_boundaries", C.c_int),
        ("enable_AB_3_order", C.c_int), ("precision", C.c_int),
    ]

    def copy(self):
        out = Params()
        C.pointer(out)[0] = self
        return out

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class OptBal(C.Structure):
    _fields_ = [
        ("period", C.c_double), ("average", C.c_double),
        ("max_itts", C.c_int), ("average_times", C.c_int),
        ("tol", C.c_double), ("enable_time_ave", C.c_int), ("adopt", C.c_int),
    ]


class DeviceView(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p), ("b", C.c_void_p),
        ("du", C.c_void_p), ("dv", C.c_void_p), ("dw", C.c_void_p), ("db", C.c_void_p),
        ("dt", C.c_double), ("Ro", C.c_double), ("itt", C.c_int), ("stream", C.c_void_p),
    ]


FORCING_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(DeviceView))

_DP = C.POINTER(C.c_double)


class Forcing(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("omega", C.c_double),
        ("u_r", _DP), ("v_r", _DP), ("w_r", _DP), ("b_r", _DP),
        ("u_i", _DP), ("v_i", _DP), ("w_i", _DP), ("b_i", _DP),
        ("u_back", _DP), ("b_back", _DP),
        ("fn", FORCING_FN), ("user", C.c_void_p),
    ]


def make_params(**kw):
    """Params with the reference's defaults (main_module.f90:16-57), overridden by kw.

    dx, dy, dz default to Lx/nx, Ly/ny, Lz/nz as every reference config sets them.
    """
    p = Params()
    defaults = dict(Ro=1.0, dsqr=1.0, eps_ab=0.0, enable_nonlinear=1,
                    enable_vertical_boundaries=0, enable_AB_3_order=0, precision=PS3D_FP64)
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(p, k, v)
    if "dx" not in kw:
        p.dx = p.Lx / p.nx
    if "dy" not in kw:
        p.dy = p.Ly / p.ny
    if "dz" not in kw:
        p.dz = p.Lz / p.nz
    return p


def halo_shape(p):
    """numpy shape (C order: z, y, x) of a halo-padded field."""
    return (p.nz + 4, p.ny + 4, p.nx + 4)


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)
