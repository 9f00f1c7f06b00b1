"""Batched ensembles over the C ABI (ps3d_ensemble_*).

Members with identical parameters share every kernel launch; all members
advance together (main-loop semantics), replayed as CUDA graphs for constant
parameters.  No counterpart in the reference, which runs one grid per job.
"""
import ctypes as C

import numpy as np

from .abi import Params, dptr, halo_shape
from .model import PS3DError, load


def _lib():
    L = load()
    if not hasattr(L, "_ens_ready"):
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.ps3d_ensemble_create.argtypes = [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.ps3d_ensemble_destroy.argtypes = [vp]
        L.ps3d_ensemble_upload.argtypes = [vp, C.c_int, dp, dp, dp, dp]
        L.ps3d_ensemble_download.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp]
        L.ps3d_ensemble_integrate.argtypes = [vp, C.c_int]
        L.ps3d_ensemble_enqueue.argtypes = [vp, C.c_int]
        L.ps3d_ensemble_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_void_p)]
        L._ens_ready = True
    return L


def _check(rc, what):
    if rc != 0:
        raise PS3DError(rc, what)


class Ensemble:
    def __init__(self, members, device=0):
        self.L = _lib()
        self.members = [m.copy() for m in members]
        arr = (Params * len(members))(*self.members)
        h = C.c_void_p()
        _check(self.L.ps3d_ensemble_create(arr, len(members), device, C.byref(h)), "ps3d_ensemble_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ps3d_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, member, u, v, w, b):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, b)]
        _check(self.L.ps3d_ensemble_upload(self.h, member, *[dptr(a) for a in arrs]), "ps3d_ensemble_upload")

    def download(self, member):
        shape = halo_shape(self.members[member])
        out = {n: np.zeros(shape) for n in ("u", "v", "w", "b", "p")}
        _check(self.L.ps3d_ensemble_download(self.h, member, *[dptr(out[n]) for n in ("u", "v", "w", "b", "p")]),
               "ps3d_ensemble_download")
        return out

    def integrate(self, nsteps):
        _check(self.L.ps3d_ensemble_integrate(self.h, nsteps), "ps3d_ensemble_integrate")

    def enqueue(self, nsteps):
        _check(self.L.ps3d_ensemble_enqueue(self.h, nsteps), "ps3d_ensemble_enqueue")

    def info(self):
        ng, nl, st = C.c_int(), C.c_longlong(), C.c_void_p()
        _check(self.L.ps3d_ensemble_info(self.h, C.byref(ng), C.byref(nl), C.byref(st)), "ps3d_ensemble_info")
        return {"groups": ng.value, "launches": nl.value, "stream": st.value or 0}
