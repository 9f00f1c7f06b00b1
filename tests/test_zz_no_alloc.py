"""ps3d_pressure_solve_noalloc: the pressure projection for callers that
cannot allocate device memory when they call it (they pass device arrays they
own; the engine works in static device arrays).  Its result must equal the
context-based ps3d_pressure_solve and the CPU oracle on the same state, call
after call, and a call must leave the device's free memory unchanged.

This file is collected last on purpose (name), so that a failing run that
stops at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from oracle.binding import Oracle
from ps3d_b200 import abi
from ps3d_b200.model import Model, load
from tests.helpers import load_oracle, random_state, rel, small_params

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the single-kernel parity tolerance of the other GPU tests


def _lib():
    L = load()
    L.ps3d_pressure_solve_noalloc.argtypes = [C.POINTER(abi.Params)] + [C.c_void_p] * 5
    L.ps3d_pressure_solve_noalloc.restype = C.c_int
    return L


def _reference(p, f):
    m = Model(p)
    m.upload(**f)
    m.pressure_solver()
    out = m.download(tendencies=False)
    m.close()
    return out


def _oracle(p, f):
    o = Oracle(p)
    load_oracle(o, f)
    o.pressure_solver()
    return {n: o.field(n).copy() for n in ("u", "v", "w", "p")}


def _noalloc(p, f, free_unchanged=False):
    import torch
    dev = {n: torch.tensor(np.ascontiguousarray(f[n][2:-2, 2:-2, 2:-2]), device="cuda:0")
           for n in ("u", "v", "w")}
    dev["p"] = torch.zeros_like(dev["u"])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    rc = _lib().ps3d_pressure_solve_noalloc(C.byref(p), *[C.c_void_p(dev[n].data_ptr()) for n in ("u", "v", "w", "p")],
                                            None)
    free1 = torch.cuda.mem_get_info(0)[0]
    assert rc == 0, rc
    if free_unchanged:
        assert free1 == free0, (free0, free1)
    return {n: dev[n].cpu().numpy() for n in dev}


@pytest.mark.parametrize("rigid", [True, False])
def test_noalloc_matches_context_two_calls(rigid):
    p = small_params(64, 48, 16, rigid=rigid)
    for seed in (1, 2):   # two calls in a row share the static arrays
        f = random_state(p, seed=seed)
        ref = _reference(p, f)
        # the first call on the device may load the module that holds the
        # static arrays; from then on a call changes no device allocation
        got = _noalloc(p, f, free_unchanged=seed > 1)
        orc = _oracle(p, f)
        for n in ("u", "v", "w", "p"):
            e = rel(got[n], ref[n][2:-2, 2:-2, 2:-2])
            assert e < TOL, (seed, n, e)
            e = rel(got[n], orc[n][2:-2, 2:-2, 2:-2])
            assert e < TOL, ("oracle", seed, n, e)


def test_noalloc_tall_columns():
    """Rigid-lid columns of 512 levels: the vertical solve's tile narrows to
    fit a block's shared memory."""
    p = small_params(16, 16, 512, rigid=True, Lz=1000.0 * 512 / 16)
    f = random_state(p, seed=3)
    ref = _reference(p, f)
    got = _noalloc(p, f)
    for n in ("u", "v", "w", "p"):
        e = rel(got[n], ref[n][2:-2, 2:-2, 2:-2])
        assert e < TOL, (n, e)


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    p = small_params(256, 256, 64)   # (nx/2+1)*ny*nz = 2.1M > 1M
    z = C.c_void_p(0)
    rc = _lib().ps3d_pressure_solve_noalloc(C.byref(p), z, z, z, z, None)
    assert rc == abi.PS3D_ERR_TOOLARGE
    # periodic columns whose z transform does not fit a block's shared memory
    q = small_params(8, 8, 512, rigid=False, Lz=1000.0 * 512 / 16)
    rc = _lib().ps3d_pressure_solve_noalloc(C.byref(q), z, z, z, z, None)
    assert rc == abi.PS3D_ERR_TOOLARGE
