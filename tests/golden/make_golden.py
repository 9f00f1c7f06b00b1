"""Regenerate tests/golden/*.npz from the CPU oracle.

These fixtures are oracle outputs, not outputs of the reference binary (which
cannot be built here); they pin the oracle against regressions and give the
GPU tests a check that needs no oracle at run time.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.binding import Oracle  # noqa: E402
from ps3d_b200 import abi  # noqa: E402
from tests.helpers import FIELDS, load_oracle, small_params, smooth_state  # noqa: E402

CASES = {
    # name: (params kwargs, steps, projection mode or None)
    "rigid_16x16x8_3steps": (dict(nx=16, ny=16, nz=8, rigid=True), 3, None),
    "periodic_16x12x8_3steps": (dict(nx=16, ny=12, nz=8, rigid=False, Kh=1e-2, Kv=1e-3), 3, None),
    "rigid_24x20x6_projection": (dict(nx=24, ny=20, nz=6, rigid=True), 0, abi.PS3D_PROJ_NORMAL_MODE),
    "periodic_16x16x8_projection": (dict(nx=16, ny=16, nz=8, rigid=False), 0, abi.PS3D_PROJ_NORMAL_MODE),
}


def make(name):
    kw, steps, proj = CASES[name]
    kw = dict(kw)
    p = small_params(kw.pop("nx"), kw.pop("ny"), kw.pop("nz"), rigid=kw.pop("rigid"), **kw)
    o = Oracle(p)
    init = smooth_state(p, seed=42)
    load_oracle(o, init)
    if steps:
        o.integrate(steps)
    if proj is not None:
        o.project(proj)
    out = {"params": np.array([getattr(p, f) for f, _ in p._fields_], dtype=np.float64)}
    for n in FIELDS:
        out["init_" + n] = init[n][2:-2, 2:-2, 2:-2]
        out[n] = o.field(n)[2:-2, 2:-2, 2:-2].copy()
    out["p"] = o.field("p")[2:-2, 2:-2, 2:-2].copy()
    return out


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **make(name))
        print("wrote", name)
