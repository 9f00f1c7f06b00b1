"""Committed golden fixtures (tests/golden/make_golden.py).

CPU: the oracle reproduces them (a regression pin of the oracle itself).
GPU: the engine reproduces them through the C ABI without the oracle.
"""
import os

import numpy as np
import pytest

from ps3d_b200 import configs as cf
from tests.golden.make_golden import CASES, make
from tests.helpers import FIELDS, rel, small_params

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(name):
    ref = load(name)
    got = make(name)
    for k in ("u", "v", "w", "b", "p"):
        scale = np.abs(ref[k]).max()
        assert np.abs(got[k] - ref[k]).max() <= 1e-13 * max(scale, 1e-300), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_reproduces_golden(name):
    from ps3d_b200.model import Model
    ref = load(name)
    kw, steps, proj = CASES[name]
    kw = dict(kw)
    p = small_params(kw.pop("nx"), kw.pop("ny"), kw.pop("nz"), rigid=kw.pop("rigid"), **kw)
    m = Model(p)
    init = {}
    for n in FIELDS:
        h = cf.empty_field(p)
        cf.interior(h)[...] = ref["init_" + n]
        init[n] = cf.halo_fill(h)
    m.upload(**init)
    if steps:
        m.run(steps)
    if proj is not None:
        m.project(proj)
    got = m.download(tendencies=False)
    names = ("u", "v", "w", "b", "p") if steps else FIELDS
    for n in names:
        if np.abs(ref[n]).max() == 0:
            continue
        e = rel(got[n][2:-2, 2:-2, 2:-2], ref[n])
        assert e < 1e-12, (n, e)
