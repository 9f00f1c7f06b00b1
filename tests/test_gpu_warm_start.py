"""The mixed path's warm-started projection.

From the second step on, PS3D_MIXED solves once per step, for the FP64
residual div(u - dt grad p0)/dt against the previous step's pressure p0, and
adds the result to p (the cold start, after create or any upload, and every
step of PS3D_MIXED_REFINED, is a full FP32 solve and one FP64-residual
refinement).  In exact arithmetic both give pressure_solver's p
(pressure_solver.f90:2-120): p0 lies in the solver's gauge (a solver output,
or zero), so only the FP32 rounding of the step's change of p differs.  These
tests check that the warm start runs, that it agrees with the refined solves,
how divergence-free each leaves the velocity, and that an uploaded p (outside
the solver's gauge) cannot leak into the result.
"""
import numpy as np
import pytest

from ps3d_b200 import abi
from ps3d_b200 import configs as cf
from ps3d_b200.model import Model
from tests.helpers import rel

pytestmark = pytest.mark.gpu

NAMES = ("u", "v", "w", "b", "p")


def _eddy(precision=abi.PS3D_MIXED):
    p = cf.eddy_params(64, 64, 32, precision=precision)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=0)
    return p, f


def _interior(a):
    return a[2:-2, 2:-2, 2:-2]


def _div(p, s):
    u, v, w = (_interior(s[n]) for n in ("u", "v", "w"))
    du = (u - np.roll(u, 1, axis=2)) / p.dx
    dv = (v - np.roll(v, 1, axis=1)) / p.dy
    wm = np.roll(w, 1, axis=0)
    wm[0] = 0.0   # rigid lid
    return du + dv + (w - wm) / p.dz


@pytest.mark.parametrize("precision,first,later",
                         [(abi.PS3D_MIXED, 2, 1), (abi.PS3D_MIXED_REFINED, 2, 2), (abi.PS3D_FP64, 1, 1)])
def test_solves_per_step(precision, first, later):
    """Forward transforms per step (profile_read counts since its last read)."""
    p, f = _eddy(precision)
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    m.profile(True)
    m.run(1)
    assert m.profile_read()["fft_fwd"][1] == first
    m.run(4)
    assert m.profile_read()["fft_fwd"][1] == 4 * later
    m.upload(b=f["b"])   # any upload: the next step starts cold again
    m.run(1)
    assert m.profile_read()["fft_fwd"][1] == first
    m.close()


def _run(p, f, nsteps):
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    m.run(nsteps)
    s = m.download(tendencies=False)
    m.close()
    return s


def test_warm_start_matches_refined_solves():
    """60 steps warm (graphs included) against PS3D_MIXED_REFINED: the step's
    change of p rounded to FP32 moves the fields by < 1e-6 (w, whose
    buoyancy and pressure terms nearly cancel, the most); the refined
    projection leaves the divergence at FP64 roundoff, the warm one at the
    FP32 rounding of the change of p."""
    p, f = _eddy()
    pr = p.copy()
    pr.precision = abi.PS3D_MIXED_REFINED
    sw = _run(p, f, 60)
    sr = _run(pr, f, 60)
    err = {n: rel(_interior(sw[n]), _interior(sr[n])) for n in NAMES}
    assert max(err.values()) < 1e-6, err
    scale = np.abs(_interior(sr["u"])).max() / p.dx
    assert np.abs(_div(p, sr)).max() < 1e-9 * scale
    assert np.abs(_div(p, sw)).max() < 4e-6 * scale


def test_step_parameters_keep_the_warm_start():
    """The drop-in integrate sets the step parameters before every ps3d_step
    (the balance drivers ramp them); new parameters do not replace the state,
    so the mixed path stays warm: one forward transform per step after the
    first, and the trajectory of ps3d_integrate."""
    p, f = _eddy()
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    m.profile(True)
    for _ in range(6):
        m.set_step_params(p.dt, p.Ro)
        m.run(1)
    assert m.profile_read()["fft_fwd"][1] == 2 + 5
    s1 = m.download(tendencies=False)
    m.close()
    s2 = _run(p, f, 6)
    err = {n: rel(_interior(s1[n]), _interior(s2[n])) for n in NAMES}
    assert max(err.values()) < 1e-13, err


def test_uploaded_pressure_does_not_leak():
    """The reference recomputes p from scratch every step, so an uploaded p
    (here random, with a mean: outside the solver's gauge) must not change the
    pressure after the first step."""
    p, f = _eddy()
    rng = np.random.default_rng(3)
    p_up = 1.0 + rng.standard_normal(f["u"].shape)
    out = []
    for pin in (None, p_up):
        m = Model(p)
        fields = {n: f[n] for n in "uvwb"}
        if pin is not None:
            fields["p"] = pin
        m.upload(**fields)
        m.run(12)
        out.append(m.download(tendencies=False))
        m.close()
    err = {n: rel(_interior(out[1][n]), _interior(out[0][n])) for n in NAMES}
    assert max(err.values()) < 1e-12, err
