"""Batched ensembles: every member of a batched launch ends where the same
grid run alone ends (the member index only selects memory)."""
import numpy as np
import pytest

from ps3d_b200 import abi
from ps3d_b200 import configs as cf
from ps3d_b200.ensemble import Ensemble
from ps3d_b200.model import Model
from tests.helpers import rel

pytestmark = pytest.mark.gpu


def _member_fields(p, amp, seed):
    f = cf.eddy_fields(p, amp=amp)
    return cf.add_noise(p, f, "b", rel=1e-3, seed=seed)


@pytest.mark.parametrize("impl", ["0", "1", "2"])
@pytest.mark.parametrize("precision", [abi.PS3D_FP64, abi.PS3D_MIXED])
def test_ensemble_members_match_single_runs(precision, impl, monkeypatch):
    monkeypatch.setenv("PS3D_PLANE_IMPL", impl)
    # untuned defaults on both sides: the batched group and a lone member
    # would otherwise be tuned separately and may take different radix
    # schedules, whose rounding differs at 1e-13
    monkeypatch.setenv("PS3D_AUTOTUNE", "0")
    sizes = [(32, 32, 16), (64, 32, 16), (32, 32, 16), (64, 32, 16), (32, 32, 16)]
    members = [cf.eddy_params(*s, precision=precision) for s in sizes]
    amps = [0.05, 0.1, 0.15, 0.2, 0.12]
    fields = [_member_fields(p, a, seed=i) for i, (p, a) in enumerate(zip(members, amps))]
    ens = Ensemble(members)
    assert ens.info()["groups"] == 2
    for i, f in enumerate(fields):
        ens.upload(i, f["u"], f["v"], f["w"], f["b"])
    nsteps = 11      # eager start, graph replays, eager remainder
    ens.integrate(nsteps)
    for i, (p, f) in enumerate(zip(members, fields)):
        m = Model(p)
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
        m.run(nsteps)
        ref = m.download(tendencies=False)
        got = ens.download(i)
        for n in ("u", "v", "w", "b", "p"):
            assert rel(got[n], ref[n]) < 1e-13, (i, n)
        m.close()
    ens.close()


@pytest.mark.parametrize("precision,tol", [(abi.PS3D_FP64, 1e-11), (abi.PS3D_MIXED, 1e-5)])
def test_ensemble_members_match_oracle(precision, tol):
    """Every member of an ensemble of two sizes, stepped in batched launches
    replayed as CUDA graphs, against the CPU oracle run on that member alone
    (FP64 at the parity tolerance of many steps, mixed at 1e-5)."""
    from oracle.binding import Oracle
    sizes = [(32, 32, 16), (64, 32, 16), (32, 32, 16)]
    members = [cf.eddy_params(*s, precision=precision) for s in sizes]
    amps = [0.08, 0.15, 0.2]
    fields = [_member_fields(p, a, seed=10 + i) for i, (p, a) in enumerate(zip(members, amps))]
    ens = Ensemble(members)
    for i, f in enumerate(fields):
        ens.upload(i, f["u"], f["v"], f["w"], f["b"])
    nsteps = 20
    ens.integrate(nsteps)
    for i, (p, f) in enumerate(zip(members, fields)):
        o = Oracle(cf.eddy_params(*sizes[i]))
        for n in ("u", "v", "w", "b"):
            o.field(n)[...] = f[n]
        o.integrate(nsteps)
        got = ens.download(i)
        for n in ("u", "v", "w", "b", "p"):
            assert rel(got[n], o.field(n)) < tol, (i, n, rel(got[n], o.field(n)))
    ens.close()


@pytest.mark.parametrize("precision,tol_single,tol_oracle",
                         [(abi.PS3D_FP64, 1e-11, 1e-11), (abi.PS3D_MIXED, 1e-8, 1e-5)])
def test_grouped_step_launch(precision, tol_single, tol_oracle, monkeypatch):
    """PS3D_ENSEMBLE_GROUPED=1: the step kernels of all size groups run as one
    launch (the groups' arguments in a table).  That kernel is compiled apart
    from the single-grid one, so its floating-point contractions may differ:
    members agree with lone runs to round-off (FP64; the mixed path's FP32
    history carries a flipped rounding further) and with the oracle at the
    parity tolerances."""
    from oracle.binding import Oracle
    monkeypatch.setenv("PS3D_AUTOTUNE", "0")
    monkeypatch.setenv("PS3D_ENSEMBLE_GROUPED", "1")
    sizes = [(32, 32, 16), (64, 32, 16), (32, 32, 16), (64, 64, 16)]
    members = [cf.eddy_params(*s, precision=precision) for s in sizes]
    amps = [0.08, 0.15, 0.2, 0.1]
    fields = [_member_fields(p, a, seed=20 + i) for i, (p, a) in enumerate(zip(members, amps))]
    ens = Ensemble(members)
    assert ens.info()["groups"] == 3
    for i, f in enumerate(fields):
        ens.upload(i, f["u"], f["v"], f["w"], f["b"])
    nsteps = 11      # eager start, graph replays, eager remainder
    l0 = ens.info()["launches"]
    ens.integrate(nsteps)
    per_step = (ens.info()["launches"] - l0) / nsteps
    for i, (p, f) in enumerate(zip(members, fields)):
        m = Model(p)
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
        m.run(nsteps)
        ref = m.download(tendencies=False)
        got = ens.download(i)
        o = Oracle(cf.eddy_params(*sizes[i]))
        for n in ("u", "v", "w", "b"):
            o.field(n)[...] = f[n]
        o.integrate(nsteps)
        for n in ("u", "v", "w", "b", "p"):
            assert rel(got[n], ref[n]) < tol_single, (i, n, rel(got[n], ref[n]))
            assert rel(got[n], o.field(n)) < tol_oracle, (i, n, rel(got[n], o.field(n)))
        m.close()
    ens.close()
    monkeypatch.setenv("PS3D_ENSEMBLE_GROUPED", "0")
    ens = Ensemble(members)
    for i, f in enumerate(fields):
        ens.upload(i, f["u"], f["v"], f["w"], f["b"])
    l0 = ens.info()["launches"]
    ens.integrate(nsteps)
    # one step-kernel launch per step instead of one per group
    assert (ens.info()["launches"] - l0) / nsteps == pytest.approx(per_step + 2)
    ens.close()


def test_graph_replay_matches_eager():
    """ps3d_integrate replays 3-step CUDA graphs; the result equals stepping
    one call at a time."""
    p = cf.eddy_params(64, 64, 32)
    f = _member_fields(p, 0.1, seed=3)
    a = Model(p)
    b = Model(p)
    for m in (a, b):
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
    a.run(20)
    for _ in range(20):
        b.run(1)
    ra, rb = a.download(tendencies=False), b.download(tendencies=False)
    for n in ("u", "v", "w", "b", "p"):
        assert np.array_equal(ra[n], rb[n]), n


@pytest.mark.parametrize("precision", [abi.PS3D_FP64, abi.PS3D_MIXED])
def test_graph_replay_across_calls_of_any_length(precision):
    """Calls whose step counts are not multiples of the graph period (3)
    leave the (tau, state buffer) cycle at another phase: each phase replays
    its own graph, and the result equals one call of the summed length and
    stepping one step per call."""
    p = cf.eddy_params(64, 64, 32, precision=precision)
    f = _member_fields(p, 0.1, seed=5)
    ms = [Model(p) for _ in range(3)]
    for m in ms:
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
    for n in (7, 8, 5, 11, 4):
        ms[0].run(n)
    ms[1].run(35)
    for _ in range(35):
        ms[2].run(1)
    r = [m.download(tendencies=False) for m in ms]
    for m in ms:
        m.close()
    for q in (1, 2):
        for n in ("u", "v", "w", "b", "p"):
            assert np.array_equal(r[0][n], r[q][n]), (q, n)


@pytest.mark.parametrize("precision", [abi.PS3D_FP64, abi.PS3D_MIXED])
def test_ensemble_calls_of_any_length(precision, monkeypatch):
    """An ensemble advanced by calls of 7, 8, 5 and 11 steps ends where one
    call of 31 steps ends: a call that starts at another phase of the cycle
    captures a graph for that phase instead of replaying the old one."""
    monkeypatch.setenv("PS3D_AUTOTUNE", "0")
    sizes = [(32, 32, 16), (64, 32, 16), (32, 32, 16)]
    members = [cf.eddy_params(*s, precision=precision) for s in sizes]
    fields = [_member_fields(p, 0.05 + 0.05 * i, seed=i) for i, p in enumerate(members)]
    ens = [Ensemble(members) for _ in range(2)]
    for e in ens:
        for i, f in enumerate(fields):
            e.upload(i, f["u"], f["v"], f["w"], f["b"])
    for n in (7, 8, 5, 11):
        ens[0].integrate(n)
    ens[1].integrate(31)
    for i in range(len(members)):
        a, b = ens[0].download(i), ens[1].download(i)
        for n in ("u", "v", "w", "b", "p"):
            assert np.array_equal(a[n], b[n]), (i, n)
    for e in ens:
        e.close()


def test_plane_implementations_agree():
    """The cluster kernels and the rows + y-lines kernels compute the same
    transforms with the same radix schedules: 30 steps agree to 1e-12."""
    import os
    p = cf.eddy_params(64, 64, 32)
    f = _member_fields(p, 0.1, seed=4)
    out = []
    for impl in ("0", "1", "2"):
        os.environ["PS3D_PLANE_IMPL"] = impl
        try:
            m = Model(p)
        finally:
            del os.environ["PS3D_PLANE_IMPL"]
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
        m.run(30)
        out.append(m.download(tendencies=False))
        m.close()
    for q in (1, 2):
        for n in ("u", "v", "w", "b", "p"):
            assert rel(out[q][n], out[0][n]) < 1e-12, (q, n)
