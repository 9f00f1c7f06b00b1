"""One grid in z-slabs (ps3d_slab_*) against the same grid on one context.

The slab phases (the step kernel on a level window, the per-level 2D
transforms, the all-to-all transposes to column slabs, the column-slab
vertical solves, the halo planes) must reproduce the single-grid engine: the
arithmetic per level and per column is the same, so the tolerance is the
single-kernel one.  Ranks run as contexts of one process on one GPU, moved
between by device copies (ps3d_slab_group_step); no kernel waits on another.
"""

import numpy as np
import pytest

from ps3d_b200 import abi
from ps3d_b200 import configs as cf
from ps3d_b200.model import Model, PS3DError
from ps3d_b200.slab import SlabGroup, Slab
from tests.helpers import random_state, rel, small_params

pytestmark = pytest.mark.gpu

TOL = 1e-12
NAMES = ("u", "v", "w", "b", "p")


def _interior(a):
    return np.ascontiguousarray(a[2:-2, 2:-2, 2:-2])


def _single(p, f, nsteps, monkeypatch):
    monkeypatch.setenv("PS3D_PLANE_IMPL", "1")   # the slabs' plane implementation
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    m.run(nsteps)
    got = m.download(tendencies=False)
    m.close()
    return {n: _interior(got[n]) for n in NAMES}


@pytest.mark.parametrize("nranks", [1, 2, 4, 8])
def test_slabs_match_single_grid(nranks, monkeypatch):
    p = small_params(64, 32, 32, rigid=True)
    f = random_state(p, seed=7, amp=0.05)
    ref = _single(p, f, 6, monkeypatch)
    g = SlabGroup(p, nranks)
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(6)
    got = g.download()
    g.close()
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < TOL, err


def test_slabs_jets_config(monkeypatch):
    """The jets case (rigid lid, AB3, Laplacian friction) at 128x128x64 on
    four slabs, 20 steps.  Both sides use one pinned plane configuration: the
    autotuner could otherwise pick different radix schedules for the two
    grid shapes, whose rounding the unstable jets amplify."""
    monkeypatch.setenv("PS3D_TUNE", "im1,C1,rc8,tj16,ly16,pol0,kc8")
    p = cf.jets_params(128, 128, 64)
    f = cf.add_noise(p, cf.jets_fields(p), "b", rel=1e-3, seed=1)
    ref = _single(p, f, 20, monkeypatch)
    g = SlabGroup(p, 4)
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(20)
    got = g.download()
    g.close()
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < 1e-11, err


def test_slab_download_per_rank(monkeypatch):
    """Each rank hands back its own levels, pressure included."""
    p = small_params(32, 32, 16, rigid=True)
    f = random_state(p, seed=3)
    ref = _single(p, f, 3, monkeypatch)
    g = SlabGroup(p, 2)
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(3)
    for s in g.ranks:
        d = s.download()
        sl = slice(s.k0, s.k0 + s.nzl)
        for n in NAMES:
            assert rel(d[n], ref[n][sl]) < TOL, (s.rank, n)
    g.close()


@pytest.mark.parametrize("precision", [abi.PS3D_MIXED, abi.PS3D_MIXED_REFINED])
@pytest.mark.parametrize("nranks", [2, 4])
def test_mixed_slabs_match_single_grid(nranks, precision, monkeypatch):
    """The mixed path: FP32 transforms; the first step solves twice (a full
    solve and the FP64-residual refinement, with a p-halo exchange between
    them), every later one once (the residual against the previous step's
    p).  The single grid reads its Thomas factors from a table; the column
    slabs form the same FP64 values on the fly."""
    monkeypatch.setenv("PS3D_TUNE", "im1,C1,rc8,tj16,ly16,pol0,kc8")
    p = small_params(64, 32, 32, rigid=True, precision=precision)
    f = random_state(p, seed=11, amp=0.05)
    ref = _single(p, f, 6, monkeypatch)
    g = SlabGroup(p, nranks)
    assert g.ranks[0].passes == 2
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(6)
    # warm: the residual solve only; refined: both solves at every step
    assert all(s.step_passes() == (1 if precision == abi.PS3D_MIXED else 2) for s in g.ranks)
    got = g.download()
    g.close()
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < 1e-10, err


@pytest.mark.parametrize("precision,tol", [(abi.PS3D_FP64, TOL), (abi.PS3D_MIXED, 1e-10)])
@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_periodic_slabs_match_single_grid(nranks, precision, tol, monkeypatch):
    """Triply periodic grids: the halo planes wrap from the top rank to the
    bottom one, and the column slabs run the z transform, the spectral
    division and the inverse z transform (pressure_solver.f90:58-70) on
    whole columns of the global grid."""
    monkeypatch.setenv("PS3D_TUNE", "im1,C1,rc8,tj16,ly16,pol0,kc8")
    p = small_params(64, 32, 32, rigid=False, precision=precision)
    f = random_state(p, seed=13, amp=0.05)
    ref = _single(p, f, 6, monkeypatch)
    g = SlabGroup(p, nranks)
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(6)
    got = g.download()
    g.close()
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < tol, err


@pytest.mark.parametrize("precision,tol", [(abi.PS3D_FP64, TOL), (abi.PS3D_MIXED, 1e-10)])
@pytest.mark.parametrize("nranks", [2, 4])
def test_forced_slabs_match_single_grid(nranks, precision, tol, monkeypatch):
    """The lee-wave case (triply periodic, background flow and wavemaker,
    lee_wave1.f90:232-332) in z-slabs: each rank holds the forcing fields of
    its levels and one halo level each side (the background terms read the
    levels above and below)."""
    monkeypatch.setenv("PS3D_TUNE", "im1,C1,rc8,tj16,ly16,pol0,kc8")
    p = cf.lee_wave_params(64, 32, 32, precision=precision)
    fr = cf.lee_wave_forcing(p, seed=3, amp=1e-4)
    f = random_state(p, seed=19, amp=0.02)
    kind = abi.PS3D_FORCE_WAVEMAKER | abi.PS3D_FORCE_BACKGROUND
    monkeypatch.setenv("PS3D_PLANE_IMPL", "1")
    m = Model(p)
    m.set_forcing(kind, fr["omega"], **{n: fr[n] for n in ("w_r", "w_i", "u_back", "b_back")})
    m.upload(**{n: f[n] for n in "uvwb"})
    m.run(8)
    ref = {n: _interior(a) for n, a in m.download(tendencies=False).items() if n in NAMES}
    m.close()
    g = SlabGroup(p, nranks)
    g.set_forcing(kind, fr["omega"], **{n: _interior(fr[n]) for n in ("w_r", "w_i", "u_back", "b_back")})
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(8)
    got = g.download()
    g.close()
    assert np.abs(got["w"]).max() > 0.0
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < tol, err


def test_slab_forcing_rejects_callback_and_background_with_friction():
    p = small_params(32, 32, 16, rigid=True)   # Laplacian friction on
    s = Slab(p, 2, 0)
    z = np.zeros((16, 32, 32))
    with pytest.raises(PS3DError) as e:
        s.set_forcing(abi.PS3D_FORCE_BACKGROUND, 0.0, u_back=z)
    assert e.value.status == abi.PS3D_ERR_UNSUPPORTED
    with pytest.raises(PS3DError) as e:
        s.set_forcing(abi.PS3D_FORCE_CALLBACK)
    assert e.value.status == abi.PS3D_ERR_UNSUPPORTED
    s.set_forcing(abi.PS3D_FORCE_WAVEMAKER, 1e-3, w_r=z)   # the wavemaker alone takes the fused step
    s.close()


@pytest.mark.parametrize("rigid", [True, False])
def test_slabs_match_oracle(rigid):
    """Four slabs of one grid against the CPU oracle, 10 AB3 steps."""
    from oracle.binding import Oracle
    p = small_params(32, 32, 16, rigid=rigid)
    f = random_state(p, seed=17, amp=0.05)
    o = Oracle(p)
    for n in "uvwb":
        o.field(n)[...] = f[n]
    o.integrate(10)
    g = SlabGroup(p, 4)
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(10)
    got = g.download()
    g.close()
    err = {n: rel(got[n], _interior(o.field(n))) for n in NAMES}
    assert max(err.values()) < 1e-11, err


def test_slab_rejects_periodic_depth_without_fft():
    p = small_params(32, 32, 22, rigid=False)   # 22 = 2 x 11: no FFT plan of that length
    with pytest.raises(PS3DError) as e:
        Slab(p, 2, 0)
    assert e.value.status == abi.PS3D_ERR_BADPARAM


def test_slab_rejects_uneven_levels():
    p = small_params(32, 32, 16, rigid=True)
    with pytest.raises(PS3DError) as e:
        Slab(p, 3, 0)
    assert e.value.status == abi.PS3D_ERR_BADPARAM


@pytest.mark.parametrize("precision", [abi.PS3D_FP64, abi.PS3D_MIXED])
def test_dist_slab_nccl_single_rank(precision, monkeypatch):
    """The torch.distributed driver (NCCL, bound torch buffers, collectives on
    the slab's stream) with one rank: the transports reduce to local copies
    and an all-to-all with itself."""
    import torch
    import torch.distributed as dist
    from ps3d_b200.slab import DistSlab
    monkeypatch.setenv("PS3D_TUNE", "im1,C1,rc8,tj16,ly16,pol0,kc8")
    p = small_params(64, 32, 16, rigid=True, precision=precision)
    f = random_state(p, seed=5, amp=0.05)
    ref = _single(p, f, 4, monkeypatch)
    monkeypatch.setenv("MASTER_ADDR", "127.0.0.1")
    monkeypatch.setenv("MASTER_PORT", "29653")
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        d = DistSlab(p, 0)
        d.upload(*[_interior(f[n]) for n in "uvwb"])
        d.step(4)
        diag = d.diagnose()
        got = d.download()
        d.close()
    finally:
        dist.destroy_process_group()
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < (TOL if precision == abi.PS3D_FP64 else 1e-10), err
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    m.run(4)
    want = m.diagnose()
    m.close()
    assert np.allclose(diag, want, rtol=1e-10, atol=0.0), (diag, want)


@pytest.mark.parametrize("n0", [1e-3, 0.0])
@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_slab_diagnose_matches_single_grid(nranks, n0, monkeypatch):
    """diagnose of a grid in slabs: the ranks' partial sums and maxima over
    their levels, combined, against diagnose of the grid on one context
    (with N0 = 0 the potential energy weighs b by the global level)."""
    monkeypatch.setenv("PS3D_PLANE_IMPL", "1")
    p = small_params(64, 32, 32, rigid=True, N0=n0)
    f = random_state(p, seed=23, amp=0.05)
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    m.run(5)
    want = m.diagnose()
    m.close()
    g = SlabGroup(p, nranks)
    g.upload(*[_interior(f[n]) for n in "uvwb"])
    g.step(5)
    got = g.diagnose()
    g.close()
    assert np.allclose(got, want, rtol=1e-11, atol=0.0), (got, want)
