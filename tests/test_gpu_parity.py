"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Tolerances are the ones the engine is specified against: relative L2 over
the interior <= 1e-11 for the FP64 path and <= 1e-5 for the mixed path after
the stated number of steps; single kernels (one pressure solve, one
projection) are held to 1e-12.
"""
import numpy as np
import pytest

from oracle.binding import Oracle
from ps3d_b200 import abi
from ps3d_b200 import configs as cf
from ps3d_b200.model import Model, PS3DError
from tests.helpers import (FIELDS, compare_state, load_oracle, random_state, rel, small_params,
                           smooth_state, upload_from_oracle)

pytestmark = pytest.mark.gpu

TOL64 = 1e-11
TOL_KERNEL = 1e-12
TOL_MIXED = 1e-5


@pytest.fixture(autouse=True, params=["cluster", "rows+lines", "pipe+lines"])
def plane_impl(request, monkeypatch):
    """Every parity case runs on the three plane-transform implementations:
    the one-cluster-per-plane kernels, the rows pass + y-lines pass, and the
    latter with the forward rows pass pipelined by bulk copies."""
    monkeypatch.setenv("PS3D_PLANE_IMPL", {"cluster": "0", "rows+lines": "1", "pipe+lines": "2"}[request.param])
    return request.param



def _pair(p, fields, pfield=None):
    o = Oracle(p)
    load_oracle(o, fields, pfield)
    m = Model(p)
    upload_from_oracle(m, o)
    return o, m


@pytest.mark.parametrize("rigid", [True, False])
@pytest.mark.parametrize("shape", [(32, 32, 16), (48, 40, 12), (256, 256, 8), (128, 64, 8), (64, 128, 8), (64, 256, 4)])
def test_pressure_solver(rigid, shape, plane_impl):
    p = small_params(*shape, rigid=rigid)
    o, m = _pair(p, random_state(p, seed=1))
    assert "plane_impl=" + plane_impl in m.describe()
    o.pressure_solver()
    m.pressure_solver()
    err = compare_state(m, o)
    assert max(err.values()) < TOL_KERNEL, err


@pytest.mark.parametrize("thomas_form", ["0", "2", "2g", "3", "3g"])
@pytest.mark.parametrize("nz", [40, 64, 100, 128, 129])
def test_pressure_solver_tall_columns(nz, thomas_form, monkeypatch):
    """Rigid-lid solve on columns split into several segments: nz = 64 and
    128 fill every segment (the full-chunk instantiation), 40 and 100 leave
    the last one short, 129 leaves trailing segments empty; every form of
    the vertical solve: one-ended (0), two-ended (2), two-ended with its
    pivot table (3), the two-ended ones also in their bounds-tested
    instantiation on every grid (g)."""
    monkeypatch.setenv("PS3D_THOMAS_FORM", thomas_form[0])
    monkeypatch.setenv("PS3D_THOMAS_FULL", "0" if thomas_form.endswith("g") else "1")
    p = small_params(32, 16, nz, rigid=True, Lz=1000.0 * nz / 16)
    o, m = _pair(p, random_state(p, seed=3))
    o.pressure_solver()
    m.pressure_solver()
    err = compare_state(m, o)
    assert max(err.values()) < TOL_KERNEL, err


@pytest.mark.parametrize("precision", [abi.PS3D_FP64, abi.PS3D_MIXED])
def test_vertical_solve_forms_bit_identical(precision, monkeypatch):
    """The two-ended vertical solve's instantiations (bounds-tested or full
    chunks; pivots formed in both sweeps or parked in a table by the
    forward sweep) run the same FP64 operations in the same order, so they
    give the same bits, on FP64 and on FP32 spectra."""
    p = small_params(64, 32, 128, rigid=True, Lz=8000.0)
    p.precision = precision
    f = random_state(p, seed=5)
    out = {}
    for form, full in (("2", "0"), ("2", "1"), ("3", "0"), ("3", "1")):
        monkeypatch.setenv("PS3D_THOMAS_FORM", form)
        monkeypatch.setenv("PS3D_THOMAS_FULL", full)
        m = Model(p)
        m.upload(**f)
        m.pressure_solver()
        out[form + full] = m.download(tendencies=False)
        m.close()
    for k, v in out.items():
        for n in ("u", "v", "w", "p"):
            assert np.array_equal(v[n], out["20"][n]), (k, n)


def test_pressure_solver_divergence_free():
    p = small_params(64, 32, 16, rigid=True)
    _, m = _pair(p, random_state(p, seed=2))
    m.pressure_solver()
    s = m.download(tendencies=False)
    u, v, w = s["u"], s["v"], s["w"]
    div = ((u[2:-2, 2:-2, 2:-2] - u[2:-2, 2:-2, 1:-3]) / p.dx + (v[2:-2, 2:-2, 2:-2] - v[2:-2, 1:-3, 2:-2]) / p.dy
           + (w[2:-2, 2:-2, 2:-2] - w[1:-3, 2:-2, 2:-2]) / p.dz)
    scale = np.abs(u).max() / p.dx
    assert np.abs(div).max() < 1e-12 * scale


@pytest.mark.parametrize("rigid", [True, False])
def test_one_step(rigid):
    p = small_params(32, 32, 16, rigid=rigid)
    o, m = _pair(p, smooth_state(p))
    o.integrate(1)
    m.run(1)
    err = compare_state(m, o)
    assert max(err.values()) < TOL_KERNEL, err
    got = m.download()
    itt, tau, *_ = o.get_time()
    # tendency stored in the slot of the step that was just taken
    slot = (tau - 2) % 3
    for n in ("du", "dv", "dw", "db"):
        e = rel(got[n][slot], o.field(n, slot + 1))
        assert e < TOL_KERNEL, (n, e)


def test_eddy_200_steps_fp64():
    """The 64x64x32 eddy case, AB3, 200 steps."""
    p = cf.eddy_params(64, 64, 32)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=0)
    o, m = _pair(p, f)
    o.integrate(200)
    m.run(200)
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err
    assert m.download(tendencies=False)["itt"] == 200


def test_periodic_ab2_eps_nonlinear():
    p = small_params(32, 32, 16, rigid=False, enable_AB_3_order=0, eps_ab=0.01, Kh=1e-2, Kv=1e-3)
    o, m = _pair(p, smooth_state(p, seed=3))
    o.integrate(20)
    m.run(20)
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err


def test_linear_model():
    p = small_params(32, 32, 16, rigid=True, enable_nonlinear=0)
    o, m = _pair(p, smooth_state(p, seed=4))
    o.integrate(20)
    m.run(20)
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err


@pytest.mark.parametrize("rigid", [True, False])
def test_biharmonic_stale_halos(rigid):
    """harmonic + biharmonic_h + biharmonic_v in sequence without halo
    exchange (integrate.f90:59-78): the generic friction path."""
    p = small_params(32, 32, 16, rigid=rigid, Kh=1e-2, Kv=1e-3, Ahbi=1e7, Avbi=1e1, Khbi=1e7, Kvbi=1e1)
    o, m = _pair(p, random_state(p, seed=5, amp=0.05))
    o.integrate(5)
    m.run(5)
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err


def test_forcing_background_and_wavemaker():
    p = small_params(32, 32, 16, rigid=False)
    p.Ah = p.Av = 0.0
    fr = cf.lee_wave_forcing(p, amp=1e-6, seed=2)
    fr["u_back"] += 0.02 * cf.halo_fill(np.sin(np.arange(np.prod(cf.empty_field(p).shape))).reshape(cf.empty_field(p).shape))
    cf.halo_fill(fr["u_back"])
    fr["b_back"] = cf.halo_fill(1e-4 * np.cos(np.arange(np.prod(cf.empty_field(p).shape))).reshape(cf.empty_field(p).shape))
    o, m = _pair(p, smooth_state(p, seed=6))
    from ps3d_b200.abi import Forcing, dptr
    kind = abi.PS3D_FORCE_BACKGROUND | abi.PS3D_FORCE_WAVEMAKER
    f = Forcing()
    f.kind = kind
    f.omega = fr["omega"]
    f.w_r, f.w_i, f.u_back, f.b_back = dptr(fr["w_r"]), dptr(fr["w_i"]), dptr(fr["u_back"]), dptr(fr["b_back"])
    o.set_forcing(f, keep=fr)
    m.set_forcing(kind, omega=fr["omega"], w_r=fr["w_r"], w_i=fr["w_i"], u_back=fr["u_back"], b_back=fr["b_back"])
    o.integrate(10)
    m.run(10)
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err


def test_forcing_with_friction_generic_path():
    p = small_params(32, 32, 16, rigid=True)
    fr = cf.lee_wave_forcing(p, amp=1e-6, seed=9)
    o, m = _pair(p, smooth_state(p, seed=8))
    from ps3d_b200.abi import Forcing, dptr
    kind = abi.PS3D_FORCE_BACKGROUND | abi.PS3D_FORCE_WAVEMAKER
    f = Forcing()
    f.kind = kind
    f.omega = fr["omega"]
    f.w_r, f.w_i, f.u_back = dptr(fr["w_r"]), dptr(fr["w_i"]), dptr(fr["u_back"])
    o.set_forcing(f, keep=fr)
    m.set_forcing(kind, omega=fr["omega"], w_r=fr["w_r"], w_i=fr["w_i"], u_back=fr["u_back"])
    o.integrate(8)
    m.run(8)
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err


def test_step_with_caller_time_levels():
    """ps3d_step is integrate.f90 as called from main.f90: the host rotates."""
    p = small_params(32, 32, 16)
    f = smooth_state(p, seed=10)
    o, m = _pair(p, f)
    itt, tau, t1, t2 = 0, 3, 2, 1
    for _ in range(4):
        o.set_time(itt, tau, t1, t2)
        o.step()
        m.integrate(itt, tau, t1, t2)
        tau, t1, t2 = tau % 3 + 1, t1 % 3 + 1, t2 % 3 + 1
        itt += 1
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err


@pytest.mark.parametrize("rigid", [True, False])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_projection(rigid, mode):
    p = small_params(32, 32, 16, rigid=rigid)
    o, m = _pair(p, smooth_state(p, seed=11))
    if mode == abi.PS3D_PROJ_EXCHANGE:   # needs a stored base point
        o.project(abi.PS3D_PROJ_BASE_POINT)
        m.project(abi.PS3D_PROJ_BASE_POINT)
        rs = random_state(p, seed=12, amp=0.02)
        load_oracle(o, rs)
        m.upload(**{n: rs[n] for n in FIELDS})
    o.project(mode)
    m.project(mode)
    if mode in (abi.PS3D_PROJ_NORMAL_MODE, abi.PS3D_PROJ_EXCHANGE):
        err = compare_state(m, o, names=FIELDS)
    else:
        which = abi.PS3D_FIELDS_BASE if mode == abi.PS3D_PROJ_BASE_POINT else abi.PS3D_FIELDS_ZERO
        got = m.get_fields(which)
        suffix = "_base" if mode == abi.PS3D_PROJ_BASE_POINT else "0"
        err = {n: rel(got[n], o.field(n + suffix)) for n in FIELDS if np.abs(o.field(n + suffix)).max() > 0}
    assert max(err.values()) < TOL_KERNEL, err


@pytest.mark.parametrize("form", ["fft", "fft2n", "dense"])
@pytest.mark.parametrize("nz", [33, 60, 64, 128])
def test_normal_mode_projection_tall_rigid(nz, form, monkeypatch):
    """Rigid-lid projection through the vertical-mode transforms at nz = 128,
    64 and 60, by FFT (PS3D_VMODE_FORM=2, the default where 2 nz factors:
    the mode matrices are sampled sines and cosines; phi and psib by FFTs of
    length nz, psi by one of length 2 nz; =3 every field by length 2 nz) or
    as the dense FP64 product (PS3D_VMODE_FORM=1), and an odd 33 (2 nz = 66
    has a factor 11: the dense product, its unpaired-load path, in every
    case)."""
    monkeypatch.setenv("PS3D_VMODE_FORM", {"dense": "1" if nz % 2 == 0 else "0", "fft": "2", "fft2n": "3"}[form])
    p = small_params(32, 16, nz, rigid=True, Lz=1000.0 * nz / 16)
    o, m = _pair(p, smooth_state(p, seed=15))
    assert ("vmode=fft" in m.describe()) == (form != "dense" and nz != 33), m.describe()
    o.project(abi.PS3D_PROJ_NORMAL_MODE)
    m.project(abi.PS3D_PROJ_NORMAL_MODE)
    err = compare_state(m, o, names=FIELDS)
    assert max(err.values()) < TOL_KERNEL, err


def test_opt_balance_tall_rigid():
    """Optimal balance on a rigid-lid grid of 96 levels, whose vertical-mode
    transforms run by FFT, against the oracle's dense products."""
    p = small_params(32, 16, 96, rigid=True, dt=600.0, Lz=6000.0)
    f = smooth_state(p, seed=21)
    o, m = _pair(p, f)
    opt = abi.OptBal(period=5.5 * p.dt, average=3.5 * p.dt, max_itts=2, average_times=2, tol=0.0,
                     enable_time_ave=0, adopt=0)
    n_o, it_o = o.opt_balance(opt)
    n_m, it_m = m.diag_opt_balance(opt)
    assert it_o == it_m == 2
    assert abs(n_m - n_o) <= 1e-9 * abs(n_o) + 1e-300
    got = m.get_fields(abi.PS3D_FIELDS_BALANCED)
    err = {n: rel(got[n], o.field(n + "_bal")) for n in FIELDS if np.abs(o.field(n + "_bal")).max() > 0}
    assert max(err.values()) < TOL64, err


@pytest.mark.parametrize("time_ave", [False, True])
def test_opt_balance(time_ave):
    p = small_params(32, 32, 8, rigid=True, dt=600.0)
    f = smooth_state(p, seed=13)
    o, m = _pair(p, f)
    opt = abi.OptBal(period=5.5 * p.dt, average=3.5 * p.dt, max_itts=3, average_times=2, tol=0.0,
                     enable_time_ave=int(time_ave), adopt=0)
    n_o, it_o = o.opt_balance(opt)
    n_m, it_m = m.diag_opt_balance(opt)
    assert it_o == it_m == 3
    assert abs(n_m - n_o) <= 1e-9 * abs(n_o) + 1e-300
    got = m.get_fields(abi.PS3D_FIELDS_BALANCED)
    err = {n: rel(got[n], o.field(n + "_bal")) for n in FIELDS if np.abs(o.field(n + "_bal")).max() > 0}
    assert max(err.values()) < TOL64, err
    # the model state is restored
    err = compare_state(m, o)
    assert max(err.values()) < TOL_KERNEL, err


def test_diagnose_and_nonfinite():
    p = small_params(32, 32, 16)
    f = smooth_state(p, seed=14)
    o, m = _pair(p, f)
    st, ke, pe, um, wm = o.diagnose()
    ke2, pe2, um2, wm2 = m.diagnose()
    assert st == 0
    assert abs(ke2 - ke) <= 1e-13 * ke and abs(pe2 - pe) <= 1e-13 * pe
    assert um2 == um and wm2 == wm
    bad = f["b"].copy()
    bad[5, 5, 5] = np.nan
    m.upload(b=bad)
    with pytest.raises(PS3DError) as ei:
        m.diagnose()
    assert ei.value.status == abi.PS3D_ERR_NONFINITE


@pytest.mark.parametrize("precision", [abi.PS3D_FP64, abi.PS3D_MIXED])
def test_long_lines_steps(precision):
    """FFT lengths 128 (radix 16 x 8) and 256 (16 x 16) in a short run."""
    p = small_params(256, 256, 16, rigid=True, Lx=256e3, Ly=256e3)
    p.precision = precision
    p64 = p.copy()
    p64.precision = abi.PS3D_FP64
    o = Oracle(p64)
    load_oracle(o, smooth_state(p64, seed=21))
    m = Model(p)
    upload_from_oracle(m, o)
    o.integrate(6)
    m.run(6)
    err = compare_state(m, o)
    assert max(err.values()) < (TOL64 if precision == abi.PS3D_FP64 else TOL_MIXED), err


def test_lazy_correction_observers():
    """The pressure-gradient correction is applied by the next step's stencil
    kernel; every observer (download, diagnose, projection, a later explicit
    pressure solve) must see the corrected state."""
    p = small_params(32, 32, 16)
    o, m = _pair(p, smooth_state(p, seed=22))
    o.integrate(5)
    m.run(5)
    st, ke, pe, um, wm = o.diagnose()
    ke2, pe2, um2, wm2 = m.diagnose()
    assert abs(ke2 - ke) <= 1e-12 * ke and abs(um2 - um) <= 1e-12 * um
    err = compare_state(m, o)
    assert max(err.values()) < TOL64, err
    o.integrate(3)
    m.run(3)
    o.project(abi.PS3D_PROJ_NORMAL_MODE)
    m.project(abi.PS3D_PROJ_NORMAL_MODE)
    err = compare_state(m, o, names=FIELDS)
    assert max(err.values()) < TOL64, err


def test_mixed_precision_200_steps():
    p = cf.eddy_params(64, 64, 32, precision=abi.PS3D_MIXED)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=0)
    p64 = p.copy()
    p64.precision = abi.PS3D_FP64
    o = Oracle(p64)
    load_oracle(o, f)
    m = Model(p)
    upload_from_oracle(m, o)
    o.integrate(200)
    m.run(200)
    err = compare_state(m, o)
    assert max(err.values()) < TOL_MIXED, err


@pytest.mark.parametrize("ysplit", ["1", "0"])
@pytest.mark.parametrize("shape", [(128, 64, 32), (128, 128, 48), (256, 32, 17)])
def test_mixed_ysplit_solve(shape, ysplit, plane_impl, monkeypatch):
    """The mixed rigid-lid solve with the y transforms split at the rows
    passes and run inside k_colsolve together with the vertical solve (odd
    nz included), against the oracle after 20 steps, and the same solve on
    the y-lines passes and k_thomas2.  The split applies to the rows + y-lines
    implementation only."""
    if ysplit == "1" and plane_impl != "rows+lines":
        pytest.skip("the y-split solve runs on the rows + y-lines implementation")
    monkeypatch.setenv("PS3D_YSPLIT", ysplit)
    p = cf.eddy_params(*shape, precision=abi.PS3D_MIXED)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=2)
    p64 = p.copy()
    p64.precision = abi.PS3D_FP64
    o = Oracle(p64)
    load_oracle(o, f)
    m = Model(p)
    assert ("rows+colsolve" in m.describe()) == (ysplit == "1"), m.describe()
    upload_from_oracle(m, o)
    o.integrate(20)
    m.run(20)
    err = compare_state(m, o)
    assert max(err.values()) < TOL_MIXED, err
    # an explicit (cold) solve of the stepped state: the velocity is already
    # divergence free to round-off, so the new p is round-off too and only
    # the velocity and buoyancy are compared
    o.pressure_solver()
    m.pressure_solver()
    err = compare_state(m, o, names=FIELDS)
    assert max(err.values()) < TOL_MIXED, err


@pytest.mark.parametrize("shape", [(128, 64, 32), (128, 32, 17), (128, 64, 2), (128, 32, 3)])
def test_colsolve_two_cta_form_matches_one_cta(shape, monkeypatch):
    """k_colsolve2 splits each half-line's levels over a cluster of two CTAs
    (each eliminates one end, the ends meet through distributed shared
    memory); it runs the same operations as the one-CTA k_colsolve, so the
    steps and an explicit solve agree bit for bit (odd nz and nz = 2, 3
    included)."""
    monkeypatch.setenv("PS3D_YSPLIT", "1")
    monkeypatch.setenv("PS3D_PLANE_IMPL", "1")
    monkeypatch.setenv("PS3D_AUTOTUNE", "0")
    p = cf.eddy_params(*shape, precision=abi.PS3D_MIXED)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=5)
    out = {}
    for form in ("1", "2"):
        monkeypatch.setenv("PS3D_COLSOLVE", form)
        m = Model(p)
        assert "rows+colsolve" in m.describe(), m.describe()
        m.upload(**{n: f[n] for n in ("u", "v", "w", "b")})
        m.run(7)
        st = m.download(tendencies=False)
        m.pressure_solver()
        out[form] = (st, m.download(tendencies=False))
        m.close()
    for a, b in zip(out["1"], out["2"]):
        for n in ("u", "v", "w", "b", "p"):
            assert np.array_equal(a[n], b[n]), (shape, n, rel(a[n], b[n]))


def test_bad_params_rejected():
    p = small_params(33, 32, 16)
    with pytest.raises(PS3DError) as ei:
        Model(p)
    assert ei.value.status == abi.PS3D_ERR_BADPARAM
    p = small_params(28, 32, 16)   # nx/2 = 14 = 2*7 has a factor 7
    with pytest.raises(PS3DError):
        Model(p)
