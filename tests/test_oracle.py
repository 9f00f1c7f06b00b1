"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests or golden vectors and cannot be built here, so
the oracle is pinned against the reference's own mathematics:
  * its FFT against numpy.fft (pocketfft), with the ps3D scalings
    (my_fft.f90:159-205);
  * eigenvector bi-orthogonality p^s . q^s' = delta (eigenvectors.f90);
  * idempotence of the geostrophic projection (diag_opt_balance.f90:288-310);
  * the Thomas solver's residual and its agreement with a DCT-II solve of the
    same Neumann operator (pressure_solver.f90:33-53);
  * zero divergence after the pressure projection;
  * energy neutrality of the inviscid tendency (advection.f90 is the
    energy-conserving form; Coriolis and buoyancy exchange are neutral);
  * the discrete dispersion relation: a single normal mode of the linear
    model rotates at omega (eigenvectors.f90:6-24/110-123).
"""
import numpy as np
import pytest
import scipy.fft as sfft

from oracle import binding as ob
from oracle.binding import Oracle
from ps3d_b200 import abi
from ps3d_b200 import configs as cf
from tests.helpers import FIELDS, load_oracle, random_state, small_params, smooth_state


@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 8, 10, 12, 15, 16, 24, 30, 40, 48, 60, 64, 100, 120, 128, 256, 512, 7, 14])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    assert np.abs(ob.fft(x, -1) - ref).max() <= 1e-14 * np.abs(ref).max()
    assert np.abs(ob.fft(x, +1) - np.fft.ifft(x) * n).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("three_d", [False, True])
@pytest.mark.parametrize("shape", [(16, 8, 4), (24, 20, 6)])
def test_field_fft_scaling_and_round_trip(three_d, shape):
    nx, ny, nz = shape
    p = small_params(nx, ny, nz, rigid=not three_d)
    o = Oracle(p)
    rng = np.random.default_rng(0)
    q = rng.standard_normal((nz, ny, nx))
    spec = o.fft_field(q, three_d)
    if three_d:
        ref = np.fft.rfftn(q, axes=(0, 1, 2)) * p.dx * p.dy * p.dz
    else:
        ref = np.fft.rfft2(q, axes=(1, 2)) * p.dx * p.dy
    assert np.abs(spec - ref).max() <= 1e-13 * np.abs(ref).max()
    back = o.ifft_field(spec, three_d)
    assert np.abs(back - q).max() <= 1e-13 * np.abs(q).max()


@pytest.mark.parametrize("rigid", [True, False])
def test_eigenvectors_biorthogonal(rigid):
    p = small_params(32, 32, 16, rigid=rigid)
    o = Oracle(p)
    kx, ky, kz = o.wavenumbers(0), o.wavenumbers(1), o.wavenumbers(2)
    rng = np.random.default_rng(1)
    for _ in range(40):
        i, j, k = rng.integers(0, len(kx)), rng.integers(0, len(ky)), rng.integers(0, len(kz))
        if (i == 0 and j == 0) or i == p.nx // 2 or j == p.ny // 2 or (not rigid and k == p.nz // 2):
            continue   # mean flow and Nyquist columns: hat_epm = 0 there and the modes degenerate
        Q, P = {}, {}
        for s in (0.0, 1.0, -1.0):
            Q[s], P[s], _ = o.eigen(kx[i], ky[j], kz[k], s)
        if rigid and kz[k] == 0.0:
            # barotropic column: only the geostrophic mode exists; the wave
            # vectors of the reference vanish (p^+- = 0)
            assert abs(np.sum(P[0.0] * Q[0.0]) - 1) < 1e-12
            assert np.abs(P[1.0]).max() == 0 and np.abs(P[-1.0]).max() == 0
            continue
        for s in Q:
            for t in Q:
                d = np.sum(P[s] * Q[t])
                assert abs(d - (1.0 if s == t else 0.0)) < 1e-11, (i, j, k, s, t, d)


def test_dispersion_relation_omega():
    """omega2_discrete against the continuous limit for a long wave."""
    p = small_params(64, 64, 64, rigid=False, Lx=1e6, Ly=1e6, Lz=1e3)
    o = Oracle(p)
    kx, ky, kz = 2 * np.pi / p.Lx, 0.0, 2 * np.pi / p.Lz
    _, _, om2 = o.eigen(kx, ky, kz, 1.0)
    hk = lambda k, d: 2 * (1 - np.cos(k * d)) / d ** 2
    he = lambda k, d: 0.5 * (1 + np.cos(k * d))
    k2 = hk(kx, p.dx) + hk(ky, p.dy)
    disc = (he(kz, p.dz) * p.N0 ** 2 * k2 + p.f0 ** 2 * hk(kz, p.dz) * he(kx, p.dx) * he(ky, p.dy)) / (p.dsqr * k2 + hk(kz, p.dz))
    assert abs(om2 - disc) / disc < 1e-13
    cont = (p.N0 ** 2 * kx ** 2 + p.f0 ** 2 * kz ** 2) / (kx ** 2 + kz ** 2)
    assert abs(om2 - cont) / cont < 1e-2


@pytest.mark.parametrize("rigid", [True, False])
def test_projection_idempotent(rigid):
    p = small_params(32, 32, 16, rigid=rigid)
    o = Oracle(p)
    load_oracle(o, smooth_state(p, seed=2))
    o.project(abi.PS3D_PROJ_NORMAL_MODE)
    once = {n: o.field(n).copy() for n in FIELDS}
    o.project(abi.PS3D_PROJ_NORMAL_MODE)
    for n in FIELDS:
        scale = np.abs(once[n]).max()
        if scale > 0:
            assert np.abs(o.field(n) - once[n]).max() <= 1e-12 * scale, n


def test_thomas_residual_and_dct():
    nz, dz, dsqr = 64, 7.8125, 1.0
    fxa = 1.0 / dz ** 2 / dsqr
    rng = np.random.default_rng(3)
    for ks in (1e-9, 1e-6, 1e-3, 1.0):
        a = np.full(nz, fxa)
        c = np.full(nz, fxa)
        b = np.full(nz, -ks - 2 * fxa)
        b[0] = b[-1] = -ks - fxa
        d = rng.standard_normal(nz) + 1j * rng.standard_normal(nz)
        x = ob.tridiag(a, b, c, d)
        r = b * x
        r[1:] += a[1:] * x[:-1]
        r[:-1] += c[:-1] * x[1:]
        assert np.abs(r - d).max() <= 1e-12 * np.abs(d).max() * max(1.0, fxa / ks) ** 0.5
        # Neumann operator diagonalised by DCT-II
        lam = -ks - 4 * fxa * np.sin(np.pi * np.arange(nz) / (2 * nz)) ** 2
        xd = sfft.idct(sfft.dct(d.real, type=2, norm="ortho") / lam, type=2, norm="ortho") + \
            1j * sfft.idct(sfft.dct(d.imag, type=2, norm="ortho") / lam, type=2, norm="ortho")
        assert np.abs(x - xd).max() <= 1e-9 * np.abs(xd).max()


@pytest.mark.parametrize("rigid", [True, False])
def test_pressure_projection_divergence_free(rigid):
    p = small_params(32, 24, 16, rigid=rigid)
    o = Oracle(p)
    load_oracle(o, random_state(p, seed=4))
    o.pressure_solver()
    u, v, w = o.field("u"), o.field("v"), o.field("w")
    div = ((u[2:-2, 2:-2, 2:-2] - u[2:-2, 2:-2, 1:-3]) / p.dx + (v[2:-2, 2:-2, 2:-2] - v[2:-2, 1:-3, 2:-2]) / p.dy
           + (w[2:-2, 2:-2, 2:-2] - w[1:-3, 2:-2, 2:-2]) / p.dz)
    assert np.abs(div).max() <= 1e-12 * np.abs(u).max() / p.dx


def test_inviscid_tendency_is_energy_neutral():
    p = small_params(32, 32, 16, rigid=False, Ah=0.0, Av=0.0)
    o = Oracle(p)
    load_oracle(o, random_state(p, seed=5, amp=0.1, wamp=0.01, bamp=1e-3))
    o.pressure_solver()                       # divergence-free velocity
    st = {n: o.field(n).copy() for n in FIELDS}
    o.set_time(0, 3, 2, 1)
    o.step()                                  # Euler step; tendency in slot 3
    t = {n: o.field("d" + n, 3) for n in FIELDS}
    I = (slice(2, -2),) * 3
    terms = (st["u"][I] * t["u"][I] + st["v"][I] * t["v"][I] + st["w"][I] * t["w"][I]
             + st["b"][I] * t["b"][I] / p.N0 ** 2)
    assert abs(terms.sum()) <= 1e-12 * np.abs(terms).sum()


@pytest.mark.parametrize("rigid", [True, False])
def test_single_mode_rotates_at_omega(rigid):
    """Linear, inviscid model started on q^+ of one wavenumber: the mode
    amplitude p^+ . Z(t) turns by omega*t (AB3 phase error O(dt^4))."""
    p = small_params(16, 16, 8, rigid=rigid, Ah=0.0, Av=0.0, enable_nonlinear=0, dt=20.0)
    o = Oracle(p)
    kx, ky, kz = o.wavenumbers(0), o.wavenumbers(1), o.wavenumbers(2)
    i, j, k = 1, 1, 1
    q, pv, om2 = o.eigen(kx[i], ky[j], kz[k], 1.0)
    # build the real field whose spectral coefficients are q at (i,j,k)
    spec = [np.zeros((p.nz, p.ny, p.nx // 2 + 1), complex) for _ in range(4)]
    for c in range(4):
        spec[c][k, j, i] = q[c]
    if rigid:
        fields = _backward_rigid(o, p, spec)
    else:
        fields = [o.ifft_field(s, True) for s in spec]
    for c, n in enumerate(FIELDS):
        h = cf.empty_field(p)
        cf.interior(h)[...] = fields[c]
        o.field(n)[...] = cf.halo_fill(h)
    om = np.sqrt(om2)
    nsteps = 60
    o.integrate(nsteps)
    o.forward_transform()
    Z = [o.spectral(w)[k, j, i] for w in (1, 2, 3, 4)]
    _, p0, _ = o.eigen(kx[i], ky[j], kz[k], 0.0)
    amp = np.sum(pv * np.array(Z))
    geo = np.sum(p0 * np.array(Z))
    assert abs(abs(amp) - 1.0) < 1e-3
    assert abs(geo) < 1e-6
    phase = np.angle(amp)
    expect = om * p.dt * nsteps
    d = (abs(phase) - (expect % (2 * np.pi))) % (2 * np.pi)
    assert min(d, 2 * np.pi - d) < 1e-3


def _backward_rigid(o, p, spec):
    """my_ifft_vert_mode on numpy arrays with the oracle's mode matrices."""
    out = []
    mats = [o.modes(0), o.modes(0), o.modes(1), o.modes(2)]   # [k, mode]
    for c in range(4):
        q = np.einsum("km,mji->kji", mats[c], spec[c])
        out.append(o.ifft_field(q, False))
    return out


def test_ramp_function():
    assert ob.ramp(0.0) == 0.0
    assert abs(ob.ramp(1.0) - 1.0) < 1e-300 + 1e-15
    assert abs(ob.ramp(0.5) - 0.5) < 1e-15
    xs = np.linspace(0.01, 0.99, 50)
    r = [ob.ramp(x) for x in xs]
    assert all(np.diff(r) > 0)


@pytest.mark.parametrize("rigid", [True, False])
def test_warn_balance_orders_scale_with_rossby_number(rigid):
    """u_n of the Warn-et-al. balance is O(Ro^n) with u0 fixed: doubling Ro
    doubles u1 and quadruples u2 (diag_balance.f90:168-171, 262-265), and the
    components shrink order by order for a weakly nonlinear eddy."""
    from ps3d_b200 import configs as cf
    res = {}
    for ro in (1.0, 2.0):
        p = cf.eddy_params(32, 32, 16, rigid=rigid)
        p.Ro = ro
        f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=0)
        o = Oracle(p)
        for n in "uvwb":
            o.field(n)[...] = f[n]
        o.diag_balance(2)
        res[ro] = {k: o.field(k).copy() for k in ("u0", "u1", "u2", "b1", "b2")}
    assert np.array_equal(res[1.0]["u0"], res[2.0]["u0"])
    for k, s in (("u1", 2.0), ("b1", 2.0), ("u2", 4.0), ("b2", 4.0)):
        a, b = res[1.0][k], res[2.0][k]
        assert np.linalg.norm(b - s * a) <= 1e-12 * np.linalg.norm(b), k
    n0, n1, n2 = (np.abs(res[1.0][k]).max() for k in ("u0", "u1", "u2"))
    assert n0 > n1 > n2 > 0
