"""Experiment recipes: parameters and initial conditions.

In the reference an experiment is a Fortran file providing set_parameter,
set_initial_conditions and set_forcing (for_config/*.f90, copied over
for_src/config.f90).  These are their Python counterparts for the workloads
this package is measured on.  Fields are returned halo-padded in the
reference's layout (numpy shape (nz+4, ny+4, nx+4), x fastest) with the halos
filled periodically (parallel_mpi.f90:70-211 on one rank).

Random perturbations use splitmix64 -> uniform [-1, 1) so that any host
(Python, C, Fortran) can regenerate them bit for bit.
"""
import math

import numpy as np

from .abi import make_params, PS3D_FP64

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64_uniform(seed, n):
    """n uniform doubles in [-1, 1) from splitmix64 (Steele et al. 2014)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53) * 2.0 - 1.0


def halo_fill(a):
    """Periodic fill of the two halo layers on every side, in place.

    Same result as border_exchg_3D on one rank (parallel_mpi.f90:70-81:
    z, then y, then x planes copied from the opposite interior edge)."""
    for ax in range(3):
        n = a.shape[ax] - 4
        sl = [slice(None)] * 3
        for h in (1, 2):
            sl[ax] = n + 1 + h; src = list(sl); src[ax] = 1 + h
            a[tuple(sl)] = a[tuple(src)]
            sl[ax] = 2 - h; src[ax] = n + 2 - h
            a[tuple(sl)] = a[tuple(src)]
    return a


def empty_field(p):
    return np.zeros((p.nz + 4, p.ny + 4, p.nx + 4))


def interior(a):
    return a[2:-2, 2:-2, 2:-2]


def zero_rigid_lid_w(p, w):
    """main.f90:119-122: w = 0 on the bottom halo levels and at/above level nz."""
    if p.enable_vertical_boundaries:
        w[0:2] = 0.0           # k = -1, 0
        w[p.nz + 1:] = 0.0     # k = nz, nz+1, nz+2
    return w


# --------------------------------------------------------------------------
# parameter sets
# --------------------------------------------------------------------------
def eddy_params(nx=64, ny=64, nz=32, precision=PS3D_FP64, rigid=True, dt=None):
    """Gaussian baroclinic eddy (template: for_config/eddy1.f90:10-43).

    N0 = 1e-3, f0 = 1e-4, Lz = 1000 m, Lx = Ly = 20 Rossby radii, Laplacian
    viscosity 1e-2 m^2/s, AB3.  dt = 0.3 * min(dx/0.1 m/s, 1/N0) (CFL 0.3)."""
    N0, f0, Lz = 1e-3, 1e-4, 1000.0
    c = N0 * Lz / math.pi
    L = 20.0 * c / f0
    p = make_params(nx=nx, ny=ny, nz=nz, Lx=L, Ly=L, Lz=Lz, f0=f0, N0=N0,
                    Ah=1e-2, Av=1e-2, enable_vertical_boundaries=int(rigid),
                    enable_AB_3_order=1, precision=precision)
    p.dt = dt if dt is not None else 0.3 * min(p.dx / 0.1, 1.0 / N0)
    return p


def jets_params(nx=256, ny=256, nz=128, precision=PS3D_FP64):
    """Two opposing zonal jets (template: for_config/jets_unscaled.f90:3-31).

    Lx = Ly = 500 km, N0 = 2e-3, f0 = 1e-4, dt = 0.5/N0, AB3, Laplacian
    viscosity 1e-2 m^2/s, rigid lid.  The depth is Lz = 4000 m rather than the
    template's 1000 m: with 0.5 m/s jets of width Ly/16 the thermal-wind
    buoyancy gives b_z ~ f U W pi^2 / Lz^2, which at Lz = 1000 m exceeds N0^2
    by a factor of ~6 (statically unstable; the explicit scheme overturns and
    blows up within ~100 steps, in the CPU restatement as on the GPU).  At
    Lz = 4000 m the minimum of N0^2 + b_z stays at ~0.6 N0^2."""
    N0, f0 = 2e-3, 1e-4
    return make_params(nx=nx, ny=ny, nz=nz, Lx=500e3, Ly=500e3, Lz=4000.0, f0=f0, N0=N0,
                       dt=0.5 / N0, Ah=1e-2, Av=1e-2, enable_vertical_boundaries=1,
                       enable_AB_3_order=1, precision=precision)


def lee_wave_params(nx=512, ny=256, nz=128, precision=PS3D_FP64):
    """Forced lee-wave-like case, triply periodic (template: for_config/lee_wave1.f90).

    dx = dy = 100 m, dz = 10 m, N0 = 1e-3, f0 = 1e-4, U = 0.1 m/s, dt = 100 s, AB3."""
    return make_params(nx=nx, ny=ny, nz=nz, Lx=100.0 * nx, Ly=100.0 * ny, Lz=10.0 * nz,
                       f0=1e-4, N0=1e-3, dt=100.0, enable_vertical_boundaries=0,
                       enable_AB_3_order=1, precision=precision)


# --------------------------------------------------------------------------
# initial conditions
# --------------------------------------------------------------------------
def _centres(p):
    i = np.arange(1, p.nx + 1)
    j = np.arange(1, p.ny + 1)
    k = np.arange(1, p.nz + 1)
    return i, j, k


def eddy_fields(p, amp=0.1, radius_frac=1.0 / 8.0):
    """Unbalanced analytic eddy: psi = exp(-r^2/R^2) cos(pi z/Lz) sampled on
    the C-grid (u at east faces, v at north faces, b at centres), with
    u = -psi_y, v = psi_x, b = f0 psi_z (thermal wind), w = 0, scaled so that
    max|u| = amp.  Balance it with the zero-order normal-mode projection
    (diag_balance.f90:109-132) as for_config/eddy1.f90:304-316 does."""
    i, j, k = _centres(p)
    R = radius_frac * p.Lx
    z = (k - 0.5) * p.dz
    cz = np.cos(np.pi * z / p.Lz)[:, None, None]
    sz = np.sin(np.pi * z / p.Lz)[:, None, None]

    def g(x, y):
        X, Y = np.meshgrid(x - 0.5 * p.Lx, y - 0.5 * p.Ly)   # (ny, nx)
        return X, Y, np.exp(-(X ** 2 + Y ** 2) / R ** 2)[None]

    X, Y, e = g(i * p.dx, (j - 0.5) * p.dy)
    u = -(-2.0 * Y[None] / R ** 2) * e * cz
    X, Y, e = g((i - 0.5) * p.dx, j * p.dy)
    v = (-2.0 * X[None] / R ** 2) * e * cz
    X, Y, e = g((i - 0.5) * p.dx, (j - 0.5) * p.dy)
    b = p.f0 * (-np.pi / p.Lz) * e * sz
    s = amp / np.abs(u).max()
    out = {}
    for name, a in (("u", u * s), ("v", v * s), ("w", np.zeros_like(u)), ("b", b * s)):
        h = empty_field(p)
        interior(h)[...] = a
        out[name] = halo_fill(h)
    zero_rigid_lid_w(p, out["w"])
    return out


def add_noise(p, fields, name="b", rel=1e-3, seed=0):
    """Add seeded white noise of amplitude rel*max|field| to the interior."""
    a = fields[name]
    amp = rel * np.abs(interior(a)).max()
    noise = splitmix64_uniform(seed, p.nx * p.ny * p.nz).reshape(p.nz, p.ny, p.nx)
    interior(a)[...] += amp * noise
    halo_fill(a)
    return fields


def jets_fields(p, amp=0.5, width_frac=1.0 / 16.0):
    """Two opposing Gaussian zonal jets at y = Ly/4 and 3Ly/4 with vertical
    structure cos(pi z/Lz) and b in thermal-wind balance built by a y prefix
    sum (for_config/jets_unscaled.f90:52-95, rigid-lid branch)."""
    i, j, k = _centres(p)
    y = (j - 1) * p.dy
    z = (k - 1) * p.dz
    W = width_frac * p.Ly
    prof = np.exp(-(y - 3 * p.Ly / 4.0) ** 2 / W ** 2) - np.exp(-(y - p.Ly / 4.0) ** 2 / W ** 2)
    u = amp * prof[None, :, None] * np.cos(z / p.Lz * np.pi)[:, None, None] * np.ones(p.nx)[None, None, :]
    uh = halo_fill(_pad(p, u))
    b = np.zeros_like(u)
    for kk in range(p.nz):
        K = kk + 2
        if kk == 0:
            b[kk] = -p.dy * (uh[K + 1, 2:-2, 2:-2] - uh[K, 2:-2, 2:-2]) / p.dz * p.f0
        elif kk == p.nz - 1:
            b[kk] = -p.dy * (uh[K, 2:-2, 2:-2] - uh[K - 1, 2:-2, 2:-2]) / p.dz * p.f0
        else:
            b[kk] = -p.dy * (uh[K + 1, 2:-2, 2:-2] - uh[K - 1, 2:-2, 2:-2]) / (2 * p.dz) * p.f0
    b = np.cumsum(b, axis=1)   # cumsum_in_y (parallel_mpi.f90:244-267) on one rank
    out = {"u": uh, "v": halo_fill(_pad(p, np.zeros_like(u))),
           "w": halo_fill(_pad(p, np.zeros_like(u))), "b": halo_fill(_pad(p, b))}
    zero_rigid_lid_w(p, out["w"])
    return out


def _pad(p, a):
    h = empty_field(p)
    interior(h)[...] = a
    return h


def lee_wave_forcing(p, U=0.1, omega_frac=0.5, amp=1e-7, nmodes=8, seed=2):
    """Background flow and wavemaker for the lee-wave-like case.

    u_back = U everywhere, b_back = 0 (for_config/lee_wave1.f90:245-312
    background terms) and a w-wavemaker w += dt*(cos(omega t) w_r +
    sin(omega t) w_i) with omega = omega_frac*N0, localised in a Gaussian of
    width Lz/20 around z = Lz/8 (cf. lee_wave1.f90:123-125), horizontally a sum
    of nmodes low modes with seeded random phases."""
    i, j, k = _centres(p)
    x = (i - 0.5) * p.dx
    y = (j - 0.5) * p.dy
    z = k * p.dz
    rnd = splitmix64_uniform(seed, 4 * nmodes)
    hr = np.zeros((p.ny, p.nx))
    hi = np.zeros((p.ny, p.nx))
    for m in range(nmodes):
        mx = 1 + int((rnd[4 * m] + 1) * 4)
        my = int((rnd[4 * m + 1] + 1) * 3)
        ph = np.pi * rnd[4 * m + 2]
        arg = 2 * np.pi * (mx * x[None, :] / p.Lx + my * y[:, None] / p.Ly) + ph
        hr += np.cos(arg)
        hi += np.sin(arg)
    gz = np.exp(-((z - p.Lz / 8.0) / (p.Lz / 20.0)) ** 2)
    w_r = amp * gz[:, None, None] * hr[None]
    w_i = amp * gz[:, None, None] * hi[None]
    u_back = np.full((p.nz, p.ny, p.nx), U)
    return {
        "omega": omega_frac * p.N0,
        "w_r": halo_fill(_pad(p, w_r)),
        "w_i": halo_fill(_pad(p, w_i)),
        "u_back": halo_fill(_pad(p, u_back)),
        "b_back": empty_field(p),
    }


def rel_l2(a, ref):
    """||a - ref||_2 / ||ref||_2 over the given arrays (interiors expected)."""
    d = np.linalg.norm((np.asarray(a) - np.asarray(ref)).ravel())
    n = np.linalg.norm(np.asarray(ref).ravel())
    return d / n if n > 0 else d
