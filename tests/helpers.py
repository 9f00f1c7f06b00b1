"""Shared test utilities: moving one state between the CPU oracle and the
engine, and error norms.  Test code only."""
import numpy as np

from ps3d_b200 import configs as cf
from ps3d_b200.abi import make_params

FIELDS = ("u", "v", "w", "b")


def random_state(p, seed=0, amp=0.1, wamp=1e-3, bamp=1e-3):
    """Seeded noisy state (interior random, halos periodic) for parity runs."""
    rng = np.random.default_rng(seed)
    out = {}
    for name, a in (("u", amp), ("v", amp), ("w", wamp), ("b", bamp)):
        h = cf.empty_field(p)
        cf.interior(h)[...] = a * rng.standard_normal((p.nz, p.ny, p.nx))
        out[name] = cf.halo_fill(h)
    cf.zero_rigid_lid_w(p, out["w"])
    cf.halo_fill(out["w"])
    return out


def smooth_state(p, seed=0):
    """Eddy + noise, a smooth flow with all four fields non-trivial."""
    f = cf.eddy_fields(p)
    f = cf.add_noise(p, f, "b", rel=1e-2, seed=seed)
    rng = np.random.default_rng(seed + 7)
    w = f["w"]
    cf.interior(w)[...] = 1e-5 * rng.standard_normal((p.nz, p.ny, p.nx))
    cf.halo_fill(w)
    cf.zero_rigid_lid_w(p, w)
    cf.halo_fill(w)
    if p.enable_vertical_boundaries:
        cf.interior(w)[-1] = 0.0
        cf.halo_fill(w)
    return f


def load_oracle(o, fields, p_field=None):
    for n in FIELDS:
        o.field(n)[...] = fields[n]
    if p_field is not None:
        o.field("p")[...] = p_field


def upload_from_oracle(m, o):
    itt, tau, t1, t2, _ = o.get_time()
    m.upload(u=o.field("u"), v=o.field("v"), w=o.field("w"), b=o.field("b"), p=o.field("p"),
             du=o.tendency("du"), dv=o.tendency("dv"), dw=o.tendency("dw"), db=o.tendency("db"),
             itt=itt, tau=tau, taum1=t1, taum2=t2)


def rel(a, b):
    a = np.asarray(a)[2:-2, 2:-2, 2:-2] if np.ndim(a) == 3 else np.asarray(a)
    b = np.asarray(b)[2:-2, 2:-2, 2:-2] if np.ndim(b) == 3 else np.asarray(b)
    n = np.linalg.norm(b.ravel())
    d = np.linalg.norm((a - b).ravel())
    return d / n if n > 0 else d


def compare_state(m, o, names=("u", "v", "w", "b", "p")):
    got = m.download(tendencies=False)
    return {n: rel(got[n], o.field(n)) for n in names}


def small_params(nx=32, ny=32, nz=16, rigid=True, **kw):
    base = dict(nx=nx, ny=ny, nz=nz, Lx=32e3, Ly=32e3, Lz=1000.0, f0=1e-4, N0=1e-3, dt=300.0,
                Ah=1e-2, Av=1e-2, enable_vertical_boundaries=int(rigid), enable_AB_3_order=1)
    base.update(kw)
    return make_params(**base)
