"""Host-side helpers of the workloads (ps3d_b200/configs.py, serve.py), CPU
only: the seeded noise that any host must regenerate bit for bit, the
periodic halo fill, the rigid-lid masking of w and the Poisson arrival
schedule of the serving workload."""
import numpy as np

from ps3d_b200 import configs as cf
from ps3d_b200.serve import SIZES, poisson_schedule


def _splitmix64_ints(seed, n):
    """splitmix64 (Steele, Lea and Flood 2014) on Python integers."""
    mask = (1 << 64) - 1
    out = []
    for i in range(1, n + 1):
        z = (seed + i * 0x9E3779B97F4A7C15) & mask
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        out.append((z >> 11) * 2.0 ** -53 * 2.0 - 1.0)
    return np.array(out)


def test_splitmix64_matches_integer_restatement():
    for seed in (0, 1, 2, 12345, 2 ** 63 + 7):
        got = cf.splitmix64_uniform(seed, 257)
        assert np.array_equal(got, _splitmix64_ints(seed, 257)), seed
        assert got.min() >= -1.0 and got.max() < 1.0


def test_halo_fill_is_periodic_wrap():
    """border_exchg_3D on one rank (parallel_mpi.f90:70-211): every halo
    layer is the opposite interior edge, corners included."""
    rng = np.random.default_rng(0)
    inner = rng.standard_normal((6, 5, 8))
    a = np.zeros((10, 9, 12))
    a[2:-2, 2:-2, 2:-2] = inner
    cf.halo_fill(a)
    assert np.array_equal(a, np.pad(inner, 2, mode="wrap"))


def test_zero_rigid_lid_w():
    """main.f90:119-122: w = 0 at k = -1, 0 and k = nz .. nz+2."""
    p = cf.eddy_params(8, 8, 6)
    w = np.ones((p.nz + 4, p.ny + 4, p.nx + 4))
    cf.zero_rigid_lid_w(p, w)
    zero = [0, 1, p.nz + 1, p.nz + 2, p.nz + 3]
    assert not w[zero].any()
    assert (w[2:p.nz + 1] == 1.0).all()
    q = cf.eddy_params(8, 8, 6, rigid=False)
    w = np.ones((q.nz + 4, q.ny + 4, q.nx + 4))
    assert (cf.zero_rigid_lid_w(q, w) == 1.0).all()


def test_poisson_schedule():
    a = poisson_schedule(2000, 50.0, seed=4)
    b = poisson_schedule(2000, 50.0, seed=4)
    assert a == b
    t = np.array([x[0] for x in a])
    assert t[0] == 0.0 and (np.diff(t) >= 0).all()
    assert abs(np.diff(t).mean() - 1 / 50.0) < 0.1 / 50.0   # exponential gaps of mean 1/rate
    assert {x[1] for x in a} <= set(SIZES)
    assert poisson_schedule(2000, 50.0, seed=5) != a
