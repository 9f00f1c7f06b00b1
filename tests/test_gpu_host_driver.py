"""The C++ host driver (ps3d_b200/ps3d_main, main.f90 over the C ABI) on the
GPU, against the CPU oracle.

A 32x32x16 eddy runs 12 steps with diagnose every 4 and a snapshot every 6
steps.  The restart file the driver writes at the end (restart.f90 layout)
and the snapshot at itt = 6 (the state after the integrate of itt = 6, i.e.
7 steps) must match the oracle's state after the same steps, and the KE it
prints at itt = 4 the oracle's diagnose.  A second run in the same directory
reads that restart file, extends runlen by its time (restart.f90:51-53) and
continues to 24 steps.  A third run writes diag_balance and diag_opt_balance
outputs, checked against the same library calls through the Python binding.
The forcing options: wavemaker and background-flow files against the same
forcing through the Python binding, and a user plugin loaded with dlopen."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from oracle.binding import Oracle
from ps3d_b200 import build
from ps3d_b200 import configs as cf
from tests.helpers import load_oracle, rel
from tests.test_gpu_restart import _records

pytestmark = pytest.mark.gpu

TOL64 = 1e-11
NAMES = ("u", "v", "w", "b", "p")


def _setup(tmp_path):
    p = cf.eddy_params(32, 32, 16)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=4)
    init = tmp_path / "init.bin"
    np.concatenate([np.ascontiguousarray(f[n], dtype="<f8").ravel() for n in "uvwb"]).tofile(init)
    par = tmp_path / "eddy.par"
    par.write_text(f"""! 32x32x16 eddy (for_config/eddy1.f90 template)
nx = {p.nx}
ny = {p.ny}
nz = {p.nz}
Lx = {p.Lx!r}
Ly = {p.Ly!r}
Lz = {p.Lz!r}
dt = {p.dt!r}
f0 = {p.f0!r}
N0 = {p.N0!r}
Ah = {p.Ah!r}
Av = {p.Av!r}
enable_vertical_boundaries = .true.
enable_AB_3_order = .true.
runlen = {12 * p.dt!r}
tsmonint = {4 * p.dt!r}
snapint = {6 * p.dt!r}
enable_diag_snap = .true.
init = {init}
outdir = {tmp_path}
""")
    return p, f, par


def _oracle_after(p, f, nsteps):
    o = Oracle(p)
    load_oracle(o, f)
    o.integrate(nsteps)
    return o


def _restart_fields(path, p):
    r1, r2, r3 = _records(path)
    nx, ny, nz, itt = struct.unpack_from("<4i", r1, 0)
    a = np.frombuffer(r3, dtype="<f8")
    n = (p.nz + 4) * (p.ny + 4) * (p.nx + 4)
    return itt, {nm: a[q * n:(q + 1) * n].reshape(p.nz + 4, p.ny + 4, p.nx + 4) for q, nm in enumerate(NAMES)}


def _snapshot(path, p):
    raw = open(path, "rb").read()
    assert raw[:8] == b"PS3DSNAP"
    nx, ny, nz, nf, itt = struct.unpack_from("<5i", raw, 8)
    (time,) = struct.unpack_from("<d", raw, 32)
    assert (nx, ny, nz, nf) == (p.nx, p.ny, p.nz, 5)
    a = np.frombuffer(raw[64:], dtype="<f8")
    n = (p.nz + 4) * (p.ny + 4) * (p.nx + 4)
    return itt, time, {nm: a[q * n:(q + 1) * n].reshape(p.nz + 4, p.ny + 4, p.nx + 4) for q, nm in enumerate(NAMES)}


def test_driver_run_and_restart(tmp_path):
    build.build()
    p, f, par = _setup(tmp_path)
    r = subprocess.run([build.DRIVER, str(par)], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout
    assert "found no restart file" in out
    assert [int(x) for x in re.findall(r"diagnosing at t=\s*\S+ itt=\s*(\d+)", out)] == [0, 4, 8]
    assert (tmp_path / "ritt").read_text().split() == ["12"]

    # the restart file after 12 steps
    itt, got = _restart_fields(tmp_path / "restart_pe=000000000.dta", p)
    assert itt == 12
    o12 = _oracle_after(p, f, 12)
    err = {n: rel(got[n], o12.field(n)) for n in NAMES}
    assert max(err.values()) < TOL64, err

    # the snapshot of itt = 6: 7 steps done, time = 6 dt
    itt, time, snap = _snapshot(tmp_path / "snap_000000006.bin", p)
    assert itt == 6 and time == pytest.approx(6 * p.dt)
    o7 = _oracle_after(p, f, 7)
    err = {n: rel(snap[n], o7.field(n)) for n in NAMES}
    assert max(err.values()) < TOL64, err
    assert (tmp_path / "snap_000000000.bin").exists()

    # diagnose at itt = 4 reports the state after 5 steps
    ke = float(re.findall(r"KE = (\S+) m\^2/s\^2", out)[1])
    _, ke_ref, _, _, _ = _oracle_after(p, f, 5).diagnose()
    assert ke == pytest.approx(ke_ref, rel=1e-3)

    # second run: reads the restart, runs to 24 steps
    r = subprocess.run([build.DRIVER, str(par)], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "reading restart file" in r.stdout and "adjusting run length" in r.stdout
    assert (tmp_path / "ritt").read_text().split() == ["24"]
    itt, got = _restart_fields(tmp_path / "restart_pe=000000000.dta", p)
    assert itt == 24
    o24 = _oracle_after(p, f, 24)
    err = {n: rel(got[n], o24.field(n)) for n in NAMES}
    assert max(err.values()) < TOL64, err


def test_driver_reports_library_errors(tmp_path):
    """A grid the engine cannot take (nz = 1 under a rigid lid) passes the
    reference's own checks but not ps3d_create: the driver prints the
    library's message and stops with 99."""
    build.build()
    r = subprocess.run([build.DRIVER, "nx=32", "ny=32", "nz=1", "Lx=1", "Ly=1", "Lz=1", "dt=1",
                        "enable_vertical_boundaries=1", f"outdir={tmp_path}"],
                       capture_output=True, text=True, timeout=120, cwd=tmp_path)
    assert r.returncode == 99
    assert "ps3d_create" in r.stderr


def _fields_file(path, p, nf):
    raw = open(path, "rb").read()
    assert raw[:8] == b"PS3DSNAP"
    assert struct.unpack_from("<4i", raw, 8) == (p.nx, p.ny, p.nz, nf)
    a = np.frombuffer(raw[64:], dtype="<f8")
    n = (p.nz + 4) * (p.ny + 4) * (p.nx + 4)
    assert a.size == nf * n
    return {nm: a[q * n:(q + 1) * n].reshape(p.nz + 4, p.ny + 4, p.nx + 4) for q, nm in enumerate("uvwb"[:nf])}


def test_driver_balance_outputs(tmp_path):
    """diag_balance and diag_opt_balance at the snapshot interval (itt = 0
    and 3): the driver's output files hold what the same library calls give
    through the Python binding after the same steps."""
    from ps3d_b200.abi import OptBal, PS3D_FIELDS_BALANCED
    from ps3d_b200.model import Model
    build.build()
    p = cf.eddy_params(32, 32, 16)
    p.Ah = p.Av = 0.0   # the backward ramp keeps harmonic friction (diag_opt_balance.f90:190-192)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=5)
    init = tmp_path / "init.bin"
    np.concatenate([np.ascontiguousarray(f[n], dtype="<f8").ravel() for n in "uvwb"]).tofile(init)
    args = [f"nx={p.nx}", f"ny={p.ny}", f"nz={p.nz}", f"Lx={p.Lx!r}", f"Ly={p.Ly!r}", f"Lz={p.Lz!r}",
            f"dt={p.dt!r}", f"f0={p.f0!r}", f"N0={p.N0!r}", "enable_vertical_boundaries=.true.",
            "enable_AB_3_order=.true.", f"runlen={4 * p.dt!r}", f"tsmonint={100 * p.dt!r}",
            f"snapint={3.5 * p.dt!r}", "enable_diag_balance=.true.", "enable_diag_opt_balance=.true.",
            f"opt_balance_period={5.5 * p.dt!r}", "opt_balance_max_Itts=2", "opt_balance_tol=0",
            f"init={init}", f"outdir={tmp_path}", "write_restart=.false."]
    r = subprocess.run([build.DRIVER, *args], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert len(re.findall(r"optimal balance: 2 iterations", r.stdout)) == 2
    assert not (tmp_path / "restart_pe=000000000.dta").exists()

    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    opt = OptBal(period=5.5 * p.dt, average=1.0, max_itts=2, average_times=1, tol=0.0, enable_time_ave=0, adopt=0)
    for itt, nrun in ((0, 1), (3, 3)):
        m.run(nrun)
        comps = m.diag_balance(3)
        bal = {n: sum(c[n] for c in comps) for n in "uvwb"}
        m.diag_opt_balance(opt)
        obal = m.get_fields(PS3D_FIELDS_BALANCED)
        got_b = _fields_file(tmp_path / f"balance_{itt:09d}.bin", p, 4)
        got_o = _fields_file(tmp_path / f"opt_balance_{itt:09d}.bin", p, 4)
        for n in "uvwb":
            assert rel(got_b[n], bal[n]) < 1e-13, (itt, "balance", n)
            assert rel(got_o[n], obal[n]) < 1e-13, (itt, "opt_balance", n)
    m.close()


def _par_args(p, runlen_steps, tmp_path, init, extra=()):
    return [f"nx={p.nx}", f"ny={p.ny}", f"nz={p.nz}", f"Lx={p.Lx!r}", f"Ly={p.Ly!r}", f"Lz={p.Lz!r}",
            f"dt={p.dt!r}", f"f0={p.f0!r}", f"N0={p.N0!r}", f"Ah={p.Ah!r}", f"Av={p.Av!r}",
            f"enable_vertical_boundaries={p.enable_vertical_boundaries}",
            f"enable_AB_3_order={p.enable_AB_3_order}", f"runlen={runlen_steps * p.dt!r}",
            f"tsmonint={1000 * p.dt!r}", f"init={init}", f"outdir={tmp_path}", *extra]


def test_driver_wavemaker_and_background_forcing(tmp_path):
    """set_forcing of the lee-wave case (config.f90:224-237 wavemaker,
    lee_wave1.f90:245-312 background flow) from files, against the same
    forcing installed through the Python binding."""
    from ps3d_b200.model import Model
    build.build()
    p = cf.lee_wave_params(32, 16, 16)
    fr = cf.lee_wave_forcing(p, seed=2)
    zero = cf.empty_field(p)
    init = tmp_path / "init.bin"
    np.concatenate([zero.ravel()] * 4).astype("<f8").tofile(init)
    wm = tmp_path / "wavemaker.bin"
    names = ("u_r", "v_r", "w_r", "b_r", "u_i", "v_i", "w_i", "b_i")
    np.concatenate([np.ascontiguousarray(fr.get(n, zero), dtype="<f8").ravel() for n in names]).tofile(wm)
    bg = tmp_path / "background.bin"
    np.concatenate([np.ascontiguousarray(fr[n], dtype="<f8").ravel() for n in ("u_back", "b_back")]).tofile(bg)
    args = _par_args(p, 10, tmp_path, init, [f"forcing_wavemaker={wm}", f"omega_forc={fr['omega']!r}",
                                             f"forcing_background={bg}"])
    r = subprocess.run([build.DRIVER, *args], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    itt, got = _restart_fields(tmp_path / "restart_pe=000000000.dta", p)
    assert itt == 10

    from ps3d_b200 import abi
    m = Model(p)
    m.set_forcing(abi.PS3D_FORCE_WAVEMAKER | abi.PS3D_FORCE_BACKGROUND, omega=fr["omega"], w_r=fr["w_r"],
                  w_i=fr["w_i"], u_back=fr["u_back"], b_back=fr["b_back"])
    m.upload(**{n: zero for n in "uvwb"})
    m.run(10)
    ref = m.download(tendencies=False)
    m.close()
    assert np.abs(ref["w"]).max() > 0.0
    err = {n: rel(got[n], ref[n]) for n in NAMES}
    assert max(err.values()) < 1e-13, err


PLUGIN = r"""
#include "ps3d_gpu.h"
/* a set_forcing that adds nothing; fails at itt = 3 when built with FAIL */
int my_forcing(void* user, const ps3d_device_view* v) {
    (void)user;
    if (v->nx != 32 || v->ny != 32 || v->nz != 16 || !(v->dt > 0) || !v->u || !v->du || !v->stream) return -2;
#ifdef FAIL
    if (v->itt == 3) return -2;
#endif
    return 0;
}
"""


def test_driver_forcing_plugin(tmp_path):
    """forcing_plugin = lib.so:symbol: the callback runs inside every step (a
    no-op callback leaves the oracle's trajectory), and its error status
    stops the run with 99."""
    build.build()
    p, f, _ = _setup(tmp_path)
    init = tmp_path / "init.bin"
    src = tmp_path / "plugin.c"
    src.write_text(PLUGIN)
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    libs = {}
    for tag, flags in (("ok", []), ("fail", ["-DFAIL"])):
        libs[tag] = tmp_path / f"libforce_{tag}.so"
        subprocess.run(["gcc", "-shared", "-fPIC", "-O2", "-I" + inc, *flags, str(src), "-o", str(libs[tag])],
                       check=True)
    r = subprocess.run([build.DRIVER, *_par_args(p, 8, tmp_path, init, [f"forcing_plugin={libs['ok']}:my_forcing"])],
                       capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    itt, got = _restart_fields(tmp_path / "restart_pe=000000000.dta", p)
    assert itt == 8
    o8 = _oracle_after(p, f, 8)
    err = {n: rel(got[n], o8.field(n)) for n in NAMES}
    assert max(err.values()) < TOL64, err

    os.remove(tmp_path / "restart_pe=000000000.dta")
    r = subprocess.run([build.DRIVER, *_par_args(p, 8, tmp_path, init,
                                                 [f"forcing_plugin={libs['fail']}:my_forcing"])],
                       capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 99
    assert "ps3d_integrate" in r.stderr
    r = subprocess.run([build.DRIVER, *_par_args(p, 8, tmp_path, init, [f"forcing_plugin={libs['ok']}:nothing"])],
                       capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 99 and "has no symbol nothing" in r.stderr
