"""The C++ host driver (ps3d_b200/host/ps3d_main.cpp), main.f90 over the C
ABI, on the CPU: its parameter reading and its main-loop schedule.

`--dry-run` runs the loop of main.f90:139-162 without a GPU and prints every
library call and diagnostic event; the schedule is checked against a direct
restatement of that loop (diagnose every max(1, int(tsmonint/dt)) steps and at
itt = 0, snapshot work every max(1, int(snapint/dt)) steps and at itt = 0,
time accumulated by time = time + dt until time >= runlen)."""
import os
import re
import subprocess

import pytest

from ps3d_b200 import build


@pytest.fixture(scope="module")
def driver():
    build.build()
    assert os.path.exists(build.DRIVER)
    return build.DRIVER


BASE = ["nx=32", "ny=32", "nz=16", "Lx=1e5", "Ly=1e5", "Lz=1000", "enable_vertical_boundaries=.true."]


def _run(driver, args, check=True):
    r = subprocess.run([driver, *args], capture_output=True, text=True, timeout=60)
    if check:
        assert r.returncode == 0, r.stdout + r.stderr
    return r


def _reference_schedule(dt, runlen, tsmonint, snapint, snap_work):
    """main.f90:139-162, event by event."""
    time, itt, ev = 0.0, 0, []
    nmon, nsnap = max(1, int(tsmonint / dt)), max(1, int(snapint / dt))
    while time < runlen:
        if itt % nmon == 0 or itt == 0:
            ev.append(("diagnose", itt, time))
        if snap_work and (itt % nsnap == 0 or itt == 0):
            ev.append(("snapshot", itt, time))
        time = time + dt
        itt += 1
    return ev, itt, time


@pytest.mark.parametrize("dt,runlen,tsmonint,snapint,snap", [
    (300.0, 3600.0, 1200.0, 1800.0, True),
    (300.0, 3600.0, 0.0, 0.0, False),        # reference defaults: diagnose every step
    (0.1, 1.0, 0.3, 0.25, True),             # runlen not a sum of exact dt: accumulated time decides
    (7.0, 100.0, 1e30, 50.0, True),          # intervals beyond int range, non-integer ratios
    (5.0, 4.0, 10.0, 10.0, False),           # one step
    (5.0, 0.0, 10.0, 10.0, True),            # no step
])
def test_dry_run_schedule(driver, dt, runlen, tsmonint, snapint, snap):
    args = BASE + [f"dt={dt!r}", f"runlen={runlen!r}", f"tsmonint={tsmonint!r}", f"snapint={snapint!r}",
                   f"enable_diag_snap={'.true.' if snap else '.false.'}", "--dry-run"]
    out = _run(driver, args).stdout
    got = [(m.group(1), int(m.group(2)), float(m.group(3)))
           for m in re.finditer(r"^(diagnose|snapshot) itt=(\d+) time=(\S+)$", out, re.M)]
    ev, itt, time = _reference_schedule(dt, runlen, tsmonint, snapint, snap)
    assert got == ev
    fin = re.search(r"^final itt=(\d+) time=(\S+) steps=(\d+) calls=(\d+)$", out, re.M)
    assert int(fin.group(1)) == itt and float(fin.group(2)) == time and int(fin.group(3)) == itt
    # the steps between events go to the library in one call each
    chunks = [int(x) for x in re.findall(r"^integrate (\d+)$", out, re.M)]
    assert sum(chunks) == itt and len(chunks) == int(fin.group(4))
    assert len(chunks) <= len({e[1] for e in ev}) + 1


def test_parameter_file(driver, tmp_path):
    """Fortran-flavoured values, comments, defaults (main_module.f90:16-57)
    and command-line overrides after the file."""
    f = tmp_path / "run.par"
    f.write_text("! eddy-like setup\nnx = 64\nny = 32   # trailing comment\nnz=16\n"
                 "Lx = 64d3\nLy = 3.2D4\nLz = 1000.\ndt = 300\nAh = 1d-2\nKv = 2.5e-3\n"
                 "enable_vertical_boundaries = .TRUE.\nenable_AB_3_order = T\nprecision = 'mixed'\n"
                 "runlen = 0\n")
    out = _run(driver, [str(f), "Ro=0.5", "--dry-run"]).stdout
    assert "nx x ny x nz =   64 x   32 x   16" in out
    assert "Delta x =  1000.00 m" in out and "Delta y =  1000.00 m" in out and "Delta z =    62.50 m" in out
    assert "Ah      = 1.000000e-02" in out and "Kv      = 2.500000e-03" in out
    assert "Ro      =     0.50" in out and "delta   =     1.00" in out
    assert "enable_AB_3_order           = T" in out and "precision                   = mixed" in out


@pytest.mark.parametrize("args,msg", [
    (["nx=33", "ny=32", "nz=16", "Lx=1", "Ly=1", "Lz=1", "dt=1", "enable_vertical_boundaries=0"],
     "nx,ny,nz need to be even or one"),
    (["nx=32", "ny=31", "nz=16", "Lx=1", "Ly=1", "Lz=1", "dt=1", "enable_vertical_boundaries=1"],
     "nx,ny need to be even or one"),
    (BASE + ["dt=1", "colour=blue"], "unknown parameter colour"),
    (BASE + ["dt=1x"], "bad number for dt"),
    (BASE + ["dt=1", "precision=half"], "bad value for precision"),
    (BASE + ["dt=1", "enable_diag_snap=maybe"], "bad logical for enable_diag_snap"),
    (BASE, "dt must be positive"),
])
def test_parameter_errors_abort_with_99(driver, args, msg):
    """The reference stops with MPI_ABORT(.., 99, ..) (main.f90:21-56)."""
    r = _run(driver, args + ["--dry-run"], check=False)
    assert r.returncode == 99
    assert msg in r.stderr


def test_driver_uses_only_the_c_abi(driver):
    """The driver links the engine library and includes nothing but the
    public header: no CUDA or torch on the host side."""
    src = open(build.DRIVER_SRC).read()
    includes = re.findall(r'#include\s+[<"]([^>"]+)[>"]', src)
    assert "ps3d_gpu.h" in includes
    assert not [i for i in includes if "cuda" in i or "torch" in i]
    out = subprocess.run(["ldd", driver], capture_output=True, text=True).stdout
    assert "libps3d_gpu.so" in out


def test_help_lists_every_key(driver):
    out = _run(driver, ["--help"]).stdout
    for key in ("nx", "lx", "dt", "n0", "ah", "enable_vertical_boundaries", "enable_ab_3_order", "precision",
                "runlen", "tsmonint", "snapint", "enable_diag_snap", "enable_diag_balance",
                "enable_diag_opt_balance", "opt_balance_period", "opt_balance_max_itts", "init", "restart",
                "forcing_wavemaker", "forcing_background", "forcing_plugin", "omega_forc", "outdir", "profile"):
        assert re.search(r"\b" + key + r"\b", out), key
