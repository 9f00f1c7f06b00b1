"""Restart files in the reference's record layout (restart.f90:2-82).

The file is parsed here by an independent reader of Fortran unformatted
sequential records (4-byte length markers around each record), and a file
written by an independent writer is read back by the engine.
"""
import struct

import numpy as np
import pytest

from ps3d_b200 import configs as cf
from ps3d_b200.model import Model, PS3DError

pytestmark = pytest.mark.gpu


def _records(path):
    out = []
    with open(path, "rb") as fh:
        data = fh.read()
    pos = 0
    while pos < len(data):
        rec = b""
        while True:
            (lead,) = struct.unpack_from("<i", data, pos)
            n = abs(lead)
            rec += data[pos + 4:pos + 4 + n]
            (trail,) = struct.unpack_from("<i", data, pos + 4 + n)
            assert abs(trail) == n
            pos += 8 + n
            if lead >= 0:
                break
        out.append(rec)
    return out


def _write_fortran(path, records):
    with open(path, "wb") as fh:
        for rec in records:
            fh.write(struct.pack("<i", len(rec)) + rec + struct.pack("<i", len(rec)))


def _model(seed=2):
    p = cf.eddy_params(32, 32, 16)
    f = cf.add_noise(p, cf.eddy_fields(p), "b", rel=1e-3, seed=seed)
    m = Model(p)
    m.upload(**{n: f[n] for n in "uvwb"})
    return p, m


def test_write_restart_layout(tmp_path):
    p, m = _model()
    m.run(7)
    path = tmp_path / "restart_pe=000000000.dta"
    m.write_restart(str(path))
    st = m.download()
    r1, r2, r3 = _records(path)
    nx, ny, nz, itt = struct.unpack_from("<4i", r1, 0)
    (time,) = struct.unpack_from("<d", r1, 16)
    taum2, taum1, tau = struct.unpack_from("<3i", r1, 24)
    assert len(r1) == 36 and (nx, ny, nz) == (p.nx, p.ny, p.nz)
    assert (itt, taum2, taum1, tau) == (st["itt"], st["taum2"], st["taum1"], st["tau"])
    assert time == pytest.approx(7 * p.dt, rel=1e-15)
    assert struct.unpack("<6i", r2) == (1, p.nx, 1, p.ny, 1, p.nz)
    arr = np.frombuffer(r3, dtype="<f8")
    n3 = (p.nx + 4) * (p.ny + 4) * (p.nz + 4)
    assert arr.size == 17 * n3
    for q, n in enumerate("uvwbp"):
        assert np.array_equal(arr[q * n3:(q + 1) * n3].reshape(st[n].shape), st[n]), n
    for q, n in enumerate(("du", "dv", "dw", "db")):
        seg = arr[(5 + 3 * q) * n3:(8 + 3 * q) * n3].reshape(st[n].shape)
        assert np.array_equal(seg, st[n]), n
    m.close()


def test_restart_round_trip_continues_identically(tmp_path):
    p, a = _model()
    a.run(9)
    path = str(tmp_path / "r.dta")
    a.write_restart(path)
    b = Model(p)
    t = b.read_restart(path)
    assert t == pytest.approx(9 * p.dt, rel=1e-15)
    a.run(6)
    b.run(6)
    sa, sb = a.download(), b.download()
    for n in ("u", "v", "w", "b", "p", "du", "dv", "dw", "db"):
        assert np.array_equal(sa[n], sb[n]), n
    assert (sa["itt"], sa["tau"]) == (sb["itt"], sb["tau"])
    a.close()
    b.close()


def test_read_restart_written_by_fortran_layout(tmp_path):
    """A file assembled record by record as the reference writes it."""
    p, m = _model(seed=5)
    st = m.download()
    n3 = (p.nx + 4) * (p.ny + 4) * (p.nz + 4)
    rng = np.random.default_rng(1)
    payload = [rng.standard_normal(n3) if n in "uvwbp" else rng.standard_normal(3 * n3) for n in
               ("u", "v", "w", "b", "p", "du", "dv", "dw", "db")]
    r1 = struct.pack("<4i", p.nx, p.ny, p.nz, 42) + struct.pack("<d", 1234.5) + struct.pack("<3i", 3, 1, 2)
    r2 = struct.pack("<6i", 1, p.nx, 1, p.ny, 1, p.nz)
    r3 = b"".join(a.astype("<f8").tobytes() for a in payload)
    path = str(tmp_path / "restart_pe=000000000.dta")
    _write_fortran(path, [r1, r2, r3])
    assert m.read_restart(path) == 1234.5
    got = m.download()
    assert (got["itt"], got["taum2"], got["taum1"], got["tau"]) == (42, 3, 1, 2)
    # interiors come back exactly; halos are the periodic copies of the interior
    for q, n in enumerate("uvwb"):
        ref = payload[q].reshape(st[n].shape)
        assert np.array_equal(got[n][2:-2, 2:-2, 2:-2], ref[2:-2, 2:-2, 2:-2]), n
    m.close()


def test_read_restart_rejects_other_grid(tmp_path):
    p, m = _model()
    path = str(tmp_path / "r.dta")
    m.write_restart(path)
    q = cf.eddy_params(64, 32, 16)
    other = Model(q)
    with pytest.raises(PS3DError):
        other.read_restart(path)
    with pytest.raises(PS3DError):
        other.read_restart(str(tmp_path / "missing.dta"))
    other.close()
    m.close()


def test_async_snapshot_is_the_state_at_the_call():
    import torch
    p, a = _model(seed=3)
    _, b = _model(seed=3)
    a.run(5)
    out = {n: torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy() for n in "uvwbp"}
    a.snapshot_begin(out)
    a.run(5)          # keeps stepping while the copies drain
    a.snapshot_wait()
    b.run(5)
    ref = b.download(tendencies=False)
    for n in "uvwbp":
        assert np.array_equal(out[n], ref[n]), n
    a.close()
    b.close()
