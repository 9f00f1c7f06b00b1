"""The C ABI library: it loads, exports every entry point include/ps3d_gpu.h
declares, and the ctypes mirrors match the C struct layouts.  No GPU needed
(no compute call is made)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from ps3d_b200 import abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ps3d_gpu.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"PS3D_API\s+[\w\s\*]+?\b(ps3d_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    return build.build()


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("ps3d_create", "ps3d_destroy", "ps3d_upload_state", "ps3d_download_state", "ps3d_step",
              "ps3d_integrate", "ps3d_pressure_solve", "ps3d_project_geostrophic", "ps3d_opt_balance",
              "ps3d_diagnose", "ps3d_set_forcing", "ps3d_strerror"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(ps3d_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_and_strerror(lib_path):
    L = C.CDLL(lib_path)
    for s in declared_symbols():
        assert hasattr(L, s)
    L.ps3d_strerror.restype = C.c_char_p
    assert L.ps3d_strerror(abi.PS3D_ERR_NONFINITE).decode().startswith("non-finite")
    assert L.ps3d_strerror(0).decode() == "ok"


def test_struct_layouts_match_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "ps3d_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(ps3d_params), sizeof(ps3d_optbal), sizeof(ps3d_forcing), sizeof(ps3d_device_view));
  printf("%zu %zu %zu %zu\n", offsetof(ps3d_params, dt), offsetof(ps3d_params, Kvbi), offsetof(ps3d_params, precision),
         offsetof(ps3d_forcing, u_back));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I" + os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    assert sizes == [C.sizeof(abi.Params), C.sizeof(abi.OptBal), C.sizeof(abi.Forcing), C.sizeof(abi.DeviceView)]
    assert offs == [abi.Params.dt.offset, abi.Params.Kvbi.offset, abi.Params.precision.offset, abi.Forcing.u_back.offset]


def test_model_fails_loudly_without_gpu(lib_path):
    """No CPU fallback: on a host without a usable GPU, creation errors out."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from ps3d_b200.model import Model, PS3DError
    from tests.helpers import small_params
    with pytest.raises(PS3DError):
        Model(small_params())


def test_constants_match_header():
    """Every numeric #define PS3D_* of the header that the Python mirror
    (ps3d_b200/abi.py) also names has the same value there."""
    text = open(HEADER).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(PS3D_\w+)\s+(-?\d+)\b", text)}
    assert "PS3D_MIXED_REFINED" in defs and "PS3D_ERR_TOOLARGE" in defs
    shared = [k for k in defs if hasattr(abi, k)]
    assert len(shared) >= 20, shared
    bad = {k: (defs[k], getattr(abi, k)) for k in shared if getattr(abi, k) != defs[k]}
    assert not bad, bad
    for k in ("PS3D_FP64", "PS3D_MIXED", "PS3D_MIXED_REFINED", "PS3D_OK", "PS3D_ERR_NONFINITE",
              "PS3D_PROJ_NORMAL_MODE", "PS3D_FIELDS_BALANCED", "PS3D_FORCE_CALLBACK"):
        assert k in shared, k


def test_phase_and_kernel_class_mirrors():
    """The slab phases (ps3d_b200/slab.py PHASE) and the profile's kernel
    classes (Model.KERNELS, indexed by PS3D_K_*) match the header."""
    from ps3d_b200.model import Model
    from ps3d_b200.slab import PHASE
    text = open(HEADER).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(PS3D_\w+)\s+(-?\d+)\b", text)}
    for name, v in PHASE.items():
        assert defs["PS3D_SLAB_" + name.upper()] == v, name
    assert len(PHASE) == len([k for k in defs if k.startswith("PS3D_SLAB_")])
    names = {"step": "STEP", "fft_fwd": "FFT_FWD", "vsolve": "VSOLVE", "fft_inv": "FFT_INV",
             "correct": "CORRECT", "other": "OTHER", "vmode": "VMODE"}
    for i, k in enumerate(Model.KERNELS):
        assert defs["PS3D_K_" + names[k]] == i, k
    assert defs["PS3D_K_COUNT"] == len(Model.KERNELS)
