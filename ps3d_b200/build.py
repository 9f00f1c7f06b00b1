"""Build the CUDA engine in-tree: ps3d_b200/libps3d_gpu.so (sm_100a), and
the C++ host driver ps3d_b200/ps3d_main (main.f90 over the C ABI) linked
against it.

Plain nvcc, one shared library with a C ABI (include/ps3d_gpu.h); no torch
extension machinery is involved, so Fortran/C hosts can link the same file.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libps3d_gpu.so")
DRIVER = os.path.join(HERE, "ps3d_main")
DRIVER_SRC = os.path.join(HERE, "host", "ps3d_main.cpp")
SOURCES = ["stencil.cu", "poisson.cu", "modes.cu", "reduce.cu", "engine.cu", "ensemble.cu", "serve.cu", "noalloc.cu", "layout.cu", "warn.cu", "restart.cu", "slab.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "ps3d_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build_driver(force=False):
    """g++ of the host driver: only include/ps3d_gpu.h and the library."""
    hdr = os.path.join(ROOT, "include", "ps3d_gpu.h")
    if (not force and os.path.exists(DRIVER) and
            os.path.getmtime(DRIVER) >= max(os.path.getmtime(p) for p in (DRIVER_SRC, hdr, LIB))):
        return DRIVER
    tmp = DRIVER + ".tmp"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include"),
                    DRIVER_SRC, "-o", tmp, "-L" + HERE, "-lps3d_gpu", "-ldl", "-Wl,-rpath,$ORIGIN"], check=True)
    os.replace(tmp, DRIVER)
    return DRIVER


def build(force=False, verbose=False):
    if not force and not needs_build():
        build_driver()
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = ["nvcc", *ARCH, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = False
    for src, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0 or verbose:
            sys.stderr.write(out.decode())
        if pr.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    subprocess.run(["nvcc", *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    build_driver(force=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
