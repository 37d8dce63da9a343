"""Build recipe for the in-tree native library (sm_100a only).

Produces ``3d_mpi_test_b200/lib/libfdtd_b200.so`` (the C ABI declared in
``include/fdtd_b200.h`` and ``include/fdtd_surrogate.h``) with explicit
nvcc calls; no JIT cache, so the built file travels with the source tree.
An object is rebuilt when its source or any header is newer.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libfdtd_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]

SOURCES = ["fdtd_k_tile_pml_f32.cu", "fdtd_k_tile_pml_f64.cu", "fdtd_k_tile_pml_f32_ter.cu", "fdtd_k_tile_pml_f64_ter.cu",
           "fdtd_k_tile_flat.cu", "fdtd_k_tile_ter.cu", "fdtd_k_tile.cu", "fdtd_k_march.cu", "mlp.cu", "fdtd_solver.cu",
           "fdtd_k_twopass.cu", "fdtd_noalloc.cu", "fdtd_spectra.cu", "fdtd_input.cpp", "fdtd_capi.cpp"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    inc = os.path.join(ROOT, "include")
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".hpp", ".cuh"))] + \
        [os.path.join(inc, f) for f in os.listdir(inc)]
    deps = [os.path.join(CSRC, f) for f in SOURCES] + headers
    if not force and not _stale(LIB, deps):
        build_host_mirror(verbose)
        return LIB
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [os.path.join(CSRC, src)] + headers):
            continue
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        cmds.append(cmd)
    # the translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    build_host_mirror(verbose)
    return LIB


HOST = os.path.join(PKG, "host")
HOST_LIB = os.path.join(LIBDIR, "libairpore_b200.so")


def build_host_mirror(verbose: bool = False) -> str:
    """The C++ host classes (host/airpore_b200.cpp) as libairpore_b200.so
    over libfdtd_b200.so, found next to it at run time."""
    src = os.path.join(HOST, "airpore_b200.cpp")
    deps = [src, os.path.join(HOST, "airpore_b200.hpp"), os.path.join(ROOT, "include", "fdtd_b200.h"), LIB]
    if not _stale(HOST_LIB, deps):
        return HOST_LIB
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"),
           src, "-o", HOST_LIB, "-L", LIBDIR, "-lfdtd_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return HOST_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv))
