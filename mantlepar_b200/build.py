"""Build the mantlepar_b200 CUDA library in-tree for sm_100a.

    python -m mantlepar_b200.build        # -> mantlepar_b200/libmantlepar_b200.so
                                          #    mantlepar_b200/libmantle_b200_host.so

Every translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared library (static CUDA runtime) that exports the C ABI of
include/mantlepar/mp.h. The C++ host layer (include/mantle/phase/
eutectic_rescaled.h, mantlepar_b200/host/) is compiled by g++ into a second
library linked against the first.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmantlepar_b200.so")
# Bounds-checked variant (-DMP_CHECKED): every stage element checks the cell
# and edge indices it derives and records a status instead of an access
# outside its arrays. Loaded instead of LIB when MP_CHECKED=1.
CHECKED_LIB = os.path.join(HERE, "libmantlepar_b200_checked.so")
# C++ host layer (mantle::phase::EutecticModel over the C ABI), linked to LIB.
HOST_LIB = os.path.join(HERE, "libmantle_b200_host.so")
HOST_SOURCES = [os.path.join(HERE, "host", "eutectic_model.cpp"), os.path.join(HERE, "host", "coupled_transport.cpp")]

SOURCES = ["phase_api.cu", "transport.cu", "tables.cpp", "mp_noalloc.cu", "batch.cu", "serve.cpp", "preheat.cu", "quad_tables.cpp", "quad_table_kernels.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the mantlepar_b200 CUDA library cannot be built")


# Per-source flags: the GPU table builder rounds every operation as the host
# builder does (no FMA contraction).
SOURCE_FLAGS = {"quad_table_kernels.cu": ["--fmad=false"]}


def _compile(src: str, verbose: bool, checked: bool = False) -> str:
    out_dir = os.path.join(BUILD, "checked") if checked else BUILD
    obj = os.path.join(out_dir, os.path.splitext(src)[0] + ".o")
    extra = ["-DMP_CHECKED"] if checked else []
    cmd = [nvcc()] + ARCH + FLAGS + extra + SOURCE_FLAGS.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build_checked(force: bool = False) -> str:
    """Compile the bounds-checked variant of the library (CHECKED_LIB)."""
    os.makedirs(os.path.join(BUILD, "checked"), exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mantlepar", "mp.h")]
    if not force and os.path.exists(CHECKED_LIB) and os.path.getmtime(CHECKED_LIB) >= max(os.path.getmtime(d) for d in deps):
        return CHECKED_LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, False, True), SOURCES))
    cmd = [nvcc()] + ARCH + ["-shared", "-o", CHECKED_LIB] + objs + ["-Xcompiler", "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return CHECKED_LIB


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mantlepar", "mp.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        hdeps = HOST_SOURCES + [LIB, os.path.join(ROOT, "include", "mantle", "phase", "eutectic_rescaled.h"),
                                os.path.join(ROOT, "include", "mantle", "couple", "coupled_transport.h")]
        if not os.path.exists(HOST_LIB) or os.path.getmtime(HOST_LIB) < max(os.path.getmtime(d) for d in hdeps):
            build_host()
        return LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_host()
    return LIB


def build_host() -> str:
    """Compile the C++ host layer (g++, C++17) against the CUDA library."""
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
           "-I", os.path.join(ROOT, "include"), *HOST_SOURCES, "-o", HOST_LIB,
           "-L", HERE, "-l:libmantlepar_b200.so", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host layer build failed:\n{r.stdout}\n{r.stderr}")
    return HOST_LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
    if "--checked" in sys.argv:
        print(build_checked(force="-f" in sys.argv))
