"""Build the CUDA C-ABI library ``anns_fhe_b200/lib/libafhe.so`` for sm_100a,
and ``lib/libafhe_accel_top.so``, the reference's ``fhe_accel_top`` symbol over
it (csrc/fhe_accel_top_shim.cpp), which a host built against the reference's
kernel ABI links in place of the HLS kernel object.

One ``nvcc -c`` per source in ``csrc/`` (in parallel), linked by ``nvcc -shared``; no torch extension, no
JIT cache: the libraries are built in-tree so they travel with the working tree.

    python -m anns_fhe_b200.build [--force] [--ptxas-verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libafhe.so")
SHIM = os.path.join(LIBDIR, "libafhe_accel_top.so")
SHIM_SRC = os.path.join(CSRC, "fhe_accel_top_shim.cpp")
OBJDIR = os.path.join(os.path.dirname(HERE), "_build", "afhe")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["api.cu", "driver.cu", "encode.cu", "ivfpq.cu", "kernels.cu", "ksfused.cu", "noalloc.cu", "tables.cpp"]
HEADERS = ["internal.h", "lanes.h", "modarith.cuh", "ntt.cuh", "tables.h"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA extension cannot be built")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "afhe.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_shim(force: bool = False) -> str:
    """Compile libafhe_accel_top.so (host C++ only, linked to libafhe.so)."""
    if not force and os.path.exists(SHIM) and os.path.getmtime(SHIM) >= max(
            os.path.getmtime(SHIM_SRC), os.path.getmtime(LIB), os.path.getmtime(os.path.join(INCLUDE, "afhe.h"))):
        return SHIM
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I", INCLUDE, "-o", SHIM + ".tmp", SHIM_SRC,
           "-L", LIBDIR, "-lafhe", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    os.replace(SHIM + ".tmp", SHIM)
    return SHIM


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> str:
    """Compile libafhe.so (and the fhe_accel_top binding) if missing or older
    than their sources; return the path of libafhe.so."""
    if not force and not _stale():
        build_shim()
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = nvcc_path()

    def compile_one(src: str):
        obj = os.path.join(OBJDIR, src + ".o")
        cmd = [nvcc, "-O3", "-std=c++17", *ARCH_FLAGS, "-lineinfo", "-Xcompiler", "-fPIC,-O3",
               "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    # one nvcc per source, side by side (the NTT and key-switch instances dominate)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, SOURCES))
    log = ""
    for src, (obj, res) in zip(SOURCES, results):
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n" + res.stdout + res.stderr)
        log += res.stdout + res.stderr
    tmp = LIB + ".tmp"
    res = subprocess.run([nvcc, *ARCH_FLAGS, "-shared", "-o", tmp, *[obj for obj, _ in results]],
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    if not quiet or ptxas_verbose:
        sys.stdout.write(log + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    build_shim(force=True)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_verbose, quiet=False))


if __name__ == "__main__":
    main()
