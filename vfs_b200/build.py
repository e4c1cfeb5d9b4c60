"""Build the vfs_b200 CUDA library in-tree (vfs_b200/_lib/libvfs_b200.so) with nvcc for sm_100a.

The library is built with ``-fmad=false``: no multiply and add is contracted into a fused
multiply-add unless the source asks for one explicitly, so every kernel's floating-point
operation order is the one written in the source.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libvfs_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]
SOURCES = ["kernels_plain.cu", "kernels_hist.cu", "kernels_fused.cu", "kernels_tb.cu", "kernels_cluster.cu", "kernels_tma.cu", "stereo_tgv.cu", "batch.cu",
           "capi.cu", "io.cpp"]


def nvcc() -> str:
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _needs(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "vfs_b200.h"))
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    jobs = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD_DIR, s + ".o")
        if force or _needs(obj, [src] + headers):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
            if s.endswith(".cpp"):
                cmd = [nvcc()] + ["-x", "cu"] + NVCC_FLAGS + ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    objs = [os.path.join(BUILD_DIR, s + ".o") for s in srcs]
    if force or jobs or _needs(LIB, objs):
        run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
