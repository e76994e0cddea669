"""In-tree build of the sm_100a shared library ``jd_lepic_b200/_lib/liblepic_gpu.so``.

Each CUDA translation unit is compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
and linked into one C-ABI shared library (no torch types cross the boundary).  The FP64
multigrid and field kernels are built with ``-fmad=false`` so that their products and sums
round exactly as the reference's Fortran expressions are written.

Usage: ``python -m jd_lepic_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "liblepic_gpu.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = {
    "api.cu": [],
    "field.cu": ["-fmad=false"],
    "mg.cu": ["-fmad=false"],
    "mg_mixed.cu": ["-fmad=false"],
    "push.cu": [],
    "sort.cu": [],
    "mcc.cu": [],
    "noalloc.cu": ["-fmad=false"],
    "cnn.cu": [],
    "sources.cu": ["-fmad=false"],
    "diag.cu": ["-fmad=false"],
    "backup.cu": [],
    "walls.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    out.append(os.path.join(ROOT, "include", "lepic_gpu.h"))
    return out


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles and links the library if any source is newer; returns its path."""
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                     "-I", os.path.join(ROOT, "include"), "-Xptxas", "-v"]
    objs = []
    log = []
    for src, extra in SOURCES.items():
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [cc, "-c", os.path.join(CSRC, src), "-o", obj] + common + extra
        r = subprocess.run(cmd, capture_output=True, text=True)
        log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [cc, "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
        f.write("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
