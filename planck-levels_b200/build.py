"""Builds libsharp_b200.so in-tree from planck-levels_b200/csrc.

Every CUDA source is compiled for sm_100a only (-gencode
arch=compute_100a,code=sm_100a); the library exports only the sharp_* C ABI
(version script) and binds its own symbols (-Bsymbolic).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "sharp_b200")
LIB = os.path.join(OUT_DIR, "libsharp_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include"), "-I", CSRC] + ARCH
SOURCES = ["sht_host.cc", "sht_execute.cu", "sht_legendre.cu", "sht_ring.cu", "sht_profile.cu", "sht_noalloc.cu", "sht_mixed.cu", "sht_mixed_anal.cu"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers):
            continue
        cmd = [nvcc(), "-c", path, "-o", obj] + NVCC_FLAGS + (extra or [])
        if src.endswith(".cc"):
            cmd = [nvcc(), "-x", "cu", "-c", path, "-o", obj] + NVCC_FLAGS + (extra or [])
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    vs = os.path.join(BUILD, "exports.map")
    with open(vs, "w") as f:
        f.write("{ global: sharp_*; local: *; };\n")
    if _stale(LIB, objs + [vs]):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + [
            "-Xlinker", f"--version-script={vs}", "-Xlinker", "-Bsymbolic", "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
