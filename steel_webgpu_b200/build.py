"""Builds libsteel_b200.so in the package directory (nvcc, sm_100a).

The float pipeline must be reproducible bit for bit: --fmad=false (no contraction), IEEE
division and square root, denormals kept.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsteel_b200.so")
BLOCK_SIZES = [32, 64, 128, 256, 512]  # prepare / solve instance sets (csrc/batch.cuh BLOCK_SIZES)
# (source, object, extra flags): prepare.cu and solve.cu are compiled once per block size.
UNITS = [("collide.cu", "collide.o", []), ("api.cu", "api.o", []), ("sort_noalloc.cu", "sort_noalloc.o", []),
         ("scene.cpp", "scene.o", []), ("hull.cpp", "hull.o", [])]
UNITS += [(f"{k}.cu", f"{k}_{n}.o", [f"-DSTEEL_BLOCK={n}"]) for k in ("prepare", "solve") for n in BLOCK_SIZES]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "--fmad=false", "-prec-div=true",
         "-prec-sqrt=true", "-ftz=false", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "steel_b200.h"))

    def compile_one(unit):
        src, obj, extra = unit
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, obj)
        if _stale(o, [s] + headers):
            r = subprocess.run([NVCC, *FLAGS, *extra, "-c", s, "-o", o], capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src} {' '.join(extra)}:\n{r.stderr}")
            if verbose:
                sys.stderr.write(r.stderr)
        return o

    # Longest compiles first (the prepare instances), so the pool ends together.
    units = sorted(UNITS, key=lambda u: (not u[0].startswith("prepare"), not u[0].startswith("solve")))
    with ThreadPoolExecutor(min(len(units), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, units))
    if _stale(LIB, objs):
        r = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs,
                            "-lcudart"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
