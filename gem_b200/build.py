"""Build recipe of the CUDA library ``gem_b200/libadz_b200.so`` (sm_100a).

nvcc cross-compiles without a GPU.  The exact translation unit (REF32, FP64)
is built with -fmad=false so that only explicit fma() calls fuse; the MIXED
unit keeps contraction on.  The host C-ABI is plain C++ (g++), built with
-ffp-contract=off.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libadz_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r.stdout + r.stderr


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cuh", ".h", ".cpp"))) + [os.path.join(ROOT, "include", "adz_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    common = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
    objs = []
    units = [("adz_exact.cu", ["-fmad=false"]), ("adz_mixed.cu", ["-fmad=true"]), ("adz_noalloc.cu", []), ("adz_batch.cu", []), ("adz_guess.cu", []), ("adz_train.cu", []), ("adz_mass.cu", []), ("adz_diag.cu", []), ("adz_ilmc.cu", ["-fmad=false"]), ("adz_halo.cu", []), ("adz_bcflux.cu", [])]
    for src, extra in units:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        out = _run([NVCC] + ARCH + common + extra + ["-Xptxas", "-v", "-c", os.path.join(CSRC, src), "-o", obj])
        if verbose:
            print(out)
        objs.append(obj)
    for src in ("adz_host.cpp",):
        obj = os.path.join(BUILD, src.replace(".cpp", ".o"))
        _run(["g++", "-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(CUDA, "include"),
              "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lquadmath"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
