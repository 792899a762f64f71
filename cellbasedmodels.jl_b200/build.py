"""Builds libcbm_b200.so, the sm_100a shared library behind include/cbm_b200.h.

`python build.py` (or `build()` from Python) runs nvcc directly, one process
per source file, and links the objects (kept in _build/) into the library,
which is written next to this file so it travels with the source tree.  Flags:
  -gencode arch=compute_100a,code=sm_100a  B200 only
  -fmad=false   no FMA contraction: the same rounding as the Julia reference
                and the CPU checker, which makes results bit-identical
  -lineinfo     source lines for ncu
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcbm_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("cbm_api.cu", "cbm_batch.cu", "cbm_adjoint.cu", "cbm_noalloc.cu", "cbm_medium.cu", "cbm_rods.cu")]
DEPS = SOURCES + [
    os.path.join(HERE, "csrc", "cbm_kernels.cuh"),
    os.path.join(HERE, "csrc", "cbm_common.cuh"),
    os.path.join(HERE, "csrc", "cbm_grid.cuh"),
    os.path.join(HERE, "..", "include", "cbm_b200.h"),
    os.path.join(HERE, "..", "include", "cbm_rng.h"),
    os.path.join(HERE, "..", "include", "cbm_rods_math.h"),
]


OBJ_DIR = os.path.join(HERE, "_build")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-fmad=false",
         "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc():
    return os.environ.get("NVCC", "nvcc")


def nvcc_cmd(extra=()):
    """One nvcc command that compiles and links every source (serial)."""
    return [_nvcc(), *FLAGS, "-shared", *extra, "-o", LIB, *SOURCES]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in DEPS)


def build(force=False, verbose=False, extra=()):
    """Compiles each source to an object in parallel, then links the library."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [_nvcc(), *FLAGS, *extra, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=("-Xptxas", "-v") if "--ptxas-v" in sys.argv else ())
