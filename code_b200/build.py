"""Build of the CUDA library ``code_b200/_lib/libgetm_b200.so`` (sm_100a) with nvcc.

The FP64 kernels are compiled with ``--fmad=false`` so that no multiply-add is contracted and
every expression rounds as written; the FP32 kernels keep contraction. Objects are rebuilt only
when a source or header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libgetm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]

# per-translation-unit flags
UNITS = {
    "kernels_f64.cu": ["--fmad=false"],
    "kernels_f32.cu": ["--fmad=true"],
    "ctx.cu": [],
    "bc.cu": ["--fmad=false"],
    "noalloc.cu": ["--fmad=false"],
    "adjoint.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_input() -> float:
    files = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h")) + [__file__]
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OUT_DIR, unit.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra_flags or []), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
