"""Compile libmiso_b200.so in-tree for sm_100a.

``python -m miso_b200.build`` (or :func:`build`) compiles each ``.cu`` file of
``miso_b200/csrc`` with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
and links ``miso_b200/lib/libmiso_b200.so``.  The FP64 kernels are compiled
with ``--fmad=false`` so their arithmetic rounds exactly as the reference's
x86-64 host build does.  Objects are rebuilt only when a source or header
is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmiso_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills", "-I" + INCLUDE, "-I" + CSRC]
# per-file extra flags
FAST32 = ["--ftz=true", "--prec-div=false", "--prec-sqrt=false"]
EXTRA = {
    "fp64_kernels.cu": ["--fmad=false"],
    "noalloc.cu": ["--fmad=false"],
    "batch64.cu": ["--fmad=false"],
    "batch32.cu": FAST32,
    "batch32_rows.cu": FAST32,
    "fp32s_kernels.cu": FAST32,
    "s32_tiled.cu": FAST32,
    "s32_flat.cu": FAST32,
    "s32_rk.cu": FAST32,
    "s32_av.cu": FAST32,
    "s32_shell.cu": FAST32,
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    objs = []
    nv = nvcc()
    for src in sources:
        base = os.path.basename(src)
        obj = os.path.join(OBJ, base.replace(".cu", ".o"))
        objs.append(obj)
        if _newer(obj, [src] + headers + [__file__]):
            cmd = [nv] + ARCH + COMMON + EXTRA.get(base, []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {base}:\n{r.stdout}\n{r.stderr}")
            if verbose and (r.stdout or r.stderr):
                print(r.stdout + r.stderr, flush=True)
    if _newer(LIB, objs):
        cmd = [nv] + ARCH + ["-shared", "--cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
