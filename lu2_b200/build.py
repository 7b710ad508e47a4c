"""Build liblu2gpu.so in-tree with nvcc for sm_100a.

The library links the CUDA runtime statically and reaches the driver API
(cuTensorMapEncodeTiled) through cudaGetDriverEntryPoint, so it loads on a
machine without a GPU driver (only its entry points then fail).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblu2gpu.so")
SOURCES = ["kernels_leaf.cu", "kernels_panel.cu", "kernels_dgemm.cu", "kernels_solve.cu", "kernels_bf16.cu", "kernels_mixed.cu",
           "kernels_batch.cu", "kernels_batch_ir.cu", "kernels_fp8.cu", "kernels_lowp.cu", "kernels_gmres.cu",
           "lu2gpu_api.cu"]
HEADERS = ["lu2gpu_internal.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "lu2gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
    if ptxas_verbose:
        flags += ["-Xptxas", "-v"]
    for s in SOURCES:
        o = os.path.join(objdir, s.replace(".cu", ".o"))
        cmd = [nvcc()] + flags + ["-c", os.path.join(CSRC, s), "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (s, r.stdout, r.stderr))
        if verbose or ptxas_verbose:
            sys.stdout.write(r.stdout + r.stderr)
        objs.append(o)
    tmp = LIB + ".tmp"
    # -Bsymbolic: the library's calls to its own exported names (lu2's
    # function names) bind to its own definitions, never to a caller's
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-Xlinker", "-Bsymbolic", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="-v" in sys.argv)
