"""Build librqcopt_gpu.so (the B200 C-ABI library) in-tree with nvcc for sm_100a.

Every ``csrc/*.cu`` file is compiled to an object under ``_build/`` (in
parallel, skipped when up to date) and linked into
``rqcopt_hpc_b200/librqcopt_gpu.so``; ``csrc/abi_real.cpp`` (host code) becomes
``rqcopt_hpc_b200/librqcopt_gpu_real.so``, the real-orthogonal build, which loads
the first library at run time.  Usage::

    python -m rqcopt_hpc_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "librqcopt_gpu.so")
REAL_LIB = os.path.join(PKG, "librqcopt_gpu_real.so")
REAL_SRC = os.path.join(CSRC, "abi_real.cpp")
CXX = os.environ.get("CXX", "g++")
NVCC = os.environ.get("NVCC", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "rqcopt_gpu.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, force, verbose, extra):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if not force and not _stale(obj, [src] + _headers()):
        return obj, None
    cmd = [NVCC] + FLAGS + extra + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{p.stdout}\n{p.stderr}"
    if verbose and (p.stdout or p.stderr):
        print(p.stdout + p.stderr, flush=True)
    return obj, None


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force or ptxas_info, verbose or ptxas_info, extra), sources))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or _stale(LIB, objs):
        # -Bsymbolic: calls between the library's own exports (and its comparisons of
        # ufunc addresses) bind inside it, also when librqcopt_gpu_real.so, which
        # exports the same names with real types, is loaded into the process
        cmd = [NVCC] + ARCH + ["-shared", "-Xlinker", "-Bsymbolic", "-o", LIB] + objs + ["-lcudart"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    real_deps = [REAL_SRC, os.path.join(ROOT, "include", "rqcopt_gpu_real.h")]
    if force or _stale(REAL_LIB, real_deps):
        cmd = [CXX, "-std=c++17", "-O2", "-fPIC", "-Wall", "-fvisibility=hidden", "-shared", "-I" + os.path.join(ROOT, "include"),
               "-o", REAL_LIB, REAL_SRC, "-ldl", "-Wl,--exclude-libs,ALL"]
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"real-build library failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv))
