"""Build the sm_100a shared library of the AKMC force path (in-tree).

    python -m akmc_b200.build [-v] [--checks]

Produces ``akmc_b200/libakmc_b200.so`` from ``akmc_b200/csrc``: every CUDA source is
compiled for ``sm_100a`` only (``-gencode arch=compute_100a,code=sm_100a``), the CUDA
runtime is linked statically, and objects are cached under ``akmc_b200/_build``
(rebuilt when a source or header is newer than its object).  ``--checks`` builds the
self-checking variant instead (``-DAKMC_CHECKS``: kernel index checks that count hits and
skip the access, read back through akmc_checks_read) as ``libakmc_b200_checks.so``, with
its objects under ``akmc_b200/_build_checks``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libakmc_b200.so")
OBJ = os.path.join(PKG, "_build")
OUT_CHECKS = os.path.join(PKG, "libakmc_b200_checks.so")
OBJ_CHECKS = os.path.join(PKG, "_build_checks")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def build(verbose: bool = False, ptxas_info: bool = False, checks: bool = False) -> str:
    obj_dir, out = (OBJ_CHECKS, OUT_CHECKS) if checks else (OBJ, OUT)
    extra = ["-DAKMC_CHECKS"] if checks else []
    os.makedirs(obj_dir, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    objs = []
    procs = []
    for src in sources:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, src):
            cmd = [NVCC] + ARCH + FLAGS + extra + (["-Xptxas", "-v"] if ptxas_info else []) + \
                  ["-x", "cu" if src.endswith(".cu") else "c++", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT, text=True)))
    for src, p in procs:
        log, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{log}")
        if verbose and log:
            print(log)
    if procs or not os.path.exists(out) or any(os.path.getmtime(o) > os.path.getmtime(out) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", out] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv, checks="--checks" in sys.argv))
