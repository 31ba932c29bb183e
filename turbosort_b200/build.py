"""Builds libturbosort_b200.so from csrc/ with nvcc for sm_100a.

    python -m turbosort_b200.build [--force] [--verbose-ptxas]

Each .cu compiles to an object under _build/ (in parallel), then one shared
library is linked in the package directory, where it travels with the tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libturbosort_b200.so")
WORKLOADS_LIB = os.path.join(PKG, "libts_workloads.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
           "-Xcompiler", "-Wall", "-Wno-deprecated-gpu-targets"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(src: str, ptxas_verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [nvcc(), *ARCH, *NVFLAGS, "-I", INCLUDE, "-c", src, "-o", obj]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if ptxas_verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = _deps()
    todo = [s for s in sources
            if force or ptxas_verbose or _stale(os.path.join(BUILD, os.path.basename(s) + ".o"), [s, *deps])]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, ptxas_verbose), todo))
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in sources]
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    wsrc = os.path.join(CSRC, "ts_workloads.c")
    if force or _stale(WORKLOADS_LIB, [wsrc]):
        cc = shutil.which("gcc") or "cc"
        r = subprocess.run([cc, "-O3", "-fPIC", "-shared", "-o", WORKLOADS_LIB, wsrc], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"gcc failed on ts_workloads.c:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.verbose_ptxas))
