"""Compile the sm_100a kernels and the C ABI into shapeextraction_b200/libshapex.so.

nvcc is called directly (no torch extension: the boundary is a plain C ABI).
Objects are compiled in parallel into _build/ and linked with the static CUDA
runtime, so the library loads with ctypes without extra search paths.

    python -m shapeextraction_b200.build [--force] [--ptxas-v]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD_DIR = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libshapex.so")
SOURCES = ["capi.cu", "capi_mlp.cu", "capi_batch.cu", "build.cu", "knn.cu", "mlp.cu", "static_sort.cu", "compat.cu"]
HEADERS = ["common.cuh", "pipeline.cuh", "eig3.cuh", "context.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cc():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _flags(ptxas_v):
    f = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden", "-ccbin", _host_cc(), "-I", INCLUDE,
         "-I", CSRC]
    if ptxas_v:
        f += ["-Xptxas", "-v"]
    return f


def _stale(force):
    if force or not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(INCLUDE, "shapex.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, ptxas_v: bool = False, verbose: bool = False) -> str:
    if not _stale(force):
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    procs = []
    objs = []
    for s in SOURCES:
        obj = os.path.join(BUILD_DIR, s.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc, *_flags(ptxas_v), "-c", os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        if out and (verbose or ptxas_v or p.returncode):
            sys.stdout.write(out)
        if p.returncode:
            failed.append(s)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-ccbin", _host_cc(), "-o", tmp, *objs, "-cudart", "static"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_v=a.ptxas_v, verbose=a.verbose))
