"""Builds fcwt_b200/lib/libfcwt_b200.so in-tree.

CUDA sources are compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); host C++ sources by g++ with
``-ffp-contract=off`` so the bit-exact host arithmetic (scale grids, truncation
lengths) keeps the reference's float operation order. The CUDA runtime is
linked statically, so the library only needs the driver at run time.

Usage: ``python -m fcwt_b200.build [--force]``
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
SRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "lib", "obj")
LIB = os.path.join(PKG, "lib", "libfcwt_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["fcwt_kernels.cu", "fcwt_fwd.cu", "fcwt_tc.cu", "fcwt_capi.cu", "fcwt_noalloc.cu", "fcwt_adjoint.cu"]
CPP_SOURCES = ["fcwt_host.cpp", "fcwt_plan.cpp", "fcwt_cpp.cpp"]
HEADERS = ["fcwt_internal.h", "fcwt_plan.h", "fcwt_fft.cuh", "fcwt_dev.cuh"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(SRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "fcwt_b200.h"),
        os.path.join(ROOT, "include", "fcwt.h"),
    ]
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            jobs.append([NVCC, "-std=c++17", "-O3", "--expt-relaxed-constexpr", *ARCH, "-lineinfo",
                         "-Xcompiler", "-fPIC,-ffp-contract=off", "-I" + os.path.join(ROOT, "include"),
                         "-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src = os.path.join(SRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            jobs.append(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                         "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA_HOME, "include"),
                         "-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for f in [ex.submit(_run, j) for j in jobs]:
                f.result()
    if force or jobs or _newer(LIB, objs):
        tmp = LIB + ".tmp"
        _run([NVCC, "-shared", *ARCH, "-o", tmp, *objs, "-Xcompiler", "-fPIC", "-cudart", "static"])
        os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


def clean() -> None:
    shutil.rmtree(os.path.join(PKG, "lib"), ignore_errors=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
