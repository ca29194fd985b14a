"""Build ``libslm_b200.so`` (all CUDA kernels + the C ABI) for sm_100a, in-tree.

Every tracing translation unit is compiled with ``--fmad=false`` and IEEE
division and square root (the nvcc defaults without fast-math), which the
bit-exact parity with the reference's arithmetic depends on.

Usage: ``python -m slm_b200.build [--force] [--verbose]``
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libslm_b200.so")
SOURCES = ["capi.cu", "trace.cu", "kde.cu", "map_kernels.cu", "scheduler.cu", "map_device.cu", "preprocess.cu",
           "seeds.cpp", "seeds_device.cu", "gemm_tc.cu", "fmm.cu"]
HEADERS = ["trace_common.cuh", "capi_util.cuh", "mt19937.hpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")


def _flags():
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true",
                   "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC",
                   "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "slm_b200.h")]
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC] + _flags() + ["-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n{}\n{}".format(" ".join(cmd), r.stderr[-6000:]))
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(run, jobs):
            if verbose and out:
                print(out)
    if force or jobs or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose or a.ptxas_info, a.ptxas_info))
