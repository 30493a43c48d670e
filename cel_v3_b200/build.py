"""Builds libcelgpu.so (sm_100a) in-tree with nvcc.

Usage: python -m cel_v3_b200.build [--verbose]
The library is written next to this file so that it travels with the
source tree; object files go to cel_v3_b200/_build/.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcelgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no multiply-add contraction anywhere in device code; the
# kernels already spell out every rounding with __dadd_rn/__dmul_rn, this
# keeps the remaining scalar code faithful too.
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
         "-I", INCLUDE, "--expt-relaxed-constexpr"]
SOURCES = ["api.cu", "spmv.cu", "blas1.cu", "pcg.cu", "krylov.cu", "ir.cu", "ru.cu", "elm.cu", "noalloc.cu",
           "batched.cu", "selftest.cu", "multirhs.cu", "adjoint.cu", "dist.cu", "dist_solve.cu", "assemble.cu",
           "blockjacobi.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "celgpu.h"))
    return hs


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _newer(o, [s] + headers) or ptxas_info:
            cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0 or verbose or ptxas_info:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(cmd[-3])
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if _newer(LIB, objs) or jobs:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
