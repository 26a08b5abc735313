"""Builds emerald_b200/libemerald_b200.so (CUDA for sm_100a + host C++).

Kernels are compiled with --fmad=false and IEEE division and square root
(nvcc's defaults otherwise), so every single-precision operation rounds
exactly as the reference's CPU code compiled with -ffp-contract=off.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libemerald_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["build_kernels.cu", "solve_kernels.cu", "sort_kernels.cu", "engine.cu", "capi.cu",
           "scene.cpp", "noalloc.cu", "reorder_kernels.cu", "server.cpp", "common_ops.cu",
           "solver_ops.cu", "sort_ops.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-O3",
]


def _nvcc():
    for cand in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.exists(cand) or cand == "nvcc":
            return cand
    return "nvcc"


def _deps():
    out = []
    for root, _, files in os.walk(CSRC):
        out += [os.path.join(root, f) for f in files]
    out.append(os.path.join(INCLUDE, "emerald_sph.h"))
    out.append(os.path.abspath(__file__))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    jobs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        cmd = [nvcc] + NVCC_FLAGS + ["-I", CSRC, "-I", INCLUDE, "-c", os.path.join(CSRC, src),
                                     "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc] + NVCC_FLAGS + ["-x", "cu", "-I", CSRC, "-I", INCLUDE, "-c",
                                         os.path.join(CSRC, src), "-o", obj]
        jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        logs = list(ex.map(run, jobs))
    if verbose:
        for log in logs:
            if log.strip():
                print(log)
    link = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
            "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
    run(link)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
