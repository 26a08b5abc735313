"""Test infrastructure: builds the checkers used by tests and bench.

1. ``oracle/liboracle_sph.so`` — the project's own C restatement of the
   reference SPH path (``oracle/sph_oracle.c``).
2. ``oracle/_ref/libemerald_ref.so`` — the UNMODIFIED emerald reference
   sources, compiled in place from the reference checkout against the
   project-written shims in ``oracle/ref_shim`` plus ``oracle/ref_harness.cpp``.
   The checkout is the directory named by ``--reference DIR`` or the
   ``EMERALD_REFERENCE_ROOT`` environment variable, else the build
   container's read-only copy at ``/root/reference``. Built only where that
   directory exists; the built file is git-ignored but travels with the
   working tree.

3. ``oracle/libfp64_oracle.so`` — the FP64 GPU oracle of the five solvers'
   sub-steps (``oracle/fp64/dfsph_fp64.cu``), which states the error of the
   FP32 results; used by tests only.

The first two are compiled ``-O2 -ffp-contract=off`` (IEEE single-precision
operations in source order, as the reference's own CMake build with
CXX_EXTENSIONS OFF gives on x86-64).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REF_ROOT = "/root/reference"


def reference_root(argv=()):
    """The reference checkout: ``--reference DIR`` in ``argv`` (this script's
    command line), else ``EMERALD_REFERENCE_ROOT``, else the build
    container's copy."""
    argv = list(argv)
    for k, a in enumerate(argv):
        if a == "--reference" and k + 1 < len(argv):
            return argv[k + 1]
        if a.startswith("--reference="):
            return a.split("=", 1)[1]
    return os.environ.get("EMERALD_REFERENCE_ROOT") or DEFAULT_REF_ROOT


REF_ROOT = reference_root()
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "liboracle_sph.so")
REF_SO = os.path.join(REF_OUT, "libemerald_ref.so")
FP64_SO = os.path.join(HERE, "libfp64_oracle.so")

REF_SOURCES = [
    "emerald/z_index/z_index.cpp",
    "emerald/sph_common/common.cpp",
    "emerald/sph_common/neighborhood.cpp",
    "emerald/sph_common/density.cpp",
    "emerald/sph_common/divergence.cpp",
    "emerald/sph_common/pressure.cpp",
    "emerald/sph_common/dynamics.cpp",
    "emerald/sph_common/cfl.cpp",
    "emerald/sph_common/volume.cpp",
    "emerald/sph2d_box/config.cpp",
    "emerald/sph2d_box/solids.cpp",
    "emerald/sph2d_box/initial_state.cpp",
    "emerald/sph2d_box/forces.cpp",
    "emerald/sph2d_box/colors.cpp",
    "emerald/sph2d_box/neighborhoods_from_state.cpp",
    "emerald/sph2d_box/iisph_ops.cpp",
    "emerald/sph2d_box/iisph_ap_ops.cpp",
    "emerald/sph2d_box/iisph_pseudo_ap_ops.cpp",
    "emerald/sph2d_box/dfsph_p_ops.cpp",
    "emerald/sph2d_box/pcisph_ops.cpp",
    "emerald/util/assert.cpp",
    "emerald/util/random.cpp",
]

CXXFLAGS = ["-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-w", "-pthread"]


def _run(cmd):
    subprocess.run(cmd, check=True)


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build_oracle(force=False):
    src = os.path.join(HERE, "sph_oracle.c")
    hdr = os.path.join(HERE, "sph_oracle.h")
    if not force and _newer(ORACLE_SO, [src, hdr, __file__]):
        return ORACLE_SO
    _run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-fopenmp",
          "-Wall", "-o", ORACLE_SO, src, "-lm"])
    return ORACLE_SO


def build_fp64(force=False):
    src = os.path.join(HERE, "fp64", "dfsph_fp64.cu")
    if not force and _newer(FP64_SO, [src, __file__]):
        return FP64_SO
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
          "-Xcompiler", "-fPIC", "-cudart", "static", "-o", FP64_SO, src])
    return FP64_SO


def build_reference(force=False):
    if not os.path.isdir(REF_ROOT):
        return REF_SO if os.path.exists(REF_SO) else None
    shim = os.path.join(HERE, "ref_shim")
    deps = [os.path.join(REF_ROOT, s) for s in REF_SOURCES]
    deps += [os.path.join(HERE, "ref_harness.cpp"), os.path.join(shim, "tbb_shim.cpp"), __file__]
    for root, _, files in os.walk(shim):
        deps += [os.path.join(root, f) for f in files]
    if not force and _newer(REF_SO, deps):
        return REF_SO
    os.makedirs(os.path.join(REF_OUT, "obj"), exist_ok=True)
    inc = ["-I", shim, "-I", REF_ROOT]
    jobs = []
    for s in REF_SOURCES:
        obj = os.path.join(REF_OUT, "obj", s.replace("/", "_") + ".o")
        jobs.append(["g++"] + CXXFLAGS + inc + ["-c", os.path.join(REF_ROOT, s), "-o", obj])
    for s in [os.path.join(HERE, "ref_harness.cpp"), os.path.join(shim, "tbb_shim.cpp")]:
        obj = os.path.join(REF_OUT, "obj", os.path.basename(s) + ".o")
        jobs.append(["g++"] + CXXFLAGS + inc + ["-c", s, "-o", obj])
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(_run, jobs))
    objs = [j[-1] for j in jobs]
    _run(["g++", "-shared", "-pthread", "-o", REF_SO] + objs)
    return REF_SO


def main():
    global REF_ROOT
    REF_ROOT = reference_root(sys.argv[1:])
    force = "--force" in sys.argv
    if os.path.exists(os.path.join(HERE, "sph_oracle.c")):
        print(build_oracle(force))
    print(build_fp64(force))
    print(build_reference(force))


if __name__ == "__main__":
    main()
