"""Builds the in-tree CUDA library ``libmgpcg_b200.so`` for sm_100a.

One translation unit (csrc/mg_plan.cu, which includes the kernel headers)
compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``.  The CUDA
runtime is linked statically, so the library needs only the driver at run
time.  The output sits next to this file so that it travels with the
repository to the GPU machine.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmgpcg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-shared",
]


def sources():
    return [os.path.join(CSRC, "mg_plan.cu"), os.path.join(CSRC, "mg_static.cu")]


def deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  [os.path.join(HERE, "..", "include", "mgpcg_b200.h"), __file__])


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [NVCC] + FLAGS + list(extra) + sources() + ["-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=True, verbose=True, extra=extra))
