"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/mgpcg_oracle.cpp`` (the solver and the pressure Strategy)
and ``oracle/simulator_oracle.cpp`` (the other Strategies and the pressure
update) into ``oracle/_build/libmgpcg_oracle.so`` with OpenMP.  ``-ffp-contract=off`` keeps every multiply and add a separate
IEEE operation, as written in the restatement.

The reference (Taichi DSL Python) has no compiled form, so ``oracle/_ref`` is
never produced.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, "mgpcg_oracle.cpp"), os.path.join(HERE, "simulator_oracle.cpp")]
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libmgpcg_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(s) for s in SRCS):
        return OUT
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           *SRCS, "-o", OUT + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
