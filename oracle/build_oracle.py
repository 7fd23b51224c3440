"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/mgpcg_oracle.cpp`` into ``oracle/_build/libmgpcg_oracle.so``
with OpenMP.  ``-ffp-contract=off`` keeps every multiply and add a separate
IEEE operation, as written in the restatement.

The reference (Taichi DSL Python) has no compiled form, so ``oracle/_ref`` is
never produced.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "mgpcg_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libmgpcg_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           SRC, "-o", OUT + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
