"""Build the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

g++ with -ffp-contract=off so single-precision expressions are evaluated operation by operation,
in the order the reference's generated WGSL writes them. OpenMP parallelises over cells /
triangles; the arithmetic of each cell does not depend on the thread count.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRC = os.path.join(HERE, "wt_oracle.cpp")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(
        os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "..", "include", "wt.h"))
    ):
        return LIB
    cmd = [
        "g++", "-std=c++17", "-O2", "-mf16c", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
        "-fPIC", "-shared", "-Wall", "-Wno-unknown-pragmas", SRC, "-o", LIB + ".tmp",
    ]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
