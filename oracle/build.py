"""Build recipe for the CPU oracle (liboracle_p4a.so), a test-only library.

g++ with -ffp-contract=off so that the only fused multiply-adds are the explicit
fmaf calls of the arithmetic contract in p4a_oracle.h; OpenMP over particles.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "p4a_oracle.cpp")
OUT = os.path.join(HERE, "liboracle_p4a.so")
FLAGS = ["-std=c++17", "-O3", "-mavx2", "-mfma", "-ffp-contract=off", "-fno-fast-math",
         "-fopenmp", "-fPIC", "-shared", "-Wall"]


def build(force=False):
    deps = [SRC, os.path.join(HERE, "p4a_oracle.h"),
            os.path.join(HERE, "..", "include", "p4a.h")]
    if not force and os.path.exists(OUT) and all(
            os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps):
        return OUT
    cmd = ["g++"] + FLAGS + ["-o", OUT, SRC]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
