"""Builds libp4a.so (the CUDA sm_100a kernels + C ABI) in-tree with nvcc.

--fmad=false keeps the device arithmetic to the explicit fmaf() calls of the
float contract (p4a_internal.h); host code is compiled with -ffp-contract=off
for the same reason. The CUDA runtime is linked statically, so the library
needs only the driver at run time.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libp4a.so")
INCLUDE = os.path.join(HERE, "..", "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler",
              "-fPIC,-fopenmp,-ffp-contract=off,-Wall", "-shared", "-cudart", "static"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(INCLUDE, "p4a.h")]


def up_to_date():
    return os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in _deps())


def build(force=False, verbose=False, ptxas_v=False):
    if not force and up_to_date():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_v else []) + \
        ["-I", CSRC, "-o", OUT] + sources() + ["-lgomp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv))
