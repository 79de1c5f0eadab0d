"""Builds libp4a.so (the CUDA sm_100a kernels + C ABI) in-tree with nvcc.

--fmad=false keeps the device arithmetic to the explicit fmaf() calls of the
float contract (p4a_internal.h); host code is compiled with -ffp-contract=off
for the same reason. The CUDA runtime is linked statically, so the library
needs only the driver at run time. Each source compiles to its own object in
_build/ (in parallel, and only when it or a header changed), then one link.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libp4a.so")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(HERE, "..", "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler",
                 "-fPIC,-fopenmp,-ffp-contract=off,-Wall"]
LINK_FLAGS = ["-shared", "-cudart", "static"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(INCLUDE, "p4a.h")]


def _deps():
    return sources() + _headers()


def up_to_date():
    return os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in _deps())


def _obj(src):
    return os.path.join(OBJ, os.path.basename(src) + ".o")


def build(force=False, verbose=False, ptxas_v=False):
    if not force and up_to_date():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in _headers())

    def compile_one(src):
        o = _obj(src)
        if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(src), newest_header):
            return None
        cmd = [nvcc] + ARCH + COMPILE_FLAGS + (["-Xptxas", "-v"] if ptxas_v else []) + \
            ["-I", CSRC, "-c", src, "-o", o]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return (src, r.returncode, r.stdout + r.stderr)

    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = [r for r in ex.map(compile_one, srcs) if r is not None]
    failed = False
    for src, rc, out in results:
        if out.strip() and (rc != 0 or verbose or ptxas_v):
            sys.stderr.write(out)
        if rc != 0:
            failed = True
            sys.stderr.write(f"build: {os.path.basename(src)} failed\n")
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc")
    cmd = [nvcc] + ARCH + LINK_FLAGS + ["-o", OUT] + [_obj(s) for s in srcs] + ["-lgomp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv))
