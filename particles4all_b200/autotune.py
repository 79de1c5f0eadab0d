"""Autotuner: picks the launch shape of each neighbour kernel per size bucket.

The library compiles lambda, delta, xsph+normals and the anisotropic pass in
several launch shapes (threads per block x minimum resident blocks per SM, i.e.
particles per block and the register budget); all shapes compute the same bits.
For every size bucket this steps a seeded dam-break scene of that size (the
served workload's scenes, with surface tension on so the normals pass runs) with
each shape of one kernel in turn and reads that kernel's device time per launch
from the library's per-kernel CUDA events. The fastest shape per (kernel,
bucket) goes into the library's table (p4a_tune_set) and into tuning.json next
to this file, which the library applies when it is loaded.

    python -m particles4all_b200.autotune            # on the GPU: measure, write tuning.json
"""
import argparse
import ctypes as C
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PATH = os.path.join(HERE, "tuning.json")

KERNELS = {"lambda": 0, "delta": 1, "xsph_normals": 2, "aniso": 3}
# bucket upper bounds (particles) and the scene size measured for each
BUCKETS = [(24_000, 12_000), (96_000, 48_000), (384_000, 192_000), (1_536_000, 768_000), (1 << 40, 2_000_000)]


def shapes(L, kernel):
    t = (C.c_int32 * 16)()
    m = (C.c_int32 * 16)()
    cnt = C.c_int32()
    L.p4a_kernel_shapes(kernel, t, m, 16, C.byref(cnt))
    return [(t[k], m[k]) for k in range(cnt.value)]


def apply(table, L=None):
    """Loads {kernel name: [[max_particles, variant], ...]} into the library."""
    if L is None:
        from ._lib import lib
        L = lib()
    for name, buckets in table.get("kernels", {}).items():
        k = KERNELS[name]
        L.p4a_tune_clear(k)
        for bound, v in buckets:
            L.p4a_tune_set(k, int(bound), int(v))


def load(path=DEFAULT_PATH, L=None):
    try:
        with open(path) as f:
            table = json.load(f)
    except (OSError, ValueError):
        return None
    apply(table, L)
    return table


def _scene_sim(n):
    from . import Sim, default_aniso
    from .loadgen import scene_params
    p = scene_params(n, tension=0.5)
    s = Sim()
    s.reset(p)
    return s, default_aniso()


def measure(sim, aniso, frames=6, warmup=2):
    """Device ms per launch of every kernel over `frames` frames (step + aniso)."""
    for _ in range(warmup):
        sim.step(1 / 60)
        sim.aniso(aniso)
    sim.synchronize()
    sim.profile(True)
    sim.profile_reset()
    for _ in range(frames):
        sim.step(1 / 60)
        sim.aniso(aniso)
    sim.synchronize()
    prof = sim.profile_read()
    sim.profile(False)
    return {k: ms / max(1, n) for k, (ms, n) in prof.items()}


def tune(buckets=BUCKETS, frames=6, path=DEFAULT_PATH, log=print):
    from ._lib import lib
    L = lib()
    L.p4a_tune_clear(-1)
    result = {"kernels": {k: [] for k in KERNELS}, "measured": {}, "shapes": {}}
    for name, k in KERNELS.items():
        result["shapes"][name] = shapes(L, k)
    t0 = time.time()
    for bound, n in buckets:
        sim, aniso = _scene_sim(n)
        real_n = sim.info()["n"]
        per = {}
        for name, k in KERNELS.items():
            times = []
            for v in range(len(result["shapes"][name])):
                L.p4a_tune_clear(k)
                L.p4a_tune_set(k, 1 << 40, v)
                t = measure(sim, aniso, frames)[name]
                times.append(t)
            best = min(range(len(times)), key=times.__getitem__)
            L.p4a_tune_clear(k)
            L.p4a_tune_set(k, 1 << 40, best)
            per[name] = {"ms_per_launch": [round(x, 5) for x in times], "best": best}
            log(f"n={real_n:>9} {name:13s} " + " ".join(f"{x * 1e3:7.1f}" for x in times) + f"  -> {best}")
        sim.close()
        result["measured"][str(real_n)] = per
        for name in KERNELS:
            result["kernels"][name].append([bound, per[name]["best"]])
    result["seconds"] = round(time.time() - t0, 1)
    L.p4a_tune_clear(-1)
    apply(result, L)
    if path:
        with open(path, "w") as f:
            json.dump(result, f, indent=1)
    return result


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--frames", type=int, default=6)
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--max-n", type=int, default=None, help="skip buckets whose scene is larger")
    a = ap.parse_args(argv)
    b = [x for x in BUCKETS if a.max_n is None or x[1] <= a.max_n]
    tune(b, a.frames, a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
