"""Autotuner: picks the launch shape of each neighbour kernel per size bucket.

The library compiles lambda, delta, xsph+normals and the anisotropic pass in
several launch shapes (threads per block x minimum resident blocks per SM, i.e.
particles per block and the register budget); all shapes compute the same bits.
For every size bucket this steps a seeded dam-break scene of that size (the
served workload's scenes, with surface tension on so the normals pass runs),
frame by frame with the shapes of one kernel taking turns, and reads that
kernel's device time per launch from the library's per-kernel CUDA events. The
fastest shape per (kernel, bucket) goes into the library's table (p4a_tune_set)
and into tuning.json next to this file, which the library applies when it is
loaded.

The batched launches of lambda, delta and xsph+normals (p4a_batch_step) have tables
of their own, keyed by the frame's total particles: their register budget differs
from the plain launches' (each warp also carries its work-item state). For each
batched bucket this admits a seeded mix of scenes (configs.batched_mix with that
many scenes) into one Batch and times the shapes, taking turns, on whole batched
frames with the batch's per-kernel events.

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
BATCHED = {"lambda_batched": 4, "delta_batched": 5, "xsph_normals_batched": 6}
PROFILE_NAME = {"lambda_batched": "lambda", "delta_batched": "delta", "xsph_normals_batched": "xsph_normals"}
# bucket upper bounds (particles) and the scene size measured for each
BUCKETS = [(24_000, 12_000), (96_000, 48_000), (384_000, 192_000), (1_536_000, 768_000), (1 << 40, 2_000_000)]
# batched buckets: upper bound of a frame's total particles and the scene count of
# the seeded mix measured for it (96 scenes: about 6.0 M particles)
BATCH_BUCKETS = [(3_000_000, 24), (1 << 40, 96)]


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
        k = KERNELS[name] if name in KERNELS else BATCHED[name]
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


def interleaved(step, profile, L, kernel, name, variants, rounds):
    """Device ms per launch of kernel `name` for each shape in `variants`: every
    round steps one frame with each shape in turn (the order rotated per round),
    so that all shapes are timed over the same stretch of the scene's motion
    (later frames of a settling scene cost more, and timing the shapes one after
    another favoured the ones timed first)."""
    ms = [0.0] * len(variants)
    launches = [0] * len(variants)
    for r in range(rounds):
        order = list(range(len(variants)))
        order = order[r % len(order):] + order[:r % len(order)]
        for q in order:
            L.p4a_tune_clear(kernel)
            L.p4a_tune_set(kernel, 1 << 40, variants[q])
            prof = profile(step)
            if name in prof:
                ms[q] += prof[name][0]
                launches[q] += prof[name][1]
    # a shape whose frames launched the kernel never is not a candidate
    return [m / n if n else float("inf") for m, n in zip(ms, launches)]


def _sim_profile(sim, aniso):
    """(run, step) for interleaved(): one frame of the Sim (step + aniso) and its
    per-kernel profile."""
    def run(step):
        sim.profile_reset()
        step()
        sim.synchronize()
        return sim.profile_read()
    sim.profile(True)
    return run, lambda: (sim.step(1 / 60), sim.aniso(aniso))


def _mix_batch(scenes):
    from . import Batch, configs
    from .batch import arena_sizes
    mix = configs.batched_mix(count=scenes)
    b = Batch(**arena_sizes(mix))
    ids = [b.add_scene(p, sc) for p, sc in mix]
    return b, ids, sum(sc["pos"].shape[0] for _, sc in mix)


def _batch_profile(b, ids):
    """(run, step) for interleaved(): one batched frame of all scenes and its
    per-kernel profile."""
    def run(step):
        b.profile_reset()
        step()
        b.synchronize()
        return b.profile_read()
    b.profile(True)
    return run, lambda: b.step(ids, 1 / 60)


def tune_batched(result, L, buckets=BATCH_BUCKETS, frames=4, log=print):
    """Fills result["kernels"] / ["measured"] for the batched tables."""
    for name in BATCHED:
        result["kernels"][name] = []
        result["shapes"][name] = shapes(L, BATCHED[name])
    for bound, scenes in buckets:
        b, ids, total = _mix_batch(scenes)
        for _ in range(2):
            b.step(ids, 1 / 60)
        run, step = _batch_profile(b, ids)
        per = {}
        for name, k in BATCHED.items():
            variants = list(range(len(result["shapes"][name])))
            times = interleaved(step, run, L, k, PROFILE_NAME[name], variants, frames)
            best = min(range(len(times)), key=times.__getitem__)
            L.p4a_tune_clear(k)
            L.p4a_tune_set(k, 1 << 40, best)
            per[name] = {"ms_per_launch": [round(x, 5) for x in times], "best": best}
            log(f"batch {total:>9} {name:21s} " + " ".join(f"{x * 1e3:7.1f}" for x in times) + f"  -> {best}")
        b.close()
        result["measured"][f"batch_{total}"] = per
        for name in BATCHED:
            result["kernels"][name].append([bound, per[name]["best"]])


def tune(buckets=BUCKETS, frames=6, path=DEFAULT_PATH, log=print, batch_buckets=BATCH_BUCKETS):
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
        for _ in range(2):
            sim.step(1 / 60)
            sim.aniso(aniso)
        run, step = _sim_profile(sim, aniso)
        per = {}
        for name, k in KERNELS.items():
            variants = list(range(len(result["shapes"][name])))
            times = interleaved(step, run, L, k, name, variants, frames)
            best = min(range(len(times)), key=times.__getitem__)
            L.p4a_tune_clear(k)
            L.p4a_tune_set(k, 1 << 40, best)
            per[name] = {"ms_per_launch": [round(x, 5) for x in times], "best": best}
            log(f"n={real_n:>9} {name:13s} " + " ".join(f"{x * 1e3:7.1f}" for x in times) + f"  -> {best}")
        sim.close()
        result["measured"][str(real_n)] = per
        for name in KERNELS:
            result["kernels"][name].append([bound, per[name]["best"]])
    if batch_buckets:
        L.p4a_tune_clear(-1)
        apply(result, L)  # the plain tables as measured, then the batched ones on top
        tune_batched(result, L, batch_buckets, log=log)
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
    ap.add_argument("--no-batched", action="store_true", help="tune the plain launches only")
    a = ap.parse_args(argv)
    b = [x for x in BUCKETS if a.max_n is None or x[1] <= a.max_n]
    tune(b, a.frames, a.out, batch_buckets=None if a.no_batched else BATCH_BUCKETS)
    return 0


if __name__ == "__main__":
    sys.exit(main())
