#!/usr/bin/env python
"""bench.py — particle-substeps/s of the Particles4All simulation step on B200.

Default workload (the headline): the seeded 96-scene mix (batched_mix_96: ~6.0 M
particles, counts log-uniform in 4k-256k, boxes of 16-64 cells, 0-6 rigid cubes,
surface tension on about half, 4 iterations, 2 substeps per 1/60 s frame) stepped
as ONE batch (one launch per pass for all scenes, CUDA-graph frames), beside the
plain per-scene loop (96 Sim handles stepped one after the other) on the same GPU.
One step = one frame of every scene. The line also carries the large single scene
with the hose (large_hose_2m) as `large_hose_2m`, the served Poisson workload, the
render passes and the CPU baseline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # the reference's algorithm on the host cores

--workload batched_mix_96 (default) | large_hose_2m | medium_bodies_264k | dam_break_32k.

Multi-GPU: scenes are independent, so N GPUs run N replicas (weak scaling); no
data-path collective. Device time is measured with CUDA events on the stream the
kernels run on, max over ranks. Prints one JSON line on rank 0.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-substeps/s"
MIX = "batched_mix_96"
L2_FLUSH_BYTES = 256 << 20
# Algorithmic bytes per particle and launch (fixed formula of the workload
# definition: neighbour re-reads are not counted).
ALGO_BYTES = {
    "key_count": 36,        # R pos, vel; W key
    "fill": 12,             # R key, rank; W unordered
    "reorder": 84,          # R key, pos, vel; W pos, vel, pred   (+64 with bodies)
    "lambda": 24,           # R pred; W density, lambda
    "delta": 36,            # R pred, lambda; W pred
    "xsph_finalize": 68,    # R pos, pred, density; W vel, pos
    "xsph_normals": 56,     # tension scenes: the extra normal pass (R pred, vel, rho; W corr, normal)
    "tension_finalize": 68,
    "aniso": 64,            # R pos; W smoothPos, G
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=MIX)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--io-groups", type=int, default=0,
                    help="frames per step of the mix's e2e run (0: chosen by p4a_batch_step_io)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-scene loop of the mix")
    ap.add_argument("--no-large", action="store_true", help="skip the large_hose_2m sub-line")
    ap.add_argument("--large-steps", type=int, default=40)
    ap.add_argument("--no-render", action="store_true", help="skip the mesh / SSFR / ray-march timings")
    ap.add_argument("--only-render", action="store_true",
                    help="profiling aid: the workload scene, a few steps, then the render-pass timings alone")
    ap.add_argument("--only-mix", choices=["batched", "plain"], default=None,
                    help="step the 96-scene mix only (one Batch, or 96 plain Sims) for --mix-frames "
                         "frames and exit; for profiling the two forms")
    ap.add_argument("--mix-frames", type=int, default=10)
    ap.add_argument("--lanes", type=int, default=2, choices=[1, 2, 3, 4],
                    help="frame lanes of the batched mix (2: a frame runs as two concurrent halves)")
    ap.add_argument("--mix-scenes", type=int, default=96,
                    help="with --only-mix: the first N scenes of the seeded mix (a smaller case for profiling)")
    ap.add_argument("--serve-seconds", type=float, default=15.0,
                    help="length of each served-workload run (batched, then plain); 0 skips it")
    ap.add_argument("--serve-budget-gb", type=float, default=160.0)
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def workload(name):
    from particles4all_b200 import configs
    params, scene = configs.WORKLOADS[name]()
    aniso = configs.medium_aniso_params() if name.startswith("medium") else None
    return params, scene, aniso


def hose_for(params, scene):
    """The workload's hose (2,048 particles per step at 3 m/s until the pour budget
    is used), or None."""
    from particles4all_b200 import configs
    budget = int(scene.get("pour_budget", 0) or 0)
    if budget <= 0:
        return None
    return configs.Hose(params["box"], params["spacing"], per_step=2048, speed=3.0, limit=budget)


def pour(sim, hose):
    """One hose layer: emitted on the device for the library's Sim (p4a_hose_emit),
    computed on the host and appended for the oracle (the same bits)."""
    if hose is None:
        return 0
    if hasattr(sim, "hoseEmit"):
        return sim.hoseEmit(hose)
    pos, vel = hose.emit()
    return 0 if pos is None else sim.appendFluid(pos, vel)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_value(kernel, wl, key):
    """The `key:` figure of the kernel's committed ncu summary for this workload."""
    path = os.path.join(ROOT, "profiles", f"ncu_{kernel}_{wl}.txt")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError):
        pass
    return None


# FP32 work of a neighbour pass that counts only the pairs within h: ~33 neighbours
# per particle at h = 2 d, ~25 flops each (distance, kernel value and gradient, sums).
NEIGHBOUR_FLOP_PER_PARTICLE = 33 * 25
NEIGHBOUR_KERNELS = ("lambda", "delta", "xsph_normals", "tension_finalize", "xsph_finalize")


def fp32_peak_tflops():
    """Nominal FP32 rate: 148 SMs x 128 FP32 lanes x 2 flops (FMA) x the max SM clock."""
    mhz = 1965.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f).get("sm_max_mhz", mhz))
    except (OSError, ValueError):
        pass
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.lines, self.proc = gpu, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for ts, line in self.lines:
            if not (t0 <= ts <= t1 + 0.05):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                sm.append(float(f[2])); mx.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _launches():
    from particles4all_b200 import _lib
    return _lib.lib().p4a_kernel_launches()


def kernel_table(kern, particles_per_launch, peak):
    """Per-kernel share, time per launch and HBM fraction (algorithmic bytes per
    launch / average launch time). particles_per_launch(k) -> (particles, bytes per
    particle) of one launch of kernel k."""
    total_ms = sum(v[0] for v in kern.values()) or 1.0
    out = {}
    for k, (ms, nl) in sorted(kern.items(), key=lambda kv: -kv[1][0]):
        row = {"ms_total": round(ms, 4), "launches": nl, "share": round(ms / total_ms, 4),
               "us_per_launch": round(ms / max(1, nl) * 1000, 2)}
        n, bpp = particles_per_launch(k)
        if bpp and n:
            gbs = bpp * n / (ms / max(1, nl) / 1000.0) / 1e9
            row.update({"algorithmic_bytes_per_launch": int(bpp * n), "algorithmic_gbs": round(gbs, 1),
                        "hbm_frac": round(gbs / peak, 4)})
        out[k] = row
    return out


def roofline_of(kern, particles_per_launch, wl):
    """Roofline of the dominant kernel of the timed region."""
    peak, peak_kind = peaks()
    name, (kms, kl) = max(kern.items(), key=lambda kv: kv[1][0])
    n, bpp = particles_per_launch(name)
    avg_s = kms / max(1, kl) / 1000.0
    algo = bpp * n
    achieved = algo / avg_s / 1e9
    traffic = committed_value(name, wl, "dram_bytes_per_launch")
    r = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
         "frac": achieved / peak, "traffic": traffic,
         "traffic_source": "committed ncu summary" if traffic is not None else None,
         "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo, "avg_launch_us": avg_s * 1e6,
         "timing": "CUDA events around every launch inside the timed steps (event-record nodes in the "
                   "replayed graphs of a batched frame)",
         "kernels": kernel_table(kern, particles_per_launch, peak)}
    issue = committed_value(name, wl, "issue_active_pct")
    l2 = committed_value(name, wl, "l2_hit_pct")
    if issue is not None or l2 is not None:
        r["ncu"] = {"issue_frac": None if issue is None else issue / 100.0, "l2_hit_pct": l2,
                    "source": "committed ncu summary", "file": f"profiles/ncu_{name}_{wl}.txt"}
    if name in NEIGHBOUR_KERNELS:
        tf = NEIGHBOUR_FLOP_PER_PARTICLE * n / avg_s / 1e12
        r["fp32"] = {"achieved_tflops": tf, "peak_tflops": fp32_peak_tflops(), "frac": tf / fp32_peak_tflops(),
                     "flop_per_particle": NEIGHBOUR_FLOP_PER_PARTICLE,
                     "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 x max SM clock",
                     "what": "FP32 work of the pairs within h only; neither this nor HBM bounds the pass"}
        r["note"] = ("the neighbour passes are bound by instruction issue and the latency of the neighbour "
                     "gathers, not HBM (their working set is mostly L2-resident)")
    return r


def bytes_per_particle_substep(iterations, bodies, tension):
    """The workload definition's fixed algorithmic bytes per particle-substep:
    sort 36 + 4 + 84, k x (lambda 24 + delta 36), finish 68, +64 with bodies,
    +56 with tension."""
    return 36 + 4 + 84 + iterations * (24 + 36) + 68 + (64 if bodies else 0) + (56 if tension else 0)


# ---------------------------------------------------------------------------
# the 96-scene mix


def mix_arenas(mix):
    """Batch arena sizes that hold the whole mix."""
    from particles4all_b200.batch import arena_sizes
    return arena_sizes(mix)


def mix_config(mix, world):
    """The workload's `config`, the same dict in both arms."""
    n = [sc["pos"].shape[0] for _, sc in mix]
    return {"workload": MIX, "scenes": len(mix), "n_particles": int(sum(n)),
            "particles_per_scene": [int(min(n)), int(max(n))],
            "scenes_with_tension": sum(1 for p, _ in mix if p["surfaceTensionK"] > 0),
            "scenes_with_bodies": sum(1 for _, sc in mix if sc["n_bodies"] > 0),
            "rigid_bodies": int(sum(sc["n_bodies"] for _, sc in mix)),
            "iterations": 4, "substeps_per_frame": 2, "seed": 12,
            "step": "one 1/60 s frame of every scene",
            "l2": "inputs larger than L2 (about 3.6 GB of state); L2 also flushed between timed steps",
            "parallelism": f"replicas x{world}"}


def mix_scene_flags(mix):
    return [(sc["pos"].shape[0], sc["n_bodies"] > 0, p["surfaceTensionK"] > 0,
             int((sc["phase"][:, 0] > 0).sum())) for p, sc in mix]


def only_mix(form, frames, scenes=96, lanes=2):
    """The mix (its first `scenes` scenes) stepped in one form only: admission (or
    reset) then `frames` frames."""
    import torch
    from particles4all_b200 import Batch, Sim, configs
    mix = configs.batched_mix(count=scenes)
    stream = torch.cuda.Stream()
    t0 = time.perf_counter()
    if form == "batched":
        b = Batch(**mix_arenas(mix))
        b.set_stream(stream.cuda_stream)
        b.set_lanes(lanes)
        ids = [b.add_scene(p, sc) for p, sc in mix]
        for _ in range(frames):
            b.step(ids, 1 / 60)
        b.synchronize()
        b.close()
    else:
        sims = []
        for p, sc in mix:
            sim = Sim()
            sim.set_stream(stream.cuda_stream)
            sim.reset_scene(p, sc)
            sims.append(sim)
        for _ in range(frames):
            for sim in sims:
                sim.step(1 / 60)
        torch.cuda.synchronize()
        for sim in sims:
            sim.close()
    print(json.dumps({"only_mix": form, "frames": frames, "scenes": len(mix),
                      "wall_s": time.perf_counter() - t0}), flush=True)
    return 0


def run_mix(args):
    import torch
    from particles4all_b200 import Batch, Sim, _lib, configs
    from particles4all_b200.replicas import Replicas
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")  # replicas only: no collective on the data path
    mix = configs.batched_mix()
    flags = mix_scene_flags(mix)
    total = sum(f[0] for f in flags)
    stream = torch.cuda.Stream()
    b = Batch(device=local, **mix_arenas(mix))
    b.set_stream(stream.cuda_stream)
    b.set_lanes(args.lanes)
    t0 = time.perf_counter()
    ids = [b.add_scene(p, sc) for p, sc in mix]
    admit_s = time.perf_counter() - t0
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    warm = max(3, args.warmup)

    def sim_times():
        return [b.info(s)["sim_time"] for s in ids]

    def particle_substeps(t_before, t_after):
        return sum(n * round((t1 - t0_) * 120.0) for (n, *_), t0_, t1 in zip(flags, t_before, t_after))

    for _ in range(warm):
        b.step(ids, 1 / 60)
    b.synchronize()

    # timed frames (two frame lanes: each frame runs as two concurrent halves)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    tb = sim_times()
    launches0 = _launches()
    rep.barrier()
    torch.cuda.synchronize()
    w0 = time.time()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()  # L2 flush between timed frames (outside the events)
            starts[k].record(stream)
            b.step(ids, 1 / 60)
            ends[k].record(stream)
    torch.cuda.synchronize()
    rep.barrier()
    w1 = time.time()
    launches = _launches() - launches0
    clocks.stop()
    done = particle_substeps(tb, sim_times())
    # per-launch times: the next frames with an event around every launch (event-record
    # nodes in the replayed graphs); profiled frames run whole, on one lane
    prof_frames = max(4, args.steps // 2)
    b.profile(True)
    b.profile_reset()
    with torch.cuda.stream(stream):
        for k in range(prof_frames):
            flush.zero_()
            b.step(ids, 1 / 60)
    torch.cuda.synchronize()
    kern = b.profile_read()
    b.profile(False)
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    dev_ms_max = rep.max(dev_ms)
    value = world * done / (dev_ms_max / 1000.0)
    subs_per_frame = done / max(1, total) / args.steps

    n_plain = sum(f[0] for f in flags if not f[2])
    n_tension = sum(f[0] for f in flags if f[2])
    n_bodies_p = sum(f[0] for f in flags if f[1])

    def per_launch(k):
        if k in ("xsph_finalize",):
            return n_plain, ALGO_BYTES[k]
        if k in ("xsph_normals", "tension_finalize"):
            return n_tension, ALGO_BYTES[k]
        if k == "reorder":
            return total, ALGO_BYTES[k] + 64 * n_bodies_p / max(1, total)
        return total, ALGO_BYTES.get(k, 0)
    roofline = roofline_of(kern, per_launch, MIX)
    if roofline:
        roofline["timing"] = (f"CUDA events around every launch of {prof_frames} whole frames (event-record nodes "
                              "in the replayed frame graphs) right after the timed frames, which run each frame "
                              "as two concurrent halves")

    # whole frame against the workload definition's fixed bytes per particle-substep
    frame_bytes = 0.0
    for (n, bod, ten, nbp), (p, _) in zip(flags, mix):
        cells = int(math.prod(math.ceil(x / (2 * p["spacing"])) for x in p["box"]))
        frame_bytes += 2 * (n * bytes_per_particle_substep(4, bod, ten) + nbp * 88 * 4 + 8 * cells)
    peak, peak_kind = peaks()
    step_ach = frame_bytes * args.steps / (dev_ms / 1000.0) / 1e9
    step_roofline = {"bound": "hbm", "achieved": step_ach, "peak": peak, "unit": "GB/s", "frac": step_ach / peak,
                     "peak_source": peak_kind, "algorithmic_bytes_per_frame": frame_bytes,
                     "what": "whole batched frame: the fixed algorithmic bytes of every scene over the "
                             "device time of the timed frames"}

    # end to end through the batch C ABI: host state in, frame, host state out
    e2e = None
    if not args.no_e2e:
        e2e = mix_e2e(b, ids, flags, max(3, min(args.steps, 10)), rep, world, args.io_groups)

    plain = None
    if world == 1 and not args.no_plain:
        plain = mix_plain(mix, stream, flush, warm, args.steps)
        plain["speedup"] = value / plain["value"]
    b.close()

    large = None
    if world == 1 and not args.no_large:
        large = single_scene("large_hose_2m", args.large_steps, warm, rep, world, local,
                             e2e_on=not args.no_e2e, render=False)

    served = None
    if world == 1 and args.serve_seconds > 0:
        try:
            served = served_bench(args.serve_seconds, args.serve_budget_gb)
        except Exception as e:  # the headline line is still printed
            served = {"error": f"{type(e).__name__}: {e}"}

    render = None
    if world == 1 and not args.no_render:
        render = medium_render(warm)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_mix(mix, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": mix_config(mix, world),
            "form": "batched: one launch per pass for all 96 scenes, persistent work-item kernels, "
                    "CUDA-graph frames",
            "substeps_per_step": subs_per_frame,
            "roofline": roofline, "step_roofline": step_roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "admit_s": admit_s,
            "plain": plain, "large_hose_2m": large, "served": served, "render": render,
            "clocks": clocks.summary(w0, w1),
        }
        print(json.dumps(line), flush=True)
    rep.close()
    return 0


def mix_e2e(b, ids, flags, frames, rep, world, groups=0):
    """Per frame through the public batch API: every scene's pos and vel written
    from pinned host memory, the batched frame, pos and vel read back to pinned
    host memory, all waited for. The state read back is the next frame's input.
    Timed twice: through p4a_batch_step_io (the scenes in `groups` frames, the
    copies of each group overlapping the frames of the others; the reported
    value) and as write_async, p4a_batch_step, read_async on the batch's stream."""
    import torch
    caps = [f[0] for f in flags]
    total = sum(caps)
    bufs = [torch.empty(total * 8, dtype=torch.float32, pin_memory=True) for _ in range(2)]
    offs = []
    o = 0
    for n in caps:
        offs.append(o)
        o += n * 8
    src = bufs[0]
    for s, n, off in zip(ids, caps, offs):
        base = src.data_ptr() + off * 4
        b.read_async(s, "pos", base, n * 16)
        b.read_async(s, "vel", base + n * 16, n * 16)
    b.synchronize()

    cur = [0]  # the buffer holding the latest state read back

    def frame(overlap):
        hin, hout = bufs[cur[0]], bufs[cur[0] ^ 1]
        cur[0] ^= 1
        if overlap:
            entries = []
            for s, n, off in zip(ids, caps, offs):
                bi, bo = hin.data_ptr() + off * 4, hout.data_ptr() + off * 4
                entries.append((s, bi, bi + n * 16, bo, bo + n * 16))
            b.step_io(entries, 1 / 60, groups)
        else:
            for s, n, off in zip(ids, caps, offs):
                base = hin.data_ptr() + off * 4
                b.write_async(s, "pos", base, n * 16)
                b.write_async(s, "vel", base + n * 16, n * 16)
            b.step(ids, 1 / 60)
            for s, n, off in zip(ids, caps, offs):
                base = hout.data_ptr() + off * 4
                b.read_async(s, "pos", base, n * 16)
                b.read_async(s, "vel", base + n * 16, n * 16)
        b.synchronize()

    # the two forms alternate frame by frame, so that both see the same stage of
    # the scenes' motion (later frames of the mix cost more); one untimed frame of
    # each first captures its frame graphs
    frame(False)
    frame(True)
    el = [0.0, 0.0]
    done = [0, 0]
    for k in range(2 * frames):
        form = k & 1
        tb = [b.info(s)["sim_time"] for s in ids]
        rep.barrier()
        t0 = time.perf_counter()
        frame(bool(form))
        t1 = time.perf_counter()
        el[form] += rep.max(t1 - t0)
        done[form] += sum(n * round((b.info(s)["sim_time"] - t) * 120.0) for s, n, t in zip(ids, caps, tb))
    serial, value = world * done[0] / el[0], world * done[1] / el[1]
    h2d = d2h = 32 * total
    return {"value": value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": frames, "io_groups": groups or "auto",
            "serial_value": serial,
            "what": "per frame through p4a_batch_step_io: every scene's pos+vel from pinned host memory, the "
                    "scenes stepped as consecutive frames of about equal particle counts with each group's "
                    "copies on two copy streams overlapping the other groups' frames, every scene's pos+vel "
                    "back to pinned host memory, p4a_batch_synchronize; wall clock, max over ranks. "
                    "serial_value: the same with write_async, one p4a_batch_step of all scenes and "
                    "read_async on the batch's stream; the two forms alternate frame by frame"}


def mix_plain(mix, stream, flush, warm, steps):
    """The same 96 scenes as 96 plain Sim handles stepped one after the other on one
    stream: device time per frame from CUDA events."""
    import torch
    from particles4all_b200 import Sim
    sims = []
    for p, sc in mix:
        sim = Sim()
        sim.set_stream(stream.cuda_stream)
        sim.reset_scene(p, sc)
        sims.append(sim)
    for _ in range(warm):
        for sim in sims:
            sim.step(1 / 60)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    done = 0
    launches0 = _launches()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            for sim in sims:
                done += sim.info()["n"] * sim.step(1 / 60)
            ends[k].record(stream)
    torch.cuda.synchronize()
    launches = _launches() - launches0
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    for sim in sims:
        sim.close()
    return {"value": done / (ms / 1000.0), "unit": METRIC, "ms_per_step": ms / steps, "steps": steps,
            "launches_per_step": launches / steps,
            "what": "the same 96 scenes as 96 Sim handles, p4a_step one after the other on one stream; "
                    "CUDA events per frame, L2 flushed between frames"}


def served_bench(seconds, budget_gb):
    """The served workload (Poisson creates at 200/s, 2k-512k particles, 60 Hz
    closed-loop step requests, exp(10 s) lifetimes, positions read back every 4th
    step) for `seconds` against the batched server, then the same trace against
    the plain per-scene server. Arenas sized for min(budget, free device memory)."""
    import torch
    from particles4all_b200 import loadgen
    from particles4all_b200.server import Server
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(budget_gb * 1e9, free - 16e9))
    out = {"workload": "poisson 200/s, n ~ logU[2k, 512k], 60 Hz closed-loop steps, exp(10 s) lifetimes, "
                       "pos readback every 4th step", "seconds": seconds, "arena_budget_bytes": budget}
    for mode in ("batched", "plain"):
        srv = Server(budget_bytes=budget, max_scenes=4096, plain=(mode == "plain"), builder_threads=10,
                     upload_bytes=4 << 30, readback_bytes=4 << 30)
        t0 = time.perf_counter()
        r = loadgen.run(srv, seconds, seed=4)
        st = srv.stats()
        srv.close()
        r.update({"server_p50_ms": st["step_p50_ms"], "server_p99_ms": st["step_p99_ms"],
                  "max_queued_creates": st["max_queued_creates"], "frames": st["frames"],
                  "mean_frame_scenes": st["mean_frame_scenes"], "gpu_seconds": st["gpu_seconds"],
                  "admit_p50_ms": st["admit_p50_ms"], "admit_p99_ms": st["admit_p99_ms"],
                  "kernel_launches": st["kernel_launches"], "wall_s": time.perf_counter() - t0})
        out[mode] = r
    out["speedup"] = out["batched"]["particle_substeps_per_s"] / max(1e-9, out["plain"]["particle_substeps_per_s"])
    return out


def render_bench(sim, params, stream, width=1920, height=1080, reps=5):
    """Device ms per call of the passes that consume the step's buffers, on the
    scene's current state: the surface mesh (resolution 128), the screen-space
    fluid rendering and the ray march at width x height (camera framing the box)."""
    import torch
    from particles4all_b200 import default_mesh, default_ray, default_ssfr
    from particles4all_b200.camera import Camera, frame_matrices
    m = frame_matrices(Camera().frame(params["box"]), width, height)
    sp = default_ssfr()
    sp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    rp = default_ray()
    rp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    mp = default_mesh()

    def timed(fn):
        for _ in range(2):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for e0, e1 in ev:
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return statistics.median(e0.elapsed_time(e1) for e0, e1 in ev)
    out = {"width": width, "height": height, "particles": sim.info()["n"],
           "mesh_ms": timed(lambda: sim.mesh(mp, wait=False)),
           "ssfr_ms": timed(lambda: sim.ssfr(sp)),
           "ray_ms": timed(lambda: sim.ray(rp)),
           "ray_field_ms": timed(lambda: sim.ray(dict(rp, use_surface=0))),
           "what": "device ms per call (median of 5): p4a_mesh at resolution 128, p4a_ssfr and p4a_ray at "
                   f"{width}x{height} on the scene after the timed steps (anisotropic pass already done); "
                   "ray_ms with the mesh surface pass (the default), ray_field_ms marching the field"}
    out["mesh_triangles"] = sim.mesh(mp)
    return out


def medium_render(warm):
    """The render passes on the medium scene after a few frames."""
    import torch
    from particles4all_b200 import Sim
    params, scene, aniso = workload("medium_bodies_264k")
    stream = torch.cuda.Stream()
    sim = Sim()
    sim.set_stream(stream.cuda_stream)
    sim.reset_scene(params, scene)
    for _ in range(warm):
        sim.step(1 / 60)
    sim.aniso(aniso)
    out = render_bench(sim, params, stream)
    out["workload"] = "medium_bodies_264k"
    sim.close()
    return out


def only_render(args):
    """The workload scene stepped a few frames (anisotropic pass included), then the
    render passes timed as in the full run."""
    import torch
    from particles4all_b200 import Sim, default_aniso
    name = "medium_bodies_264k" if args.workload == MIX else args.workload
    params, scene, aniso = workload(name)
    stream = torch.cuda.Stream()
    sim = Sim()
    sim.set_stream(stream.cuda_stream)
    sim.reset_scene(params, scene)
    for _ in range(max(1, args.warmup)):
        sim.step(1 / 60)
    sim.aniso(aniso or default_aniso())
    out = render_bench(sim, params, stream)
    sim.close()
    print(json.dumps({"only_render": out}), flush=True)
    return 0


# ---------------------------------------------------------------------------
# one scene


def single_scene(name, steps, warm, rep, world, local, e2e_on=True, render=False):
    """One scene stepped `steps` frames (hose and anisotropic pass as the workload
    has them), timed with CUDA events on the simulation's stream; per-kernel events
    inside the timed frames; e2e through the plain C ABI with host buffers."""
    import torch
    from particles4all_b200 import Sim, _lib
    params, scene, aniso = workload(name)
    stream = torch.cuda.Stream()
    sim = Sim(device=local)
    sim.set_stream(stream.cuda_stream)
    sim.reset_scene(params, scene)
    n0 = sim.info()["n"]
    hose = hose_for(params, scene)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    done = [0.0]
    appended = [0]

    def frame(between=None):
        appended[0] += pour(sim, hose)
        s = sim.step(1 / 60)
        if between is not None:
            between()
        if aniso:
            sim.aniso(aniso)
        done[0] += sim.info()["n"] * s
        return s

    for _ in range(warm):
        frame()
    sim.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    sim.profile(True)
    sim.profile_reset()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = _launches()
    rep.barrier()
    torch.cuda.synchronize()
    w0 = time.time()
    done[0] = 0.0
    subs = 0
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            subs += frame()
            ends[k].record(stream)
    torch.cuda.synchronize()
    rep.barrier()
    w1 = time.time()
    launches = _launches() - launches0
    clocks.stop()
    kern = sim.profile_read()
    sim.profile(False)
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    done_timed = done[0]
    dev_ms_max = rep.max(dev_ms)
    value = world * done_timed / (dev_ms_max / 1000.0)
    n_avg = done_timed / max(1, subs)
    info = sim.info()

    def per_launch(k):
        if k == "aniso":
            return n_avg, ALGO_BYTES[k]
        return n_avg, ALGO_BYTES.get(k, 0) + (64 if k == "reorder" and info["n_bodies"] else 0)
    roofline = roofline_of(kern, per_launch, name)

    k_it = max(1, int(params["iterations"]))
    bpp = bytes_per_particle_substep(k_it, info["n_bodies"] > 0, params.get("surfaceTensionK", 0) > 0)
    step_bytes = done_timed * bpp + subs * (info["n_body_parts"] * 88 * k_it + 8 * info["n_cells"])
    if aniso:
        step_bytes += steps * n_avg * 64
    peak, peak_kind = peaks()
    step_ach = step_bytes / (dev_ms / 1000.0) / 1e9
    step_roofline = {"bound": "hbm", "achieved": step_ach, "peak": peak, "unit": "GB/s", "frac": step_ach / peak,
                     "peak_source": peak_kind, "bytes_per_particle_substep": bpp,
                     "what": "whole step: fixed algorithmic bytes of the workload definition over the "
                             "device time of the timed steps"}

    e2e = None
    if e2e_on:
        L = _lib.lib()
        check = _lib.check
        h = sim._h
        cap = max(1, info["cap"])
        hp = torch.empty(cap * 4, dtype=torch.float32, pin_memory=True)
        hv = torch.empty(cap * 4, dtype=torch.float32, pin_memory=True)
        hs = torch.empty(8, dtype=torch.int32, pin_memory=True)
        nb0 = info["n"] * 16
        L.p4a_read(h, 0, -1, hp.data_ptr(), 0, nb0)
        L.p4a_read(h, 1, -1, hv.data_ptr(), 0, nb0)
        e_steps = max(3, min(steps, 20))
        rep.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done[0] = 0.0
        appended[0] = 0
        h2d = d2h = 0
        nb2 = [0]

        def read_state():
            # the step's pos / vel leave on the copy stream while the anisotropic
            # pass (which changes neither) runs
            nb2[0] = sim.info()["n"] * 16
            check(L.p4a_read_async(h, 0, -1, hp.data_ptr(), 0, nb2[0]), h, "read_async")
            check(L.p4a_read_async(h, 1, -1, hv.data_ptr(), 0, nb2[0]), h, "read_async")
        for _ in range(e_steps):
            nb = sim.info()["n"] * 16
            check(L.p4a_write(h, 0, -1, hp.data_ptr(), 0, nb), h, "write")
            check(L.p4a_write(h, 1, -1, hv.data_ptr(), 0, nb), h, "write")
            frame(read_state)
            check(L.p4a_read(h, 17, -1, hs.data_ptr(), 0, 32), h, "read")
            check(L.p4a_read_wait(h), h, "read_wait")
            h2d += 2 * nb
            d2h += 2 * nb2[0] + 32
        t1 = time.perf_counter()
        rep.barrier()
        el = rep.max(t1 - t0)
        e2e = {"value": world * done[0] / el, "unit": METRIC, "h2d_bytes_per_step": h2d // e_steps,
               "d2h_bytes_per_step": d2h // e_steps, "steps": e_steps,
               "what": "per step: live pos+vel written from pinned host, Sim.step (+ hose, + aniso as the "
                       "workload has them; the hose layer is emitted on the device), pos+vel read back to "
                       "pinned host on the copy stream (overlapping the anisotropic pass) and stats read back, "
                       "all waited for"}

    rend = render_bench(sim, params, stream) if render else None
    st = sim.get_stats()
    out = {"metric": METRIC, "value": value, "unit": METRIC, "steps": steps, "warmup": warm,
           "ms_per_step": dev_ms_max / steps,
           "config": {"workload": name, "n_particles": n0, "n_particles_end": info["n"],
                      "hose": "2,048 particles per step at 3 m/s" if hose else None,
                      "n_bodies": info["n_bodies"], "substeps_per_step": subs // max(1, steps),
                      "iterations": params["iterations"], "surface_tension": params["surfaceTensionK"],
                      "aniso_pass": bool(aniso),
                      "l2": "flushed between timed steps (256 MiB write outside the timed events)",
                      "parallelism": f"replicas x{world}"},
           "roofline": roofline, "step_roofline": step_roofline, "e2e": e2e, "gpu_launches": launches,
           "render": rend, "clocks": clocks.summary(w0, w1),
           "final_stats": {k: st[k] for k in ("avgRho", "maxRho", "maxSpeed")}}
    sim.close()
    return out


def run_single_line(args):
    import torch
    from particles4all_b200.replicas import Replicas
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    warm = max(3, args.warmup)
    out = single_scene(args.workload, args.steps, warm, rep, world, local, e2e_on=not args.no_e2e,
                       render=(world == 1 and not args.no_render and args.workload.startswith("medium")))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        params, scene, aniso = workload(args.workload)
        cpu = cpu_baseline_single(params, scene, aniso, args.cpu_seconds)
    if rank == 0:
        cfg = out.pop("config")
        line = {"metric": METRIC, "value": out.pop("value"), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": warm, "ms_per_step": out.pop("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": cfg, "cpu_baseline": cpu}
        for k in ("steps", "warmup", "metric", "unit"):
            out.pop(k, None)
        line.update(out)
        print(json.dumps(line), flush=True)
    rep.close()
    return 0


# ---------------------------------------------------------------------------
# the oracle on the host cores (CPU baseline and the reference arm)


def cpu_baseline_single(params, scene, aniso, seconds):
    """The oracle (a CPU restatement of the reference's passes) on one scene."""
    import oracle
    o = oracle.OracleSim()
    o.reset_scene(params, scene)
    hose = hose_for(params, scene)
    ps = 0.0
    subs = 0
    steps = 0
    t0 = time.perf_counter()
    while True:
        pour(o, hose)
        s = o.step(1 / 60)
        if aniso:
            o.aniso(aniso)
        subs += s
        ps += o.info()["n"] * s
        steps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    n = o.info()["n"]
    return {"value": ps / el, "unit": METRIC, "cores": oracle.threads(), "kind": "port",
            "sample": f"{steps} full steps ({subs} substeps{' + anisotropic pass' if aniso else ''}"
                      f"{' + hose' if hose else ''}) of the same scene ({n} particles at the end) in {el:.1f} s"}


def oracle_mix(mix):
    import oracle
    sims = []
    for p, sc in mix:
        o = oracle.OracleSim()
        o.reset_scene(p, sc)
        sims.append(o)
    return sims


def oracle_round(sims):
    """One substep (1/120 s) of every scene of the mix; returns particle-substeps."""
    ps = 0
    for o in sims:
        ps += o.info()["n"] * o.step(1 / 120)
    return ps


def cpu_baseline_mix(mix, seconds):
    """The oracle on the same 96 scenes: rounds of one substep of every scene."""
    import oracle
    sims = oracle_mix(mix)
    ps = 0
    rounds = 0
    t0 = time.perf_counter()
    while True:
        ps += oracle_round(sims)
        rounds += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    return {"value": ps / el, "unit": METRIC, "cores": oracle.threads(), "kind": "port",
            "sample": f"{rounds} rounds of one substep of each of the 96 scenes ({ps} particle-substeps) "
                      f"in {el:.1f} s, all host threads"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    import oracle
    if args.workload == MIX:
        from particles4all_b200 import configs
        mix = configs.batched_mix()
        sims = oracle_mix(mix)
        for _ in range(max(0, args.warmup)):
            oracle_round(sims)
        ps = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ps += oracle_round(sims)
        el = time.perf_counter() - t0
        value = ps / el
        sample = (f"each step one substep of every one of the 96 scenes (the mix's {ps // max(1, args.steps)} "
                  f"particle-substeps), {args.steps} steps timed, all host threads")
        config = mix_config(mix, world)
    else:
        params, scene, aniso = workload(args.workload)
        o = oracle.OracleSim()
        o.reset_scene(params, scene)
        hose = hose_for(params, scene)
        base = max(1, params["substeps"])
        # a step is the full frame, or one substep of it when K frames would not fit
        t0 = time.perf_counter()
        o.step(1 / 60)
        if aniso:
            o.aniso(aniso)
        frame_s = time.perf_counter() - t0
        frame = frame_s * (args.steps + args.warmup) <= 150.0
        dt = 1 / 60 if frame else (1 / 60) / base

        def one():
            if frame:
                pour(o, hose)
            s = o.step(dt)
            if aniso and frame:
                o.aniso(aniso)
            return o.info()["n"] * s
        for _ in range(max(0, args.warmup - 1)):
            one()
        ps = 0.0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ps += one()
        el = time.perf_counter() - t0
        value = ps / el
        n = o.info()["n"]
        sample = f"{'full frames' if frame else 'single substeps'} of the {n}-particle scene, all host threads"
        config = {"workload": args.workload, "n_particles": n}
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el * 1000 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": config,
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": oracle.threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.only_mix:
        return only_mix(args.only_mix, args.mix_frames, args.mix_scenes, args.lanes)
    if args.only_render:
        return only_render(args)
    if args.workload == MIX:
        return run_mix(args)
    return run_single_line(args)


if __name__ == "__main__":
    sys.exit(main())
