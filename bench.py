#!/usr/bin/env python
"""bench.py — particle-substeps/s of the Particles4All simulation step on B200.

One step = Sim.step(1/60) of the workload (2 substeps: grid sort, k PBF
iterations, rigid shape matching, XSPH, surface tension, finalize, stats) plus
the anisotropic-kernel pass the renderer runs per frame. Default workload: the
medium scene with rigid bodies (medium_bodies_264k: 262,144 fluid particles +
8 cubes of 216, tension, XSPH, anisotropic pass).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # the reference's algorithm on the host cores

Multi-GPU: scenes are independent, so N GPUs run N replicas (weak scaling); no
data-path collective. Device time is measured with CUDA events on the
simulation's stream, max over ranks. Prints one JSON line on rank 0.
"""
import argparse
import json
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
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="medium_bodies_264k")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mix", action="store_true", help="skip the 96-scene batched vs plain comparison")
    ap.add_argument("--no-render", action="store_true", help="skip the mesh / SSFR / ray-march timings")
    ap.add_argument("--mix-frames", type=int, default=10)
    ap.add_argument("--only-render", action="store_true",
                    help="profiling aid: the workload scene, a few steps, then the render-pass timings alone")
    ap.add_argument("--only-mix", choices=["batched", "plain"], default=None,
                    help="step the 96-scene mix only (one Batch, or 96 plain Sims) for --mix-frames "
                         "frames and exit; for profiling the two forms")
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
    if hose is None:
        return 0
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


def committed_issue(kernel, wl):
    """Issue-slot utilisation (smsp__issue_active, fraction of peak) of the kernel's
    committed ncu summary: the roof of an issue- and latency-bound pass."""
    v = committed_value(kernel, wl, "issue_active_pct")
    return None if v is None else v / 100.0


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


def committed_traffic(kernel, wl):
    """DRAM bytes per launch from the committed ncu summary of this kernel and workload."""
    path = os.path.join(ROOT, "profiles", f"ncu_{kernel}_{wl}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1].split()[0]))
    except OSError:
        pass
    return None


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


def mix_arenas(mix):
    """Batch arena sizes that hold the whole mix."""
    import math
    cap = sum((sc["pos"].shape[0] + 511) // 256 * 256 for _, sc in mix)
    cells = sum((int(math.prod(int(b) for b in p["box"])) // 2048 + 2) * 2048 for p, _ in mix)
    nbound = 0
    for p, _ in mix:
        nb = [max(2, math.ceil(b / p["spacing"]) + 1) for b in p["box"]]
        nbound += nb[0] * nb[1] * nb[2] - (nb[0] - 2) * (nb[1] - 2) * (nb[2] - 2)
    bodies = sum(sc["n_bodies"] + 1 for _, sc in mix)
    body_parts = sum(int((sc["phase"][:, 0] > 0).sum()) + 1 for _, sc in mix)
    return dict(max_particles=cap + 4096, max_cells=cells, max_scenes=len(mix) + 1, max_bodies=bodies + 8,
                max_boundary=nbound + 4096, max_body_parts=body_parts + 64)


def only_mix(form, frames):
    """The mix stepped in one form only: admission (or reset) then `frames` frames."""
    import torch
    from particles4all_b200 import Batch, Sim, configs
    mix = configs.batched_mix()
    stream = torch.cuda.Stream()
    t0 = time.perf_counter()
    if form == "batched":
        b = Batch(**mix_arenas(mix))
        b.set_stream(stream.cuda_stream)
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


def only_render(args):
    """The workload scene stepped a few frames (anisotropic pass included), then the
    render passes timed as in the full run."""
    import torch
    from particles4all_b200 import Sim, default_aniso
    params, scene, aniso = workload(args.workload)
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


def batched_mix_bench(frames, warmup):
    """The 96-scene mix stepped (a) as one batch (one launch per pass for all
    scenes, CUDA-graph frames) and (b) as the plain per-scene loop (96 Sim handles
    on the same stream, one after the other). Device time per frame from CUDA
    events; particle-substeps/s for both."""
    import torch
    from particles4all_b200 import Batch, Sim, configs
    mix = configs.batched_mix()
    total = sum(sc["pos"].shape[0] for _, sc in mix)
    stream = torch.cuda.Stream()
    b = Batch(**mix_arenas(mix))
    b.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    ids = [b.add_scene(p, sc) for p, sc in mix]
    admit_s = time.perf_counter() - t0
    sims = []
    for p, sc in mix:
        sim = Sim()
        sim.set_stream(stream.cuda_stream)
        sim.reset_scene(p, sc)
        sims.append(sim)

    def timed(fn, k):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        subs = 0
        for e0, e1 in ev:
            e0.record(stream)
            subs += fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return sum(e0.elapsed_time(e1) for e0, e1 in ev), subs

    def batched():
        b.step(ids, 1 / 60)
        return 2

    def plain():
        for sim in sims:
            sim.step(1 / 60)
        return 2
    timed(batched, warmup)
    timed(plain, warmup)
    launches0 = _launches()
    tb, sb = timed(batched, frames)
    lb = _launches() - launches0
    launches0 = _launches()
    tp, sp = timed(plain, frames)
    lp = _launches() - launches0
    for sim in sims:
        sim.close()
    b.close()
    vb = total * sb / (tb / 1000.0)
    vp = total * sp / (tp / 1000.0)
    return {"scenes": len(mix), "particles": total, "frames": frames, "substeps_per_frame": 2,
            "batched_value": vb, "plain_value": vp, "speedup": vb / vp, "unit": METRIC,
            "batched_ms_per_frame": tb / frames, "plain_ms_per_frame": tp / frames,
            "batched_launches_per_frame": lb / frames, "plain_launches_per_frame": lp / frames,
            "admit_s_total": admit_s}


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


def _launches():
    from particles4all_b200 import _lib
    return _lib.lib().p4a_kernel_launches()


def cpu_baseline(params, scene, aniso, seconds):
    """The oracle (a CPU restatement of the reference's passes) on this workload."""
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


def run_reference(args):
    rank, _, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    params, scene, aniso = workload(args.workload)
    o = oracle.OracleSim()
    o.reset_scene(params, scene)
    hose = hose_for(params, scene)
    n = o.info()["n"]
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
        return s, o.info()["n"] * s
    for _ in range(max(0, args.warmup - 1)):
        one()
    subs = 0
    ps = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s, p = one()
        subs += s
        ps += p
    el = time.perf_counter() - t0
    value = ps / el
    n = o.info()["n"]
    sample = (f"{'full frames' if frame else 'single substeps'} of the {n}-particle scene, "
              f"{subs} substeps timed, all host threads")
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el * 1000 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload, "n_particles": n, "substeps_per_step": subs // max(1, args.steps)},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": oracle.threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import numpy as np
    import torch
    from particles4all_b200 import Sim, _lib

    from particles4all_b200.replicas import Replicas
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")  # replicas only: no collective on the data path
    barrier, allmax = rep.barrier, rep.max

    params, scene, aniso = workload(args.workload)
    stream = torch.cuda.Stream()
    sim = Sim(device=local)
    sim.set_stream(stream.cuda_stream)
    sim.reset_scene(params, scene)
    n = sim.info()["n"]
    hose = hose_for(params, scene)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    done = [0.0]  # particle-substeps

    def frame(between=None):
        pour(sim, hose)
        s = sim.step(1 / 60)
        if between is not None:
            between()
        if aniso:
            sim.aniso(aniso)
        done[0] += sim.info()["n"] * s
        return s

    for _ in range(max(3, args.warmup)):
        frame()
    sim.synchronize()
    # per-kernel breakdown: a pass with a CUDA event around every launch, before the
    # timed pass (whose steps run without the extra event records)
    prof_steps = max(3, min(args.steps, 30))
    sim.profile(True)
    sim.profile_reset()
    done[0] = 0.0
    prof_subs = 0
    with torch.cuda.stream(stream):
        for _ in range(prof_steps):
            flush.zero_()
            prof_subs += frame()
    sim.synchronize()
    kern = sim.profile_read()
    sim.profile(False)
    prof_n_avg = done[0] / max(1, prof_subs)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = _lib.lib().p4a_kernel_launches()
    barrier()
    torch.cuda.synchronize()
    w0 = time.time()
    done[0] = 0.0
    subs = 0
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (not inside the events)
            starts[k].record(stream)
            subs += frame()
            ends[k].record(stream)
    torch.cuda.synchronize()
    barrier()
    w1 = time.time()
    launches = _lib.lib().p4a_kernel_launches() - launches0
    clocks.stop()
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    done_timed = done[0]
    dev_ms_max = allmax(dev_ms)
    value = world * done_timed / (dev_ms_max / 1000.0)

    # roofline of the dominant kernel (live per-kernel events of the timed region)
    top = max(kern.items(), key=lambda kv: kv[1][0])
    name, (kms, kl) = top
    total_ms = sum(x[0] for x in kern.values())

    def kernel_bytes(k):
        return ALGO_BYTES.get(k, 0) + (64 if k == "reorder" and sim.info()["n_bodies"] else 0)

    def kernel_line(k, v):
        """Per-kernel share and HBM fraction (algorithmic bytes / average launch time)."""
        out = {"ms_total": round(v[0], 4), "launches": v[1], "share": round(v[0] / total_ms, 4),
               "us_per_launch": round(v[0] / max(1, v[1]) * 1000, 2)}
        if kernel_bytes(k):
            gbs = kernel_bytes(k) * prof_n_avg / (v[0] / max(1, v[1]) / 1000.0) / 1e9
            out.update({"algorithmic_gbs": round(gbs, 1), "hbm_frac": round(gbs / peaks()[0], 4)})
        return out

    per_p = kernel_bytes(name)
    avg_s = kms / kl / 1000.0
    n_avg = done_timed / max(1, subs)  # mean particles per substep (grows with a hose)
    algo = per_p * prof_n_avg
    peak, peak_kind = peaks()
    achieved = algo / avg_s / 1e9
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": committed_traffic(name, args.workload),
                "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo,
                "issue_frac_ncu": committed_issue(name, args.workload),
                "l2_hit_pct_ncu": committed_value(name, args.workload, "l2_hit_pct"),
                "note": "the neighbour passes are bound by instruction issue and load latency, not HBM: "
                        "issue_frac_ncu is the kernel's issue-slot utilisation from its committed ncu summary",
                "avg_launch_us": avg_s * 1e6,
                "kernels": {k: kernel_line(k, v) for k, v in sorted(kern.items(), key=lambda kv: -kv[1][0])}}

    if name in NEIGHBOUR_KERNELS:
        tf = NEIGHBOUR_FLOP_PER_PARTICLE * prof_n_avg / avg_s / 1e12
        roofline["fp32"] = {"achieved_tflops": tf, "peak_tflops": fp32_peak_tflops(),
                            "frac": tf / fp32_peak_tflops(), "flop_per_particle": NEIGHBOUR_FLOP_PER_PARTICLE,
                            "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 x max SM clock",
                            "what": "FP32 work of the pairs within h only; neither this nor HBM bounds the pass"}

    # whole-step HBM roofline with the fixed per-particle-substep formula of the
    # workload definition: sort (36 + 4 + 84), k x (lambda 24 + delta 36), finish 68,
    # bodies +64 per particle and 88 x k per body particle, tension +56, scan 8 per
    # cell, and 64 per particle per frame for the anisotropic pass
    k_it = max(1, int(params["iterations"]))
    info_now = sim.info()
    bpp = 36 + 4 + 84 + k_it * (24 + 36) + 68 + (64 if info_now["n_bodies"] else 0) + \
        (56 if params.get("surfaceTensionK", 0) > 0 else 0)
    step_bytes = done_timed * bpp + subs * (info_now["n_body_parts"] * 88 * k_it + 8 * info_now["n_cells"])
    if aniso:
        step_bytes += args.steps * n_avg * 64
    step_achieved = step_bytes / (dev_ms / 1000.0) / 1e9
    step_roofline = {"bound": "hbm", "achieved": step_achieved, "peak": peak, "unit": "GB/s",
                     "frac": step_achieved / peak, "peak_source": peak_kind,
                     "bytes_per_particle_substep": bpp,
                     "what": "whole step: fixed algorithmic bytes of the workload definition over the "
                             "device time of the timed steps"}

    # end to end through the public API: host state in, step, host state out
    e2e = None
    if not args.no_e2e:
        L = _lib.lib()
        check = _lib.check
        h = sim._h
        cap = max(1, sim.info()["cap"])
        hp = torch.empty(cap * 4, dtype=torch.float32, pin_memory=True)
        hv = torch.empty(cap * 4, dtype=torch.float32, pin_memory=True)
        hs = torch.empty(8, dtype=torch.int32, pin_memory=True)
        nb0 = sim.info()["n"] * 16
        L.p4a_read(h, 0, -1, hp.data_ptr(), 0, nb0)
        L.p4a_read(h, 1, -1, hv.data_ptr(), 0, nb0)
        e_steps = max(3, min(args.steps, 50))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done[0] = 0.0
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
        barrier()
        el = allmax(t1 - t0)
        e2e = {"value": world * done[0] / el, "unit": METRIC, "h2d_bytes_per_step": h2d // e_steps,
               "d2h_bytes_per_step": d2h // e_steps, "steps": e_steps,
               "what": "per step: live pos+vel written from pinned host, Sim.step (+ hose, + aniso as the "
                       "workload has them), pos+vel read back to pinned host on the copy stream (overlapping "
                       "the anisotropic pass) and stats read back, all waited for"}

    render = None
    if world == 1 and aniso and not args.no_render:
        render = render_bench(sim, params, stream)

    mix = None
    if world == 1 and not args.no_mix:
        mix = batched_mix_bench(args.mix_frames, 3)

    served = None
    if world == 1 and args.serve_seconds > 0:
        try:
            served = served_bench(args.serve_seconds, args.serve_budget_gb)
        except Exception as e:  # the headline line is still printed
            served = {"error": f"{type(e).__name__}: {e}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(params, scene, aniso, args.cpu_seconds)

    if rank == 0:
        st = sim.get_stats()
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": dev_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": args.workload, "n_particles": n, "n_particles_end": sim.info()["n"],
                       "hose": "2,048 particles per step at 3 m/s" if hose else None,
                       "n_bodies": sim.info()["n_bodies"],
                       "substeps_per_step": subs // args.steps, "iterations": params["iterations"],
                       "surface_tension": params["surfaceTensionK"], "aniso_pass": bool(aniso),
                       "l2": "flushed between timed steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "step_roofline": step_roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches,
            "batched_mix": mix,
            "render": render,
            "served": served,
            "clocks": clocks.summary(w0, w1),
            "final_stats": {k: st[k] for k in ("avgRho", "maxRho", "maxSpeed")},
        }
        print(json.dumps(line), flush=True)
    sim.close()
    rep.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.only_mix:
        return only_mix(args.only_mix, args.mix_frames)
    if args.only_render:
        return only_render(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
