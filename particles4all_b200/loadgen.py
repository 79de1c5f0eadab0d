"""Seeded request traces for the serving loop (the served workload).

Scenes arrive as a Poisson process (`rate` per second) with particle counts
log-uniform in [n_lo, n_hi] and exponential lifetimes (mean `mean_life` s). Each
live scene has a client that wants `hz` steps per second: its next step is
submitted when the previous one has completed and 1/hz s have passed since that
one was submitted (so an overloaded server slows its clients down instead of
queueing without bound), and every `readback_every`-th step reads the scene's
positions back. A scene is destroyed when its lifetime, counted from admission,
has run out. Scenes are the reference's dam-break block (buildScene with
targetParticleCount = n) in a box sized for n, spacing 0.5, h = 1, rho0 = 1,
CFM epsilon 100, 4 iterations, 2 substeps per 1/60 s.

The trace (arrival gaps, sizes, lifetimes) depends only on the seed, so the batched
and the plain server see the same requests.
"""
import heapq
import math

import numpy as np

from .configs import _base_params


def scene_params(n, iterations=4, substeps=2, tension=0.0):
    """Params of an n-particle dam-break scene (built by the library's buildScene)."""
    d = 0.5
    s = math.ceil(n ** (1.0 / 3.0))
    box = [float(math.ceil(s * d / 0.35) + 1), 1.5 * s * d + 4.0, s * d + 2 * d + 1.0]
    p = _base_params(box, iterations=iterations, tension=tension, xsph=0.05, substeps=substeps)
    p["targetParticleCount"] = int(n)
    return p


def trace(seed, count, rate, n_lo, n_hi, mean_life):
    """(arrival offset s, particles, lifetime s) for `count` scenes."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    sizes = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), size=count)).round().astype(np.int64)
    lives = rng.exponential(mean_life, size=count)
    return list(zip(np.cumsum(gaps).tolist(), sizes.tolist(), lives.tolist()))


def run(server, duration, rate=200.0, n_lo=2000, n_hi=512000, mean_life=10.0, hz=60.0, readback_every=4,
        seed=0, drain_seconds=10.0, max_scenes=None):
    """Drives `server` with the trace for `duration` seconds of its clock, then stops
    submitting, waits for outstanding steps (at most drain_seconds) and destroys the
    live scenes. Returns client-side counts and latencies over the window."""
    arrivals = trace(seed, int(rate * duration * 1.5) + 16, rate, n_lo, n_hi, mean_life)
    if max_scenes is not None:
        arrivals = arrivals[:max_scenes]
    t0 = server.clock()
    period = 1.0 / hz
    live = {}      # sid -> dict(n, life, t_live, steps, busy, last_submit, buf)
    pending = {}   # create request -> (sid, n, life)
    due = []       # heap of (time, sid)
    lat, ps_window, done_steps = [], 0.0, 0
    created = rejected = admitted = 0
    k = 0
    end = t0 + duration

    def submit_step(sid, now):
        s = live[sid]
        s["steps"] += 1
        rb = s["steps"] % readback_every == 0
        server.step(sid, 1.0 / 60.0, pos_out=s["buf"] if rb else None)
        s["busy"] = True
        s["last_submit"] = now

    while True:
        now = server.clock()
        if now >= end:
            break
        while k < len(arrivals) and t0 + arrivals[k][0] <= now:
            _, n, life = arrivals[k]
            sid, req = server.create_scene(scene_params(n))
            pending[req] = (sid, n, life)
            created += 1
            k += 1
        next_t = min(t0 + arrivals[k][0] if k < len(arrivals) else end, due[0][0] if due else end, end)
        for c in server.poll(wait=max(0.0, min(0.002, next_t - now))):
            if c["kind"] == "create":
                sid, n, life = pending.pop(c["request"])
                if c["status"] != 0:
                    rejected += 1
                    continue
                admitted += 1
                live[sid] = dict(n=c["particles"], life=life, t_live=c["finished"], steps=0, busy=False,
                                 last_submit=-1.0, buf=np.empty((max(1, c["particles"]), 4), np.float32))
                heapq.heappush(due, (c["finished"], sid))
            elif c["kind"] == "step":
                sid = c["scene"]
                if c["status"] == 0 and c["finished"] <= end:
                    lat.append((c["finished"] - c["submitted"]) * 1e3)
                    ps_window += c["particles"] * c["substeps"]
                    done_steps += 1
                s = live.get(sid)
                if s is None:
                    continue
                s["busy"] = False
                if c["finished"] - s["t_live"] >= s["life"]:
                    server.destroy_scene(sid)
                    del live[sid]
                else:
                    heapq.heappush(due, (max(c["finished"], s["last_submit"] + period), sid))
        now = server.clock()
        while due and due[0][0] <= now:
            _, sid = heapq.heappop(due)
            if sid in live and not live[sid]["busy"]:
                submit_step(sid, now)
    # stop: let outstanding steps finish (bounded), then destroy the live scenes;
    # creates still queued are left to the server's shutdown
    t_stop = server.clock()
    while any(s["busy"] for s in live.values()) and server.clock() - t_stop < drain_seconds:
        for c in server.poll(wait=0.01):
            if c["kind"] == "create" and c["request"] in pending:
                pending.pop(c["request"])
            elif c["kind"] == "step" and c["scene"] in live:
                live[c["scene"]]["busy"] = False
    for sid in list(live):
        server.destroy_scene(sid)
    lat_a = np.array(lat) if lat else np.zeros(1)
    return dict(window_s=duration, created=created, admitted=admitted, rejected=rejected,
                steps=done_steps, particle_substeps=ps_window, particle_substeps_per_s=ps_window / duration,
                step_p50_ms=float(np.percentile(lat_a, 50)), step_p99_ms=float(np.percentile(lat_a, 99)),
                step_mean_ms=float(lat_a.mean()), still_pending_creates=len(pending))
