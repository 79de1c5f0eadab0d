"""Server — the serving loop over libp4a's p4a_server_* API (continuous batching).

Clients submit create / step / destroy requests; an engine thread inside the
library admits created scenes as scene slots and arena memory free up, packs
every live scene with a pending step into the next batched frame while the
previous frame is still on the GPU, and posts one completion per request.

    srv = Server(budget_bytes=8 << 30)
    sid, req = srv.create_scene(params)            # or (params, scene) explicit
    srv.step(sid, 1 / 60, pos_out=np.empty((n, 4), np.float32))
    for c in srv.poll(wait=0.1): ...               # dicts: request, kind, scene, status, ...
    srv.stats()                                    # p50/p99 step latency, throughput, counts

`plain=True` serves the same requests with one plain Sim per scene, stepped one
after another: the comparison for the batched form.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import P4AError, lib
from ._scene_desc import scene_desc
from .params import CParams

def _arenas(p, max_scenes):
    """Arena sizes for p particle slots: one cell and half a boundary sample per
    particle slot (the ratio of dam-break scenes), an eighth of a slot for body
    particles and 16 bodies per scene."""
    return dict(max_particles=int(p), max_cells=int(p), max_boundary=max(1, int(p) // 2),
                max_scenes=int(max_scenes), max_bodies=int(max_scenes) * 16, max_body_parts=max(1, int(p) // 8))


def arena_bytes(arenas):
    """Device bytes of the batch arenas for these sizes, as p4a_batch_create
    allocates them (p4a_batch_footprint)."""
    cfg = _abi.BatchConfig()
    for k, v in arenas.items():
        setattr(cfg, k, int(v))
    out = C.c_int64()
    rc = lib().p4a_batch_footprint(C.byref(cfg), C.byref(out))
    if rc != 0:
        raise P4AError(rc, "p4a_batch_footprint")
    return int(out.value)


def arenas_for_budget(budget_bytes, max_scenes=4096):
    """The largest arena sizes (in the ratios of _arenas) whose allocation fits in
    `budget_bytes` of device memory."""
    p0 = 1 << 20
    f0, f1 = arena_bytes(_arenas(p0, max_scenes)), arena_bytes(_arenas(2 * p0, max_scenes))
    slope = (f1 - f0) / p0
    p = int((budget_bytes - (f0 - slope * p0)) / slope)
    p = max(1, min(p, (1 << 31) - (1 << 24)))
    while p > 1 and arena_bytes(_arenas(p, max_scenes)) > budget_bytes:
        p = int(p * 0.999)
    return _arenas(p, max_scenes)


class Server:
    def __init__(self, device=0, budget_bytes=None, arenas=None, plain=False, builder_threads=4,
                 max_frames_in_flight=2, admit_timeout=0.0, max_pending_creates=0, graphs=True,
                 upload_bytes=1 << 30, readback_bytes=1 << 30, max_scenes=1024, lanes=2,
                 lane_min_particles=1_000_000):
        self._L = lib()
        cfg = _abi.ServerConfig()
        self._L.p4a_server_default_config(C.byref(cfg))
        if arenas is None:
            arenas = arenas_for_budget(budget_bytes, max_scenes) if budget_bytes else {}
        for k, v in arenas.items():
            setattr(cfg.arenas, k, int(v))
        cfg.builder_threads = int(builder_threads)
        cfg.max_frames_in_flight = int(max_frames_in_flight)
        cfg.admit_timeout = float(admit_timeout)
        cfg.max_pending_creates = int(max_pending_creates)
        cfg.use_graphs = 1 if graphs else 0
        cfg.plain = 1 if plain else 0
        cfg.upload_bytes = int(upload_bytes)
        cfg.readback_bytes = int(readback_bytes)
        cfg.frame_lanes = int(lanes)
        cfg.lane_min_particles = int(lane_min_particles)
        self.config = {k: getattr(cfg, k) for k, _ in _abi.ServerConfig._fields_ if k != "arenas"}
        self.config["arenas"] = {k: getattr(cfg.arenas, k) for k, _ in _abi.BatchConfig._fields_}
        h = C.c_void_p()
        rc = self._L.p4a_server_create(int(device), C.byref(cfg), C.byref(h))
        if rc != 0:
            raise P4AError(rc, f"p4a_server_create: {self._L.p4a_status_string(rc).decode()}")
        self._h = h
        self._outputs = {}  # request -> output arrays kept alive until its completion
        self._buf = (_abi.Completion * 4096)()

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.p4a_server_destroy(h)
        self._outputs = {}

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise P4AError(rc, f"{what}: {self._L.p4a_server_last_error(self._h).decode()}")

    def clock(self):
        return self._L.p4a_server_clock(self._h)

    def create_scene(self, params, scene=None):
        """Submits a create; returns (scene handle, request id). `scene` (the dict
        of configs.py scenes) is copied before the call returns."""
        cp = CParams(params)
        sid, req = C.c_int32(), C.c_int64()
        if scene is None:
            rc = self._L.p4a_server_create_scene(self._h, cp.ref(), None, C.byref(sid), C.byref(req))
        else:
            desc, keep = scene_desc(scene)
            rc = self._L.p4a_server_create_scene(self._h, cp.ref(), C.byref(desc), C.byref(sid), C.byref(req))
        self._check(rc, "create_scene")
        return sid.value, req.value

    def step(self, sid, frame_dt, pos_out=None, vel_out=None):
        """Submits a step; pos_out / vel_out (float32 [>= n, 4], C-contiguous) receive
        the scene's live positions / velocities when the step completes."""
        outs = [a for a in (pos_out, vel_out) if a is not None]
        for a in outs:
            if a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("outputs must be C-contiguous float32")
        nbytes = min(a.nbytes for a in outs) if outs else 0
        req = C.c_int64()
        rc = self._L.p4a_server_step(self._h, int(sid), float(frame_dt),
                                     None if pos_out is None else pos_out.ctypes.data,
                                     None if vel_out is None else vel_out.ctypes.data, nbytes, C.byref(req))
        self._check(rc, "step")
        if outs:
            self._outputs[req.value] = outs
        return req.value

    def destroy_scene(self, sid):
        req = C.c_int64()
        self._check(self._L.p4a_server_destroy_scene(self._h, int(sid), C.byref(req)), "destroy_scene")
        return req.value

    def poll(self, max_count=4096, wait=0.0):
        """Completions as dicts (request, kind, scene, status, substeps, particles,
        submitted, started, finished); waits up to `wait` s for the first."""
        cnt = C.c_int32()
        m = min(int(max_count), len(self._buf))
        rc = self._L.p4a_server_poll(self._h, self._buf, m, C.byref(cnt), float(wait))
        self._check(rc, "poll")
        out = []
        for k in range(cnt.value):
            c = self._buf[k]
            d = {f: getattr(c, f) for f, _ in _abi.Completion._fields_}
            d["kind"] = _abi.REQ_NAMES.get(d["kind"], d["kind"])
            self._outputs.pop(d["request"], None)
            out.append(d)
        return out

    def stats(self):
        s = _abi.ServerStats()
        self._check(self._L.p4a_server_get_stats(self._h, C.byref(s)), "stats")
        return {k: getattr(s, k) for k, _ in _abi.ServerStats._fields_}
