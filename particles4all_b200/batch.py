"""Batch — many independent scenes stepped together (libp4a's p4a_batch_* API).

Each scene behaves as its own `Sim` (own params, time bank, parity, iterations,
tension), but every pass of a substep is one kernel launch over all the scenes
that are stepped: the cell-key sort is one counting sort over the scenes'
disjoint key ranges and the kernels pull (scene, tile) work items. Results per
scene are bit-identical to stepping that scene alone.

    b = Batch(max_particles=8_000_000, max_cells=8_000_000, max_scenes=128)
    sid = b.add_scene(params, scene)      # admission: raises P4AError(5) when full
    b.step([sid, ...], 1 / 60)
    pos = b.read(sid, "pos")
"""
import ctypes as C
import math

import numpy as np

from . import _abi
from ._lib import P4AError, lib
from ._scene_desc import scene_desc
from .params import CParams


def arena_sizes(scenes, spare_particles=4096):
    """Batch arena sizes (keyword arguments of Batch) that hold every (params,
    scene) of `scenes` at once: particle ranges rounded to 256 with room for
    alignment, cell ranges padded to whole 2,048-cell scan tiles, the boundary
    shell of each box at the scene's spacing, and each scene's bodies."""
    cap = sum((sc["pos"].shape[0] + 511) // 256 * 256 for _, sc in scenes)
    cells = sum((int(math.prod(int(b) for b in p["box"])) // 2048 + 2) * 2048 for p, _ in scenes)
    nbound = 0
    for p, _ in scenes:
        nb = [max(2, math.ceil(b / p["spacing"]) + 1) for b in p["box"]]
        nbound += nb[0] * nb[1] * nb[2] - (nb[0] - 2) * (nb[1] - 2) * (nb[2] - 2)
    bodies = sum(sc["n_bodies"] + 1 for _, sc in scenes)
    body_parts = sum(int((sc["phase"][:, 0] > 0).sum()) + 1 for _, sc in scenes)
    return dict(max_particles=cap + spare_particles, max_cells=cells, max_scenes=len(scenes) + 1,
                max_bodies=bodies + 8, max_boundary=nbound + 4096, max_body_parts=body_parts + 64)


class Batch:
    def __init__(self, device=0, max_particles=1 << 22, max_cells=1 << 22, max_scenes=128,
                 max_bodies=1024, max_boundary=1 << 22, max_body_parts=1 << 20, graphs=True):
        self._L = lib()
        cfg = _abi.BatchConfig(int(max_particles), int(max_cells), int(max_boundary), int(max_scenes),
                               int(max_bodies), int(max_body_parts))
        h = C.c_void_p()
        rc = self._L.p4a_batch_create(int(device), C.byref(cfg), C.byref(h))
        if rc != 0:
            raise P4AError(rc, f"p4a_batch_create: {self._L.p4a_status_string(rc).decode()}")
        self._h = h
        self._keep = {}
        self.use_graphs(graphs)

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.p4a_batch_destroy(h)

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise P4AError(rc, f"{what}: {self._L.p4a_batch_last_error(self._h).decode()}")

    def use_graphs(self, on=True):
        self._check(self._L.p4a_batch_use_graphs(self._h, 1 if on else 0), "use_graphs")

    def set_stream(self, stream_handle):
        self._check(self._L.p4a_batch_set_stream(self._h, C.c_void_p(stream_handle or None)), "set_stream")

    def add_scene(self, params, scene):
        cp = CParams(params)
        desc, keep = scene_desc(scene)
        sid = C.c_int32()
        self._check(self._L.p4a_batch_add_scene(self._h, cp.ref(), C.byref(desc), C.byref(sid)), "add_scene")
        self._keep[sid.value] = (cp, desc, keep)
        return sid.value

    def add_preset(self, params):
        cp = CParams(params)
        sid = C.c_int32()
        self._check(self._L.p4a_batch_add_preset(self._h, cp.ref(), C.byref(sid)), "add_preset")
        self._keep[sid.value] = (cp,)
        return sid.value

    def remove_scene(self, sid):
        self._check(self._L.p4a_batch_remove_scene(self._h, int(sid)), "remove_scene")
        self._keep.pop(sid, None)

    def step(self, sids, frame_dt):
        ids = np.ascontiguousarray(sids, np.int32)
        self._check(self._L.p4a_batch_step(self._h, ids.ctypes.data, ids.size, float(frame_dt)), "step")

    def synchronize(self):
        self._check(self._L.p4a_batch_synchronize(self._h), "synchronize")

    def usage(self):
        u = _abi.BatchUsage()
        self._check(self._L.p4a_batch_usage_get(self._h, C.byref(u)), "usage")
        return {k: getattr(u, k) for k, _ in _abi.BatchUsage._fields_}

    def info(self, sid):
        i = _abi.Info()
        self._check(self._L.p4a_batch_scene_info(self._h, int(sid), C.byref(i)), "scene_info")
        return _abi.info_dict(i)

    def read(self, sid, name, which=_abi.LIVE, count=None):
        bid = _abi.BUF[name]
        dt, comps = _abi.BUF_LAYOUT[bid]
        inf = self.info(sid)
        if name == "cellStart":
            elems = inf["n_cells"] + 2
        elif name.startswith("body") and name != "body":
            elems = max(1, inf["n_bodies"]) * (3 if name == "bodyRot" else 1)
        else:
            elems = inf["cap"]
        if count is not None:
            elems = min(elems, int(count))
        out = np.zeros(elems * comps, dt)
        if out.nbytes:
            self._check(self._L.p4a_batch_read(self._h, int(sid), bid, which, out.ctypes.data, 0, out.nbytes), "read")
        return out.reshape(-1, comps) if comps > 1 else out

    def write(self, sid, name, data, which=_abi.LIVE, offset_elems=0):
        bid = _abi.BUF[name]
        dt, comps = _abi.BUF_LAYOUT[bid]
        a = np.ascontiguousarray(data, dt).reshape(-1)
        self._check(self._L.p4a_batch_write(self._h, int(sid), bid, which, a.ctypes.data,
                                            offset_elems * 4 * comps, a.nbytes), "write")

    def read_async(self, sid, name, host_ptr, nbytes, which=_abi.LIVE, offset=0):
        """Queue a copy of the scene's buffer into host memory at host_ptr (pinned
        for an asynchronous copy); complete after synchronize()."""
        self._check(self._L.p4a_batch_read_async(self._h, int(sid), _abi.BUF[name], which, C.c_void_p(host_ptr),
                                                 int(offset), int(nbytes)), "read_async")

    def write_async(self, sid, name, host_ptr, nbytes, which=_abi.LIVE, offset=0):
        """Queue a copy from host memory at host_ptr into the scene's buffer."""
        self._check(self._L.p4a_batch_write_async(self._h, int(sid), _abi.BUF[name], which, C.c_void_p(host_ptr),
                                                  int(offset), int(nbytes)), "write_async")

    def set_lanes(self, lanes=2, min_particles=1_000_000):
        """Frames of at least min_particles particles run as `lanes` concurrent parts
        (1-4, default 2; 1 = whole); the same bits either way."""
        self._check(self._L.p4a_batch_set_lanes(self._h, int(lanes), int(min_particles)), "set_lanes")

    def step_io(self, entries, frame_dt, groups=0):
        """One frame of the scenes of `entries` with overlapped host I/O: each entry
        is (sid, pos_in, vel_in, pos_out, vel_out), host addresses (pinned for
        overlap) of n x float4 each, or None. Same bits as write_async, step and
        read_async; the scenes run as `groups` frames (0: chosen from their size)
        so that the copies of one group overlap the frames of the others. Host
        memory stays in use until synchronize()."""
        arr = (_abi.BatchIO * max(1, len(entries)))()
        for k, (sid, pin, vin, pout, vout) in enumerate(entries):
            arr[k] = _abi.BatchIO(int(sid), pin, vin, pout, vout)
        self._check(self._L.p4a_batch_step_io(self._h, arr, len(entries), float(frame_dt), int(groups)),
                    "step_io")

    def profile(self, on=True):
        self._check(self._L.p4a_batch_profile_enable(self._h, 1 if on else 0), "profile_enable")

    def profile_reset(self):
        self._check(self._L.p4a_batch_profile_reset(self._h), "profile_reset")

    def profile_read(self):
        """{kernel name: (device ms, launches)} of the frames since profile_reset()."""
        arr = (_abi.PhaseTime * 32)()
        cnt = C.c_int32()
        self._check(self._L.p4a_batch_profile_read(self._h, arr, 32, C.byref(cnt)), "profile_read")
        return {arr[i].name.decode(): (arr[i].ms, arr[i].launches) for i in range(min(cnt.value, 32))}

    def stats(self, sid):
        s = _abi.Stats()
        self._check(self._L.p4a_batch_stats(self._h, int(sid), C.byref(s)), "stats")
        return dict(avgRho=s.avg_rho, maxRho=s.max_rho, maxSpeed=s.max_speed, ke=s.ke, raw=list(s.raw),
                    valid=s.valid)
