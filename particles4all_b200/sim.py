"""Sim — the reference's `class Sim` (src/sim.js:9-814) over libp4a's C ABI.

Same method names and argument meaning as the JS class, so code written
against the reference reads the same:

    sim = Sim(device=0)
    sim.reset(default_params("small"))
    sim.step(1 / 60)
    sim.appendFluid(pos3, vel3) -> count
    sim.applyRayImpulse(origin, dir, impulse, radius, speedLimit)
    sim.holdBody(body1, target, rate, limit); sim.releaseBody()
    sim.resizeBox([x, y, z])
    sim.livePos() / liveVel() / liveBody()   -> device pointers (ints)
    sim.n, sim.h, sim.gridDim, sim.nCells, sim.parity, sim.gen, sim.simTime,
    sim.stats, sim.bodyPose, ...

All device work runs in libp4a (CUDA sm_100a); this module only marshals
arguments. Buffers stay in device memory; read() copies one to host as numpy.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import check, lib
from .params import CParams, aniso_struct, default_aniso, default_mesh, mesh_struct


class Sim:
    def __init__(self, device=0):
        self._L = lib()
        h = C.c_void_p()
        check(self._L.p4a_create(int(device), C.byref(h)), None, "p4a_create")
        self._h = h
        self.device = device
        self.params = None
        self.bodyPhases = False  # accepted for API parity; the fused body pass has no phases

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.p4a_destroy(h)

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- reset / step --------------------------------------------------------
    def reset(self, params):
        """Sim.reset(params) (src/sim.js:66-221)."""
        self.params = dict(params)
        self._cp = CParams(self.params)
        check(self._L.p4a_reset(self._h, self._cp.ref()), self._h, "reset")

    def reset_scene(self, params, scene):
        """reset() on an explicit scene dict (pos/vel/rest/phase float4/uint4 arrays,
        n_bodies, body_density, body_centre, mass, denom_rest, pour_budget)."""
        from ._scene_desc import scene_desc
        self.params = dict(params)
        self._cp = CParams(self.params)
        self._desc, self._keep = scene_desc(scene)
        check(self._L.p4a_reset_scene(self._h, self._cp.ref(), C.byref(self._desc)), self._h, "reset_scene")

    def step(self, frameDt):
        """Sim.step(frameDt) (src/sim.js:415-656); returns the substeps taken."""
        sub = C.c_int32()
        check(self._L.p4a_step(self._h, float(frameDt), C.byref(sub)), self._h, "step")
        return sub.value

    def synchronize(self):
        check(self._L.p4a_synchronize(self._h), self._h, "synchronize")

    # ---- interactive ---------------------------------------------------------
    def appendFluid(self, pos, vel):
        """Sim.appendFluid(pos, vel) (src/sim.js:774-809): flat xyz lists/arrays."""
        p = np.ascontiguousarray(pos, np.float32).reshape(-1)
        v = np.ascontiguousarray(vel, np.float32).reshape(-1)
        added = C.c_int32()
        count = min(p.size // 3, v.size // 3)
        check(self._L.p4a_append_fluid(self._h, p.ctypes.data, v.ctypes.data, count, C.byref(added)),
              self._h, "appendFluid")
        return added.value

    def hoseEmit(self, hose):
        """One layer of the fixed-rate hose (configs.Hose) emitted on the device at
        the hose's next emission index (p4a_hose_emit): no host copy, no wait."""
        added = C.c_int32()
        check(self._L.p4a_hose_emit(self._h, C.byref(hose.c_struct()), hose.emission, C.byref(added)),
              self._h, "hoseEmit")
        hose.advance(added.value)
        return added.value

    def applyRayImpulse(self, origin, direction, impulse, radius, speedLimit):
        o, d, im = (np.asarray(x, np.float64).reshape(3) for x in (origin, direction, impulse))
        check(self._L.p4a_apply_ray_impulse(self._h, o.ctypes.data, d.ctypes.data, im.ctypes.data,
                                            float(radius), float(speedLimit)), self._h, "applyRayImpulse")

    def holdBody(self, body1Based, target, rate, limit):
        t = np.asarray(target, np.float64).reshape(3)
        check(self._L.p4a_hold_body(self._h, int(body1Based), t.ctypes.data, float(rate), float(limit)),
              self._h, "holdBody")

    def releaseBody(self):
        check(self._L.p4a_release_body(self._h), self._h, "releaseBody")

    def resizeBox(self, newBox):
        b = np.asarray(newBox, np.float64).reshape(3)
        check(self._L.p4a_resize_box(self._h, b.ctypes.data), self._h, "resizeBox")
        self.params["box"] = [float(x) for x in b]

    def aniso(self, aparams=None):
        """The anisotropic-kernel pass (src/aniso_wgsl.js, src/mesh.js:207-261)."""
        s = aniso_struct(aparams or default_aniso())
        check(self._L.p4a_aniso(self._h, C.byref(s)), self._h, "aniso")

    def mesh(self, mparams=None, wait=True):
        """SurfaceMesh.generate (src/mesh.js:99-352) on the live buffers; returns the
        triangle count (None when wait=False). Results: read('meshField'),
        read('meshNField'), read('meshVerts') (uint2 per vertex, 3 per triangle)."""
        m = mesh_struct(mparams or default_mesh())
        t = C.c_int64()
        check(self._L.p4a_mesh(self._h, C.byref(m), C.byref(t) if wait else None), self._h, "mesh")
        return t.value if wait else None

    def ssfr(self, sparams, bodies=None):
        """FluidSSFR.render (src/ssfr.js:173-356) into headless device images; needs the
        anisotropic pass of the current particles. `bodies`: float32 [count, 6, 4]
        packed rigid bodies for the composite, or None. Read results with
        ssfr_read('image' | 'eyeZ' | 'rawZ' | 'thick' | 'bodyT')."""
        from .params import ssfr_struct
        sp = ssfr_struct(sparams)
        if bodies is None or len(bodies) == 0:
            ptr, count, keep = None, 0, None
        else:
            keep = np.ascontiguousarray(bodies, dtype=np.float32).reshape(-1, 24)
            ptr, count = keep.ctypes.data, keep.shape[0]
        check(self._L.p4a_ssfr(self._h, C.byref(sp), ptr, count), self._h, "ssfr")

    def ssfr_info(self):
        i = _abi.SsfrInfo()
        check(self._L.p4a_ssfr_get_info(self._h, C.byref(i)), self._h, "ssfr_info")
        return {k: getattr(i, k) for k, _ in _abi.SsfrInfo._fields_}

    def ssfr_read(self, name):
        """A copy of an SSFR buffer: float maps [h, w], the image uint8 [height, width, 4]."""
        p, nb = C.c_void_p(), C.c_size_t()
        which = _abi.SSFR_BUF[name]
        check(self._L.p4a_ssfr_buffer(self._h, which, C.byref(p), C.byref(nb)), self._h, "ssfr_buffer")
        inf = self.ssfr_info()
        out = np.empty(nb.value, np.uint8)
        if nb.value:
            check(self._L.p4a_ssfr_read(self._h, which, out.ctypes.data, nb.value), self._h, "ssfr_read")
        if name == "image":
            return out.reshape(inf["height"], inf["width"], 4)
        w, h = (inf["thick_w"], inf["thick_h"]) if name == "thick" else (inf["map_w"], inf["map_h"])
        return out.view(np.float32).reshape(h, w)

    def set_environment(self, rgb):
        """Environment.load (src/env.js:180-236): `rgb` a float32 equirectangular
        panorama [height, width, 3] (2:1), or None to clear (Environment.clear)."""
        if rgb is None:
            check(self._L.p4a_set_environment(self._h, None, 0, 0), self._h, "set_environment")
            return
        a = np.ascontiguousarray(rgb, np.float32)
        if a.ndim != 3 or a.shape[2] != 3:
            raise ValueError("the panorama is [height, width, 3]")
        check(self._L.p4a_set_environment(self._h, a.ctypes.data, a.shape[1], a.shape[0]), self._h,
              "set_environment")

    def environment(self):
        """The cube map as uint16 half-float bits [6, size, size, 4], or None."""
        size = C.c_int32()
        check(self._L.p4a_environment_read(self._h, C.byref(size), None, 0), self._h, "environment_read")
        if size.value == 0:
            return None
        out = np.empty((6, size.value, size.value, 4), np.uint16)
        check(self._L.p4a_environment_read(self._h, C.byref(size), out.ctypes.data, out.nbytes), self._h,
              "environment_read")
        return out

    def ray(self, rparams, bodies=None):
        """RayMarch.draw (src/ray.js:30-97) on the last mesh(): its triangles as the
        surface (use_surface 1, the default) or its density field marched
        (use_surface 0); returns nothing, read the image with ray_read()."""
        from .params import ray_struct
        rp = ray_struct(rparams)
        if bodies is None or len(bodies) == 0:
            ptr, count, keep = None, 0, None
        else:
            keep = np.ascontiguousarray(bodies, dtype=np.float32).reshape(-1, 24)
            ptr, count = keep.ctypes.data, keep.shape[0]
        check(self._L.p4a_ray(self._h, C.byref(rp), ptr, count), self._h, "ray")

    def ray_read(self):
        """The last ray() image, uint8 [height, width, 4]."""
        p, nb, w, h = C.c_void_p(), C.c_size_t(), C.c_int32(), C.c_int32()
        check(self._L.p4a_ray_buffer(self._h, C.byref(p), C.byref(nb), C.byref(w), C.byref(h)), self._h,
              "ray_buffer")
        out = np.empty((h.value, w.value, 4), np.uint8)
        check(self._L.p4a_ray_read(self._h, out.ctypes.data, nb.value), self._h, "ray_read")
        return out

    def mesh_info(self):
        i = _abi.MeshInfo()
        check(self._L.p4a_mesh_get_info(self._h, C.byref(i)), self._h, "mesh_info")
        return {"vert_dim": list(i.vert_dim), "origin": list(i.origin), "voxel": i.voxel,
                "triangles": i.triangles, "mesh_gen": i.mesh_gen}

    # ---- fields --------------------------------------------------------------
    def info(self):
        i = _abi.Info()
        check(self._L.p4a_get_info(self._h, C.byref(i)), self._h, "info")
        return _abi.info_dict(i)

    def __getattr__(self, name):
        fields = {"n": "n", "h": "h", "gridDim": "grid_dim", "nCells": "n_cells", "nBodies": "n_bodies",
                  "nBodyParts": "n_body_parts", "nBoundary": "n_boundary", "cap": "cap",
                  "pourBudget": "pour_budget", "parity": "parity", "predParity": "pred_parity",
                  "gen": "gen", "simTime": "sim_time", "lastSubsteps": "last_substeps",
                  "lastAdvanced": "last_advanced", "timeBank": "time_bank", "bodyScale": "body_scale",
                  "covScale": "cov_scale", "heldBody": "held_body"}
        if name in fields and "_h" in self.__dict__:
            return self.info()[fields[name]]
        raise AttributeError(name)

    @property
    def stats(self):
        """Sim.stats (src/sim.js:619-633): the latest completed readback."""
        return self.get_stats(wait=False)

    def get_stats(self, wait=True):
        s = _abi.Stats()
        check(self._L.p4a_get_stats(self._h, 1 if wait else 0, C.byref(s)), self._h, "stats")
        return dict(avgRho=s.avg_rho, maxRho=s.max_rho, maxSpeed=s.max_speed, ke=s.ke,
                    raw=list(s.raw), valid=s.valid)

    @property
    def bodyPose(self):
        return self.get_body_pose(wait=False)

    def get_body_pose(self, wait=True):
        nb = self.info()["n_bodies"]
        c = np.zeros((max(1, nb), 3), np.float32)
        r = np.zeros((max(1, nb), 9), np.float32)
        check(self._L.p4a_body_pose(self._h, 1 if wait else 0, c.ctypes.data, r.ctypes.data, nb),
              self._h, "bodyPose")
        return [{"centre": c[i].tolist(), "rot": r[i].tolist()} for i in range(nb)]

    # ---- GPU timing (the reference's GpuTimer) --------------------------------
    def profile(self, on=True):
        check(self._L.p4a_profile_enable(self._h, 1 if on else 0), self._h, "profile_enable")

    def profile_reset(self):
        check(self._L.p4a_profile_reset(self._h), self._h, "profile_reset")

    def profile_read(self):
        """{kernel name: (device ms, launches)} accumulated since profile_reset()."""
        arr = (_abi.PhaseTime * 32)()
        cnt = C.c_int32()
        check(self._L.p4a_profile_read(self._h, arr, 32, C.byref(cnt)), self._h, "profile_read")
        return {arr[i].name.decode(): (arr[i].ms, arr[i].launches) for i in range(min(cnt.value, 32))}

    def set_stream(self, stream_handle):
        """Issue all work on an existing cudaStream_t (an int handle); 0 = own stream."""
        check(self._L.p4a_set_stream(self._h, C.c_void_p(stream_handle or None)), self._h, "set_stream")

    # ---- buffers -------------------------------------------------------------
    def buffer_ptr(self, name, which=_abi.LIVE):
        p, nbytes = C.c_void_p(), C.c_size_t()
        check(self._L.p4a_buffer(self._h, _abi.BUF[name], which, C.byref(p), C.byref(nbytes)),
              self._h, "buffer")
        return p.value or 0, nbytes.value

    def livePos(self):
        return self.buffer_ptr("pos")[0]

    def liveVel(self):
        return self.buffer_ptr("vel")[0]

    def liveBody(self):
        return self.buffer_ptr("body")[0]

    def read(self, name, which=_abi.LIVE, count=None):
        """Copy a buffer to host as numpy (rows of 4 for float4/uint4 buffers)."""
        bid = _abi.BUF[name]
        _, nbytes = self.buffer_ptr(name, which)
        dt, comps = _abi.BUF_LAYOUT[bid]
        elem = 4 * comps
        if count is not None:
            nbytes = min(nbytes, int(count) * elem)
        out = np.zeros(nbytes // 4, dt)
        if nbytes:
            check(self._L.p4a_read(self._h, bid, which, out.ctypes.data, 0, nbytes), self._h, "read")
        return out.reshape(-1, comps) if comps > 1 else out

    def read_async(self, name, host, nbytes=None, which=_abi.LIVE):
        """Start copying a buffer into `host` (a numpy array, or the address of
        pinned host memory with `nbytes`) on the sim's copy stream, after the work
        queued so far; the data is there once read_wait() returns. Keep `host`
        alive until then."""
        bid = _abi.BUF[name]
        if isinstance(host, np.ndarray):
            if not host.flags.c_contiguous:
                raise ValueError("read_async needs a contiguous array")
            ptr, nb = host.ctypes.data, host.nbytes if nbytes is None else int(nbytes)
            if nb > host.nbytes:
                raise ValueError(f"read_async of {nb} bytes into an array of {host.nbytes}")
        else:
            ptr, nb = int(host), int(nbytes)
        check(self._L.p4a_read_async(self._h, bid, which, ptr, 0, nb), self._h, "read_async")

    def read_wait(self):
        """Wait for the copies started by read_async()."""
        check(self._L.p4a_read_wait(self._h), self._h, "read_wait")

    def write(self, name, data, which=_abi.LIVE, offset_elems=0):
        bid = _abi.BUF[name]
        dt, comps = _abi.BUF_LAYOUT[bid]
        a = np.ascontiguousarray(data, dt).reshape(-1)
        check(self._L.p4a_write(self._h, bid, which, a.ctypes.data, offset_elems * 4 * comps, a.nbytes),
              self._h, "write")
