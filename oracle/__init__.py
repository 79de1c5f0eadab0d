"""CPU oracle of the Particles4All simulation step (ctypes wrapper of liboracle_p4a.so).

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use this module, as what the product's results are compared against or
as the timed CPU baseline. The product (particles4all_b200 / libp4a.so) never
imports it.

PARITY UNPINNED: the reference (JS + WGSL in a browser) cannot run in this
environment and ships no golden vectors; the restatement is pinned only by
hand-derived known answers and the reference's own verify checks
(src/main.js:853-937). See p4a_oracle.h for the arithmetic contract.
"""
import ctypes as C
import os

import numpy as np

from particles4all_b200 import _abi
from particles4all_b200._scene_desc import scene_desc
from particles4all_b200.params import CParams, aniso_struct, mesh_struct

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle_p4a.so")
_lib = None


def build(force=False):
    from .build import build as _build
    return _build(force=force)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, dbl = C.c_void_p, C.c_int32, C.c_double
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        for name, args in {
            "orc_reset": [vp, vp], "orc_reset_scene": [vp, vp, vp],
            "orc_step": [vp, dbl, C.POINTER(i32)],
            "orc_append_fluid": [vp, vp, vp, i32, C.POINTER(i32)],
            "orc_apply_ray_impulse": [vp, vp, vp, vp, dbl, dbl],
            "orc_hold_body": [vp, i32, vp, dbl, dbl], "orc_release_body": [vp],
            "orc_resize_box": [vp, vp], "orc_aniso": [vp, vp], "orc_mesh": [vp, vp, vp], "orc_get_info": [vp, vp],
            "orc_stats": [vp, vp], "orc_buffer": [vp, i32, i32, C.POINTER(vp), C.POINTER(C.c_size_t)],
            "orc_build_scene": [vp, vp, vp, vp, vp, vp, vp, vp],
            "orc_boundary": [vp, dbl, dbl, C.POINTER(i32), vp, vp],
            "orc_grid_sort": [vp, i32, C.c_float, C.c_float] + [vp] * 11,
            "orc_ssfr": [vp, vp, vp, i32], "orc_ssfr_buffer": [vp, i32, C.POINTER(vp), C.POINTER(C.c_size_t)],
            "orc_ray": [vp, vp, vp, i32], "orc_ray_image": [vp, C.POINTER(vp), C.POINTER(C.c_size_t)],
            "orc_set_environment": [vp, vp, i32, i32], "orc_environment": [vp, C.POINTER(vp), C.POINTER(i32)],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.orc_cbrt_newton.argtypes = [C.c_float]
        L.orc_cbrt_newton.restype = C.c_float
        for name in ("orc_expf", "orc_logf"):
            getattr(L, name).argtypes = [C.c_float]
            getattr(L, name).restype = C.c_float
        _lib = L
    return _lib


def set_threads(n):
    lib().orc_set_threads(int(n))


def threads():
    return lib().orc_get_threads()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


def build_scene(params):
    """buildScene(params) restated (src/scene.js:159-315)."""
    cp = CParams(params)
    cnt = _abi.SceneCounts()
    L = lib()
    _check(L.orc_build_scene(cp.ref(), C.byref(cnt), None, None, None, None, None, None), "build_scene")
    n, nb = cnt.n, cnt.n_bodies
    pos = np.zeros((n, 4), np.float32); vel = np.zeros((n, 4), np.float32)
    rest = np.zeros((n, 4), np.float32); phase = np.zeros((n, 4), np.uint32)
    centre = np.zeros((max(1, nb), 3), np.float64); dens = np.zeros(max(1, nb), np.float64)
    _check(L.orc_build_scene(cp.ref(), C.byref(cnt), _ptr(pos), _ptr(vel), _ptr(rest), _ptr(phase),
                             _ptr(centre), _ptr(dens)), "build_scene")
    return dict(n=n, n_fluid=cnt.n_fluid, n_body=cnt.n_body, n_bodies=nb, n_boundary=cnt.n_boundary,
                mass=cnt.mass, denom_rest=cnt.denom_rest, h=cnt.h, pos=pos, vel=vel, rest=rest,
                phase=phase, body_centre=centre[:nb], body_density=dens[:nb])


def boundary(params, d, h):
    """boundaryParticles(p, d, h) restated (src/scene.js:76-135)."""
    cp = CParams(params)
    cnt = C.c_int32()
    L = lib()
    _check(L.orc_boundary(cp.ref(), d, h, C.byref(cnt), None, None), "boundary")
    pts = np.zeros((cnt.value, 3), np.float64); psi = np.zeros(max(1, cnt.value), np.float32)
    _check(L.orc_boundary(cp.ref(), d, h, C.byref(cnt), _ptr(pts), _ptr(psi)), "boundary")
    return pts, psi[:cnt.value]


def cbrt_newton(x):
    return lib().orc_cbrt_newton(float(x))


def grid_sort(grid, dt, gravity, pos, vel, body=None, rest=None):
    """predict + grid pass on host arrays; returns the sorted outputs."""
    n = pos.shape[0]
    g = _abi.Grid()
    for k in range(3):
        g.box_min[k] = grid["box_min"][k]; g.dim[k] = grid["dim"][k]
    g.h = grid["h"]
    ncells = grid["dim"][0] * grid["dim"][1] * grid["dim"][2]
    out = dict(pos=np.zeros((n, 4), np.float32), vel=np.zeros((n, 4), np.float32),
               pred=np.zeros((n, 4), np.float32),
               body=np.zeros((n, 4), np.uint32) if body is not None else None,
               rest=np.zeros((n, 4), np.float32) if rest is not None else None,
               cell_start=np.zeros(ncells + 1, np.uint32), slot=np.zeros(n, np.uint32))
    pos = np.ascontiguousarray(pos, np.float32); vel = np.ascontiguousarray(vel, np.float32)
    _check(lib().orc_grid_sort(C.byref(g), n, dt, gravity, _ptr(pos), _ptr(vel),
                               _ptr(body), _ptr(rest), _ptr(out["pos"]), _ptr(out["vel"]),
                               _ptr(out["pred"]), _ptr(out["body"]), _ptr(out["rest"]),
                               _ptr(out["cell_start"]), _ptr(out["slot"])), "grid_sort")
    return out


class OracleSim:
    """The reference's Sim (src/sim.js) restated on the CPU, same method names."""

    def __init__(self):
        self._L = lib()
        self._h = self._L.orc_create()

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.orc_destroy(h)

    def reset(self, params):
        self._cp = CParams(params)
        _check(self._L.orc_reset(self._h, self._cp.ref()), "reset")

    def reset_scene(self, params, scene):
        self._cp = CParams(params)
        self._desc, self._keep = scene_desc(scene)
        _check(self._L.orc_reset_scene(self._h, self._cp.ref(), C.byref(self._desc)), "reset_scene")

    def step(self, frame_dt):
        sub = C.c_int32()
        _check(self._L.orc_step(self._h, frame_dt, C.byref(sub)), "step")
        return sub.value

    def appendFluid(self, pos3, vel3):
        p = np.ascontiguousarray(pos3, np.float32).reshape(-1)
        v = np.ascontiguousarray(vel3, np.float32).reshape(-1)
        added = C.c_int32()
        _check(self._L.orc_append_fluid(self._h, _ptr(p), _ptr(v), min(p.size, v.size) // 3,
                                        C.byref(added)), "appendFluid")
        return added.value

    def applyRayImpulse(self, origin, direction, impulse, radius, speed_limit):
        o, d, im = (np.asarray(x, np.float64) for x in (origin, direction, impulse))
        _check(self._L.orc_apply_ray_impulse(self._h, _ptr(o), _ptr(d), _ptr(im), radius, speed_limit),
               "applyRayImpulse")

    def holdBody(self, body1, target, rate, limit):
        t = np.asarray(target, np.float64)
        _check(self._L.orc_hold_body(self._h, int(body1), _ptr(t), rate, limit), "holdBody")

    def releaseBody(self):
        _check(self._L.orc_release_body(self._h), "releaseBody")

    def resizeBox(self, box):
        b = np.asarray(box, np.float64)
        _check(self._L.orc_resize_box(self._h, _ptr(b)), "resizeBox")

    def aniso(self, aparams):
        s = aniso_struct(aparams)
        _check(self._L.orc_aniso(self._h, C.byref(s)), "aniso")

    def mesh(self, mparams):
        m = mesh_struct(mparams)
        t = C.c_int64()
        _check(self._L.orc_mesh(self._h, C.byref(m), C.byref(t)), "mesh")
        return t.value

    def ssfr(self, sparams, bodies=None):
        """FluidSSFR.render restated on the CPU (same parameters as Sim.ssfr)."""
        from particles4all_b200.params import ssfr_struct
        sp = ssfr_struct(sparams)
        self._ssfr_dims = None
        if bodies is None or len(bodies) == 0:
            ptr, count, self._keep_bodies = None, 0, None
        else:
            self._keep_bodies = np.ascontiguousarray(bodies, dtype=np.float32).reshape(-1, 24)
            ptr, count = self._keep_bodies.ctypes.data, self._keep_bodies.shape[0]
        _check(self._L.orc_ssfr(self._h, C.byref(sp), ptr, count), "ssfr")
        rs = min(1.0, max(0.25, sp.render_scale))
        w, h = max(1, int(np.floor(sp.width * rs + 0.5))), max(1, int(np.floor(sp.height * rs + 0.5)))
        half = sp.thickness_half_res and sp.thickness_filter_size >= 4
        self._ssfr_dims = {"width": sp.width, "height": sp.height, "map_w": w, "map_h": h,
                           "thick_w": (w + 1) >> 1 if half else w, "thick_h": (h + 1) >> 1 if half else h}

    def ssfr_read(self, name):
        p, nb = C.c_void_p(), C.c_size_t()
        _check(self._L.orc_ssfr_buffer(self._h, _abi.SSFR_BUF[name], C.byref(p), C.byref(nb)), "ssfr_buffer")
        raw = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), (nb.value,)).copy() if nb.value else \
            np.zeros(0, np.uint8)
        dm = self._ssfr_dims
        if name == "image":
            return raw.reshape(dm["height"], dm["width"], 4)
        w, h = (dm["thick_w"], dm["thick_h"]) if name == "thick" else (dm["map_w"], dm["map_h"])
        return raw.view(np.float32).reshape(h, w)

    def ray(self, rparams, bodies=None):
        """RayMarch.draw restated on the CPU (same parameters as Sim.ray); returns the
        RGBA8 image [height, width, 4]."""
        from particles4all_b200.params import ray_struct
        rp = ray_struct(rparams)
        if bodies is None or len(bodies) == 0:
            ptr, count, keep = None, 0, None
        else:
            keep = np.ascontiguousarray(bodies, dtype=np.float32).reshape(-1, 24)
            ptr, count = keep.ctypes.data, keep.shape[0]
        _check(self._L.orc_ray(self._h, C.byref(rp), ptr, count), "ray")
        p, nb = C.c_void_p(), C.c_size_t()
        _check(self._L.orc_ray_image(self._h, C.byref(p), C.byref(nb)), "ray_image")
        raw = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), (nb.value,)).copy()
        return raw.reshape(rp.height, rp.width, 4)

    def set_environment(self, rgb):
        """Environment.load restated (same arguments as Sim.set_environment)."""
        if rgb is None:
            _check(self._L.orc_set_environment(self._h, None, 0, 0), "set_environment")
            return
        a = np.ascontiguousarray(rgb, np.float32)
        _check(self._L.orc_set_environment(self._h, a.ctypes.data, a.shape[1], a.shape[0]), "set_environment")

    def environment(self):
        """The cube map as uint16 half-float bits [6, size, size, 4], or None."""
        p, size = C.c_void_p(), C.c_int32()
        _check(self._L.orc_environment(self._h, C.byref(p), C.byref(size)), "environment")
        if size.value == 0:
            return None
        n = 6 * size.value * size.value * 4
        raw = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint16)), (n,)).copy()
        return raw.reshape(6, size.value, size.value, 4)

    def info(self):
        i = _abi.Info()
        _check(self._L.orc_get_info(self._h, C.byref(i)), "info")
        return _abi.info_dict(i)

    def stats(self):
        s = _abi.Stats()
        _check(self._L.orc_stats(self._h, C.byref(s)), "stats")
        return dict(avgRho=s.avg_rho, maxRho=s.max_rho, maxSpeed=s.max_speed, ke=s.ke,
                    raw=list(s.raw), valid=s.valid)

    def write(self, name, data, which=_abi.LIVE):
        """Overwrite the start of a buffer with `data` (as Sim.write)."""
        bid = _abi.BUF[name]
        p, nbytes = C.c_void_p(), C.c_size_t()
        _check(self._L.orc_buffer(self._h, bid, which, C.byref(p), C.byref(nbytes)), "buffer")
        a = np.ascontiguousarray(data, _abi.BUF_LAYOUT[bid][0]).reshape(-1)
        if a.nbytes > nbytes.value:
            raise ValueError(f"write of {a.nbytes} bytes into a buffer of {nbytes.value}")
        C.memmove(p, a.ctypes.data, a.nbytes)

    def buffer(self, name, which=_abi.LIVE):
        """A numpy copy of a buffer (name as in _abi.BUF)."""
        bid = _abi.BUF[name]
        p, nbytes = C.c_void_p(), C.c_size_t()
        _check(self._L.orc_buffer(self._h, bid, which, C.byref(p), C.byref(nbytes)), "buffer")
        dt, comps = _abi.BUF_LAYOUT[bid]
        if nbytes.value == 0:
            return np.zeros((0, comps) if comps > 1 else 0, dt)
        raw = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), (nbytes.value,)).copy()
        arr = raw.view(dt)
        return arr.reshape(-1, comps) if comps > 1 else arr
