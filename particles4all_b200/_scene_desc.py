"""Builds the p4a_scene_desc struct (include/p4a.h) over numpy arrays."""
import numpy as np

from . import _abi


def scene_desc(scene):
    """A p4a_scene_desc over the arrays of a scene dict (kept alive by the caller)."""
    keep = {}
    d = _abi.SceneDesc()
    n = int(scene["pos"].shape[0])
    d.n = n
    for k in ("pos", "vel", "rest"):
        if scene.get(k) is not None:
            keep[k] = np.ascontiguousarray(scene[k], np.float32).reshape(n, 4)
            setattr(d, k, keep[k].ctypes.data)
    if scene.get("phase") is not None:
        keep["phase"] = np.ascontiguousarray(scene["phase"], np.uint32).reshape(n, 4)
        d.phase = keep["phase"].ctypes.data
    nb = int(scene.get("n_bodies", 0))
    d.n_bodies = nb
    keep["bd"] = np.ascontiguousarray(scene.get("body_density", np.zeros(max(1, nb))), np.float64)
    keep["bc"] = np.ascontiguousarray(scene.get("body_centre", np.zeros((max(1, nb), 3))), np.float64)
    d.body_density = keep["bd"].ctypes.data
    d.body_centre = keep["bc"].ctypes.data
    d.mass = float(scene.get("mass", 0.0))
    d.denom_rest = float(scene.get("denom_rest", 0.0))
    d.pour_budget = int(scene.get("pour_budget", 0))
    return d, keep
