"""particles4all_b200 — B200-native (sm_100a CUDA) Particles4All simulation step.

The product is libp4a.so (C ABI in include/p4a.h); this package is its Python
host: `Sim` mirrors the reference's `class Sim` (src/sim.js), `default_params`
its `defaultParams` (src/scene.js:11-39), `Batch` steps many scenes per launch,
`Server` is the continuous-batching request loop, `autotune` picks kernel launch
shapes per size bucket, `camera` restates the viewer's matrices for the
screen-space fluid rendering (`Sim.ssfr`, `default_ssfr`) and the ray-marched
surface (`Sim.ray`, `default_ray`), and `configs` /
`loadgen` are the seeded workloads.
"""
from ._lib import P4AError, device_available, lib  # noqa: F401
from .params import PRESETS, default_aniso, default_mesh, default_params, default_ray, default_ssfr  # noqa: F401
from .batch import Batch  # noqa: F401
from .server import Server  # noqa: F401
from .sim import Sim  # noqa: F401

__all__ = ["Sim", "Batch", "Server", "default_params", "default_aniso", "default_mesh", "default_ssfr", "default_ray", "PRESETS",
           "P4AError", "device_available", "lib"]
