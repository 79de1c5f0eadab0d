"""Writes the golden fixtures of tests/golden from float64 transcriptions of the
reference written from its WGSL / JS text, which share no code with the oracle or
the library. The reference itself (a browser WebGPU app) cannot run here, so these
are the fixed float64 answers the float32 paths are held to.

Scene inputs come from tests/scene_f64.py (buildScene, src/scene.js:159-315, with
the JS number semantics), not from either scene builder under test.

transcription_small.npz: positions, velocities and densities of four tiny scenes
  (fluid, a rigid body, surface tension, both) after one or two substeps
  (tests/test_oracle_transcription.py Transcription).
ops_small.npz: the passes the step fixtures do not reach (tests/ops_f64.py):
  the anisotropic pass on the reset state and on displaced positions; the stats
  words after two substeps; a ray impulse on written velocities, then a substep;
  a held body dragged over two substeps; a box resize between two substeps; a
  fluid layer appended, then a substep.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
sys.path.insert(0, TESTS)
sys.path.insert(0, os.path.dirname(TESTS))

from ops_f64 import aniso_f64, impulse_f64, stats_f64  # noqa: E402
from scene_f64 import boundary_f64, build_scene_f64  # noqa: E402
from test_oracle_transcription import Transcription  # noqa: E402

from particles4all_b200.params import default_params  # noqa: E402

CASES = [("fluid", 2), ("bodies", 2), ("tension", 2), ("bodies_tension", 1)]
ANISO = {"ratio": 4.0, "ks": 1.0, "stretch": 2.0, "lonely": 1.0, "min_neighbours": 25, "lambda": 0.9,
         "radius_scale": 2.0, "min_extent": 0.0}
IMPULSE = ([0.0, 0.1, 0.1], [1.0, 0.05, 0.0], [6.0, 2.0, 0.0], 0.3, 4.0)
HOLD = (1, [0.15, 0.2, 0.1], 2.0, 0.5)
RESIZED = [0.22, 0.27, 0.2]
APPEND_BUDGET = 100


def case_params(case):
    p = default_params("small")
    p.update({"targetParticleCount": 350, "box": [0.25, 0.3, 0.21], "bodies": [], "substeps": 2})
    if "bodies" in case:
        p.update({"bodies": ["box:0.5"], "bodySize": 0.03})
    if "tension" in case:
        p.update({"surfaceTensionK": 0.4})
    return p


def scene_for(p):
    """The scene of buildScene(p) from the float64 transcription, as a scene dict."""
    return build_scene_f64(p)


def transcription(p, sc):
    d = p["spacing"]
    bpts, bpsi = boundary_f64(p, d, 2 * d)
    return Transcription(p, sc, bpts, bpsi)


def moved_positions(pos):
    """Displaced positions for the second anisotropic case (float32): a shear along
    x growing with height and a 7 % squeeze in y."""
    out = pos.copy()
    out[:, 0] += (0.3 * (out[:, 1].astype(np.float64) - 0.1) ** 2).astype(np.float32)
    out[:, 1] *= np.float32(0.93)
    return out


def written_velocities(pos):
    """Velocities written before the impulse case (float32)."""
    x = pos[:, :3].astype(np.float64)
    v = np.zeros((len(x), 4), np.float32)
    v[:, 0] = 0.5 * np.sin(70 * x[:, 0])
    v[:, 1] = 0.5 * np.cos(50 * x[:, 1])
    v[:, 2] = 0.15
    return v


def appended_layer():
    """A 7 x 7 layer of fluid beside the block, moving down and along x; like the
    block, every coordinate is a quarter cell or more off the cell faces, so float32
    and float64 bin it the same."""
    iy, iz = np.meshgrid(np.arange(7), np.arange(7), indexing="ij")
    pos = np.zeros((49, 3))
    pos[:, 0] = 0.17
    pos[:, 1] = 0.15 + 0.02 * iy.ravel()
    pos[:, 2] = 0.05 + 0.02 * iz.ravel()
    vel = np.tile([0.5, -0.2, 0.0], (49, 1))
    return pos.astype(np.float32), vel.astype(np.float32)


def ops_fixtures():
    out = {}
    dt = (1 / 60) / 2
    # anisotropic pass: reset state (sorted by the prime sort) and displaced positions
    p = case_params("bodies")
    sc = scene_for(p)
    t = transcription(p, sc)
    pos = np.zeros((len(t.pos), 4), np.float32)
    pos[:, :3] = t.pos
    pos[:, 3] = 1.0
    cs = t.cs.astype(np.uint32)
    for name, pin in (("reset", pos), ("moved", moved_positions(pos))):
        sm, G = aniso_f64(pin, cs, [0.0, 0.0, 0.0], t.dim, t.h, ANISO)
        out[f"aniso_{name}_pos"] = pin
        out[f"aniso_{name}_smooth"] = sm
        out[f"aniso_{name}_G"] = G
    out["aniso_cs"] = cs
    # stats after two substeps of the fluid scene
    p = case_params("fluid")
    sc = scene_for(p)
    t = transcription(p, sc)
    for _ in range(2):
        t.substep(dt)
    raw, exact = stats_f64(t.rho.astype(np.float32), t.vel.astype(np.float32), len(t.pos), p["restDensity"],
                           sc["mass"])
    out["stats_raw"] = np.array(raw, np.int64)
    out["stats_exact"] = np.array(exact)
    # ray impulse on written velocities, then one substep
    t = transcription(p, sc)
    pos = t.pos.astype(np.float32)
    vin = written_velocities(pos)
    t.vel = vin[:, :3].astype(np.float64)
    t.vel = impulse_f64(pos, vin, *IMPULSE)
    out["impulse_vel_in"] = vin
    out["impulse_vel"] = t.vel.copy()
    t.substep(dt)
    out["impulse_step_pos"], out["impulse_step_vel"] = t.pos.copy(), t.vel.copy()
    # a held body dragged for two substeps
    pb = case_params("bodies")
    t = transcription(pb, scene_for(pb))
    t.hold(*HOLD)
    for _ in range(2):
        t.substep(dt)
    out["drag_pos"], out["drag_vel"], out["drag_centre"] = t.pos.copy(), t.vel.copy(), t.centre.copy()
    # box resize between two substeps
    t = transcription(p, sc)
    t.substep(dt)
    pr = dict(p, box=list(RESIZED))
    t.resize(RESIZED, boundary_f64(pr, p["spacing"], 2 * p["spacing"]))
    t.substep(dt)
    out["resize_pos"], out["resize_vel"] = t.pos.copy(), t.vel.copy()
    # a fluid layer appended, then one substep
    t = transcription(p, sc)
    t.substep(dt)
    lp, lv = appended_layer()
    t.append(lp, lv)
    t.substep(dt)
    out["append_pos"], out["append_vel"] = t.pos.copy(), t.vel.copy()
    return out


def main():
    out = {}
    for case, substeps in CASES:
        p = case_params(case)
        t = transcription(p, scene_for(p))
        dt = (1 / 60) / p["substeps"]
        for _ in range(substeps):
            t.substep(dt)
        out[f"{case}_pos"] = t.pos
        out[f"{case}_vel"] = t.vel
        out[f"{case}_rho"] = t.rho
        out[f"{case}_body"] = t.body.astype(np.uint32)
        out[f"{case}_substeps"] = np.array(substeps)
    np.savez_compressed(os.path.join(HERE, "transcription_small.npz"), **out)
    np.savez_compressed(os.path.join(HERE, "ops_small.npz"), **ops_fixtures())


if __name__ == "__main__":
    main()
