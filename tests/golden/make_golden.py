"""Writes transcription_small.npz: positions, velocities and densities of four tiny
scenes (fluid, a rigid body, surface tension, both) after one or two substeps, from
the float64 NumPy transcription of the reference's passes in
tests/test_oracle_transcription.py (written from the WGSL / JS text; it shares no
code with the oracle or the library). The reference itself (a browser WebGPU app)
cannot run here, so these are the fixed float64 answers the float32 paths are held
to. Scene inputs come from the scene builder both paths use.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from test_oracle_transcription import Transcription  # noqa: E402

from particles4all_b200.params import default_params  # noqa: E402

CASES = [("fluid", 2), ("bodies", 2), ("tension", 2), ("bodies_tension", 1)]


def case_params(case):
    p = default_params("small")
    p.update({"targetParticleCount": 350, "box": [0.25, 0.3, 0.21], "bodies": [], "substeps": 2})
    if "bodies" in case:
        p.update({"bodies": ["box:0.5"], "bodySize": 0.03})
    if "tension" in case:
        p.update({"surfaceTensionK": 0.4})
    return p


def main():
    out = {}
    for case, substeps in CASES:
        p = case_params(case)
        sc = oracle.build_scene(p)
        bpts, bpsi = oracle.boundary(p, p["spacing"], 2 * p["spacing"])
        t = Transcription(p, sc, bpts, bpsi)
        dt = (1 / 60) / p["substeps"]
        for _ in range(substeps):
            t.substep(dt)
        out[f"{case}_pos"] = t.pos
        out[f"{case}_vel"] = t.vel
        out[f"{case}_rho"] = t.rho
        out[f"{case}_body"] = t.body.astype(np.uint32)
        out[f"{case}_substeps"] = np.array(substeps)
    np.savez_compressed(os.path.join(HERE, "transcription_small.npz"), **out)


if __name__ == "__main__":
    main()
