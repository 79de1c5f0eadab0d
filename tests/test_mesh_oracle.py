"""CPU checks of the oracle's surface mesh (src/mesh_wgsl.js:23-238): the density
field against a float64 brute-force splat of the same particles, and the packed
vertices' layout (grid positions in range, octahedral normals of unit L1 norm)."""
import math

import numpy as np

import oracle
from particles4all_b200 import configs
from particles4all_b200.params import default_mesh


def test_field_and_vertices(built):
    p, sc = configs.dam_break_32k(side=8)
    o = oracle.OracleSim()
    o.reset_scene(p, sc)
    o.step(1 / 60)
    m = default_mesh()
    m["resolution"] = 48
    tris = o.mesh(m)
    assert tris > 0
    f = o.buffer("meshField")
    info = o.info()
    box = np.array(p["box"], np.float64)
    voxel = box.max() / 48
    dim = [int(math.ceil(b / voxel)) + 3 for b in box]
    assert f.size == dim[0] * dim[1] * dim[2]
    # float64 splat: every particle within h of a vertex, volume m / max(rho, rho0 / 2)
    h = info["h"]
    n = info["n"]
    pos = o.buffer("pos")[:n, :3].astype(np.float64)
    rho = o.buffer("density")[:n].astype(np.float64)
    mass = info["mass"]
    vol = mass / np.maximum(rho, 0.5 * p["restDensity"])
    poly6 = 315 / (64 * math.pi * h ** 9)
    rng = np.random.default_rng(0)
    for idx in rng.choice(f.size, 400, replace=False).tolist() + [int(np.argmax(f))]:
        x, y, z = idx % dim[0], (idx // dim[0]) % dim[1], idx // (dim[0] * dim[1])
        v = -voxel + voxel * np.array([x, y, z], np.float64)
        r2 = ((pos - v) ** 2).sum(1)
        t = np.clip(h * h - r2, 0, None)
        want = float((vol * poly6 * t ** 3).sum())
        assert abs(f[idx] - want) <= 1e-4 * max(1.0, abs(want)), (idx, f[idx], want)
    v = o.buffer("meshVerts").reshape(-1, 2)
    assert v.shape[0] == 3 * tris
    q = np.stack([v[:, 0] & 0xFFFF, v[:, 0] >> 16, v[:, 1] & 0xFFFF], 1)
    assert q.max() <= 65535
    e = np.stack([(v[:, 1] >> 16) & 0xFF, v[:, 1] >> 24], 1) / 255.0 * 2 - 1
    assert np.all(np.abs(e).sum(1) <= 2.0 + 1e-6)
