"""The surface mesh (src/mesh.js:99-352, src/mesh_wgsl.js:23-238) on the GPU is bit-
identical to the oracle: the density field, the blurred normal field and the packed
triangle vertices (both in voxel order), and the triangle total, for both blur-axis
modes, with field passes, and with a triangle cap."""
import numpy as np
import pytest

import oracle
from particles4all_b200 import Sim, _lib, configs
from particles4all_b200.params import default_mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def pair(p, sc, frames):
    g = Sim()
    g.reset_scene(p, sc)
    o = oracle.OracleSim()
    o.reset_scene(p, sc)
    for _ in range(frames):
        g.step(1 / 60)
        o.step(1 / 60)
    return g, o


CASES = [
    ("medium_bodies", dict(resolution=64)),
    ("medium_bodies", dict(resolution=96, blur_axes=1, field_passes=1)),
    ("dam_break", dict(resolution=128)),
    ("dam_break", dict(resolution=80, normal_passes=0, iso=0.6)),
]


@pytest.mark.parametrize("scene,over", CASES)
def test_mesh_matches_oracle(scene, over):
    p, sc = (configs.medium_bodies_264k(side=16, n_cubes=2) if scene == "medium_bodies"
             else configs.dam_break_32k(side=14))
    g, o = pair(p, sc, 4)
    m = default_mesh()
    m.update(over)
    tg = g.mesh(m)
    to = o.mesh(m)
    assert tg == to and tg > 0
    assert np.array_equal(g.read("meshField"), o.buffer("meshField"))
    assert np.array_equal(g.read("meshNField"), o.buffer("meshNField"))
    assert np.array_equal(g.read("meshVerts"), o.buffer("meshVerts").reshape(-1, 2))
    info = g.mesh_info()
    assert info["triangles"] == tg and np.prod(info["vert_dim"]) == g.read("meshField").size
    g.close()


def test_mesh_triangle_cap():
    p, sc = configs.dam_break_32k(side=12)
    g, o = pair(p, sc, 2)
    m = default_mesh()
    m["resolution"] = 64
    full = g.mesh(m)
    verts = g.read("meshVerts").copy()
    m["max_triangles"] = full // 3
    assert g.mesh(m) == full == o.mesh(m)  # the total counts every triangle
    capped = g.read("meshVerts")
    assert capped.shape[0] == 3 * (full // 3)
    assert np.array_equal(capped, verts[: capped.shape[0]])
    assert np.array_equal(capped, o.buffer("meshVerts").reshape(-1, 2))
    g.close()
