"""The ray-marched surface (src/ray.js:30-97, src/ray_wgsl.js) on the GPU is bit-
identical to the oracle: the shaded image with the mesh surface pass (the default)
and with the field march, with and without rigid bodies, at two iso levels and
field resolutions, and every debug view in both modes. The surface pass's depth
test does not depend on the order of its atomics."""
import math

import numpy as np
import pytest

import oracle
from particles4all_b200 import Sim, _lib, configs
from particles4all_b200.camera import Camera, frame_matrices
from particles4all_b200.params import default_mesh, default_ray

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


@pytest.fixture(scope="module")
def block():
    p, sc = configs.dam_break_32k(side=10)
    g, o = Sim(), oracle.OracleSim()
    g.reset_scene(p, sc)
    o.reset_scene(p, sc)
    for _ in range(3):
        g.step(1 / 60)
        o.step(1 / 60)
    yield p, g, o
    g.close()


def params_for(w, h, **over):
    cam = Camera()
    cam.target = [2.5, 1.5, 2.5]
    cam.az, cam.el, cam.dist = -0.5, 0.4, 10.0
    m = frame_matrices(cam, w, h)
    rp = default_ray()
    rp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    rp.update(over)
    return rp


def bodies():
    b = np.zeros((2, 6, 4), np.float32)
    b[0, 0] = [1.5, 1.0, 1.5, 1.0]
    b[0, 1] = [0.7, 0.7, 0.7, 0.0]
    b[0, 2:5, :3] = np.eye(3)
    b[0, 5, :3] = [0.60, 0.88, 0.66]
    c, s = math.cos(0.4), math.sin(0.4)
    b[1, 0] = [4.0, 0.6, 2.0, 2.0]          # shape 2 = torus
    b[1, 1] = [0.6, 0.2, 0.0, 0.0]
    b[1, 2, :3] = [1.0, 0.0, 0.0]
    b[1, 3, :3] = [0.0, c, -s]
    b[1, 4, :3] = [0.0, s, c]
    b[1, 5, :3] = [0.96, 0.60, 0.62]
    return b


CASES = [
    ("default", dict(resolution=48), dict(), False),
    ("field", dict(resolution=48), dict(use_surface=0), False),
    ("iso", dict(resolution=64, field_passes=1), dict(iso=0.6, thickness_steps=24, use_surface=0), False),
    ("iso_surface", dict(resolution=64, field_passes=1), dict(iso=0.6, thickness_steps=24), False),
    ("bodies", dict(resolution=48), dict(floor_plane=0, ground_reflection=0.5), True),
    ("bodies_field", dict(resolution=48), dict(floor_plane=0, ground_reflection=0.5, use_surface=0), True),
]


@pytest.mark.parametrize("name,mesh,over,with_bodies", CASES, ids=[c[0] for c in CASES])
def test_ray_matches_oracle(block, name, mesh, over, with_bodies):
    p, g, o = block
    mp = default_mesh()
    mp.update(mesh)
    g.mesh(mp)
    o.mesh(mp)
    rp = params_for(80, 60, **over)
    b = bodies() if with_bodies else None
    g.ray(rp, b)
    a = g.ray_read()
    e = o.ray(rp, b)
    assert a.shape == e.shape == (60, 80, 4)
    bad = np.argwhere(a != e)
    assert bad.size == 0, f"{bad.shape[0]} mismatches, first {bad[:3].tolist()}"
    dbg = params_for(80, 60, **dict(over, debug=2))
    g.ray(dbg, b)
    d = g.ray_read()
    assert d[..., :3].any() and not d[..., :3].all()  # the surface is in view, with background around it


@pytest.mark.parametrize("surface", [1, 0])
@pytest.mark.parametrize("debug", [1, 2, 3, 4, 5, 6])
def test_ray_debug_views_match_oracle(block, debug, surface):
    p, g, o = block
    mp = default_mesh()
    mp["resolution"] = 48
    g.mesh(mp)
    o.mesh(mp)
    rp = params_for(48, 36, debug=debug, use_surface=surface)
    g.ray(rp, bodies())
    assert np.array_equal(g.ray_read(), o.ray(rp, bodies()))


def test_ray_surface_repeatable(block):
    p, g, _ = block
    mp = default_mesh()
    mp["resolution"] = 64
    g.mesh(mp)
    rp = params_for(160, 120, debug=1)
    g.ray(rp)
    first = g.ray_read()
    for _ in range(3):
        g.ray(rp)
        assert np.array_equal(first, g.ray_read())


def test_ray_surface_cut_by_the_near_plane(block):
    """The eye just above the block's top face: the near plane cuts the mesh, and
    the clipped triangles' visible parts come out bit-identical to the oracle."""
    p, g, o = block
    mp = default_mesh()
    mp["resolution"] = 48
    g.mesh(mp)
    o.mesh(mp)
    verts = g.read("meshVerts").view(np.uint32).reshape(-1, 2)
    info = g.mesh_info()
    pos = np.stack([verts[:, 0] & 0xFFFF, verts[:, 0] >> 16, verts[:, 1] & 0xFFFF], 1) / 65535.0
    pos = pos * (np.array(info["vert_dim"]) - 1) * info["voxel"] + np.array(info["origin"])
    near = (np.abs(pos[:, 0] - 2.5) < 1.0) & (np.abs(pos[:, 2] - 2.5) < 1.0)
    cam = Camera()
    cam.target = [2.5, float(pos[near, 1].max()), 2.5]  # the top face above the block's centre
    cam.az, cam.el, cam.dist = 0.3, 0.6, 0.05
    m = frame_matrices(cam, 64, 48)
    for debug in (0, 1, 2):
        rp = default_ray()
        rp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
        rp["debug"] = debug
        g.ray(rp)
        a, e = g.ray_read(), o.ray(rp)
        bad = np.argwhere(a != e)
        assert bad.size == 0, f"debug {debug}: {bad.shape[0]} mismatches, first {bad[:3].tolist()}"
