"""The environment map on the GPU (src/env.js, envSample in src/ssfr_composite_wgsl.js
and src/ray_wgsl.js): the library's cube map is the oracle's bit for bit, and the
screen-space fluid rendering and the ray pass (mesh surface and field march) that
sample it for the sky, the floor's far colour and reflections give the oracle's
images, with a yaw and an intensity, with the floor plane on and off; clearing the
map brings back the built-in sky."""
import numpy as np
import pytest

import oracle
from particles4all_b200 import Sim, _lib, configs
from particles4all_b200.camera import Camera, frame_matrices
from particles4all_b200.params import default_aniso, default_mesh, default_ray, default_ssfr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def panorama(w, h):
    rng = np.random.default_rng(11)
    y, x = np.mgrid[0:h, 0:w]
    lon = (x + 0.5) / w * 2 * np.pi
    lat = np.pi / 2 - (y + 0.5) / h * np.pi
    base = np.stack([0.6 + 0.4 * np.cos(lon) * np.cos(lat), 0.5 + 0.3 * np.sin(2 * lon), 0.7 + 0.5 * np.sin(lat)], -1)
    return (base * (1 + 0.3 * rng.random((h, w, 1)))).astype(np.float32)


@pytest.fixture(scope="module")
def scene():
    p, sc = configs.dam_break_32k(side=10)
    g, o = Sim(), oracle.OracleSim()
    g.reset_scene(p, sc)
    o.reset_scene(p, sc)
    for _ in range(2):
        g.step(1 / 60)
        o.step(1 / 60)
    for s in (g, o):
        s.aniso(default_aniso())
        s.set_environment(panorama(160, 80))
    yield g, o
    g.close()


def matrices(w, h):
    cam = Camera()
    cam.target = [2.5, 1.5, 2.5]
    cam.az, cam.el, cam.dist = -0.5, 0.3, 11.0
    m = frame_matrices(cam, w, h)
    return {k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")}


def test_cube_map_matches_oracle(scene):
    g, o = scene
    a, b = g.environment(), o.environment()
    assert a.shape == b.shape == (6, 40, 40, 4)
    assert np.array_equal(a, b)


def bodies():
    """A sphere and a box in the renderers' packed layout: their shading reflects the
    environment (envReflect)."""
    b = np.zeros((2, 6, 4), np.float32)
    b[0, 0] = [1.2, 0.9, 1.0, 1.0]
    b[0, 1] = [0.6, 0.6, 0.6, 0.0]
    b[0, 2:5, :3] = np.eye(3)
    b[0, 5, :3] = [0.60, 0.88, 0.66]
    b[1, 0] = [3.5, 0.7, 3.0, 0.0]
    b[1, 1] = [0.5, 0.3, 0.4, 0.0]
    b[1, 2:5, :3] = np.eye(3)
    b[1, 5, :3] = [0.55, 0.72, 0.95]
    return b


@pytest.mark.parametrize("floor,debug,with_bodies", [(0, 0, False), (1, 0, True), (0, 4, False), (0, 0, True)])
def test_ssfr_with_environment(scene, floor, debug, with_bodies):
    g, o = scene
    sp = default_ssfr()
    sp.update(matrices(80, 60))
    sp.update(env_intensity=1.4, env_yaw=0.9, floor_plane=floor, debug=debug)
    b = bodies() if with_bodies else None
    g.ssfr(sp, b)
    o.ssfr(sp, b)
    a, b = g.ssfr_read("image"), o.ssfr_read("image")
    assert np.array_equal(a, b), np.argwhere(a != b)[:3].tolist()


@pytest.mark.parametrize("surface", [1, 0])
def test_ray_with_environment(scene, surface):
    g, o = scene
    mp = default_mesh()
    mp["resolution"] = 48
    g.mesh(mp)
    o.mesh(mp)
    for floor, debug, packed in ((0, 0, None), (1, 6, None), (0, 0, bodies())):
        rp = default_ray()
        rp.update(matrices(64, 48))
        rp.update(env_intensity=0.8, env_yaw=-2.0, floor_plane=floor, debug=debug, use_surface=surface)
        g.ray(rp, packed)
        a, b = g.ray_read(), o.ray(rp, packed)
        assert np.array_equal(a, b), (floor, debug, np.argwhere(a != b)[:3].tolist())


def test_clearing_restores_the_sky(scene):
    g, o = scene
    sp = default_ssfr()
    sp.update(matrices(48, 36))
    g.ssfr(sp)
    with_env = g.ssfr_read("image").copy()
    for s in (g, o):
        s.set_environment(None)
    assert g.environment() is None
    g.ssfr(sp)
    o.ssfr(sp)
    plain = g.ssfr_read("image")
    assert np.array_equal(plain, o.ssfr_read("image"))
    assert not np.array_equal(plain, with_env)
    for s in (g, o):
        s.set_environment(panorama(160, 80))
    with pytest.raises(_lib.P4AError):
        g.set_environment(np.zeros((10, 30, 3), np.float32))  # not 2:1
    assert g.environment().shape == (6, 40, 40, 4)  # a rejected panorama keeps the map
