"""Screen-space fluid rendering (src/ssfr.js:173-356, src/ssfr_wgsl.js,
src/ssfr_composite_wgsl.js) on the GPU is bit-identical to the oracle: the
unfiltered and filtered eye-space depth maps, the blurred thickness map, the
body-depth map and the RGBA8 image, for the default settings, the other filter
modes, a reduced render scale with a full-resolution thickness map, rigid bodies
in the composite, and every debug view. Two runs give the same bits."""
import math

import numpy as np
import pytest

import oracle
from particles4all_b200 import Sim, _lib, configs
from particles4all_b200.camera import Camera, frame_matrices
from particles4all_b200.params import default_aniso, default_ssfr

pytestmark = pytest.mark.gpu

BUFFERS = ("rawZ", "eyeZ", "thick", "bodyT", "image")


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


@pytest.fixture(scope="module")
def block():
    """A 10^3-particle dam-break block after 3 frames, anisotropic pass done."""
    p, sc = configs.dam_break_32k(side=10)
    g, o = Sim(), oracle.OracleSim()
    g.reset_scene(p, sc)
    o.reset_scene(p, sc)
    for _ in range(3):
        g.step(1 / 60)
        o.step(1 / 60)
    g.aniso(default_aniso())
    o.aniso(default_aniso())
    yield p, g, o
    g.close()


def params_for(p, w, h, **over):
    cam = Camera()
    cam.target = [2.5, 1.5, 2.5]
    cam.az, cam.el, cam.dist = -0.5, 0.35, 11.0
    m = frame_matrices(cam, w, h)
    sp = default_ssfr()
    sp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    sp.update(over)
    return sp


def packed_bodies():
    """Two rigid bodies in the composite's packed layout: a sphere and a rotated box."""
    b = np.zeros((2, 6, 4), np.float32)
    b[0, 0] = [1.2, 0.9, 1.0, 1.0]          # centre, shape 1 = sphere
    b[0, 1] = [0.6, 0.6, 0.6, 0.0]          # radius
    b[0, 2:5, :3] = np.eye(3)
    b[0, 5, :3] = [0.60, 0.88, 0.66]
    c, s = math.cos(0.5), math.sin(0.5)
    b[1, 0] = [3.5, 0.7, 3.0, 0.0]          # shape 0 = box
    b[1, 1] = [0.5, 0.3, 0.4, 0.0]          # half extents
    b[1, 2, :3] = [c, 0.0, -s]
    b[1, 3, :3] = [0.0, 1.0, 0.0]
    b[1, 4, :3] = [s, 0.0, c]
    b[1, 5, :3] = [0.55, 0.72, 0.95]
    return b


def compare(g, o):
    for name in BUFFERS:
        a, b = g.ssfr_read(name), o.ssfr_read(name)
        assert a.shape == b.shape, (name, a.shape, b.shape)
        if a.dtype == np.float32:
            bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
        else:
            bad = np.argwhere(a != b)
        assert bad.size == 0, f"{name}: {bad.shape[0]} mismatches, first {bad[:3].tolist()}"


CASES = [
    ("default", dict(), False),
    ("gaussian", dict(filter=0, filter_iterations=1), False),
    ("bilateral", dict(filter=1, cleanup_pass=0), False),
    ("scaled", dict(render_scale=0.6, thickness_half_res=0, thickness_filter_size=5, depth_cull_neighbours=200),
     False),
    ("bodies", dict(floor_plane=0, ground_reflection=0.3, exposure=1.4), True),
]


@pytest.mark.parametrize("name,over,bodies", CASES, ids=[c[0] for c in CASES])
def test_ssfr_matches_oracle(block, name, over, bodies):
    p, g, o = block
    sp = params_for(p, 96, 72, **over)
    b = packed_bodies() if bodies else None
    g.ssfr(sp, b)
    o.ssfr(sp, b)
    compare(g, o)
    z = g.ssfr_read("eyeZ")
    assert (z > -1e3).any() and (z < -1e3).any()  # the block is in view, with background around it
    if bodies:
        assert (g.ssfr_read("bodyT") < 1e29).any()


@pytest.mark.parametrize("debug", [1, 2, 3, 4, 5])
def test_ssfr_debug_views_match_oracle(block, debug):
    p, g, o = block
    sp = params_for(p, 64, 48, debug=debug)
    g.ssfr(sp, packed_bodies())
    o.ssfr(sp, packed_bodies())
    a, b = g.ssfr_read("image"), o.ssfr_read("image")
    assert np.array_equal(a, b), np.argwhere(a != b)[:3].tolist()


def test_ssfr_repeatable(block):
    """Depth ties and the thickness sums do not depend on the order of the atomics."""
    p, g, _ = block
    sp = params_for(p, 128, 96)
    g.ssfr(sp)
    first = {k: g.ssfr_read(k) for k in BUFFERS}
    g.ssfr(sp)
    for k in BUFFERS:
        assert np.array_equal(first[k], g.ssfr_read(k)), k
