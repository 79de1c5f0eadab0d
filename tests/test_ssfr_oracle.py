"""CPU checks of the oracle's screen-space fluid rendering (src/ssfr.js,
src/ssfr_wgsl.js, src/ssfr_composite_wgsl.js): the exp / log the render passes use
against float64, the splats of a particle pair against the analytic spheres
(nearest depth, silhouette, per-pixel thickness chords), composite pixels that
see no fluid against a float64 transcription of the sky / floor shading and tone
map, and the depth filter's narrow range on a particle block."""
import math

import numpy as np

import oracle
import render_f64
from particles4all_b200 import configs
from particles4all_b200.camera import Camera, frame_matrices
from particles4all_b200.params import default_aniso, default_ssfr


def test_exp_log_against_float64(built):
    L = oracle.lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-87, 88, 20000), rng.uniform(-2, 2, 20000), [0.0, -0.0, 1.0, -1.0]])
    xs = xs.astype(np.float32)
    worst = 0.0
    for x in xs.tolist():
        got = L.orc_expf(x)
        want = math.exp(float(np.float32(x)))
        worst = max(worst, abs(got - want) / want)
    assert worst < 3.0e-7, worst
    ys = np.concatenate([np.exp(rng.uniform(-80, 80, 20000)), rng.uniform(0.5, 2.0, 20000), [1.0, 2.0, 1e-40]])
    ys = ys.astype(np.float32)
    worst = 0.0
    for y in ys.tolist():
        got = L.orc_logf(y)
        want = math.log(float(np.float32(y)))
        worst = max(worst, abs(got - want) / max(1.0, abs(want)))
    assert worst < 2.0e-7, worst
    assert L.orc_expf(100.0) == math.inf and L.orc_expf(-200.0) == 0.0
    assert L.orc_logf(0.0) == -math.inf and math.isnan(L.orc_logf(-1.0))


def pair_sim():
    """Two fluid particles 0.5 apart in an 8 x 6 x 5 box. Each sees only the other
    within the anisotropic radius, far fewer than N_eps, so its kernel is the
    isotropic G = (kn / h) I: a sphere of radius splatRadius x spacing around
    its smoothed centre. (A particle with no neighbour at all gets a NaN G, in the
    reference as here: its covariance is zero and 1 / extent is infinite.)"""
    p = configs._base_params([8.0, 6.0, 5.0], iterations=2, tension=0.0, xsph=0.0)
    fluid = np.array([[3.75, 3.0, 2.5], [4.25, 3.0, 2.5]], np.float64)
    sc = configs._assemble(fluid, [], p, configs.lattice_mass(0.5, 1.0))
    o = oracle.OracleSim()
    o.reset_scene(p, sc)
    o.aniso(default_aniso())
    return o, p


def camera_for(p, w, h, az=0.0, el=0.0, dist=6.0):
    cam = Camera()
    cam.target = [4.0, 3.0, 2.5]
    cam.az, cam.el, cam.dist = az, el, dist
    m = frame_matrices(cam, w, h)
    sp = default_ssfr()
    sp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    return sp, m


def test_particle_pair_depth_and_thickness(built):
    o, p = pair_sim()
    w = h = 96
    sp, m = camera_for(p, w, h)
    sp.update({"filter_iterations": 0, "thickness_filter_size": 0, "thickness_half_res": 0})
    o.ssfr(sp)
    raw = o.ssfr_read("rawZ")
    thick = o.ssfr_read("thick")
    assert raw.shape == (h, w) and thick.shape == (h, w)
    g = o.buffer("aniso")[:4]
    assert np.allclose(g[0], [1, 0, 0, 1]) and np.allclose(g[1, :3], [0, 1, 1])  # G = I
    centres = o.buffer("smoothPos")[:2, :3].astype(np.float64)
    eye = np.array(m["eye"])
    radius = 0.5  # splatRadius x spacing
    hit = raw > -1e3
    assert hit.any()
    # nearest surface: eye-space z of the spheres' front points (camera looks along -z)
    front = -(eye[2] - centres[:, 2].max() - radius)
    assert abs(raw.max() - front) < 2e-2, (raw.max(), front)
    # silhouette height: angular radius asin(r / d) against the projection's pixel footprint
    dist = np.linalg.norm(centres.mean(0) - eye)
    proj11 = m["proj"][5]
    half_px = math.tan(math.asin(radius / dist)) * proj11 * h / 2
    rows = np.nonzero(hit.any(1))[0]
    assert abs((rows[-1] - rows[0] + 1) / 2 - half_px) <= 1.0, (rows, half_px)
    # thickness: the chords of both spheres of radius 0.62 x spacing along every
    # pixel's ray, summed, against float64 (pixels within one pixel of a silhouette
    # may differ in coverage and are skipped)
    tr = 0.62 * 0.5
    ivp = np.array(m["inv_view_proj"], np.float64).reshape(4, 4).T
    want = np.zeros((h, w))
    margin = np.zeros((h, w), bool)
    for py in range(h):
        for px in range(w):
            nx, ny = (px + 0.5) / w * 2 - 1, 1 - (py + 0.5) / h * 2
            a, b = ivp @ [nx, ny, -1, 1], ivp @ [nx, ny, 1, 1]
            ro = a[:3] / a[3]
            rd = b[:3] / b[3] - ro
            rd /= np.linalg.norm(rd)
            for c in centres:
                oc = ro - c
                bb, cc = oc @ rd, oc @ oc - tr * tr
                disc = bb * bb - cc
                if disc > 0:
                    want[py, px] += 2 * math.sqrt(disc)
                margin[py, px] |= abs(disc) < 2e-3
    ok = ~margin
    # float32 rays: b^2 - c cancels (b ~ 6, c ~ 36), so chords carry ~1e-4 absolute error
    assert np.abs(thick[ok] - want[ok]).max() < 1e-3, np.abs(thick[ok] - want[ok]).max()
    assert np.count_nonzero(want) > 50


def test_composite_background_against_float64(built):
    o, p = pair_sim()
    sp, m = camera_for(p, 64, 48, az=0.6, el=0.25, dist=9.0)
    o.ssfr(sp)
    img = o.ssfr_read("image")
    assert img.shape == (48, 64, 4) and (img[..., 3] == 255).all()
    z = o.ssfr_read("eyeZ")
    checked = 0
    for py in range(0, 48, 5):
        for px in range(0, 64, 7):
            if z[py, px] > -1e3:
                continue
            ro, rd = render_f64.pixel_ray(m, sp["width"], sp["height"], px, py)
            want = render_f64.rgba8(render_f64.background(sp, ro, rd), sp["exposure"])
            assert np.abs(img[py, px, :3].astype(np.float64) - want).max() <= 1.0, (px, py, img[py, px], want)
            checked += 1
    assert checked > 30


def test_depth_filter_keeps_background_and_smooths(built):
    """A block of particles: the filtered depth keeps the empty pixels empty and
    stays within the narrow range of the raw depth around every covered pixel."""
    p, sc = configs.dam_break_32k(side=6)
    o = oracle.OracleSim()
    o.reset_scene(p, sc)
    o.step(1 / 60)
    o.aniso(default_aniso())
    cam = Camera().frame(p["box"])
    cam.target = [2.0, 1.5, 1.5]
    cam.dist = 9.0
    mm = frame_matrices(cam, 80, 60)
    sp = default_ssfr()
    sp.update({k: mm[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    o.ssfr(sp)
    raw, z = o.ssfr_read("rawZ"), o.ssfr_read("eyeZ")
    empty = raw < -1e3
    assert empty.any() and (~empty).any()
    assert np.array_equal(z < -1e3, empty)
    delta = sp["narrow_delta"] * 0.5 * 0.5
    assert np.all(np.abs(z[~empty] - raw[~empty]) <= 4 * delta + 1.0)
