"""float64 transcriptions of the render passes' shading (the sky, floor and
background functions and the tone map that src/ssfr_composite_wgsl.js and
src/ray_wgsl.js share), for checking the oracle's images pixel by pixel."""
import math

import numpy as np

HAZE = np.array([0.62, 0.74, 0.90])


def pixel_ray(m, w, h, px, py, from_eye=False):
    """The fragment's ray: near/far points through inv_view_proj at the pixel
    centre; origin the near point (SSFR) or the eye (ray march)."""
    nx = (px + 0.5) / w * 2 - 1
    ny = 1 - (py + 0.5) / h * 2
    ivp = np.array(m["inv_view_proj"], np.float64).reshape(4, 4).T
    nh = ivp @ np.array([nx, ny, -1, 1])
    fh = ivp @ np.array([nx, ny, 1, 1])
    near, far = nh[:3] / nh[3], fh[:3] / fh[3]
    rd = far - near
    rd /= np.linalg.norm(rd)
    return (np.array(m["eye"], np.float64) if from_eye else near), rd


def smooth(e0, e1, x):
    t = min(max((x - e0) / (e1 - e0), 0.0), 1.0)
    return t * t * (3 - 2 * t)


def sun_dir(p):
    el, az = math.radians(p["sun_elevation"]), math.radians(p["sun_azimuth"])
    s = np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
    return s / np.linalg.norm(s)


def sky(p, d):
    hh = min(max(d[1], 0.0), 1.0)
    c = HAZE * (1 - smooth(0, 0.16, hh)) + np.array([0.25, 0.48, 0.85]) * smooth(0, 0.16, hh)
    t = smooth(0.10, 0.85, hh)
    c = c * (1 - t) + np.array([0.09, 0.28, 0.72]) * t
    s = max(float(d @ sun_dir(p)), 0.0)
    return c + np.array([1.0, 0.96, 0.88]) * s ** 3000 * 14 + np.array([1.0, 0.92, 0.78]) * s ** 24 * 0.2


def floor_color(q):
    g = np.abs(q[[0, 2]] - np.floor(q[[0, 2]]) - 0.5)
    line = 1 - smooth(0, 0.015, g.min())
    c = np.array([0.30, 0.305, 0.315]) * (1 - line * 0.8) + np.array([0.50, 0.51, 0.52]) * line * 0.8
    fs = math.floor(q[0]) + math.floor(q[2])
    chk = fs - 2 * math.floor(fs * 0.5)
    return c * (0.88 * (1 - chk) + 1.10 * chk)


def background(p, ro, rd):
    if p["floor_plane"] and rd[1] < -1e-4 and (0 - ro[1]) / rd[1] > 0:
        t = (0 - ro[1]) / rd[1]
        fade = 1 - math.exp(-0.02 * t)
        return floor_color(ro + rd * t) * (1 - fade) + HAZE * fade
    return sky(p, rd)


def rgba8(col, exposure=1.0):
    col = np.asarray(col, np.float64) * exposure
    col = col / (1 + col.max() * 0.35)
    col = np.maximum(col, 0.0) ** (1 / 2.2)
    return np.floor(np.clip(col, 0, 1) * 255 + 0.5)
