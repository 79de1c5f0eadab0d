"""CPU checks of the environment map (src/env.js, envSample in src/ray_wgsl.js and
src/ssfr_composite_wgsl.js): the .hdr reader on RGBE files written here in both
scanline encodings, the oracle's cube map against a float64 resampling of the
panorama with the reference's half rounding, and the composite's sky pixels
against float64 cube sampling (and, for a smooth panorama, against the panorama
itself in the yaw-rotated direction)."""
import math
import struct

import numpy as np

import oracle
import render_f64
from particles4all_b200.camera import Camera, frame_matrices
from particles4all_b200.hdr import decode_hdr
from particles4all_b200.params import default_aniso, default_ssfr
from test_ssfr_oracle import pair_sim


def rgbe_of(rgb):
    """Exact RGBE bytes of values that are m * 2^k with m < 256."""
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    for idx in np.ndindex(rgb.shape[:-1]):
        v = rgb[idx]
        big = float(v.max())
        if big <= 0:
            continue
        e = math.frexp(big)[1]
        out[idx][:3] = np.round(v / 2.0 ** (e - 8)).astype(np.uint8)
        out[idx][3] = e + 128
    return out


def hdr_bytes(rgbe, rle):
    h, w, _ = rgbe.shape
    head = b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode()
    body = bytearray()
    for y in range(h):
        if rle:
            body += bytes([2, 2, w >> 8, w & 255])
            for c in range(4):
                row, x = rgbe[y, :, c], 0
                while x < w:
                    n = 1
                    while x + n < w and n < 127 and row[x + n] == row[x]:
                        n += 1
                    if n > 2:
                        body += bytes([128 + n, row[x]])
                    else:
                        n = min(w - x, 64)
                        body += bytes([n]) + bytes(row[x:x + n])
                    x += n
        else:
            x = 0
            while x < w:
                body += bytes(rgbe[y, x])
                run = 1
                while x + run < w and run < 255 and (rgbe[y, x + run] == rgbe[y, x]).all():
                    run += 1
                if run > 2:  # the old repeat marker: 1 1 1 n copies the previous pixel n times
                    body += bytes([1, 1, 1, run - 1])
                    x += run
                else:
                    x += 1
    return head + bytes(body)


def test_hdr_reader_both_encodings():
    rng = np.random.default_rng(2)
    h, w = 5, 24
    mant = rng.integers(1, 256, (h, w, 3)).astype(np.float64)
    mant[:, 8:14] = mant[:, 8:9]  # runs
    expo = rng.integers(-6, 6, (h, w, 1))
    rgb = mant * 2.0 ** (expo - 8)
    rgb[1, 3] = 0.0
    rgbe = rgbe_of(rgb)
    e = rgbe[..., 3:].astype(np.float64)
    want = np.where(e > 0, rgbe[..., :3] * 2.0 ** (e - 136), 0.0).astype(np.float32)
    for rle in (True, False):
        got = decode_hdr(hdr_bytes(rgbe, rle))
        assert got.shape == (h, w, 3) and np.array_equal(got, want), rle


def to_half_ref(v):
    """toHalf (src/env.js:125-147) in Python, on float32 values."""
    x = struct.unpack("<I", struct.pack("<f", float(v)))[0]
    s = (x >> 16) & 0x8000
    e = ((x >> 23) & 0xFF) - 112
    m = x & 0x7FFFFF
    if e <= 0:
        if e < -10:
            return s
        m = (m | 0x800000) >> (1 - e)
        return s | ((m + 0x1000) >> 13)
    if e >= 0x1F:
        return s | 0x7C00
    return s | (e << 10) | ((m + 0x1000) >> 13)


def panorama(w, h, kind):
    y, x = np.mgrid[0:h, 0:w]
    lon = (x + 0.5) / w * 2 * np.pi - np.pi
    lat = np.pi / 2 - (y + 0.5) / h * np.pi
    if kind == "smooth":
        r = 0.55 + 0.35 * np.cos(lon) * np.cos(lat)
        g = 0.55 + 0.35 * np.sin(lon) * np.cos(lat)
        b = 0.55 + 0.35 * np.sin(lat)
        return np.stack([r, g, b], -1).astype(np.float32)
    rng = np.random.default_rng(5)
    return (rng.random((h, w, 3)) * np.array([4.0, 1.0, 0.25])).astype(np.float32)


def face_dirs(size):
    t, s = np.meshgrid(2 * (np.arange(size) + 0.5) / size - 1, 2 * (np.arange(size) + 0.5) / size - 1,
                       indexing="ij")
    one = np.ones_like(s)
    return [np.stack(v, -1) for v in ((one, -t, -s), (-one, -t, s), (s, one, t), (s, -one, -t), (s, -t, one),
                                      (-s, -t, -one))]


def equirect_f64(src, d):
    h, w, _ = src.shape
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)
    u = 0.5 + np.arctan2(d[..., 0], d[..., 2]) / (2 * np.pi)
    v = np.arccos(np.clip(d[..., 1], -1, 1)) / np.pi
    fx, fy = u * w - 0.5, v * h - 0.5
    x0, y0 = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
    tx, ty = (fx - x0)[..., None], (fy - y0)[..., None]

    def at(x, y):
        return src[np.clip(y, 0, h - 1), x % w].astype(np.float64)
    a = at(x0, y0) * (1 - tx) + at(x0 + 1, y0) * tx
    b = at(x0, y0 + 1) * (1 - tx) + at(x0 + 1, y0 + 1) * tx
    return (a * (1 - ty) + b * ty).astype(np.float32)


def test_cube_map_against_float64(built):
    src = panorama(96, 48, "noise")
    o = oracle.OracleSim()
    o.set_environment(src)
    cube = o.environment()
    size = 24
    assert cube.shape == (6, size, size, 4)
    half = np.vectorize(to_half_ref, otypes=[np.uint16])
    mism = 0
    for f, d in enumerate(face_dirs(size)):
        want = half(equirect_f64(src, d))
        got = cube[f, ..., :3]
        diff = np.abs(got.astype(np.int64) - want.astype(np.int64))
        assert diff.max() <= 1, (f, diff.max())  # a last-bit libm difference at most
        mism += int((diff > 0).sum())
        assert (cube[f, ..., 3] == 0x3C00).all()
    assert mism <= cube.size // 1000, mism
    o.set_environment(None)
    assert o.environment() is None
    assert to_half_ref(65520.0) == 0x7C00 and to_half_ref(1e-9) == 0


def half_to_f64(bits):
    return bits.astype(np.uint16).view(np.float16).astype(np.float64)


def cube_sample_f64(cube, d, footprint=None):
    size = cube.shape[1]
    ax, ay, az = np.abs(d)
    if ax >= ay and ax >= az:
        face, ma, sc, tc = (0 if d[0] >= 0 else 1), ax, (-d[2] if d[0] >= 0 else d[2]), -d[1]
    elif ay >= az:
        face, ma, sc, tc = (2 if d[1] >= 0 else 3), ay, d[0], (d[2] if d[1] >= 0 else -d[2])
    else:
        face, ma, sc, tc = (4 if d[2] >= 0 else 5), az, (d[0] if d[2] >= 0 else -d[0]), -d[1]
    u = 0.5 * (sc / ma + 1) * size - 0.5
    v = 0.5 * (tc / ma + 1) * size - 0.5
    x0, y0 = math.floor(u), math.floor(v)
    tx, ty = u - x0, v - y0
    def c(y, x):
        y, x = min(max(y, 0), size - 1), min(max(x, 0), size - 1)
        if footprint is not None:
            footprint.append((face, y, x))
        return half_to_f64(cube[face, y, x, :3])
    top = c(y0, x0) * (1 - tx) + c(y0, x0 + 1) * tx
    bot = c(y0 + 1, x0) * (1 - tx) + c(y0 + 1, x0 + 1) * tx
    return top * (1 - ty) + bot * ty


def sky_view(kind, yaw, intensity):
    o, p = pair_sim()
    src = panorama(128, 64, kind)
    o.set_environment(src)
    cam = Camera()
    cam.target = [4.0, 3.0, 2.5]
    cam.az, cam.el, cam.dist = 0.7, -0.35, 6.0  # looking up: mostly sky
    m = frame_matrices(cam, 64, 48)
    sp = default_ssfr()
    sp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    sp.update(env_intensity=intensity, env_yaw=yaw, floor_plane=0)
    o.aniso(default_aniso())
    o.ssfr(sp)
    return o, src, sp, m


def rotate(d, yaw):
    c, s = math.cos(yaw), math.sin(yaw)
    return np.array([c * d[0] + s * d[2], d[1], -s * d[0] + c * d[2]])


def test_composite_sky_from_the_cube_map(built):
    yaw, gain = 0.8, 1.3
    o, src, sp, m = sky_view("noise", yaw, gain)
    img, z, cube = o.ssfr_read("image"), o.ssfr_read("eyeZ"), o.environment()
    checked = 0
    for py in range(0, 48, 3):
        for px in range(0, 64, 3):
            if z[py, px] > -1e3:
                continue
            ro, rd = render_f64.pixel_ray(m, sp["width"], sp["height"], px, py)
            want = render_f64.rgba8(cube_sample_f64(cube, rotate(rd, yaw)) * gain, sp["exposure"])
            assert np.abs(img[py, px, :3] - want).max() <= 1, (px, py, img[py, px], want)
            checked += 1
    assert checked > 100


def test_composite_sky_follows_the_panorama(built):
    """End to end on a smooth panorama: the sky pixel in direction d is the
    panorama's value at d turned by the yaw. The reference's half rounding ORs a
    mantissa carry into the exponent field, so a value just below a power of two
    with an odd half exponent (0.49995 -> 0.25) comes out halved; the cube keeps
    that, and pixels that sample such a texel are left out here."""
    assert to_half_ref(np.float32(0.49995)) == 0x3400 and to_half_ref(np.float32(0.99995)) == 0x3C00
    yaw = -1.1
    o, src, sp, m = sky_view("smooth", yaw, 1.0)
    img, z, cube = o.ssfr_read("image"), o.ssfr_read("eyeZ"), o.environment()
    rounded = half_to_f64(cube[..., :3])
    size = cube.shape[1]
    true = np.stack([equirect_f64(src, d) for d in face_dirs(size)]).astype(np.float16).astype(np.float64)
    halved = (rounded < 0.75 * true).any(-1)
    assert halved.any()
    checked = 0
    for py in range(0, 48, 4):
        for px in range(0, 64, 4):
            if z[py, px] > -1e3:
                continue
            ro, rd = render_f64.pixel_ray(m, sp["width"], sp["height"], px, py)
            used = []
            cube_sample_f64(cube, rotate(rd, yaw), used)
            if any(halved[t] for t in used):
                continue
            want = render_f64.rgba8(equirect_f64(src, rotate(rd, yaw)[None])[0].astype(np.float64), sp["exposure"])
            assert np.abs(img[py, px, :3] - want).max() <= 3, (px, py, img[py, px], want)
            checked += 1
    assert checked > 50
