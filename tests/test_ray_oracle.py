"""CPU checks of the oracle's ray-marched surface (src/ray_wgsl.js): the distance to
the iso surface (debug view 2) against a float64 march of the same trilinear field
along each pixel's ray, pixels that miss the field against the float64 sky / floor
shading and tone map, and the mesh surface pass (src/mesh.js:380-396): distance and
normal (debug views 2 and 1) against float64 ray / triangle intersections with the
mesh's decoded vertices and perspective-correct normal interpolation."""
import math

import numpy as np

import oracle
import render_f64
from particles4all_b200 import configs
from particles4all_b200.camera import Camera, frame_matrices
from particles4all_b200.params import default_mesh, default_ray


def block_with_field():
    p, sc = configs.dam_break_32k(side=8)
    o = oracle.OracleSim()
    o.reset_scene(p, sc)
    o.step(1 / 60)
    m = default_mesh()
    m["resolution"] = 40
    o.mesh(m)
    return o, p


def ray_params(w, h, **over):
    cam = Camera()
    cam.target = [2.0, 1.5, 2.0]
    cam.az, cam.el, cam.dist = -0.6, 0.45, 9.0
    m = frame_matrices(cam, w, h)
    rp = default_ray()
    rp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    rp["use_surface"] = 0
    rp.update(over)
    return rp, m


def field_hit_f64(o, p, ro, rd, iso):
    """First iso crossing of the trilinear field along ro + t rd inside the field's
    volume, by fine sampling and bisection in float64; None on a miss."""
    info_box = np.array(p["box"], np.float64)
    voxel = info_box.max() / 40
    dim = np.array([int(math.ceil(b / voxel)) + 3 for b in info_box])
    f = o.buffer("meshField").astype(np.float64).reshape(dim[2], dim[1], dim[0])
    origin = -voxel

    def field(t):
        g = (ro + rd * t - origin) / voxel
        c = np.floor(g).astype(int)
        u = np.clip(g - c, 0, 1)

        def F(x, y, z):
            return f[min(max(z, 0), dim[2] - 1), min(max(y, 0), dim[1] - 1), min(max(x, 0), dim[0] - 1)]
        x, y, z = c
        v = 0.0
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = (u[0] if dx else 1 - u[0]) * (u[1] if dy else 1 - u[1]) * (u[2] if dz else 1 - u[2])
                    v += w * F(x + dx, y + dy, z + dz)
        return v - iso

    lo, hi = origin, origin + voxel * (dim - 1)
    with np.errstate(divide="ignore"):
        inv = 1.0 / rd
    a, b = (lo - ro) * inv, (hi - ro) * inv
    t0, t1 = np.minimum(a, b).max(), np.maximum(a, b).min()
    if not t1 > max(t0, 0):
        return None
    step = voxel * 1e-3
    t = max(t0, 0) + 1e-5
    prev = field(t)
    while t < t1:
        tn = min(t + step, t1)
        cur = field(tn)
        if prev == 0 or (prev < 0) != (cur < 0):
            lo_t, hi_t = t, tn
            for _ in range(60):
                mid = 0.5 * (lo_t + hi_t)
                if (field(mid) < 0) == (prev < 0):
                    lo_t = mid
                else:
                    hi_t = mid
            return 0.5 * (lo_t + hi_t)
        t, prev = tn, cur
    return None


def test_surface_distance_against_float64(built):
    o, p = block_with_field()
    w, h = 40, 30
    rp, m = ray_params(w, h, debug=2)
    img = o.ray(rp)
    hits = misses = 0
    for py in range(0, h, 3):
        for px in range(0, w, 3):
            ro, rd = render_f64.pixel_ray(m, w, h, px, py, from_eye=True)
            t = field_hit_f64(o, p, ro, rd, rp["iso"])
            if t is None:
                assert (img[py, px, :3] == 0).all(), (px, py, img[py, px])
                misses += 1
                continue
            frac = t - math.floor(t)
            if min(frac, 1 - frac) < 0.01 or min(t * 0.1 % 1, 1 - t * 0.1 % 1) < 0.01:
                continue  # fract() wraps within the tolerance
            want = render_f64.rgba8([frac, (t * 0.1) % 1.0, 0.0])
            assert np.abs(img[py, px, :3] - want).max() <= 2, (px, py, img[py, px], want, t)
            hits += 1
    assert hits > 10 and misses > 10


def test_background_against_float64(built):
    o, p = block_with_field()
    w, h = 48, 36
    rp, m = ray_params(w, h)
    img = o.ray(rp)
    dbg = o.ray(dict(rp, debug=2))
    checked = 0
    for py in range(0, h, 4):
        for px in range(0, w, 5):
            if dbg[py, px, :3].any():
                continue  # the ray met the surface
            ro, rd = render_f64.pixel_ray(m, w, h, px, py, from_eye=True)
            want = render_f64.rgba8(render_f64.background(rp, ro, rd), rp["exposure"])
            assert np.abs(img[py, px, :3] - want).max() <= 1, (px, py, img[py, px], want)
            checked += 1
    assert checked > 20


def mesh_triangles(o, p):
    """The mesh's triangles decoded as meshDrawWGSL's vs does (src/mesh_wgsl.js:268-286),
    in float64: positions (T, 3, 3) and unit vertex normals (T, 3, 3)."""
    box = np.array(p["box"], np.float64)
    voxel = float(np.float32(box.max() / 40))
    dim = np.array([int(math.ceil(b / (box.max() / 40))) + 3 for b in box])
    v = o.buffer("meshVerts").view(np.uint32).reshape(-1, 3, 2).astype(np.int64)
    pn = np.stack([v[..., 0] & 0xFFFF, v[..., 0] >> 16, v[..., 1] & 0xFFFF], -1) / 65535.0
    pos = -voxel + pn * (dim - 1) * voxel
    oct = v[..., 1] >> 16
    e = np.stack([oct & 0xFF, oct >> 8], -1) / 255.0 * 2 - 1
    n = np.concatenate([e, (1 - np.abs(e).sum(-1))[..., None]], -1)
    neg = n[..., 2] < 0
    fx = (1 - np.abs(n[..., 1])) * np.where(n[..., 0] >= 0, 1, -1)
    fy = (1 - np.abs(n[..., 0])) * np.where(n[..., 1] >= 0, 1, -1)
    n[..., 0] = np.where(neg, fx, n[..., 0])
    n[..., 1] = np.where(neg, fy, n[..., 1])
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    return pos, n


def nearest_triangle(pos, ro, rd):
    """Moller-Trumbore against every triangle: (t, barycentrics, index) of the
    nearest hit, or None."""
    a, b, c = pos[:, 0], pos[:, 1], pos[:, 2]
    e1, e2 = b - a, c - a
    pv = np.cross(rd, e2)
    det = (e1 * pv).sum(1)
    ok = np.abs(det) > 1e-14
    inv = np.where(ok, 1 / np.where(ok, det, 1), 0)
    tv = ro - a
    u = (tv * pv).sum(1) * inv
    qv = np.cross(tv, e1)
    v = (qv @ rd) * inv
    t = (qv * e2).sum(1) * inv
    hit = ok & (u >= 0) & (v >= 0) & (u + v <= 1) & (t > 0)
    if not hit.any():
        return None
    i = np.flatnonzero(hit)[np.argmin(t[hit])]
    return t[i], np.array([1 - u[i] - v[i], u[i], v[i]]), i


def test_mesh_surface_against_float64(built):
    o, p = block_with_field()
    pos, nrm = mesh_triangles(o, p)
    assert len(pos) > 500
    w, h = 48, 36
    rp, m = ray_params(w, h, debug=2, use_surface=1)
    dist = o.ray(rp)
    normals = o.ray(dict(rp, debug=1))
    # the f64 hit map first, so that pixels at the silhouette (a neighbour differs) are skipped
    hits = {}
    for py in range(h):
        for px in range(w):
            ro, rd = render_f64.pixel_ray(m, w, h, px, py, from_eye=True)
            hits[px, py] = (nearest_triangle(pos, ro, rd), rd)
    checked = misses = 0
    for py in range(1, h - 1):
        for px in range(1, w - 1):
            near = [hits[px + dx, py + dy][0] is None for dx in (-1, 0, 1) for dy in (-1, 0, 1)]
            if any(near) != all(near):
                continue
            hit, rd = hits[px, py]
            if hit is None:
                assert (dist[py, px, :3] == 0).all(), (px, py, dist[py, px])
                misses += 1
                continue
            t, bc, i = hit
            frac = t - math.floor(t)
            if min(frac, 1 - frac) > 0.01 and min(t * 0.1 % 1, 1 - t * 0.1 % 1) > 0.01:
                want = render_f64.rgba8([frac, (t * 0.1) % 1.0, 0.0])
                assert np.abs(dist[py, px, :3] - want).max() <= 2, (px, py, dist[py, px], want, t)
            n = bc @ nrm[i]
            n /= np.linalg.norm(n)
            if n @ rd > 0:
                n = -n
            want = render_f64.rgba8(n * 0.5 + 0.5)
            assert np.abs(normals[py, px, :3] - want).max() <= 2, (px, py, normals[py, px], want)
            checked += 1
    assert checked > 100 and misses > 100, (checked, misses)


def test_mesh_surface_clipped_at_the_near_plane(built):
    """The eye just above the block's top face, looking down across it: the near
    plane cuts the triangles of the face in front of the eye, and the pixels there
    show what lies beyond the plane (the block's far faces, seen from inside), as
    a rasteriser that clips does. Distance and normal against float64 ray /
    triangle intersections restricted to 0 <= z <= w in clip space."""
    o, p = block_with_field()
    pos, nrm = mesh_triangles(o, p)
    c = pos.reshape(-1, 3)
    top = c[(np.abs(c[:, 0] - 2.0) < 1.0) & (np.abs(c[:, 2] - 2.0) < 1.0), 1].max()
    w, h = 48, 36
    cam = Camera()
    cam.target = [2.0, float(top), 2.0]
    cam.az, cam.el, cam.dist = 0.3, 0.6, 0.05  # eye 0.03 above the face; the cut lies ~0.1 ahead
    m = frame_matrices(cam, w, h)
    rp = default_ray()
    rp.update({k: m[k] for k in ("view", "proj", "inv_view_proj", "inv_view", "eye", "width", "height")})
    rp.update(debug=2, use_surface=1)
    dist = o.ray(rp)
    normals = o.ray(dict(rp, debug=1))
    pv = (np.array(m["proj"], np.float64).reshape(4, 4).T @ np.array(m["view"], np.float64).reshape(4, 4).T)

    def visible_hit(ro, rd):
        a, b, cc = pos[:, 0], pos[:, 1], pos[:, 2]
        e1, e2 = b - a, cc - a
        pvec = np.cross(rd, e2)
        det = (e1 * pvec).sum(1)
        ok = np.abs(det) > 1e-14
        inv = np.where(ok, 1 / np.where(ok, det, 1), 0)
        tv = ro - a
        u = (tv * pvec).sum(1) * inv
        qv = np.cross(tv, e1)
        v = (qv @ rd) * inv
        t = (qv * e2).sum(1) * inv
        hit = ok & (u >= 0) & (v >= 0) & (u + v <= 1) & (t > 0)
        pts = ro + t[:, None] * rd
        clip = np.c_[pts, np.ones(len(pts))] @ pv.T
        front = hit & (clip[:, 2] < 0)                      # cut away by the near plane
        vis = hit & (clip[:, 2] >= 0) & (clip[:, 2] <= clip[:, 3])
        margin = np.abs(clip[:, 2]) < 1e-3 * clip[:, 3]
        if not vis.any():
            return None, front.any(), False
        i = np.flatnonzero(vis)[np.argmin(t[vis])]
        return (t[i], np.array([1 - u[i] - v[i], u[i], v[i]]), i), front.any(), bool((hit & margin).any())

    hits = {}
    for py in range(h):
        for px in range(w):
            ro, rd = render_f64.pixel_ray(m, w, h, px, py, from_eye=True)
            hits[px, py] = visible_hit(ro, rd) + (rd,)
    checked = clipped = 0
    for py in range(1, h - 1):
        for px in range(1, w - 1):
            hit, front, edge, rd = hits[px, py]
            ts = [hits[px + dx, py + dy][0] for dx in (-1, 0, 1) for dy in (-1, 0, 1)]
            if edge or any(x is None for x in ts) or max(x[0] for x in ts) - min(x[0] for x in ts) > 0.3:
                continue  # near the silhouette, the cut line or a depth jump
            t, bc, i = hit
            frac = t - math.floor(t)
            if min(frac, 1 - frac) > 0.01 and min(t * 0.1 % 1, 1 - t * 0.1 % 1) > 0.01:
                want = render_f64.rgba8([frac, (t * 0.1) % 1.0, 0.0])
                assert np.abs(dist[py, px, :3] - want).max() <= 2, (px, py, dist[py, px], want, t)
            n = bc @ nrm[i]
            n /= np.linalg.norm(n)
            if n @ rd > 0:
                n = -n
            want = render_f64.rgba8(n * 0.5 + 0.5)
            assert np.abs(normals[py, px, :3] - want).max() <= 2, (px, py, normals[py, px], want)
            checked += 1
            clipped += front
    assert checked > 200 and clipped > 50, (checked, clipped)
