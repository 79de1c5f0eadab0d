"""Float64 transcriptions, written from the reference's WGSL / JS text, of the passes
the step transcription (test_oracle_transcription.Transcription) does not cover:

  aniso_f64    the anisotropic-kernel pass (src/aniso_wgsl.js:64-158) with the
               uniform packing of SurfaceMesh.buildAnisotropy (src/mesh.js:207-261)
  stats_f64    the stats pass (src/wgsl.js:785-832): 256-particle workgroup sums
               and maxima, truncated to u32 at x1024, summed / maxed over groups
  impulse_f64  applyRayImpulse (src/sim.js:658-676, src/wgsl.js:216-248)
  resize_f64   the resize pass of resizeBox (src/sim.js:687-772, src/wgsl.js:125-157)

They share no code with the oracle or the library. Small inputs only.
"""
import math

import numpy as np


def _f32(x):
    return float(np.float32(x))


# ---- anisotropic kernel -----------------------------------------------------

def _jacobi(a):
    """The reference's 6-sweep cyclic Jacobi (mat[col][row] indexing, as WGSL)."""
    a = [row[:] for row in a]
    v = [[1.0 if r == c else 0.0 for r in range(3)] for c in range(3)]

    def mul(x, y):  # column-major: (x*y)[c][r] = sum_k x[k][r] y[c][k]
        return [[sum(x[k][r] * y[c][k] for k in range(3)) for r in range(3)] for c in range(3)]

    def tr(x):
        return [[x[r][c] for r in range(3)] for c in range(3)]
    for _ in range(6):
        for p in range(2):
            for q in range(p + 1, 3):
                apq = a[q][p]
                if abs(apq) < 1e-12:
                    continue
                theta = (a[q][q] - a[p][p]) / (2.0 * apq)
                t = math.copysign(1.0, theta) / (abs(theta) + math.sqrt(theta * theta + 1.0))
                if theta == 0.0:
                    t = 1.0
                cth = 1.0 / math.sqrt(t * t + 1.0)
                s = t * cth
                r = [[1.0 if rr == cc else 0.0 for rr in range(3)] for cc in range(3)]
                r[p][p] = cth
                r[q][q] = cth
                r[q][p] = s
                r[p][q] = -s
                a = mul(mul(tr(r), a), r)
                v = mul(v, r)
    return a, v


def aniso_f64(pos, cell_start, box_min, grid_dim, h, A):
    """smoothPos (n x 3) and the packed G (n x 8: G00, G10, G20, G11, G21, G22, det, n)
    of the anisotropic pass. pos: the live positions (float32 values), cell_start:
    the sim's cellStart; A: the aniso settings (ratio, ks, stretch, lonely,
    min_neighbours, lambda, radius_scale, min_extent) mapped to the uniform as
    buildAnisotropy maps them, each stored as float32."""
    support = h
    radius = A["radius_scale"] * support
    cells = int(math.ceil(A["radius_scale"]))
    sigma_bulk = 0.15 * radius * radius
    U = {"lambda": _f32(A["lambda"]), "inv": _f32(1 / support), "support": _f32(support),
         "radius": _f32(radius), "kr": _f32(A["ratio"]), "kn": _f32(A["lonely"]),
         "ks": _f32(A["ks"] / sigma_bulk), "stretch": _f32(A["stretch"]), "minext": _f32(A["min_extent"]),
         "neps": int(A["min_neighbours"])}
    dim = [int(x) for x in grid_dim]
    n = pos.shape[0]
    P = pos[:, :3].astype(np.float64)
    smooth = np.zeros((n, 3))
    G = np.zeros((n, 8))
    r2max = U["radius"] * U["radius"]
    inv_r = 1.0 / U["radius"]
    for i in range(n):
        xi = P[i]
        c = [min(max(int(math.floor((xi[k] - box_min[k]) * U["inv"])), 0), dim[k] - 1) for k in range(3)]
        x0, x1 = max(c[0] - cells, 0), min(c[0] + cells, dim[0] - 1)
        rel = xi - np.asarray(box_min, np.float64)
        sd = np.zeros(3)
        m2 = np.zeros((3, 3))  # m2[col] = sum d * (d[col] * w)
        wsum = 0.0
        nn = 0
        for dz in range(-cells, cells + 1):
            z = c[2] + dz
            if z < 0 or z >= dim[2]:
                continue
            dzmin = max(max(z * U["support"] - rel[2], rel[2] - (z + 1) * U["support"]), 0.0)
            dz2 = dzmin * dzmin
            if dz2 >= r2max:
                continue
            for dy in range(-cells, cells + 1):
                y = c[1] + dy
                if y < 0 or y >= dim[1]:
                    continue
                dymin = max(max(y * U["support"] - rel[1], rel[1] - (y + 1) * U["support"]), 0.0)
                if dz2 + dymin * dymin >= r2max:
                    continue
                base = (z * dim[1] + y) * dim[0]
                for j in range(int(cell_start[base + x0]), int(cell_start[base + x1 + 1])):
                    d = P[j] - xi
                    r2 = float(d @ d)
                    if r2 >= r2max:
                        continue
                    t = math.sqrt(r2) * inv_r
                    w = 1.0 - t * t * t
                    sd += d * w
                    for col in range(3):
                        m2[col] += d * (d[col] * w)
                    wsum += w
                    nn += 1
        if wsum <= 0.0:
            smooth[i] = xi
            g = U["kn"] / U["support"]
            G[i] = [g, 0.0, 0.0, g, 0.0, g, g * g * g, 0.0]
            continue
        dbar = sd / wsum
        smooth[i] = xi + dbar * U["lambda"]
        cov = [[m2[col][r] / wsum - dbar[r] * dbar[col] for r in range(3)] for col in range(3)]
        ea, ev = _jacobi(cov)
        sig = np.array([ea[0][0], ea[1][1], ea[2][2]])
        s1 = sig.max()
        sig_t = np.maximum(sig, s1 / U["kr"])
        ext = U["ks"] * sig_t
        ext = ext / max(1.0, ext.max() / U["stretch"])
        ext = np.maximum(ext, U["minext"])
        inv = 1.0 / (U["support"] * ext)
        R = np.array(ev).T  # row r, col c = ev[c][r]
        Gan = R @ np.diag(inv) @ R.T
        giso = U["kn"] / U["support"]
        lo, hi = U["neps"] * 0.4, U["neps"] * 1.6
        tt = min(max((nn - lo) / (hi - lo), 0.0), 1.0)
        w = tt * tt * (3.0 - 2.0 * tt)
        Gm = np.eye(3) * giso * (1.0 - w) + Gan * w
        G[i] = [Gm[0, 0], Gm[0, 1], Gm[0, 2], Gm[1, 1], Gm[1, 2], Gm[2, 2], np.linalg.det(Gm), nn]
    return smooth, G


# ---- stats -------------------------------------------------------------------

def stats_f64(density, vel, n, rho0, mass):
    """The four u32 words of the stats pass before the host scales them: per
    256-particle workgroup the sum of rho / rho0, max rho / rho0, max |v| and sum of
    0.5 m |v|^2, each truncated at x1024, then added (0, 3) or maxed (1, 2) over
    the workgroups. Also the untruncated float64 totals."""
    out = [0, 0, 0, 0]
    exact = [0.0, 0.0, 0.0, 0.0]
    inv = _f32(1.0 / rho0)  # P.invRho0 and P.mass are float32 uniforms
    m = _f32(mass)
    for g0 in range(0, n, 256):
        rho = density[g0:min(n, g0 + 256)].astype(np.float64) * inv
        v = vel[g0:min(n, g0 + 256), :3].astype(np.float64)
        v2 = np.sum(v * v, 1)
        s = [rho.sum(), rho.max(), np.sqrt(v2).max(), (0.5 * m * v2).sum()]
        exact[0] += s[0]
        exact[3] += s[3]
        exact[1] = max(exact[1], s[1])
        exact[2] = max(exact[2], s[2])
        w = [int(x * 1024.0) for x in s]
        out[0] += w[0]
        out[3] += w[3]
        out[1] = max(out[1], w[1])
        out[2] = max(out[2], w[2])
    return out, exact


# ---- interactive passes --------------------------------------------------------

def impulse_f64(pos, vel, origin, direction, impulse, radius, speed_limit):
    """Velocities after applyRayImpulse: the uniform as the host packs it (float32
    copies of origin, dir / |dir|, impulse, radius, speedLimit), the pass in float64."""
    dl = math.hypot(*direction) or 1.0
    o = np.array([_f32(x) for x in origin])
    d = np.array([_f32(x / dl) for x in direction])
    im = np.array([_f32(x) for x in impulse])
    rad, lim = _f32(radius), _f32(speed_limit)
    out = vel[:, :3].astype(np.float64).copy()
    for i in range(pos.shape[0]):
        to_p = pos[i, :3].astype(np.float64) - o
        along = float(to_p @ d)
        if along <= 0.0:
            continue
        radial = to_p - along * d
        d2 = float(radial @ radial)
        if d2 >= rad * rad:
            continue
        x = 1.0 - math.sqrt(d2) / rad
        v = out[i].copy()
        old = math.sqrt(float(v @ v))
        nv = v + (x * x) * im
        ns = math.sqrt(float(nv @ nv))
        allowed = max(old, lim)
        if ns > allowed:
            nv = nv * (allowed / ns)
        out[i] = nv
    return out


def resize_f64(pos, old_box, new_box, spacing):
    """Live positions after the resize pass of resizeBox (min corners at the origin;
    the clamp box inset by half a spacing), uniform values stored as float32."""
    half = 0.5 * spacing
    old = [_f32(x) for x in old_box]
    new = [_f32(x) for x in new_box]
    cmin = [_f32(half)] * 3
    cmax = [_f32(b - half) for b in new_box]
    out = pos[:, :3].astype(np.float64).copy()
    for a in range(3):
        if new[a] < old[a]:
            t = np.clip(out[:, a] / old[a], 0.0, 1.0)
            out[:, a] = t * new[a]
        out[:, a] = np.clip(out[:, a], cmin[a], cmax[a])
    return out
