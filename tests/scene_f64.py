"""buildScene (src/scene.js:159-315) transcribed from the JS text into Python with
the JS number semantics: IEEE double arithmetic throughout, values stored into
Float32Array where the reference stores them (positions, rest offsets, psi), and
Map buckets iterated in the reference's neighbour order (dc, db, da outer to inner,
particles of a cell in insertion order). It shares no code with the oracle or the
library, so its scenes are independent inputs for the golden fixtures and a check
of both scene builders. Small scenes only (pure Python loops).
"""
import math

import numpy as np


def _lcg_block(p, d):
    """fluidBlock (src/scene.js:43-64): the lattice block with the JS LCG jitter
    (seed 12345, the product rounded to double before the 31-bit mask)."""
    bx, by, bz = p["box"]
    margin = d
    nx = max(1, math.floor(bx * 0.35 / d))
    nz = max(1, math.floor((bz - 2 * margin) / d))
    max_layers = max(1, math.floor((by - 2 * margin) / d))
    target = p["targetParticleCount"]
    layers = min(math.ceil(target / (nx * nz)), max_layers)
    out = []
    seed = 12345

    def rnd():
        nonlocal seed
        seed = int(float(seed) * 1103515245.0 + 12345.0) & 0x7FFFFFFF
        return (seed / 0x7FFFFFFF - 0.5) * 0.002 * d
    for iy in range(layers):
        if len(out) >= target:
            break
        for ix in range(nx):
            if len(out) >= target:
                break
            for iz in range(nz):
                if len(out) >= target:
                    break
                x = margin + (ix + 0.5) * d + rnd()
                y = margin + (iy + 0.5) * d + rnd()
                z = margin + (iz + 0.5) * d + rnd()
                out.append((x, y, z))
    return out


def _sample_body(shape, size, d):
    """sampleBody (src/scene.js:137-157)."""
    if shape == "sphere":
        ext = [size, size, size]
    elif shape == "torus":
        ext = [size + 0.4 * size, 0.4 * size, size + 0.4 * size]
    else:
        ext = [size * 0.9, size * 0.7, size * 0.9]
    steps = [max(1, math.ceil(e / d)) for e in ext]
    local = []
    for ix in range(-steps[0], steps[0] + 1):
        for iy in range(-steps[1], steps[1] + 1):
            for iz in range(-steps[2], steps[2] + 1):
                x, y, z = ix * d, iy * d, iz * d
                if shape == "sphere":
                    inside = x * x + y * y + z * z <= size * size
                elif shape == "torus":
                    planar = math.sqrt(x * x + z * z) - size
                    inside = planar * planar + y * y <= (0.4 * size) * (0.4 * size)
                else:
                    inside = abs(x) <= size * 0.9 and abs(y) <= size * 0.7 and abs(z) <= size * 0.9
                if inside:
                    local.append((x, y, z))
    return local


def boundary_f64(p, d, h):
    """boundaryParticles (src/scene.js:76-135): the shell samples (doubles) and
    psi = rho0 / (poly6 sum), stored as float32."""
    size = p["box"]
    nb = [max(2, math.ceil(s / d) + 1) for s in size]
    step = [s / (nb[k] - 1) for k, s in enumerate(size)]
    pts = []
    for ix in range(nb[0]):
        for iy in range(nb[1]):
            for iz in range(nb[2]):
                if ix in (0, nb[0] - 1) or iy in (0, nb[1] - 1) or iz in (0, nb[2] - 1):
                    pts.append((ix * step[0], iy * step[1], iz * step[2]))
    dim = [max(1, math.ceil(s / h)) for s in size]

    def cell(x):
        return [min(dim[k] - 1, max(0, math.floor(x[k] / h))) for k in range(3)]
    buckets = {}
    for i, x in enumerate(pts):
        a, b, c = cell(x)
        buckets.setdefault((c * dim[1] + b) * dim[0] + a, []).append(i)
    coef = 315 / (64 * math.pi * math.pow(h, 9))
    h2 = h * h
    psi = np.zeros(max(1, len(pts)), np.float32)
    for i, x in enumerate(pts):
        a, b, c = cell(x)
        s = 0.0
        for dc in (-1, 0, 1):
            if not 0 <= c + dc < dim[2]:
                continue
            for db in (-1, 0, 1):
                if not 0 <= b + db < dim[1]:
                    continue
                for da in (-1, 0, 1):
                    if not 0 <= a + da < dim[0]:
                        continue
                    for j in buckets.get(((c + dc) * dim[1] + b + db) * dim[0] + a + da, ()):
                        y = pts[j]
                        dx, dy, dz = x[0] - y[0], x[1] - y[1], x[2] - y[2]
                        r2 = dx * dx + dy * dy + dz * dz
                        if r2 >= h2:
                            continue
                        t = h2 - r2
                        s += t * t * t
        s *= coef
        psi[i] = p["restDensity"] / s if s > 0 else 0.0
    return np.array(pts, np.float64).reshape(-1, 3), psi[:len(pts)]


def build_scene_f64(p):
    """The scene of buildScene(p): float32 pos / rest / phase arrays (n x 4), body
    centres and densities, mass and denomRest (doubles), boundary samples."""
    d = p["spacing"]
    h = 2 * d
    bx, by, bz = p["box"]
    fluid = _lcg_block(p, d)
    n_fluid = len(fluid)
    specs = []
    for s in p["bodies"]:
        bits = s.split(":")

        def num(k, dflt):
            try:
                v = float(bits[k]) if len(bits) > k else dflt
            except ValueError:
                v = 0.0
            return v if v else dflt   # Number(x) || default
        specs.append((bits[0], num(1, 0.5), num(2, 0.75)))
    sz = p["bodySize"] if p["bodySize"] > 0 else 0.12 * min(bx, by, bz)
    step = min(2.5 * sz, bx * 0.25)
    span = step * (len(specs) - 1)
    body_pts, body_rest, body_phase, centres, dens = [], [], [], [], []
    for r, (shape, density, start_y) in enumerate(specs):
        local = _sample_body(shape, sz, d)
        if not local:
            continue
        centre = [0.5 * bx - 0.5 * span + step * r, by * start_y, bz * 0.5]
        cx = cy = cz = 0.0
        for x, y, z in local:
            cx += x
            cy += y
            cz += z
        cx /= len(local)
        cy /= len(local)
        cz /= len(local)
        bid = len(centres) + 1
        for x, y, z in local:
            body_pts.append((centre[0] + x, centre[1] + y, centre[2] + z))
            body_rest.append((x - cx, y - cy, z - cz))
            body_phase.append(bid)
        centres.append(centre)
        dens.append(density)
    n = n_fluid + len(body_pts)
    pos = np.zeros((n, 4), np.float32)
    rest = np.zeros((n, 4), np.float32)
    phase = np.zeros((n, 4), np.uint32)
    if n_fluid:
        pos[:n_fluid, :3] = np.array(fluid, np.float64)
    if body_pts:
        pos[n_fluid:, :3] = np.array(body_pts, np.float64)
        rest[n_fluid:, :3] = np.array(body_rest, np.float64)
        phase[n_fluid:, 0] = body_phase
    bpts, bpsi = boundary_f64(p, d, h)

    # mass calibration and denomRest on the float32-stored positions (read back as doubles)
    P = pos[:, :3].astype(np.float64)
    coef = 315 / (64 * math.pi * math.pow(h, 9))
    h2 = h * h
    spiky = -45 / (math.pi * math.pow(h, 6))
    dim = [max(1, math.floor(bx / h)), max(1, math.floor(by / h)), max(1, math.floor(bz / h))]

    def cell(i):
        return [min(dim[k] - 1, max(0, math.floor(P[i, k] / h))) for k in range(3)]
    buckets = {}
    for i in range(n_fluid):
        a, b, c = cell(i)
        buckets.setdefault((c * dim[1] + b) * dim[0] + a, []).append(i)

    def neighbours(i):
        a, b, c = cell(i)
        for dc in (-1, 0, 1):
            if not 0 <= c + dc < dim[2]:
                continue
            for db in (-1, 0, 1):
                if not 0 <= b + db < dim[1]:
                    continue
                for da in (-1, 0, 1):
                    if not 0 <= a + da < dim[0]:
                        continue
                    for j in buckets.get(((c + dc) * dim[1] + b + db) * dim[0] + a + da, ()):
                        if j != i:
                            yield j

    def density_at(i, m):
        rho = m * coef * h2 * h2 * h2
        xi = P[i]
        for j in neighbours(i):
            r2 = (xi[0] - P[j, 0]) ** 2 + (xi[1] - P[j, 1]) ** 2 + (xi[2] - P[j, 2]) ** 2
            if r2 >= h2:
                continue
            t = h2 - r2
            rho += m * coef * t * t * t
        return rho
    rho0 = p["restDensity"]
    mass = rho0 * d * d * d
    max_rho = 0.0
    for i in range(n_fluid):
        max_rho = max(max_rho, density_at(i, mass))
    if max_rho > 0.5 * rho0:
        mass *= rho0 / max_rho
    denom = 0.0
    volume = mass / rho0
    for i in range(n_fluid):
        if density_at(i, mass) < 0.99 * rho0:
            continue
        gx = gy = gz = g2 = 0.0
        xi = P[i]
        for j in neighbours(i):
            rx, ry, rz = xi[0] - P[j, 0], xi[1] - P[j, 1], xi[2] - P[j, 2]
            r2 = rx * rx + ry * ry + rz * rz
            if r2 < 1e-12 or r2 >= h2:
                continue
            r = math.sqrt(r2)
            hr = h - r
            s = volume * spiky * hr * hr / r
            gx += s * rx
            gy += s * ry
            gz += s * rz
            g2 += s * s * r2
        denom = max(denom, gx * gx + gy * gy + gz * gz + g2)
        if i > 2000 and denom > 0:
            break
    return {"n": n, "n_fluid": n_fluid, "n_bodies": len(centres), "pos": pos,
            "vel": np.zeros((n, 4), np.float32), "rest": rest, "phase": phase,
            "body_centre": np.array(centres, np.float64).reshape(-1, 3),
            "body_density": np.array(dens, np.float64), "mass": mass, "denom_rest": denom,
            "boundary_pts": bpts, "boundary_psi": bpsi, "pour_budget": 0}
