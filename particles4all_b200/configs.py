"""Seeded synthetic scenes for the benchmark workloads.

The reference has no benchmark scenes of its own (its presets are browser
settings); these generators build the scenes the workload definitions name,
as explicit scenes for Sim.reset_scene:

  dam_break_32k     32,768 fluid particles on a 32^3 lattice, d = 0.5, jitter
                    U(+-0.01 d), in the corner of a [0,40]x[0,24]x[0,20] box;
                    h = 2d = 1; rho0 = 1 with the mass normalised on the
                    unjittered lattice; CFM epsilon 100 (absolute); 4
                    iterations; 2 substeps per 1/60 s; g = 9.8; no bodies,
                    no tension.
  medium_bodies_264k  262,144 fluid particles on a 64^3 lattice in the box
                    scaled x2, plus 8 rigid 6x6x6 cubes (1,728 particles) at
                    density 0.5 rho0 with seeded orientations and positions
                    above the water; surface tension 0.5; XSPH c = 0.01;
                    anisotropic pass k_r = 4, N_eps = 25, lambda = 0.9.
  large_hose_2m     2,097,152 fluid particles on a 128^3 lattice in the box
                    scaled x4, 64 seeded boxes/spheres 4-10 particles across
                    at densities U[0.3, 1.5] rho0, tension on, 8 iterations,
                    and a hose of 2,048 particles per step at 3 m/s until the
                    total reaches 2.5M.

Values the workloads leave open take the dam-break values (rho0 = 1,
epsilon = 100, g = 9.8, 2 substeps).
"""
import math

import numpy as np

KERNEL_POLY6 = 315.0 / (64.0 * math.pi)


def lattice_mass(d, h, rho0=1.0):
    """Particle mass that makes the density of an unjittered cubic lattice of
    spacing d equal rho0 with the poly6 kernel of radius h (self term included)."""
    m = int(math.ceil(h / d)) + 1
    r = np.arange(-m, m + 1) * d
    x, y, z = np.meshgrid(r, r, r, indexing="ij")
    r2 = (x * x + y * y + z * z).ravel()
    h2 = h * h
    t = h2 - r2[r2 < h2]
    w = KERNEL_POLY6 / h ** 9 * np.sum(t * t * t)
    return rho0 / w


def _rotation(rng):
    """A uniformly random rotation matrix (from a normalised Gaussian quaternion)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _fluid_lattice(nx, ny, nz, d, jitter, rng, origin):
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1).astype(np.float64)
    pos = origin + (base + 0.5) * d
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    return pos


def _body_points(shape, across, d):
    """Local lattice points of a box (across^3) or a sphere of diameter across."""
    r = (np.arange(across) - (across - 1) / 2.0) * d
    x, y, z = np.meshgrid(r, r, r, indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    if shape == "sphere":
        rad = across * d / 2.0
        pts = pts[np.sum(pts * pts, 1) <= rad * rad + 1e-9]
    return pts - pts.mean(0)


def _assemble(fluid, bodies, params, mass, pour_budget=0):
    """Scene dict: fluid first, then each body's particles (rest = world offset)."""
    n_f = fluid.shape[0]
    n_b = sum(b["offsets"].shape[0] for b in bodies)
    n = n_f + n_b
    pos = np.zeros((n, 4), np.float32)
    rest = np.zeros((n, 4), np.float32)
    phase = np.zeros((n, 4), np.uint32)
    pos[:n_f, :3] = fluid
    o = n_f
    for k, b in enumerate(bodies):
        m = b["offsets"].shape[0]
        pos[o:o + m, :3] = b["centre"] + b["offsets"]
        rest[o:o + m, :3] = b["offsets"]
        phase[o:o + m, 0] = k + 1
        o += m
    return {
        "pos": pos, "vel": np.zeros((n, 4), np.float32), "rest": rest, "phase": phase,
        "n_bodies": len(bodies),
        "body_density": np.array([b["density"] for b in bodies], np.float64),
        "body_centre": np.array([b["centre"] for b in bodies], np.float64).reshape(-1, 3),
        "mass": mass, "denom_rest": 0.0, "pour_budget": pour_budget, "n_fluid": n_f,
    }


def _place_bodies(rng, count, lo, hi, min_dist):
    centres = []
    tries = 0
    while len(centres) < count and tries < 100000:
        tries += 1
        c = rng.uniform(lo, hi)
        if all(np.linalg.norm(c - e) >= min_dist for e in centres):
            centres.append(c)
    if len(centres) < count:
        raise ValueError("could not place the bodies without overlap")
    return centres


def _base_params(box, iterations, tension, xsph, substeps=2):
    return {
        "spacing": 0.5, "restDensity": 1.0, "gravity": 9.8, "substeps": substeps,
        "iterations": iterations, "cfmEpsilonRel": 0.01, "cfmEpsilonAbs": 100.0,
        "sCorrK": 0.1, "sCorrDq": 0.3, "xsphC": xsph, "omega": 1.0, "sorAverage": False,
        "surfaceTensionK": tension, "box": [float(b) for b in box], "bodies": [], "bodySize": 0,
        "noBoundary": False, "pour": False,
    }


def dam_break_32k(seed=0, side=32):
    """The plain single-scene dam break (side^3 lattice; side = 32 is the workload)."""
    d, h = 0.5, 1.0
    rng = np.random.default_rng(seed)
    fluid = _fluid_lattice(side, side, side, d, 0.01 * d, rng, np.array([d, d, d]))
    params = _base_params([40.0, 24.0, 20.0], iterations=4, tension=0.0, xsph=0.05)
    return params, _assemble(fluid, [], params, lattice_mass(d, h))


def medium_bodies_264k(seed=1, side=64, n_cubes=8, cube=6):
    """The medium scene with 8 floating cubes (side = 64 is the workload)."""
    d, h = 0.5, 1.0
    rng = np.random.default_rng(seed)
    top = d + side * d
    span = cube * d
    box = np.array([80.0, 48.0, 40.0]) * (side / 64.0)
    # room above the water for the cubes at reduced sizes (no change at side = 64)
    box = np.maximum(box, [4 * span + 4.0, top + 4 * span + 2.0, 4 * span + 4.0])
    fluid = _fluid_lattice(side, side, side, d, 0.01 * d, rng, np.array([d, d, d]))
    lo = np.array([span + 1.0, top + span, span + 1.0])
    hi = np.array([box[0] - span - 1.0, min(box[1] - span - 1.0, top + 3 * span), box[2] - span - 1.0])
    centres = _place_bodies(rng, n_cubes, lo, hi, min_dist=2.0 * span)
    local = _body_points("box", cube, d)
    bodies = [{"centre": c, "offsets": local @ _rotation(rng).T, "density": 0.5} for c in centres]
    params = _base_params(box, iterations=4, tension=0.5, xsph=0.01)
    return params, _assemble(fluid, bodies, params, lattice_mass(d, h))


def medium_aniso_params():
    """Anisotropic-kernel settings of the medium workload: k_r = 4, N_eps = 25,
    lambda = 0.9. Yu & Turk's k_s = 1400 is the constant that makes k_s * sigma
    about 1 for a full neighbourhood at their particle scale; the reference
    expresses the same normalisation as anisoKs / sigma_bulk with anisoKs = 1
    (src/mesh.js:226,238), which is what is used here."""
    return {"ratio": 4.0, "ks": 1.0, "stretch": 2.0, "lonely": 1.0, "min_neighbours": 25,
            "lambda": 0.9, "radius_scale": 2.0, "min_extent": 0.0}


def large_hose_2m(seed=2, side=128, n_bodies=64, target_total=2_500_000):
    """The large scene with 64 mixed bodies and a hose (side = 128 is the workload)."""
    d, h = 0.5, 1.0
    rng = np.random.default_rng(seed)
    top = d + side * d
    box = np.array([160.0, 96.0, 80.0]) * (side / 128.0)
    box = np.maximum(box, [40.0, top + 20.0, 40.0])  # room for the bodies at reduced sizes
    fluid = _fluid_lattice(side, side, side, d, 0.01 * d, rng, np.array([d, d, d]))
    bodies = []
    lo = np.array([6.0, top + 6.0, 6.0])
    hi = np.array([box[0] - 6.0, box[1] - 6.0, box[2] - 6.0])
    centres = _place_bodies(rng, n_bodies, lo, hi, min_dist=6.0)
    for c in centres:
        shape = "box" if rng.random() < 0.5 else "sphere"
        across = int(rng.integers(4, 11))
        local = _body_points(shape, across, d) @ _rotation(rng).T
        bodies.append({"centre": c, "offsets": local, "density": float(rng.uniform(0.3, 1.5))})
    params = _base_params(box, iterations=8, tension=0.5, xsph=0.01)
    scene = _assemble(fluid, bodies, params, lattice_mass(d, h))
    scene["pour_budget"] = max(0, target_total - scene["pos"].shape[0])
    return params, scene


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011) on numpy uint32
    counter arrays with key (k0, k1): the generator of the device hose
    (csrc/kernels_hose.cu), restated word for word."""
    m0, m1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    mask = np.uint64(0xFFFFFFFF)
    c0, c1, c2, c3 = (np.asarray(c, np.uint32) for c in (c0, c1, c2, c3))
    for _ in range(10):
        p0 = m0 * c0.astype(np.uint64)
        p1 = m1 * c2.astype(np.uint64)
        hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & mask).astype(np.uint32)
        hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & mask).astype(np.uint32)
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint32(k0), lo1, hi0 ^ c3 ^ np.uint32(k1), lo0
        k0 = (k0 + 0x9E3779B9) & 0xFFFFFFFF
        k1 = (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return c0, c1, c2, c3


class Hose:
    """A hose emitting `per_step` particles per step at `speed` along +x from the
    near wall: square k x k lattice layers (k = ceil(sqrt(per_step))) with jitter,
    the layered emitter of src/main.js:106-160 at a fixed rate, up to `limit`
    particles in total. The jitter of emission e, slot q and axis a is uniform in
    [-0.001 d, 0.001 d) from Philox4x32-10 keyed by (seed, e, q), so a layer is a
    function of its emission index: Sim.hoseEmit computes it on the device, and
    emit() computes the same float32 bits on the host (the oracle's input)."""

    def __init__(self, box, d, per_step=2048, speed=3.0, height=0.6, seed=22222, limit=None):
        self.box, self.d, self.per_step, self.speed = box, d, per_step, speed
        self.k = int(math.ceil(math.sqrt(per_step)))
        self.nozzle = np.array([2.0 * d + d, height * box[1], 0.5 * box[2]]).astype(np.float32)
        self.spacing = np.float32(d)
        self.jitter = np.float32(0.001 * d)
        self.seed = int(seed) & 0xFFFFFFFF
        self.left = limit
        self.emission = 0

    def c_struct(self):
        from ._abi import Hose as CHose
        h = CHose()
        for a in range(3):
            h.nozzle[a] = float(self.nozzle[a])
        h.spacing, h.jitter, h.speed = float(self.spacing), float(self.jitter), float(self.speed)
        h.per_step = self.per_step
        h.count = self.per_step if self.left is None else max(0, min(self.per_step, self.left))
        h.seed = self.seed
        return h

    def advance(self, n):
        """Book one emission of n particles."""
        self.emission += 1
        if self.left is not None:
            self.left -= n

    def layer(self, emission, n):
        """Positions and velocities (float32, n x 3) of slots [0, n) of an emission."""
        q = np.arange(n, dtype=np.uint32)
        e = np.uint64(emission)
        w = philox4x32_10(np.full(n, e & np.uint64(0xFFFFFFFF), np.uint32),
                          np.full(n, e >> np.uint64(32), np.uint32), q, np.zeros(n, np.uint32),
                          self.seed, 0x5EED5EED)
        f32 = np.float32
        j = [((w[a] >> np.uint32(8)).astype(f32) * f32(2.0 ** -24) * f32(2.0) - f32(1.0)) * self.jitter
             for a in range(3)]
        iy, iz = (q // np.uint32(self.k)).astype(f32), (q % np.uint32(self.k)).astype(f32)
        c = f32((self.k - 1) * 0.5)
        pos = np.zeros((n, 3), f32)
        pos[:, 0] = self.nozzle[0] + j[0]
        pos[:, 1] = (self.nozzle[1] + (iy - c) * self.spacing) + j[1]
        pos[:, 2] = (self.nozzle[2] + (iz - c) * self.spacing) + j[2]
        vel = np.zeros((n, 3), f32)
        vel[:, 0] = f32(self.speed)
        return pos, vel

    def emit(self):
        """The next layer on the host (None, None once the limit is reached)."""
        n = self.per_step if self.left is None else min(self.per_step, self.left)
        if n <= 0:
            return None, None
        pos, vel = self.layer(self.emission, n)
        self.advance(n)
        return pos, vel


def batched_mix(seed=12, count=96, n_lo=4000, n_hi=256000, cube=6):
    """The batched mix: `count` scenes with particle counts log-uniform in
    [n_lo, n_hi] (about 6 M in total for 96), boxes of 16-64 cells per axis, 0-6
    rigid 6x6x6 cubes (density 0.5) with seeded orientations above the water,
    surface tension 0.5 on half of the scenes, 4 iterations. Returns a list of
    (params, scene). Seed 12 gives 6,003,226 particles for the 96 scenes."""
    d, h = 0.5, 1.0
    rng = np.random.default_rng(seed)
    mass = lattice_mass(d, h)
    span = cube * d
    out = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        side = int(math.ceil(n ** (1.0 / 3.0)))
        lo_cells = max(16, int(math.ceil(side * d)) + 6)
        box = np.array([float(rng.integers(lo_cells, 65)) for _ in range(3)])
        n_cubes = int(rng.integers(0, 7))
        tension = 0.5 if rng.random() < 0.5 else 0.0
        # the block fills layer by layer (y outermost), as the reference's fluidBlock
        iy, ix, iz = np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij")
        lat = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1)[:n].astype(np.float64)
        fluid = d + (lat + 0.5) * d + rng.uniform(-0.01 * d, 0.01 * d, size=lat.shape)
        top = d + (lat[:, 1].max() + 1) * d
        bodies = []
        if n_cubes:
            box = np.maximum(box, [4 * span + 4.0, top + 4 * span + 2.0, 4 * span + 4.0])
            lo = np.array([span + 1.0, top + span, span + 1.0])
            hi = np.array([box[0] - span - 1.0, min(box[1] - span - 1.0, top + 3 * span), box[2] - span - 1.0])
            local = _body_points("box", cube, d)
            for c in _place_bodies(rng, n_cubes, lo, hi, min_dist=2.0 * span):
                bodies.append({"centre": c, "offsets": local @ _rotation(rng).T, "density": 0.5})
        params = _base_params(box, iterations=4, tension=tension, xsph=0.01)
        out.append((params, _assemble(fluid, bodies, params, mass)))
    return out


WORKLOADS = {
    "dam_break_32k": dam_break_32k,
    "medium_bodies_264k": medium_bodies_264k,
    "large_hose_2m": large_hose_2m,
}
