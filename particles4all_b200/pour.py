"""The viewer's hose (pourStep and its helpers, src/main.js:89-160) on the host, as
the reference runs it: every call extrudes `speed * sim_dt` of jet from the nozzle
at (h + d, height * box_y, box_z / 2), emits each new k x k lattice layer
(k = round(width / d), layers d * 1.25 apart, at most 32 per call) advanced
ballistically for the time since it left the nozzle, with the reference's jitter
(a JS LCG from seed 22222 whose product is rounded in double) on every coordinate,
drops particles outside the box's inner band, and appends them with appendFluid
until the pour budget is spent.

    hose = Pour(budget=sim.info()["pour_budget"])
    while hose.pouring:
        sim.step(slice_dt)                       # the frame split into substep slices,
        hose.step(sim, sim.info()["last_advanced"])   # as src/main.js:986-997 does

The arithmetic is JavaScript's: doubles throughout, rounded to float32 when
appended (the reference's Float32Array upload).
"""
import math

import numpy as np

POUR_SLACK = 1.25  # layer pitch in spacings (src/main.js:89)


def lattice_across(width, spacing):
    """pourLatticeAcross (src/main.js:91-93): particles across the nozzle."""
    return max(1, math.floor(width / max(spacing, 1e-4) + 0.5))  # Math.round


def rate_per_second(width, speed, spacing):
    """pourRatePerSecond (src/main.js:95-98)."""
    k = lattice_across(width, spacing)
    return math.floor(k * k * speed / max(spacing * POUR_SLACK, 1e-4))


class Pour:
    """The hose state of the viewer's `ui` (pourSpeed, pourWidth, pourHeight,
    pourTilt in degrees, pourLeft, pourExtruded, pourNextLayer) and its jitter
    generator. Defaults are the viewer's (src/main.js:303-307)."""

    def __init__(self, budget, speed=3.0, width=0.24, height=0.85, tilt=0.0, seed=22222):
        self.speed, self.width, self.height, self.tilt = speed, width, height, tilt
        self.left = int(budget)
        self.pouring = self.left > 0
        self.extruded = 0.0
        self.next_layer = 0
        self.seed = seed

    def jitter(self, step):
        """pourJitter (src/main.js:101-104): the product is a rounded double, then
        ToInt32 and the low 31 bits."""
        s = float(self.seed) * 1103515245.0 + 12345.0
        self.seed = int(s) & 0x7FFFFFFF
        return (((self.seed >> 8) & 0xFFFF) / 65535 - 0.5) * 0.002 * step

    def emit(self, params, h, sim_dt):
        """The particles pourStep would emit for `sim_dt` seconds of the simulation
        with `params` (spacing, box, gravity) and support `h`: (pos, vel) float64
        [n, 3] arrays, or (None, None). Advances the hose state as pourStep does
        before its appendFluid."""
        if not self.pouring or self.left <= 0 or sim_dt <= 0:
            return None, None
        d = params["spacing"]
        box = params["box"]
        step = d
        layer_step = d * POUR_SLACK
        self.extruded += self.speed * sim_dt
        layers = 0
        m = self.next_layer
        while m * layer_step <= self.extruded:
            layers += 1
            m += 1
        if layers <= 0:
            return None, None
        layers = min(layers, 32)
        k = lattice_across(self.width, d)
        span = (k - 1) * step
        nozzle = [h + d, self.height * box[1], 0.5 * box[2]]
        tilt = self.tilt * math.pi / 180
        jet = [self.speed * math.cos(tilt), -self.speed * math.sin(tilt), 0.0]
        g = params["gravity"]
        pos, vel = [], []
        for layer in range(layers):
            if len(pos) >= self.left:
                break
            m = self.next_layer + layer
            behind = self.extruded - m * layer_step
            t = behind / max(self.speed, 1e-6)
            cx = nozzle[0] + jet[0] * t
            cy = nozzle[1] + jet[1] * t - 0.5 * g * t * t
            vy = jet[1] - g * t
            if cx >= box[0] - d or cy <= d:
                break
            for iy in range(k):
                if len(pos) >= self.left:
                    break
                for iz in range(k):
                    if len(pos) >= self.left:
                        break
                    y = cy - 0.5 * span + iy * step + self.jitter(step)
                    if y <= d or y >= box[1] - d:
                        continue
                    x = cx + self.jitter(step)
                    z = nozzle[2] - 0.5 * span + iz * step + self.jitter(step)
                    pos.append((x, y, z))
                    vel.append((jet[0], vy, 0.0))
        self.next_layer += layers
        if not pos:
            return None, None
        return np.array(pos, np.float64), np.array(vel, np.float64)

    def step(self, sim, sim_dt, params=None):
        """pourStep: emit for `sim_dt` and append to `sim` (a Sim, or anything with
        info() and appendFluid(); pass its `params` when it has no .params);
        returns the number appended."""
        pos, vel = self.emit(params if params is not None else sim.params, sim.info()["h"], sim_dt)
        if pos is None:
            return 0
        added = sim.appendFluid(pos.astype(np.float32), vel.astype(np.float32))
        self.left = max(0, self.left - added)
        if self.left == 0:
            self.pouring = False
        return added
