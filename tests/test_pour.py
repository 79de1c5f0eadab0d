"""The viewer's hose (pourStep, src/main.js:89-160) restated on the host: the jitter
generator's JS-double LCG, the layer schedule and ballistic pre-advance of one
call, the inner-band drop, the budget, and appends into the oracle."""
import math

import numpy as np

import oracle
from particles4all_b200.params import default_params
from particles4all_b200.pour import Pour, lattice_across, rate_per_second


def test_jitter_generator():
    hose = Pour(budget=10)
    j = hose.jitter(0.5)
    first = (22222 * 1103515245 + 12345) & 0x7FFFFFFF  # exact: the product is below 2^53
    assert hose.seed == first
    assert j == (((first >> 8) & 0xFFFF) / 65535 - 0.5) * 0.002 * 0.5
    seeds = []
    for _ in range(2000):
        hose.jitter(1.0)
        seeds.append(hose.seed)
    assert all(0 <= s < 2 ** 31 for s in seeds)
    # later products exceed 2^53 and are rounded to double before the mask, as in JS
    s, want = first, []
    for _ in range(2000):
        s = int(float(s * 1103515245) + 12345.0) & 0x7FFFFFFF
        want.append(s)
    assert seeds == want
    assert lattice_across(0.24, 0.02) == 12 and lattice_across(0.25, 0.1) == 3  # Math.round: 2.5 -> 3
    assert rate_per_second(0.24, 3.0, 0.02) == math.floor(144 * 3.0 / 0.025)


def test_one_call_emits_a_ballistic_layer():
    p = {"spacing": 0.02, "box": [2.0, 1.0, 1.0], "gravity": 9.81}
    hose = Pour(budget=10 ** 6)
    pos, vel = hose.emit(p, 0.04, 1 / 240)  # extrudes 0.0125: layer 0 only (pitch 0.025)
    k, d = 12, 0.02
    assert pos.shape == (k * k, 3) and hose.next_layer == 1
    t = 0.0125 / 3.0
    assert np.allclose(pos[:, 0], 0.04 + d + 3.0 * t, atol=0.001 * d)
    ys = 0.85 - 0.5 * 9.81 * t * t - 0.5 * (k - 1) * d + np.repeat(np.arange(k), k) * d
    zs = 0.5 - 0.5 * (k - 1) * d + np.tile(np.arange(k), k) * d
    assert np.abs(pos[:, 1] - ys).max() <= 0.001 * d and np.abs(pos[:, 2] - zs).max() <= 0.001 * d
    assert np.allclose(vel, [[3.0, -9.81 * t, 0.0]] * (k * k))
    pos2, _ = hose.emit(p, 0.04, 1 / 240)  # 0.025 extruded: layer 1 is exactly due
    assert pos2.shape == (k * k, 3) and hose.next_layer == 2
    assert hose.emit(p, 0.04, 1 / 2400) == (None, None)  # not a full layer more
    # a tall nozzle in a low box: rows outside the inner band are dropped
    low = {"spacing": 0.02, "box": [2.0, 0.2, 1.0], "gravity": 9.81}
    pos3, _ = Pour(budget=10 ** 6, width=0.4, height=0.5).emit(low, 0.04, 1 / 240)
    assert 0 < pos3.shape[0] < 20 * 20 and (pos3[:, 1] > 0.02).all() and (pos3[:, 1] < 0.18).all()


def test_budget_and_appends_into_the_oracle(built):
    p = default_params("small")
    p.update({"targetParticleCount": 2000, "box": [0.6, 0.5, 0.3], "bodies": [], "pour": True})
    o = oracle.OracleSim()
    o.reset(p)
    info = o.info()
    budget = min(info["pour_budget"], 300)
    hose = Pour(budget=budget)
    added = 0
    for _ in range(40):
        o.step(1 / 240)
        added += hose.step(o, o.info()["last_advanced"], params=p)
        if not hose.pouring:
            break
    assert added == budget and hose.left == 0 and not hose.pouring
    assert o.info()["n"] == info["n"] + budget
