"""The larger workloads at their full stated sizes against the oracle, bit for bit.

Smaller cases elsewhere pin every pass; these reach what only large scenes reach:
32-bit index arithmetic over millions of particles, grids of 1.2 M cells (the large
scene's dense grid) with scan tile counts in the hundreds, crowded neighbour lists,
and the 96-scene mix's segmented sort with its per-scene key offsets.

  - medium_bodies_264k (263,872 particles, 8 cubes, tension, XSPH): one full step
    (2 substeps) and the anisotropic pass;
  - large_hose_2m (2,097,152 fluid particles + 64 bodies, 8 iterations, tension):
    one hose layer (emitted on the device for the library, on the host for the
    oracle), then one substep;
  - batched_mix_96 (96 scenes, 6.0 M particles) stepped as one batch for one frame:
    every scene against its own oracle.

Each oracle leg runs in seconds with all host threads.
"""
import numpy as np
import pytest

import oracle
from particles4all_b200 import Batch, Sim, _lib, configs
from particles4all_b200.batch import arena_sizes

pytestmark = pytest.mark.gpu

NAMES = ("pos", "vel", "pred", "body", "rest", "density", "lambda_")


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def same(a, b, what):
    bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
    assert bad.size == 0, f"{what}: {bad.shape[0]} mismatches, first at {bad[:3].tolist()}"


def compare_sim(g, o):
    gi, oi = g.info(), o.info()
    for k in ("n", "parity", "pred_parity", "n_cells", "n_boundary", "n_bodies", "last_substeps"):
        assert gi[k] == oi[k], (k, gi[k], oi[k])
    n, c = gi["n"], gi["n_cells"]
    for name in NAMES:
        same(g.read(name)[:n], o.buffer(name)[:n], name)
    same(g.read("cellStart")[:c + 1], o.buffer("cellStart")[:c + 1], "cellStart")
    if gi["n_bodies"]:
        for name in ("bodyCentre", "bodyRot", "bodyRef"):
            same(g.read(name), o.buffer(name), name)
    assert g.get_stats()["raw"] == o.stats()["raw"]


def test_medium_full_size_step_and_aniso():
    params, scene = configs.medium_bodies_264k()
    g, o = Sim(), oracle.OracleSim()
    g.reset_scene(params, scene)
    o.reset_scene(params, scene)
    assert g.info()["n"] == 263872
    assert g.step(1 / 60) == o.step(1 / 60) == 2
    compare_sim(g, o)
    a = configs.medium_aniso_params()
    g.aniso(a)
    o.aniso(a)
    n = g.info()["n"]
    same(g.read("smoothPos")[:n], o.buffer("smoothPos")[:n], "smoothPos")
    same(g.read("aniso")[: 2 * n], o.buffer("aniso")[: 2 * n], "aniso")
    g.close()


def test_large_hose_full_size_append_and_substep():
    params, scene = configs.large_hose_2m()
    g, o = Sim(), oracle.OracleSim()
    g.reset_scene(params, scene)
    o.reset_scene(params, scene)
    info = g.info()
    assert info["n"] == scene["pos"].shape[0] and info["n_cells"] == 160 * 96 * 80
    assert info["n_bodies"] == 64
    # the layer emitted on the device for the library, computed on the host for the oracle
    hg, ho = (configs.Hose(params["box"], params["spacing"], per_step=2048, speed=3.0,
                           limit=int(scene["pour_budget"])) for _ in range(2))
    pos, vel = ho.emit()
    assert g.hoseEmit(hg) == o.appendFluid(pos, vel) == 2048
    dt = (1 / 60) / params["substeps"]
    assert g.step(dt) == o.step(dt) == 1
    compare_sim(g, o)
    g.close()


def test_batched_mix_full_size_one_frame():
    mix = configs.batched_mix()
    assert sum(sc["pos"].shape[0] for _, sc in mix) == 6003226
    b = Batch(**arena_sizes(mix))
    ids = [b.add_scene(p, sc) for p, sc in mix]
    b.step(ids, 1 / 60)
    b.synchronize()
    for sid, (p, sc) in zip(ids, mix):
        o = oracle.OracleSim()
        o.reset_scene(p, sc)
        assert o.step(1 / 60) == 2
        bi, oi = b.info(sid), o.info()
        for k in ("n", "parity", "n_cells", "n_bodies", "last_substeps"):
            assert bi[k] == oi[k], (sid, k, bi[k], oi[k])
        n, c = bi["n"], bi["n_cells"]
        for name in NAMES:
            same(b.read(sid, name)[:n], o.buffer(name)[:n], f"scene {sid} {name}")
        same(b.read(sid, "cellStart")[:c + 1], o.buffer("cellStart")[:c + 1], f"scene {sid} cellStart")
        assert b.stats(sid)["raw"] == o.stats()["raw"], sid
    b.close()
