"""Batched multi-scene stepping: every scene stepped inside a batch (one launch
per pass for all scenes, segmented sort, (scene, tile) work items, CUDA-graph
replay) must give the bits it gives when stepped alone through the plain Sim,
whatever else shares the batch. Also: admission by arena capacity, removal and
reuse of arena ranges."""
import numpy as np
import pytest

from particles4all_b200 import Batch, P4AError, Sim, _lib, configs
from particles4all_b200.params import default_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def mixed_scenes():
    out = []
    p = default_params("small")
    p.update({"targetParticleCount": 2500, "box": [0.5, 0.4, 0.3], "bodies": ["sphere:0.5", "box:1.4"],
              "bodySize": 0.05, "surfaceTensionK": 0.4, "substeps": 2})
    out.append((p, None))
    p = default_params("small")
    p.update({"targetParticleCount": 1800, "box": [0.4, 0.3, 0.3], "bodies": [], "iterations": 3,
              "sorAverage": True, "omega": 1.2})
    out.append((p, None))
    out.append(configs.dam_break_32k(side=10))
    out.append(configs.medium_bodies_264k(side=12, n_cubes=2))
    p = default_params("small")
    p.update({"targetParticleCount": 900, "box": [0.3, 0.3, 0.2], "bodies": ["torus:0.8"],
              "bodySize": 0.06, "substeps": 1, "noBoundary": True})
    out.append((p, None))
    return out


def run_alone(params, scene, frames):
    s = Sim()
    if scene is None:
        s.reset(params)
    else:
        s.reset_scene(params, scene)
    for fd in frames:
        s.step(fd)
    return s


NAMES = ("pos", "vel", "pred", "body", "rest", "density", "lambda_")


def assert_same(sim, batch, sid):
    n = sim.info()["n"]
    bi = batch.info(sid)
    assert bi["n"] == n and bi["parity"] == sim.info()["parity"]
    for name in NAMES:
        a, b = sim.read(name)[:n], batch.read(sid, name)[:n]
        assert np.array_equal(a, b), name
    c = sim.info()["n_cells"]
    assert np.array_equal(sim.read("cellStart")[: c + 1], batch.read(sid, "cellStart")[: c + 1])
    if sim.info()["n_bodies"]:
        for name in ("bodyCentre", "bodyRot"):
            assert np.array_equal(sim.read(name)[: sim.info()["n_bodies"] * (3 if name == "bodyRot" else 1)],
                                  batch.read(sid, name)[: sim.info()["n_bodies"] * (3 if name == "bodyRot" else 1)])
    assert sim.get_stats()["raw"] == batch.stats(sid)["raw"]


@pytest.mark.parametrize("graphs,lanes", [(True, 1), (False, 1), (True, 2), (False, 2), (True, 4)])
def test_batch_equals_alone_bit_exact(graphs, lanes):
    """lanes > 1 with no size threshold: every frame runs as concurrent parts."""
    scenes = mixed_scenes()
    frames = [1 / 60] * 6 + [1 / 45, 1 / 90, 1 / 60]
    b = Batch(max_particles=200_000, max_cells=400_000, max_scenes=16, graphs=graphs)
    b.set_lanes(lanes, 0)
    ids = []
    for p, sc in scenes:
        ids.append(b.add_preset(p) if sc is None else b.add_scene(p, sc))
    for fd in frames:
        b.step(ids, fd)
    b.synchronize()
    for (p, sc), sid in zip(scenes, ids):
        assert_same(run_alone(p, sc, frames), b, sid)


def test_subset_steps_and_arena_reuse():
    scenes = mixed_scenes()
    b = Batch(max_particles=60_000, max_cells=200_000, max_scenes=8)
    ids = [b.add_preset(p) if sc is None else b.add_scene(p, sc) for p, sc in scenes[:3]]
    # step only some scenes in some frames: the others must not move
    b.step(ids, 1 / 60)
    b.step(ids[:1], 1 / 60)
    b.step(ids[1:], 1 / 60)
    b.synchronize()
    p0, s0 = scenes[0]
    assert_same(run_alone(p0, s0, [1 / 60, 1 / 60]), b, ids[0])
    p1, s1 = scenes[1]
    assert_same(run_alone(p1, s1, [1 / 60, 1 / 60]), b, ids[1])
    # remove one, admit another into the freed ranges
    free0 = b.usage()["free_particles"]
    b.remove_scene(ids[1])
    assert b.usage()["free_particles"] > free0
    p4, s4 = scenes[4]
    sid = b.add_preset(p4)
    b.step([sid, ids[0]], 1 / 60)
    b.synchronize()
    assert_same(run_alone(p4, s4, [1 / 60]), b, sid)
    assert_same(run_alone(p0, s0, [1 / 60] * 3), b, ids[0])


def test_admission_rejects_when_full():
    p, sc = configs.dam_break_32k(side=12)  # 1,728 particles
    b = Batch(max_particles=4000, max_cells=100_000, max_scenes=4)
    b.add_scene(p, sc)
    b.add_scene(p, sc)
    with pytest.raises(P4AError) as e:
        b.add_scene(p, sc)
    assert e.value.status == 5
    assert b.usage()["live_scenes"] == 2


@pytest.mark.parametrize("groups", [1, 2, 0, 7])
def test_step_io_equals_write_step_read(groups):
    """p4a_batch_step_io (host inputs, the scenes in `groups` frames with the copies
    on their own streams) gives the bits of write_async + step + read_async."""
    import torch
    scenes = mixed_scenes()
    b = Batch(max_particles=400_000, max_cells=800_000, max_scenes=16)
    add = lambda p, sc: b.add_preset(p) if sc is None else b.add_scene(p, sc)
    a_ids = [add(p, sc) for p, sc in scenes]
    b_ids = [add(p, sc) for p, sc in scenes]
    ns = [b.info(s)["n"] for s in a_ids]
    rng = np.random.default_rng(5)
    pin = lambda n: torch.zeros(n * 4, dtype=torch.float32, pin_memory=True)
    inputs = []
    for s, n in zip(a_ids, ns):
        pos, vel = b.read(s, "pos")[:n].copy(), b.read(s, "vel")[:n].copy()
        pos[:, :3] += rng.uniform(-2e-4, 2e-4, (n, 3)).astype(np.float32)
        vel[:, :3] += rng.uniform(-0.3, 0.3, (n, 3)).astype(np.float32)
        inputs.append((torch.from_numpy(pos.reshape(-1)).pin_memory(), torch.from_numpy(vel.reshape(-1)).pin_memory()))
    outs_a = [(pin(n), pin(n)) for n in ns]
    outs_b = [(pin(n), pin(n)) for n in ns]
    for f, fd in enumerate([1 / 60, 1 / 45, 1 / 60]):
        # frame 0 from the perturbed inputs, later frames from the previous outputs;
        # velocities only in frame 1 (pos_in None), nothing read back in frame 2 for
        # the odd scenes
        src_a = inputs if f == 0 else outs_a
        src_b = inputs if f == 0 else outs_b
        if f > 0:
            src_a = [(p.clone().pin_memory(), v.clone().pin_memory()) for p, v in src_a]
            src_b = [(p.clone().pin_memory(), v.clone().pin_memory()) for p, v in src_b]
        for k, (s, n) in enumerate(zip(a_ids, ns)):
            if f != 1:
                b.write_async(s, "pos", src_a[k][0].data_ptr(), n * 16)
            b.write_async(s, "vel", src_a[k][1].data_ptr(), n * 16)
        b.step(a_ids, fd)
        for k, (s, n) in enumerate(zip(a_ids, ns)):
            if f == 2 and k % 2:
                continue
            b.read_async(s, "pos", outs_a[k][0].data_ptr(), n * 16)
            b.read_async(s, "vel", outs_a[k][1].data_ptr(), n * 16)
        entries = []
        for k, (s, n) in enumerate(zip(b_ids, ns)):
            skip = f == 2 and k % 2
            entries.append((s, None if f == 1 else src_b[k][0].data_ptr(), src_b[k][1].data_ptr(),
                            None if skip else outs_b[k][0].data_ptr(), None if skip else outs_b[k][1].data_ptr()))
        b.step_io(entries, fd, groups)
        b.synchronize()
        for k in range(len(ns)):
            assert torch.equal(outs_a[k][0], outs_b[k][0]) and torch.equal(outs_a[k][1], outs_b[k][1]), (f, k)
    for sa, sb in zip(a_ids, b_ids):
        n = b.info(sa)["n"]
        assert b.info(sa)["parity"] == b.info(sb)["parity"]
        for name in NAMES:
            assert np.array_equal(b.read(sa, name)[:n], b.read(sb, name)[:n]), name
        assert b.stats(sa)["raw"] == b.stats(sb)["raw"]


def test_lanes_with_subsets_and_arena_reuse():
    """Two-lane frames over changing scene subsets, across a removal and a new
    admission, give each scene the bits it gets alone."""
    scenes = mixed_scenes()
    b = Batch(max_particles=200_000, max_cells=400_000, max_scenes=8)
    b.set_lanes(2, 0)
    ids = [b.add_preset(p) if sc is None else b.add_scene(p, sc) for p, sc in scenes[:4]]
    b.step(ids, 1 / 60)
    b.step(ids[1:], 1 / 60)
    b.step(ids[:2], 1 / 45)
    b.synchronize()
    steps = {0: [1 / 60, 1 / 45], 1: [1 / 60, 1 / 60, 1 / 45], 2: [1 / 60, 1 / 60], 3: [1 / 60, 1 / 60]}
    for k, sid in enumerate(ids):
        p, sc = scenes[k]
        assert_same(run_alone(p, sc, steps[k]), b, sid)
    b.remove_scene(ids[2])
    p4, s4 = scenes[4]
    sid = b.add_preset(p4)
    b.step([ids[0], sid, ids[3]], 1 / 60)
    b.synchronize()
    assert_same(run_alone(p4, s4, [1 / 60]), b, sid)
    assert_same(run_alone(scenes[3][0], scenes[3][1], [1 / 60] * 3), b, ids[3])
    with pytest.raises(P4AError):
        b.set_lanes(5, 0)
    with pytest.raises(P4AError):
        b.set_lanes(0, 0)


def test_step_io_rejects_bad_lists():
    p, sc = configs.dam_break_32k(side=8)
    b = Batch(max_particles=20_000, max_cells=100_000, max_scenes=4)
    s = b.add_scene(p, sc)
    with pytest.raises(P4AError):
        b.step_io([(s, None, None, None, None), (s, None, None, None, None)], 1 / 60)
    with pytest.raises(P4AError):
        b.step_io([(s + 1, None, None, None, None)], 1 / 60)
    with pytest.raises(P4AError):
        b.step_io([(s, None, None, None, None)], 1 / 60, groups=-1)
    b.step_io([], 1 / 60)
    b.step_io([(s, None, None, None, None)], 1 / 60, groups=3)  # more groups than scenes
    b.synchronize()
    assert b.info(s)["sim_time"] > 0
