"""The serving loop (continuous batching): a scene's results are the same bits
whether it is served alone through the plain Sim or in the mix with scenes that
arrive, step and leave while its own frames are on the GPU; admission waits for
room (or rejects after the timeout); requests to gone scenes fail cleanly."""
import time

import numpy as np
import pytest

from particles4all_b200 import Sim, _lib, configs
from particles4all_b200.server import Server
from particles4all_b200.params import default_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def scenes():
    out = []
    p = default_params("small")
    p.update({"targetParticleCount": 2500, "box": [0.5, 0.4, 0.3], "bodies": ["sphere:0.5", "box:1.4"],
              "bodySize": 0.05, "surfaceTensionK": 0.4, "substeps": 2})
    out.append((p, None))
    out.append(configs.dam_break_32k(side=10))
    out.append(configs.medium_bodies_264k(side=12, n_cubes=2))
    p = default_params("small")
    p.update({"targetParticleCount": 1800, "box": [0.4, 0.3, 0.3], "bodies": [], "iterations": 3})
    out.append((p, None))
    return out


def alone(params, scene, steps):
    """Positions and velocities after each of `steps` 1/60 s frames, stepped alone."""
    s = Sim()
    if scene is None:
        s.reset(params)
    else:
        s.reset_scene(params, scene)
    out = []
    n = s.info()["n"]
    for _ in range(steps):
        s.step(1 / 60)
        out.append((s.read("pos")[:n].copy(), s.read("vel")[:n].copy()))
    s.close()
    return out


def wait_for(srv, want, timeout=60.0):
    """Polls until every request id in `want` has completed; returns {request: completion}."""
    got = {}
    t0 = time.time()
    while not want <= set(got):
        for c in srv.poll(wait=0.05):
            got[c["request"]] = c
        assert time.time() - t0 < timeout, "server did not complete the requests"
    return got


def step_with_readback(srv, sid, outs, rows=20_000):
    pos = np.zeros((rows, 4), np.float32)
    vel = np.zeros((rows, 4), np.float32)
    outs.setdefault(sid, []).append((pos, vel))
    return srv.step(sid, 1 / 60, pos_out=pos, vel_out=vel)


def serve_mix(plain, lanes=2):
    sc = scenes()
    steps = 4
    # lane_min_particles 0: with lanes > 1 every batched frame runs as concurrent parts
    srv = Server(arenas=dict(max_particles=100_000, max_cells=400_000, max_boundary=400_000, max_scenes=8,
                             max_bodies=64, max_body_parts=20_000),
                 plain=plain, builder_threads=2, upload_bytes=64 << 20, readback_bytes=64 << 20,
                 lanes=lanes, lane_min_particles=0)
    outs = {}
    reqs = set()
    # two scenes first; the others arrive while those are stepping
    sids = []
    for k, (p, s) in enumerate(sc):
        sid, r = srv.create_scene(p, s)
        sids.append(sid)
        reqs.add(r)
        if k == 1:
            for _ in range(2):
                for q in sids:
                    reqs.add(step_with_readback(srv, q, outs))
    for q in sids:
        while len(outs.get(q, [])) < steps:
            reqs.add(step_with_readback(srv, q, outs))
    got = wait_for(srv, reqs)
    assert all(c["status"] == 0 for c in got.values()), [c for c in got.values() if c["status"]]
    n = {c["scene"]: c["particles"] for c in got.values() if c["kind"] == "create"}
    st = srv.stats()
    gone = {srv.destroy_scene(q) for q in sids}
    done = wait_for(srv, gone)
    assert all(c["status"] == 0 for c in done.values())
    assert st["steps"] == steps * len(sc) and st["admitted"] == len(sc)
    srv.close()
    return sc, sids, n, outs, st


@pytest.mark.parametrize("plain,lanes", [(False, 1), (False, 2), (True, 1)])
def test_served_equals_alone_bit_exact(plain, lanes):
    sc, sids, n, outs, st = serve_mix(plain, lanes)
    for (p, s), sid in zip(sc, sids):
        ref = alone(p, s, len(outs[sid]))
        for k, ((pos, vel), (rp, rv)) in enumerate(zip(outs[sid], ref)):
            assert np.array_equal(pos[: n[sid]], rp), (sid, k, "pos")
            assert np.array_equal(vel[: n[sid]], rv), (sid, k, "vel")
    assert st["frames"] <= st["steps"]


def test_admission_waits_for_room_then_rejects():
    p, s = configs.dam_break_32k(side=12)  # 1,728 particles
    arenas = dict(max_particles=2000, max_cells=100_000, max_boundary=100_000, max_scenes=4, max_bodies=8,
                  max_body_parts=16)
    srv = Server(arenas=arenas, builder_threads=1, admit_timeout=0.0, upload_bytes=16 << 20,
                 readback_bytes=16 << 20)
    a, ra = srv.create_scene(p, s)
    b, rb = srv.create_scene(p, s)  # no room until a is destroyed
    got = wait_for(srv, {ra})
    assert got[ra]["status"] == 0
    time.sleep(0.3)
    assert not any(c["request"] == rb for c in srv.poll())
    assert srv.stats()["queued_creates"] == 1
    rd = srv.destroy_scene(a)
    got = wait_for(srv, {rb, rd})
    assert got[rb]["status"] == 0 and got[rd]["status"] == 0
    srv.close()
    # with a timeout the waiting create is rejected
    srv = Server(arenas=arenas, builder_threads=1, admit_timeout=0.2, upload_bytes=16 << 20,
                 readback_bytes=16 << 20)
    a, ra = srv.create_scene(p, s)
    b, rb = srv.create_scene(p, s)
    got = wait_for(srv, {ra, rb})
    assert got[ra]["status"] == 0 and got[rb]["status"] == 5
    st = srv.stats()
    assert st["rejected"] == 1 and st["admitted"] == 1
    srv.close()


def test_requests_to_gone_scenes_fail_cleanly():
    p, s = configs.dam_break_32k(side=8)
    srv = Server(arenas=dict(max_particles=10_000, max_cells=100_000, max_boundary=100_000, max_scenes=4,
                             max_bodies=8, max_body_parts=16),
                 builder_threads=1, upload_bytes=16 << 20, readback_bytes=16 << 20)
    sid, rc = srv.create_scene(p, s)
    assert wait_for(srv, {rc})[rc]["status"] == 0
    r1 = srv.step(sid, 1 / 60)
    rd = srv.destroy_scene(sid)
    r2 = srv.step(sid, 1 / 60)          # after the destroy: refused
    r3 = srv.step(12345, 1 / 60)        # never created
    r4 = srv.destroy_scene(sid)         # twice
    got = wait_for(srv, {r1, rd, r2, r3, r4})
    assert got[r1]["status"] == 0 and got[rd]["status"] == 0
    assert got[r2]["status"] == 6 and got[r3]["status"] == 6 and got[r4]["status"] == 6
    # the step submitted before the destroy ran first
    assert got[r1]["finished"] <= got[rd]["finished"]
    srv.close()
