"""Asynchronous readback (p4a_read_async / p4a_read_wait): the copy sees the buffer
as it was when the copy was queued, later calls that change the buffer (a step, a
write, the anisotropic pass on its own outputs) wait for it on the device, calls
that reallocate wait for it on the host, and the data equals a synchronous read."""
import numpy as np
import pytest
import torch

from particles4all_b200 import Sim, _lib, configs
from particles4all_b200.params import default_aniso

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def pinned(n):
    """Pinned float32 host memory as a torch tensor and its numpy view."""
    t = torch.empty(n, dtype=torch.float32, pin_memory=True)
    return t, t.numpy()


@pytest.fixture()
def sim():
    p, sc = configs.dam_break_32k(side=16)
    g = Sim()
    g.reset_scene(p, sc)
    for _ in range(2):
        g.step(1 / 60)
    yield g
    g.close()


def test_async_read_equals_sync_read(sim):
    n = sim.info()["n"]
    _, hp = pinned(n * 4)
    _, hv = pinned(n * 4)
    sim.read_async("pos", hp)
    sim.read_async("vel", hv)
    sim.read_wait()
    assert np.array_equal(hp.reshape(-1, 4), sim.read("pos")[:n])
    assert np.array_equal(hv.reshape(-1, 4), sim.read("vel")[:n])


def test_copy_sees_the_buffer_before_later_calls(sim):
    n = sim.info()["n"]
    before = sim.read("pos")[:n].copy()
    _, hp = pinned(n * 4)
    sim.read_async("pos", hp)
    sim.write("pos", np.zeros_like(before))  # same buffer, queued after the copy
    sim.read_wait()
    assert np.array_equal(hp.reshape(-1, 4), before)
    assert not sim.read("pos")[:n].any()


def test_steps_and_aniso_queued_behind_copies(sim):
    n = sim.info()["n"]
    pos0 = sim.read("pos")[:n].copy()
    _, hp = pinned(n * 4)
    sim.read_async("pos", hp)
    for _ in range(3):
        sim.step(1 / 60)
    sim.read_wait()
    assert np.array_equal(hp.reshape(-1, 4), pos0)
    sim.aniso(default_aniso())
    g0 = sim.read("aniso")[:2 * n].copy()
    _, hg = pinned(n * 8)
    sim.read_async("aniso", hg)
    sim.step(1 / 60)
    sim.aniso(default_aniso())  # rewrites G after the copy
    sim.read_wait()
    assert np.array_equal(hg.reshape(-1, 4), g0)


def test_reset_and_close_with_copies_in_flight():
    p, sc = configs.dam_break_32k(side=12)
    g = Sim()
    g.reset_scene(p, sc)
    n = g.info()["n"]
    _, hp = pinned(n * 4)
    g.read_async("pos", hp)
    g.reset_scene(p, sc)  # frees and reallocates: waits for the copy first
    assert np.array_equal(hp.reshape(-1, 4), g.read("pos")[:n])
    g.read_async("vel", hp)
    g.synchronize()
    g.read_async("pos", hp)
    g.close()


def test_read_async_rejects_bad_ranges(sim):
    n = sim.info()["n"]
    _, hp = pinned(n * 4)
    with pytest.raises(ValueError):
        sim.read_async("pos", hp, nbytes=hp.nbytes + 16)
    with pytest.raises(_lib.P4AError):
        sim.read_async("pos", hp.ctypes.data, nbytes=sim.info()["cap"] * 16 + 16)
