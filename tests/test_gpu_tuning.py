"""Launch shapes: every shape of every tuned kernel (threads per block x minimum
blocks per SM) gives the same bits, in plain steps, in the anisotropic pass and in
batched frames, so the autotuner can only change speed."""
import numpy as np
import pytest

from particles4all_b200 import Batch, Sim, _lib, configs, default_aniso
from particles4all_b200 import autotune

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")
    yield
    L = _lib.lib()
    L.p4a_tune_clear(-1)
    autotune.load(L=L)


NAMES = ("pos", "vel", "pred", "density", "lambda_", "smoothPos", "aniso")


def run(p, sc, frames=3):
    s = Sim()
    s.reset_scene(p, sc)
    for _ in range(frames):
        s.step(1 / 60)
        s.aniso(default_aniso())
    n = s.info()["n"]
    out = {k: s.read(k)[: n * (2 if k == "aniso" else 1)].copy() for k in NAMES}
    out["stats"] = s.get_stats()["raw"]
    s.close()
    return out


def force(kernel, variant):
    L = _lib.lib()
    L.p4a_tune_clear(-1)
    L.p4a_tune_set(kernel, 1 << 40, variant)


def test_every_shape_same_bits_plain():
    p, sc = configs.medium_bodies_264k(side=16, n_cubes=2)  # tension on: the normals pass runs
    L = _lib.lib()
    L.p4a_tune_clear(-1)
    ref = run(p, sc)
    for kernel in range(4):
        for v in range(1, 6):
            force(kernel, v)
            got = run(p, sc)
            for k in ref:
                assert np.array_equal(np.asarray(ref[k]), np.asarray(got[k])), (kernel, v, k)


@pytest.mark.parametrize("variant", [2, 3])
def test_batched_frames_in_other_shapes(variant):
    scenes = [configs.dam_break_32k(side=10), configs.medium_bodies_264k(side=12, n_cubes=2)]
    L = _lib.lib()
    L.p4a_tune_clear(-1)
    alone = [run(p, sc, frames=2) for p, sc in scenes]
    for k in range(3):
        L.p4a_tune_set(k, 1 << 40, variant)
    b = Batch(max_particles=50_000, max_cells=200_000, max_scenes=4)
    ids = [b.add_scene(p, sc) for p, sc in scenes]
    for _ in range(2):
        b.step(ids, 1 / 60)
    b.synchronize()
    for sid, ref in zip(ids, alone):
        n = b.info(sid)["n"]
        for name in ("pos", "vel", "density", "lambda_"):
            assert np.array_equal(b.read(sid, name)[:n], ref[name]), (variant, name)
    b.close()
    L.p4a_tune_clear(-1)
