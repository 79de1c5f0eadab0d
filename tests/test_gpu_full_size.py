"""The large workload at its full size (2,097,152 fluid particles + 64 rigid bodies,
the hose, 8 iterations, tension; 2^22-cell grid), where the oracle is too slow to
follow: the properties that do not depend on size. After each frame the cell
offsets are monotone and end at n, every particle's sort cell matches its range,
positions stay in the clamp box, nothing is non-finite, and n grows by exactly what
the hose appended; two runs from the same state give the same bits."""
import numpy as np
import pytest

from particles4all_b200 import Sim, _lib, configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")


def run(params, scene, frames):
    s = Sim()
    s.reset_scene(params, scene)
    hose = configs.Hose(params["box"], params["spacing"], per_step=2048, speed=3.0,
                        limit=int(scene.get("pour_budget", 0)))
    d = params["spacing"]
    box = np.array(params["box"])
    for _ in range(frames):
        n0 = s.info()["n"]
        added = s.hoseEmit(hose)
        s.step(1 / 60)
        info = s.info()
        n, c = info["n"], info["n_cells"]
        assert n == n0 + added and added == 2048
        cs = s.read("cellStart")[: c + 1].astype(np.int64)
        assert np.all(np.diff(cs) >= 0) and cs[c] == n
        pred = s.read("pred")[:n, :3]
        assert np.isfinite(pred).all() and np.isfinite(s.read("vel")[:n, :3]).all()
        assert np.isfinite(s.read("density")[:n]).all()
        half = 0.5 * d
        assert (pred >= half - 1e-5).all() and (pred <= box - half + 1e-5).all()
    # the last substep's sort: particle i sits in the range of the cell its predicted
    # position was binned into; since then only the iterations moved it, so its
    # final position's cell is that cell or a neighbour of it
    h = info["h"]
    dim = np.array(info["grid_dim"])
    cell = np.clip(np.floor(s.read("pos")[:n, :3] / h).astype(np.int64), 0, dim - 1)
    owner = np.searchsorted(cs, np.arange(n), side="right") - 1  # the cell whose range holds i
    oc = np.stack([owner % dim[0], (owner // dim[0]) % dim[1], owner // (dim[0] * dim[1])], 1)
    assert np.abs(oc - cell).max() <= 1
    out = {k: s.read(k)[:n].copy() for k in ("pos", "vel", "density")}
    out["stats"] = s.get_stats(wait=1)["raw"]
    s.close()
    return out


def test_large_workload_properties_and_determinism():
    params, scene = configs.large_hose_2m()
    a = run(params, scene, 3)
    b = run(params, scene, 3)
    for k in ("pos", "vel", "density"):
        assert np.array_equal(a[k], b[k]), k
    assert a["stats"] == b["stats"]
