"""The benchmark hose's generator and layer on the host (CPU only): Philox4x32-10
against the published known-answer vectors of its authors' Random123 library, and
the layer's lattice, jitter range, limit and emission bookkeeping."""
import numpy as np

from particles4all_b200.configs import Hose, philox4x32_10


def _one(c, k):
    return [int(x[0]) for x in philox4x32_10(*[np.array([v], np.uint32) for v in c], k[0], k[1])]


def test_philox_known_answers():
    assert _one([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert _one([0xFFFFFFFF] * 4, [0xFFFFFFFF, 0xFFFFFFFF]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert _one([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_layer_lattice_jitter_and_limit():
    d = 0.5
    h = Hose([160.0, 96.0, 80.0], d, per_step=2048, speed=3.0, limit=5000)
    assert h.k == 46
    pos, vel = h.emit()
    assert pos.dtype == np.float32 and pos.shape == (2048, 3)
    q = np.arange(2048)
    iy, iz = q // 46, q % 46
    ideal = np.stack([np.full(2048, h.nozzle[0], np.float64),
                      h.nozzle[1] + (iy - 22.5) * d, h.nozzle[2] + (iz - 22.5) * d], 1)
    dev = pos.astype(np.float64) - ideal
    assert np.abs(dev).max() <= 0.001 * d * (1 + 1e-3) + 1e-5
    assert np.abs(dev).max() > 0.0009 * d  # the jitter spans its range
    assert np.all(vel == np.array([3.0, 0.0, 0.0], np.float32))
    assert h.emission == 1 and h.left == 2952
    p2, _ = h.emit()
    assert not np.array_equal(p2, pos)  # each emission draws new jitter
    p3, _ = h.emit()
    assert p3.shape == (904, 3) and h.left == 0
    assert h.emit() == (None, None)
    # a layer is a function of its emission index
    again = Hose([160.0, 96.0, 80.0], d, per_step=2048, speed=3.0).layer(1, 2048)[0]
    assert np.array_equal(again, p2)
    assert h.c_struct().count == 0 and h.c_struct().per_step == 2048  # the lattice stays 46 x 46
