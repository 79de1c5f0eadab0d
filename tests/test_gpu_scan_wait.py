"""The cell scan's bounded wait, made to run out on purpose.

The scan's decoupled lookback polls its predecessor tiles' state words with a
bounded spin; when the limit runs out it sets the error word and stops waiting,
so the kernel returns and every access stays in bounds (the outputs are then
invalid). Here the operators' test hook starts the tile tickets at 1: tile 0 is
never scanned, so tile 1 (and any tile that looks back past it) waits on a flag
that nothing sets, with a limit of 1,024 polls (~0.1 ms). The calls must report
it (P4A_ERR_TIMEOUT, or a nonzero device status word), and the context must stay
usable: with the hook off again, the same call is bit-exact against the oracle.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from particles4all_b200 import _abi, _lib

pytestmark = pytest.mark.gpu


def _case(n=20000, dims=(40, 30, 20), h=0.5, seed=3):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0.0, np.array(dims) * h, size=(n, 3))
    vel = rng.normal(size=(n, 4)).astype(np.float32)
    return list(dims), h, pos, vel


def _call(torch, entry, dims, h, pos, vel, status=None):
    L = _lib.lib()
    n = pos.shape[0]
    ncells = dims[0] * dims[1] * dims[2]
    assert ncells > 2048  # at least two scan tiles, so tile 1 looks back at tile 0
    g = _abi.Grid()
    g.h = h
    for k in range(3):
        g.dim[k] = dims[k]
    t_in = [torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda()]
    t_out = [torch.zeros((n, 4), dtype=torch.float32, device="cuda") for _ in range(3)]
    cs = torch.zeros(ncells + 1, dtype=torch.int32, device="cuda")
    slot = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    ptrs = [t_in[0].data_ptr(), t_in[1].data_ptr(), None, None, t_out[0].data_ptr(), t_out[1].data_ptr(),
            t_out[2].data_ptr(), None, None, cs.data_ptr(), slot.data_ptr()]
    sp = None if status is None else status.data_ptr()
    if entry == "p4a_grid_sort":
        wsz = L.p4a_grid_sort_workspace_size(n, ncells)
        ws = torch.zeros(wsz, dtype=torch.uint8, device="cuda")
        rc = L.p4a_grid_sort(C.byref(g), n, 1 / 240, 9.81, *ptrs, ws.data_ptr(), wsz, sp, st)
    else:
        rc = L.p4a_grid_sort_noalloc(C.byref(g), n, 1 / 240, 9.81, *ptrs, sp, st)
    torch.cuda.synchronize()
    return rc, cs.cpu().numpy().view(np.uint32), slot.cpu().numpy().view(np.uint32)


def test_scan_wait_that_runs_out_is_reported_and_the_context_stays_usable(built):
    import torch
    L = _lib.lib()
    dims, h, pos, vel = _case()
    try:
        assert L.p4a_test_scan_wait(1024, 1) == 0
        for entry in ("p4a_grid_sort", "p4a_grid_sort_noalloc"):
            rc, _, _ = _call(torch, entry, dims, h, pos, vel)
            assert rc == _abi.P4A_ERR_TIMEOUT, (entry, rc)
            status = torch.zeros(1, dtype=torch.int32, device="cuda")
            rc, _, _ = _call(torch, entry, dims, h, pos, vel, status=status)
            assert rc == 0, (entry, rc)
            assert int(status.item()) & 1, (entry, "the device status word must carry the timeout")
    finally:
        assert L.p4a_test_scan_wait(0, 0) == 0
    grid = {"box_min": [0.0, 0.0, 0.0], "h": h, "dim": dims}
    want = oracle.grid_sort(grid, 1 / 240, 9.81, pos, vel, None, None)
    for entry in ("p4a_grid_sort", "p4a_grid_sort_noalloc"):
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        rc, cs, slot = _call(torch, entry, dims, h, pos, vel, status=status)
        assert rc == 0 and int(status.item()) == 0, entry
        assert np.array_equal(cs, want["cell_start"]), entry
        assert np.array_equal(slot, want["slot"]), entry
        rc, cs, _ = _call(torch, entry, dims, h, pos, vel)
        assert rc == 0 and np.array_equal(cs, want["cell_start"]), entry


def test_scan_wait_hook_rejects_bad_arguments(built):
    L = _lib.lib()
    assert L.p4a_test_scan_wait(0, 2) == _abi.P4A_ERR_ARG
    assert L.p4a_test_scan_wait(0, -1) == _abi.P4A_ERR_ARG
    assert L.p4a_test_scan_wait(0, 0) == 0
