"""p4a_grid_sort_noalloc — the grid-sort operator for callers that cannot allocate
device memory (hosts that own every allocation through their own arena, frame
loops that must not stall on cudaMalloc). It takes the same inputs and outputs
as p4a_grid_sort but uses the library's fixed device scratch array instead of a
caller workspace. Checked against p4a_grid_sort on two calls in a row, through
the C ABI. This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from particles4all_b200 import _abi, _lib

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 524288
MAX_CELLS = 524288


def _inputs(rng, n, dims, h, crowd=None):
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-0.5, np.array(dims) * h + 0.5, size=(n, 3))
    pos[: n // 5 if crowd is None else crowd, :3] = 1.3 * h  # a crowded cell
    vel = rng.normal(size=(n, 4)).astype(np.float32)
    body = rng.integers(0, 4, size=(n, 4)).astype(np.uint32)
    rest = rng.normal(size=(n, 4)).astype(np.float32)
    return pos, vel, body, rest


def _run(torch, fn_name, grid, n, ncells, arrays, workspace=None, status=None):
    L = _lib.lib()
    t_in = [torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda() for a in arrays]
    t_out = [torch.full((max(n, 1), 4), -7, dtype=t.dtype, device="cuda") for t in t_in]
    t_out.insert(2, torch.full((max(n, 1), 4), -7.0, dtype=torch.float32, device="cuda"))
    cs = torch.full((ncells + 1,), -7, dtype=torch.int32, device="cuda")
    slot = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    ptrs = [t.data_ptr() for t in t_in] + [t.data_ptr() for t in t_out] + [cs.data_ptr(), slot.data_ptr()]
    sp = None if status is None else status.data_ptr()
    if fn_name == "p4a_grid_sort":
        rc = L.p4a_grid_sort(C.byref(grid), n, 1 / 240, 9.81, *ptrs, workspace.data_ptr(),
                             workspace.numel(), sp, st)
    else:
        rc = L.p4a_grid_sort_noalloc(C.byref(grid), n, 1 / 240, 9.81, *ptrs, sp, st)
    assert rc == 0, (fn_name, rc)
    torch.cuda.synchronize()
    if status is not None:
        assert int(status.item()) == 0, (fn_name, "scan error word set")
    return [t.cpu().numpy()[:n] for t in t_out] + [cs.cpu().numpy(), slot.cpu().numpy()[:n]]


def test_noalloc_matches_workspace_entry_on_two_calls(built):
    import torch
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0")
    h = 0.5
    cases = [(30000, [17, 11, 13], 11), (4000, [9, 40, 5], 12)]
    rng_results = []
    for n, dims, seed in cases:
        grid = _abi.Grid()
        grid.h = h
        for k in range(3):
            grid.dim[k] = dims[k]
        ncells = dims[0] * dims[1] * dims[2]
        arrays = _inputs(np.random.default_rng(seed), n, dims, h)
        ws = torch.zeros(_lib.lib().p4a_grid_sort_workspace_size(n, ncells), dtype=torch.uint8, device="cuda")
        want = _run(torch, "p4a_grid_sort", grid, n, ncells, arrays, ws)
        rng_results.append((grid, n, ncells, arrays, want))
    # two calls in a row on the shared scratch, then compare both with the workspace entry
    got = [_run(torch, "p4a_grid_sort_noalloc", g, n, c, a) for g, n, c, a, _ in rng_results]
    for (_, _, _, _, want), res in zip(rng_results, got):
        for a, b in zip(want, res):
            assert np.array_equal(a, b)
    # and once more on the first input after the second call left its contents behind,
    # this time with the error word delivered to a device status word
    g, n, c, a, want = rng_results[0]
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    again = _run(torch, "p4a_grid_sort_noalloc", g, n, c, a, status=status)
    for x, y in zip(want, again):
        assert np.array_equal(x, y)


def test_noalloc_at_its_maximum_sizes(built):
    """Exactly P4A_NOALLOC_MAX_PARTICLES particles on exactly P4A_NOALLOC_MAX_CELLS
    cells (128 x 64 x 64), so every region of the fixed scratch array is used to
    its end; bit-exact against the workspace entry, twice in a row."""
    import torch
    h = 0.5
    dims = [128, 64, 64]
    assert dims[0] * dims[1] * dims[2] == MAX_CELLS
    n = MAX_PARTICLES
    grid = _abi.Grid()
    grid.h = h
    for k in range(3):
        grid.dim[k] = dims[k]
    arrays = _inputs(np.random.default_rng(21), n, dims, h, crowd=2000)
    ws = torch.zeros(_lib.lib().p4a_grid_sort_workspace_size(n, MAX_CELLS), dtype=torch.uint8, device="cuda")
    want = _run(torch, "p4a_grid_sort", grid, n, MAX_CELLS, arrays, ws)
    del ws
    for _ in range(2):
        got = _run(torch, "p4a_grid_sort_noalloc", grid, n, MAX_CELLS, arrays)
        for a, b in zip(want, got):
            assert np.array_equal(a, b)


def test_noalloc_rejects_sizes_beyond_its_scratch(built):
    L = _lib.lib()
    g = _abi.Grid()
    g.h = 1.0
    g.dim[0], g.dim[1], g.dim[2] = 64, 64, 64
    dummy = [C.c_void_p(256)] * 11
    assert L.p4a_grid_sort_noalloc(C.byref(g), MAX_PARTICLES + 1, 0.0, 0.0, *dummy, None,
                                   None) == _abi.P4A_ERR_CAPACITY
    g.dim[0], g.dim[1], g.dim[2] = 128, 64, 65  # 532,480 cells
    assert L.p4a_grid_sort_noalloc(C.byref(g), 16, 0.0, 0.0, *dummy, None, None) == _abi.P4A_ERR_CAPACITY
