"""The C-ABI library loads, exports every entry point include/p4a.h declares, and
fails loudly (no fallback) where a GPU is needed but absent. CPU only."""
import ctypes as C
import os
import re
import subprocess

import pytest

from particles4all_b200 import _abi, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "p4a.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(p4a_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "p4a_step" in syms and "p4a_reset" in syms and "p4a_grid_sort" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol(built):
    L = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_ctypes_signatures_cover_header(built):
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_abi_version_and_status_strings(built):
    L = _lib.lib()
    assert L.p4a_abi_version() == 1
    assert L.p4a_status_string(0) == b"ok"
    assert L.p4a_status_string(4) == b"device wait timed out"


def test_struct_layouts_match_c_compiler(tmp_path):
    """Every ctypes mirror has the size and field offsets gcc gives the C struct."""
    structs = {"p4a_body_spec": _abi.BodySpec, "p4a_params": _abi.Params,
               "p4a_scene_desc": _abi.SceneDesc, "p4a_info": _abi.Info, "p4a_stats": _abi.Stats,
               "p4a_aniso_params": _abi.AnisoParams, "p4a_grid": _abi.Grid,
               "p4a_scene_counts": _abi.SceneCounts, "p4a_batch_config": _abi.BatchConfig,
               "p4a_batch_usage": _abi.BatchUsage, "p4a_phase_time": _abi.PhaseTime,
               "p4a_server_config": _abi.ServerConfig, "p4a_completion": _abi.Completion,
               "p4a_server_stats": _abi.ServerStats, "p4a_mesh_params": _abi.MeshParams,
               "p4a_mesh_info": _abi.MeshInfo, "p4a_ssfr_params": _abi.SsfrParams,
               "p4a_ssfr_info": _abi.SsfrInfo, "p4a_ray_params": _abi.RayParams,
               "p4a_batch_io": _abi.BatchIO, "p4a_hose": _abi.Hose}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "p4a.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            cf = "lambda" if fname == "lambda_" else fname
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {cf}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        cname, field, val = line.split()
        cls = structs[cname]
        got = C.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert got == int(val), (cname, field, got, val)


def test_default_params_match_reference(built):
    p = _abi.Params()
    assert _lib.lib().p4a_default_params(b"small", C.byref(p)) == 0
    # src/scene.js:14-31
    assert (p.spacing, p.rest_density, p.gravity, p.substeps, p.iterations) == (0.02, 1000, 9.81, 4, 4)
    assert (p.cfm_epsilon_rel, p.s_corr_k, p.s_corr_dq, p.xsph_c, p.omega) == (0.01, 0.1, 0.3, 0.05, 1.0)
    assert (p.target_particle_count, list(p.box), p.n_bodies) == (60000, [1.5, 1.5, 1.0], 3)
    assert [(p.bodies[i].shape, p.bodies[i].density) for i in range(3)] == [(0, 0.5), (1, 0.8), (2, 1.4)]


def test_no_device_fails_loudly(built):
    if _lib.device_available():
        pytest.skip("a GPU is present")
    L = _lib.lib()
    h = C.c_void_p()
    rc = L.p4a_create(0, C.byref(h))
    assert rc == _abi.P4A_ERR_NODEV and not h.value
    from particles4all_b200 import Sim, P4AError
    with pytest.raises(P4AError):
        Sim()
    cfg = _abi.ServerConfig()
    assert L.p4a_server_default_config(C.byref(cfg)) == 0
    assert cfg.max_frames_in_flight == 2 and cfg.use_graphs == 1 and cfg.arenas.max_scenes == 1024
    assert L.p4a_server_create(0, C.byref(cfg), C.byref(h)) == _abi.P4A_ERR_NODEV and not h.value
    from particles4all_b200.server import Server
    with pytest.raises(P4AError):
        Server(budget_bytes=1 << 30)


def test_grid_sort_rejects_bad_arguments(built):
    L = _lib.lib()
    g = _abi.Grid()
    g.h = 1.0
    for k in range(3):
        g.dim[k] = 4
    assert L.p4a_grid_sort_workspace_size(100, 64) > 0
    assert L.p4a_grid_sort_workspace_size(-1, 64) == 0
    # missing workspace -> capacity error before any device work
    rc = L.p4a_grid_sort(C.byref(g), 0, 0.0, 0.0, *([None] * 9), C.c_void_p(16), None, None, 0, None, None)
    assert rc == _abi.P4A_ERR_CAPACITY
    g.dim[0] = 0
    assert L.p4a_grid_sort(C.byref(g), 0, 0.0, 0.0, *([None] * 11), None, 0, None, None) == _abi.P4A_ERR_ARG


@pytest.mark.parametrize("dims", [(2**31 - 1, 2**31 - 1, 2**31 - 1), (2**20, 2**20, 2**20), (65536, 65536, 1),
                                  (1, 2**16, 2**16), (2**31 - 1, 2, 1), (3, 2**30, 2**30)])
def test_grid_sort_entries_reject_huge_dims_without_overflow(built, dims):
    """A cell count beyond an entry's limit is rejected before any device work,
    whatever the dims: the product is checked factor by factor, so it cannot wrap
    to a small or negative count that would pass the check."""
    L = _lib.lib()
    g = _abi.Grid()
    g.h = 1.0
    for k in range(3):
        g.dim[k] = dims[k]
    assert dims[0] * dims[1] * dims[2] > 2**31 - 1  # beyond both entries' limits
    dummy = [C.c_void_p(256)] * 11
    rc = L.p4a_grid_sort_noalloc(C.byref(g), 16, 0.0, 0.0, *dummy, None, None)
    assert rc == _abi.P4A_ERR_CAPACITY
    rc = L.p4a_grid_sort(C.byref(g), 16, 0.0, 0.0, *dummy, C.c_void_p(256), 1 << 40, None, None)
    assert rc == _abi.P4A_ERR_CAPACITY


def test_tuning_table_host_side(built, tmp_path):
    """The launch-shape table is host state: set / get / clear and the JSON round
    trip of the autotuner work without a GPU."""
    from particles4all_b200 import autotune
    L = _lib.lib()
    cnt = C.c_int32()
    t = (C.c_int32 * 8)()
    m = (C.c_int32 * 8)()
    assert L.p4a_kernel_shapes(0, t, m, 8, C.byref(cnt)) == 0 and cnt.value == 6
    assert (t[0], m[0]) == (256, 4) and all(t[k] in (64, 128, 256) for k in range(6))
    assert L.p4a_kernel_shapes(9, t, m, 8, C.byref(cnt)) == _abi.P4A_ERR_ARG
    v = C.c_int32()
    try:
        L.p4a_tune_clear(-1)
        assert L.p4a_tune_set(1, 1000, 3) == 0 and L.p4a_tune_set(1, 100, 2) == 0
        for n, want in ((50, 2), (100, 2), (101, 3), (1000, 3), (1001, 0)):
            assert L.p4a_tune_get(1, n, C.byref(v)) == 0 and v.value == want, n
        assert L.p4a_tune_set(1, 100, 7) == _abi.P4A_ERR_ARG
        path = tmp_path / "t.json"
        path.write_text('{"kernels": {"aniso": [[10, 5], [1000000, 1]]}}')
        autotune.load(str(path), L)
        assert L.p4a_tune_get(3, 5, C.byref(v)) == 0 and v.value == 5
        assert L.p4a_tune_get(3, 500, C.byref(v)) == 0 and v.value == 1
        L.p4a_tune_clear(3)
        assert L.p4a_tune_get(3, 5, C.byref(v)) == 0 and v.value == 0
    finally:
        L.p4a_tune_clear(-1)
        autotune.load(L=L)



def test_batched_tuning_tables_fall_back_to_the_plain_ones(built):
    """The batched launches' tables (kernels 4-6) are their own; while one is empty,
    a batched launch of that kernel uses the plain kernel's table."""
    L = _lib.lib()
    v = C.c_int32()
    t = (C.c_int32 * 8)()
    m = (C.c_int32 * 8)()
    cnt = C.c_int32()
    assert L.p4a_kernel_shapes(4, t, m, 8, C.byref(cnt)) == 0 and cnt.value == 6
    assert L.p4a_kernel_shapes(7, t, m, 8, C.byref(cnt)) == _abi.P4A_ERR_ARG
    try:
        L.p4a_tune_clear(-1)
        assert L.p4a_tune_set(0, 1 << 40, 2) == 0
        assert L.p4a_tune_get(4, 5_000_000, C.byref(v)) == 0 and v.value == 2  # falls back to lambda's
        assert L.p4a_tune_set(4, 1 << 40, 3) == 0
        assert L.p4a_tune_get(4, 5_000_000, C.byref(v)) == 0 and v.value == 3
        assert L.p4a_tune_get(0, 5_000_000, C.byref(v)) == 0 and v.value == 2  # plain table unchanged
        L.p4a_tune_clear(4)
        assert L.p4a_tune_get(4, 5_000_000, C.byref(v)) == 0 and v.value == 2
    finally:
        L.p4a_tune_clear(-1)
        from particles4all_b200 import autotune
        autotune.load()

def test_server_default_config(built):
    """p4a_server_default_config (host only): the documented defaults, frame lanes
    included."""
    L = _lib.lib()
    cfg = _abi.ServerConfig()
    assert L.p4a_server_default_config(C.byref(cfg)) == 0
    assert (cfg.frame_lanes, cfg.lane_min_particles) == (2, 1_000_000)
    assert (cfg.builder_threads, cfg.max_frames_in_flight, cfg.use_graphs, cfg.plain) == (4, 2, 1, 0)
    assert cfg.upload_bytes == cfg.readback_bytes == 1 << 30


def test_batch_footprint_sizes_server_arenas(built):
    """p4a_batch_footprint counts the arenas p4a_batch_create would allocate (no
    device needed), and the serving loop's arena sizing stays within its budget."""
    from particles4all_b200 import server
    L = _lib.lib()
    out = C.c_int64()
    cfg = _abi.BatchConfig()
    assert L.p4a_batch_footprint(C.byref(cfg), C.byref(out)) == _abi.P4A_ERR_ARG
    small, big = server._arenas(1 << 16, 64), server._arenas(1 << 17, 64)
    fs, fb = server.arena_bytes(small), server.arena_bytes(big)
    # per particle slot at least the ten float4 ping-pong arrays, six float4 solver
    # arrays (corr, normal, start positions, packed gathers), seven 4-byte ones and
    # the neighbour list (96 entries of 4 B)
    assert (fb - fs) / (1 << 16) >= 160 + 6 * 16 + 7 * 4 + 96 * 4
    for budget in (1 << 30, 8 << 30, 160_000_000_000):
        a = server.arenas_for_budget(budget, 4096)
        assert server.arena_bytes(a) <= budget
        assert server.arena_bytes(server._arenas(int(a["max_particles"] * 1.01), 4096)) > budget
