"""GPU parity: libp4a (CUDA sm_100a) against the CPU oracle on the same inputs.

Both sides follow the same float contract (explicit fma only in dot products and
accumulations, IEEE division/sqrt, fixed-point integer reductions), so the
expected agreement is bit-exact for every buffer: cell keys, the sort
permutation and cellStart (integer work), and positions, velocities, densities,
lambdas, body poses and the fixed-point stats (float work). The looser
tolerance of the workload definition (1e-5 h absolute on positions and
velocities after one substep) is asserted as well, so a failure says which bar
broke.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from particles4all_b200 import Sim, _abi, _lib, configs
from particles4all_b200.params import default_params

pytestmark = pytest.mark.gpu

TOL_H = 1e-5  # positions / velocities after one substep, times h


@pytest.fixture(scope="module", autouse=True)
def need_gpu(built):
    if not _lib.device_available():
        pytest.fail("libp4a cannot use GPU 0 (no sm_100 device or the library failed to load)")


def small_params(**kw):
    p = default_params("small")
    p.update({"targetParticleCount": 3000, "box": [0.5, 0.4, 0.3], "bodies": []})
    p.update(kw)
    return p


def pair(params, scene=None):
    g, o = Sim(), oracle.OracleSim()
    if scene is None:
        g.reset(params)
        o.reset(params)
    else:
        g.reset_scene(params, scene)
        o.reset_scene(params, scene)
    return g, o


PARTICLE_BUFS = ("pos", "vel", "pred", "body", "rest")


def compare(g, o, names=PARTICLE_BUFS + ("density", "lambda_"), h=None, exact=True):
    gi, oi = g.info(), o.info()
    for k in ("n", "parity", "pred_parity", "n_cells", "n_boundary", "n_bodies", "last_substeps"):
        assert gi[k] == oi[k], (k, gi[k], oi[k])
    n = gi["n"]
    for name in names:
        a = g.read(name)[:n]
        b = o.buffer(name)[:n]
        if exact:
            bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
            assert bad.size == 0, f"{name}: {bad.shape[0]} mismatches, first {bad[:3].tolist()} " \
                                  f"gpu {a[tuple(bad[0][:1])]} oracle {b[tuple(bad[0][:1])]}"
        if h is not None and name in ("pos", "vel", "pred"):
            assert np.max(np.abs(a.astype(np.float64) - b)) <= TOL_H * h, name
    c = gi["n_cells"]
    assert np.array_equal(g.read("cellStart")[:c + 1], o.buffer("cellStart")[:c + 1])


def test_grid_sort_operator_matches_oracle():
    import torch
    rng = np.random.default_rng(5)
    dims = [13, 7, 9]
    h = 0.7
    for n in (0, 1, 257, 5000, 40000):
        pos = np.zeros((n, 4), np.float32)
        pos[:, :3] = rng.uniform(-1.0, np.array(dims) * h + 1.0, size=(n, 3))  # some outside: clamped
        if n >= 5000:
            pos[: n // 4, :3] = 2.1  # a crowded cell: many particles share one key
        vel = rng.normal(size=(n, 4)).astype(np.float32)
        body = rng.integers(0, 5, size=(n, 4)).astype(np.uint32)
        rest = rng.normal(size=(n, 4)).astype(np.float32)
        grid = {"box_min": [0.0, 0.0, 0.0], "h": h, "dim": dims}
        want = oracle.grid_sort(grid, 1 / 240, 9.81, pos, vel, body, rest)
        dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
        t_in = [dev(pos), dev(vel), dev(body.view(np.int32)), dev(rest)]
        t_out = [torch.zeros((max(n, 1), 4), dtype=t.dtype, device="cuda") for t in t_in]
        t_out.insert(2, torch.zeros((max(n, 1), 4), dtype=torch.float32, device="cuda"))
        ncells = dims[0] * dims[1] * dims[2]
        cs = torch.zeros(ncells + 1, dtype=torch.int32, device="cuda")
        slot = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
        L = _lib.lib()
        wsz = L.p4a_grid_sort_workspace_size(n, ncells)
        ws = torch.zeros(wsz, dtype=torch.uint8, device="cuda")
        g = _abi.Grid()
        g.h = h
        for k in range(3):
            g.dim[k] = dims[k]
        st = torch.cuda.current_stream().cuda_stream
        rc = L.p4a_grid_sort(C.byref(g), n, 1 / 240, 9.81, *[t.data_ptr() for t in t_in],
                             *[t.data_ptr() for t in t_out], cs.data_ptr(), slot.data_ptr(),
                             ws.data_ptr(), wsz, None, st)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(cs.cpu().numpy().view(np.uint32), want["cell_start"])
        assert np.array_equal(slot.cpu().numpy()[:n].view(np.uint32), want["slot"])
        for t, k in zip(t_out, ("pos", "vel", "pred", "body", "rest")):
            got = t.cpu().numpy()[:n]
            if k == "body":
                got = got.view(np.uint32)
            assert np.array_equal(got, want[k]), k


@pytest.mark.parametrize("case", ["fluid", "bodies_tension", "odd_k_sor", "no_boundary"])
def test_reset_and_one_substep_bit_exact(case):
    if case == "fluid":
        p = small_params()
    elif case == "bodies_tension":
        p = small_params(bodies=["sphere:0.5", "torus:0.8", "box:1.4"], bodySize=0.05,
                         surfaceTensionK=0.4, xsphC=0.066, omega=1.03, targetParticleCount=4000)
    elif case == "odd_k_sor":
        p = small_params(iterations=3, sorAverage=True, omega=1.2, bodies=["box:0.6"], bodySize=0.05)
    else:
        p = small_params(noBoundary=True, substeps=2)
    g, o = pair(p)
    compare(g, o, names=PARTICLE_BUFS)
    dt = (1 / 60) / p["substeps"]
    assert g.step(dt) == o.step(dt) == 1
    compare(g, o, h=2 * p["spacing"])
    assert g.get_stats()["raw"] == o.stats()["raw"]
    if case != "fluid" and case != "no_boundary":
        for name in ("bodyCentre", "bodyRot", "bodyRef"):
            assert np.array_equal(g.read(name), o.buffer(name)), name


def test_many_frames_bit_exact():
    p = small_params(bodies=["sphere:0.5", "box:1.4"], bodySize=0.05, surfaceTensionK=0.3,
                     targetParticleCount=2500, substeps=2)
    g, o = pair(p)
    for frame in range(30):
        fd = 1 / 60 if frame % 7 else 1 / 45  # uneven frames exercise the time bank
        assert g.step(fd) == o.step(fd)
    compare(g, o)
    assert g.get_stats()["raw"] == o.stats()["raw"]
    gp = g.get_body_pose()
    op_c = o.buffer("bodyCentre")
    for b, pose in enumerate(gp):
        assert np.array_equal(np.float32(pose["centre"]), op_c[b, :3])


def test_workload_scenes_one_step():
    for gen, kw in ((configs.dam_break_32k, {"side": 12}), (configs.medium_bodies_264k, {"side": 16, "n_cubes": 3})):
        params, scene = gen(**kw)
        g, o = pair(params, scene)
        compare(g, o, names=PARTICLE_BUFS)
        assert g.step(1 / 60) == o.step(1 / 60) == 2
        compare(g, o, h=1.0)
        assert g.get_stats()["raw"] == o.stats()["raw"]


def test_aniso_bit_exact():
    params, scene = configs.medium_bodies_264k(side=14, n_cubes=2)
    g, o = pair(params, scene)
    g.step(1 / 60); o.step(1 / 60)
    a = configs.medium_aniso_params()
    g.aniso(a); o.aniso(a)
    n = g.info()["n"]
    assert np.array_equal(g.read("smoothPos")[:n], o.buffer("smoothPos")[:n])
    assert np.array_equal(g.read("aniso")[: 2 * n], o.buffer("aniso")[: 2 * n])
    a["min_extent"] = 0.3
    a["ratio"] = 2.3
    g.aniso(a); o.aniso(a)
    assert np.array_equal(g.read("aniso")[: 2 * n], o.buffer("aniso")[: 2 * n])


def test_aniso_after_many_frames_and_moves():
    """The anisotropic pass after every frame of a splashing scene whose box is not
    a whole number of cells (particles beyond the grid are binned into the end
    cells), after a resize and after positions are written: the cells it skips
    as out of reach never change a bit."""
    p = small_params(bodies=["sphere:0.5"], bodySize=0.06, targetParticleCount=4000)
    g, o = pair(p)
    a = configs.medium_aniso_params()
    n = g.info()["n"]

    def check():
        for s in (g, o):
            s.aniso(a)
        assert np.array_equal(g.read("smoothPos")[:n], o.buffer("smoothPos")[:n])
        assert np.array_equal(g.read("aniso")[: 2 * n], o.buffer("aniso")[: 2 * n])
    for f in range(12):
        for s in (g, o):
            s.step(1 / 60)
            if f == 4:
                s.applyRayImpulse([0.0, 0.1, 0.15], [1.0, 0.0, 0.0], [6.0, 2.0, 0.0], 0.3, 4.0)
        check()
    for s in (g, o):
        s.resizeBox([0.42, 0.4, 0.3])
    check()
    pos = g.read("pos")[:n].copy()
    pos[: n // 2, 1] += 0.05
    g.write("pos", pos)
    o.write("pos", pos)
    check()


def test_interactive_calls_bit_exact():
    p = small_params(bodies=["sphere:0.5", "box:1.4"], bodySize=0.05, targetParticleCount=2000)
    g, o = pair(p)
    for s in (g, o):
        s.step(1 / 60)
        s.applyRayImpulse([0.0, 0.1, 0.15], [1.0, 0.0, 0.0], [3.0, 1.0, 0.0], 0.2, 2.0)
        s.holdBody(1, [0.25, 0.3, 0.15], 10.0, 4.0)
        s.step(1 / 60)
        s.releaseBody()
        rng = np.random.default_rng(3)
        pos3 = rng.uniform([0.05, 0.2, 0.05], [0.2, 0.3, 0.2], size=(300, 3)).astype(np.float32)
        vel3 = np.tile(np.float32([1.0, 0.0, 0.0]), (300, 1))
        assert s.appendFluid(pos3, vel3) == 300
        s.step(1 / 60)
        s.resizeBox([0.45, 0.4, 0.3])
        s.step(1 / 60)
    compare(g, o)


def test_viewer_hose_bit_exact():
    """The reference's frame loop while pouring (src/main.js:986-997): the frame
    split into substep slices, pourStep after each with the time advanced, on the
    GPU and the oracle alike."""
    from particles4all_b200.pour import Pour
    p = small_params(targetParticleCount=1500, pour=True)
    g, o = pair(p)
    hoses = [Pour(budget=g.info()["pour_budget"], height=0.7), Pour(budget=o.info()["pour_budget"], height=0.7)]
    for _ in range(6):
        for s, hose in zip((g, o), hoses):
            want = 1 / 60
            for _guard in range(64):
                if want <= 1e-6:
                    break
                sl = min(want, 1 / 60 / max(1, p["substeps"]))
                s.step(sl)
                hose.step(s, s.info()["last_advanced"], params=p)
                want -= sl
    assert hoses[0].left == hoses[1].left < g.info()["pour_budget"]
    compare(g, o)


def test_append_clamps_to_capacity():
    p = small_params(targetParticleCount=500, pour=True)
    g, o = pair(p)
    cap, n = g.info()["cap"], g.info()["n"]
    big = np.full((cap, 3), 0.1, np.float32)
    assert g.appendFluid(big, big) == o.appendFluid(big, big) == cap - n
    assert g.appendFluid(big, big) == 0
    g.step(1 / 60); o.step(1 / 60)
    compare(g, o)


def test_run_to_run_deterministic():
    p = small_params(bodies=["torus:0.8"], bodySize=0.06, surfaceTensionK=0.4)
    outs = []
    for _ in range(2):
        g = Sim()
        g.reset(p)
        for _ in range(5):
            g.step(1 / 60)
        outs.append([g.read(k) for k in ("pos", "vel", "density", "lambda_")] + [g.get_stats()["raw"]])
        g.close()
    for a, b in zip(*outs):
        assert np.array_equal(np.asarray(a), np.asarray(b))


def test_edge_cases():
    # no particles at all (no fluid, no bodies)
    g, o = pair(small_params(targetParticleCount=0))
    assert g.info()["n"] == 0
    assert g.step(1 / 60) == o.step(1 / 60)
    compare(g, o)
    # one particle; a frame shorter than a substep takes no substep
    g, o = pair(small_params(targetParticleCount=1))
    assert g.step(0.001) == 0 and g.info()["last_advanced"] == 0
    g.step(1 / 60); o.step(1 / 60)
    compare(g, o)
    # the spiral-of-death cap (src/sim.js:422-423)
    assert g.step(10.0) == 8 * 4 and g.info()["time_bank"] == 0


def test_crowded_lists_take_the_direct_walk():
    """A cluster far denser than rest density (spacing 0.15 h): every particle has
    more than the list capacity (96) of candidates within h + skin, so lambda,
    delta and the finishing passes all take the reference's direct loop; a sparse
    part of the same scene keeps using lists. Both stay bit-identical to the
    oracle, with tension (normals pass + tension walk) and without."""
    rng = np.random.default_rng(3)
    for tension in (0.0, 0.5):
        p = configs._base_params([12.0, 8.0, 10.0], iterations=4, tension=tension, xsph=0.01)
        side = np.arange(8) * 0.15
        x, y, z = np.meshgrid(side, side, side, indexing="ij")
        dense = np.stack([x.ravel(), y.ravel(), z.ravel()], 1) + [3.0, 1.0, 3.0]
        sparse = rng.uniform([6.0, 1.0, 2.0], [10.0, 5.0, 8.0], size=(1500, 3))
        fluid = np.concatenate([dense, sparse]) + rng.uniform(-0.005, 0.005, size=(512 + 1500, 3))
        sc = configs._assemble(fluid, [], p, configs.lattice_mass(0.5, 1.0))
        g, o = pair(p, sc)
        for _ in range(2):
            assert g.step(1 / 60) == o.step(1 / 60)
        compare(g, o, names=PARTICLE_BUFS + ("density", "lambda_"))
        if tension > 0:
            compare(g, o, names=("normal", "corr"))


def test_verify_harness_checks():
    """The reference's own ?verify=1 checks (src/main.js:853-937) on the GPU state."""
    p = small_params(targetParticleCount=5000, bodies=["sphere:0.5"], bodySize=0.05)
    g = Sim()
    g.reset(p)
    g.step(1 / 60)
    info = g.info()
    n, c = info["n"], info["n_cells"]
    cs = g.read("cellStart")[: c + 1].astype(np.int64)
    assert np.all(np.diff(cs) >= 0) and cs[c] == n
    pred = g.read("pred")[:n]
    dens = g.read("density")[:n]
    lam = g.read("lambda_")[:n]
    assert np.isfinite(pred).all() and np.isfinite(dens).all() and np.isfinite(lam).all()
    half = 0.5 * p["spacing"]
    assert (pred[:, :3] >= half - 1e-6).all() and (pred[:, :3] <= np.array(p["box"]) - half + 1e-6).all()


def _long_run_stats(sim, n_bodies, rest, body, mass, rho0, body_density):
    """Mean / max density constraint error (rho/rho0 - 1)^+, particle count and the
    rigid-body volumes (N_b m / rho_body plus the extent of the oriented bounding box
    of the body's rest offsets under its pose)."""
    n = sim.info()["n"]
    rho = (sim.read("density") if hasattr(sim, "read") else sim.buffer("density"))[:n].astype(np.float64)
    err = np.maximum(rho / rho0 - 1.0, 0.0)
    out = {"n": n, "mean_err": float(err.mean()), "max_err": float(err.max()), "volumes": []}
    rot = (sim.read("bodyRot") if hasattr(sim, "read") else sim.buffer("bodyRot"))[: 3 * n_bodies, :3]
    for b in range(n_bodies):
        sel = body[:n, 0] == b + 1
        R = rot[3 * b: 3 * b + 3].astype(np.float64)
        q = rest[:n, :3][sel].astype(np.float64) @ R.T
        ext = float(np.prod(q.max(0) - q.min(0)))
        out["volumes"].append(sel.sum() * mass / (body_density[b] * rho0) + ext)
    return out


@pytest.mark.parametrize("workload", ["dam_break_32k", "bodies_small"])
def test_thousand_steps_statistics(workload):
    """1,000 steps on the GPU and in the oracle: mean and max density-constraint
    error, particle count and rigid-body volumes agree within 2 % (they are in fact
    bit-identical, since every step is)."""
    if workload == "dam_break_32k":
        p, sc = configs.dam_break_32k()
    else:
        p, sc = configs.medium_bodies_264k(side=12, n_cubes=2)
    g, o = pair(p, sc)
    for _ in range(1000):
        g.step(1 / 60)
        o.step(1 / 60)
    gi = g.info()
    nb = gi["n_bodies"]
    dens = list(sc.get("body_density", [])) if nb else []
    sg = _long_run_stats(g, nb, g.read("rest"), g.read("body"), gi["mass"], p["restDensity"], dens)
    so = _long_run_stats(o, nb, o.buffer("rest"), o.buffer("body"), gi["mass"], p["restDensity"], dens)
    assert sg["n"] == so["n"]
    for k in ("mean_err", "max_err"):
        assert abs(sg[k] - so[k]) <= 0.02 * max(abs(so[k]), 1e-6), (k, sg[k], so[k])
    for vg, vo in zip(sg["volumes"], so["volumes"]):
        assert abs(vg - vo) <= 0.02 * abs(vo)
    assert sg == so  # bit-identical state gives identical statistics
    assert g.get_stats()["raw"] == o.stats()["raw"]
    compare(g, o)
    g.close()


def test_device_hose_layers_match_the_host_restatement():
    """p4a_hose_emit writes each layer on the device from its emission index: the
    appended positions, velocities and the appendFluid fields (pred = pos, density
    rho0, zero lambda / body / rest) must equal the host restatement bit for bit,
    over several emissions and up to the capacity limit."""
    params, scene = configs.dam_break_32k(side=12)
    scene = dict(scene, pour_budget=5000)
    g, o = pair(params, scene)
    hg, ho = (configs.Hose(params["box"], params["spacing"], per_step=2048, speed=3.0, limit=5000)
              for _ in range(2))
    for k in range(4):
        n0 = g.info()["n"]
        pos, vel = ho.emit()
        added_o = 0 if pos is None else o.appendFluid(pos, vel)
        added_g = g.hoseEmit(hg)
        assert added_g == added_o == [2048, 2048, 904, 0][k]
        n = g.info()["n"]
        assert n == n0 + added_g
        if added_g:
            assert np.array_equal(g.read("pos")[n0:n, :3], pos)
            assert np.all(g.read("pos")[n0:n, 3] == 1.0)
            assert np.array_equal(g.read("vel")[n0:n, :3], vel)
        compare(g, o, names=PARTICLE_BUFS + ("density", "lambda_"))
        g.step(1 / 60)
        o.step(1 / 60)
        compare(g, o, h=1.0)
