"""Scene setup (src/scene.js): the product's host builder (libp4a) against the
oracle, and the oracle against independent Python transcriptions of the JS for
small scenes. CPU only."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from particles4all_b200 import _abi, _lib
from particles4all_b200.params import CParams, apply_ini, default_params


def product_scene(params):
    cp = CParams(params)
    cnt = _abi.SceneCounts()
    L = _lib.lib()
    assert L.p4a_build_scene(cp.ref(), C.byref(cnt), None, None, None, None, None, None) == 0
    n, nb = cnt.n, cnt.n_bodies
    pos = np.zeros((n, 4), np.float32); vel = np.zeros((n, 4), np.float32)
    rest = np.zeros((n, 4), np.float32); phase = np.zeros((n, 4), np.uint32)
    cen = np.zeros((max(1, nb), 3)); den = np.zeros(max(1, nb))
    assert L.p4a_build_scene(cp.ref(), C.byref(cnt), pos.ctypes.data, vel.ctypes.data, rest.ctypes.data,
                             phase.ctypes.data, cen.ctypes.data, den.ctypes.data) == 0
    return dict(n=n, n_fluid=cnt.n_fluid, n_bodies=nb, n_boundary=cnt.n_boundary, mass=cnt.mass,
                denom_rest=cnt.denom_rest, pos=pos, rest=rest, phase=phase, body_centre=cen[:nb],
                body_density=den[:nb])


SMALL_INI = """substeps=2
iterations=4
xsph=0.066
tension=0.4
omega=1.03
box=1.5 1 1
particles=30000
body=sphere:0.5,torus:0.5,box:0.5
bodysize=0.1
"""


@pytest.mark.parametrize("preset,count", [("small", 3000), ("small", 20000), ("extreme", 5000)])
def test_product_scene_matches_oracle(built, preset, count):
    p = default_params(preset)
    p["targetParticleCount"] = count
    a, b = product_scene(p), oracle.build_scene(p)
    for k in ("n", "n_fluid", "n_bodies", "n_boundary"):
        assert a[k] == b[k], k
    assert a["mass"] == b["mass"] and a["denom_rest"] == b["denom_rest"]
    for k in ("pos", "rest", "phase"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["body_centre"], b["body_centre"])
    assert np.array_equal(a["body_density"], b["body_density"])


def test_ini_preset_scene(built):
    p = apply_ini(default_params("small"), SMALL_INI)
    p["targetParticleCount"] = 4000
    assert p["box"] == [1.5, 1.0, 1.0] and p["bodySize"] == 0.1 and p["surfaceTensionK"] == 0.4
    a, b = product_scene(p), oracle.build_scene(p)
    assert a["n_bodies"] == 3 and np.array_equal(a["pos"], b["pos"]) and a["mass"] == b["mass"]


# ---- independent transcriptions of src/scene.js (float64, JS semantics) ----

def js_fluid_block(p, d):
    """fluidBlock (src/scene.js:43-64) in Python floats (IEEE doubles, like JS)."""
    bx, by, bz = p["box"]
    margin = d
    nx = max(1, math.floor(bx * 0.35 / d))
    nz = max(1, math.floor((bz - 2 * margin) / d))
    max_layers = max(1, math.floor((by - 2 * margin) / d))
    target = p["targetParticleCount"]
    layers = min(math.ceil(target / (nx * nz)), max_layers)
    out = []
    seed = 12345

    def rnd():
        nonlocal seed
        s = float(seed) * 1103515245.0 + 12345.0   # double product, as JS
        seed = int(s) & 0x7fffffff                  # ToInt32 then mask
        return (seed / 0x7fffffff - 0.5) * 0.002 * d
    iy = 0
    while iy < layers and len(out) // 3 < target:
        ix = 0
        while ix < nx and len(out) // 3 < target:
            iz = 0
            while iz < nz and len(out) // 3 < target:
                out += [margin + (ix + 0.5) * d + rnd(), margin + (iy + 0.5) * d + rnd(),
                        margin + (iz + 0.5) * d + rnd()]
                iz += 1
            ix += 1
        iy += 1
    return np.array(out).reshape(-1, 3)


def test_fluid_block_matches_js_transcription(built):
    p = default_params("small")
    p["targetParticleCount"] = 2500
    p["bodies"] = []
    sc = oracle.build_scene(p)
    ref = js_fluid_block(p, p["spacing"]).astype(np.float32)
    assert sc["n_fluid"] == ref.shape[0] == 2500
    assert np.array_equal(sc["pos"][:, :3], ref)


def test_lcg_first_values():
    # first draws of the JS LCG (seed 12345): exact integer products below 2^53
    seed = 12345
    seq = []
    for _ in range(3):
        s = float(seed) * 1103515245.0 + 12345.0
        seed = int(s) & 0x7fffffff
        seq.append(seed)
    assert seq[0] == (12345 * 1103515245 + 12345) & 0x7fffffff == 1406932606


def test_boundary_counts_and_psi(built):
    p = default_params("small")
    p["box"] = [0.3, 0.2, 0.25]
    d, h = 0.02, 0.04
    pts, psi = oracle.boundary(p, d, h)
    nb = [max(2, math.ceil(s / d) + 1) for s in p["box"]]
    assert pts.shape[0] == nb[0] * nb[1] * nb[2] - (nb[0] - 2) * (nb[1] - 2) * (nb[2] - 2)
    # psi = rho0 / sum_j W(r_ij) by brute force (src/scene.js:105-133)
    coef = 315 / (64 * math.pi * h ** 9)
    r2 = np.sum((pts[:, None, :] - pts[None, :, :]) ** 2, -1)
    t = np.where(r2 < h * h, h * h - r2, 0.0)
    want = (1000.0 / (coef * np.sum(t ** 3, 1))).astype(np.float32)
    assert np.allclose(psi, want, rtol=2e-7, atol=0)


def test_mass_calibration_brute_force(built):
    p = default_params("small")
    p["targetParticleCount"] = 1500
    p["bodies"] = []
    sc = oracle.build_scene(p)
    d = p["spacing"]; h = 2 * d
    x = sc["pos"][:, :3].astype(np.float64)
    coef = 315 / (64 * math.pi * h ** 9)
    r2 = np.sum((x[:, None] - x[None]) ** 2, -1)
    np.fill_diagonal(r2, np.inf)
    t = np.where(r2 < h * h, h * h - r2, 0.0)
    m0 = 1000 * d ** 3
    rho = m0 * coef * h ** 6 + m0 * coef * np.sum(t ** 3, 1)
    want = m0 * 1000 / rho.max() if rho.max() > 500 else m0
    assert math.isclose(sc["mass"], want, rel_tol=1e-12)
    assert sc["denom_rest"] > 0


RENDER_INI = """
display=4
meshres=96
meshiso=0.35
fieldsmooth=2
raysurface=0
cubemap="D:\\\\panoramas\\\\sky_2k.hdr"
cubemapintensity=1.5
cubemapyaw=90
floorplane=0
anisoradius=2.5
anisonbrs=20
ior=1.5
transmit=0.1 0.2 0.3
sunelev=20
ssfrradius=0.7
ssfrfilter=1
ssfrcleanup=0
ssfrdepthcull=0.5
soraverage=1
"""


def test_ini_render_settings():
    """The render keys of a preset reach the pass parameters as the reference's
    viewer applies them (src/settingsini.js:3-93, src/main.js:320-400, 955-970)."""
    from particles4all_b200.params import render_from_ini
    p = apply_ini(default_params("small"), RENDER_INI)
    assert p["sorAverage"] is False  # soraverage is on the reference's unsupported list
    r = render_from_ini(RENDER_INI, p)
    assert r["view"] == "ssfr"
    assert (r["mesh"]["resolution"], r["mesh"]["iso"], r["mesh"]["field_passes"]) == (96, 0.35, 2)
    assert r["ray"]["use_surface"] == 0 and r["ray"]["iso"] == 0.35
    assert r["env"] == {"file": "sky_2k.hdr", "intensity": 1.5, "yaw": math.pi / 2}
    for g in ("ssfr", "ray"):
        assert r[g]["floor_plane"] == 0 and r[g]["env_intensity"] == 1.5 and r[g]["env_yaw"] == math.pi / 2
        assert r[g]["ior"] == 1.5 and r[g]["transmit"] == [0.1, 0.2, 0.3] and r[g]["sun_elevation"] == 20
    assert (r["aniso"]["radius_scale"], r["aniso"]["min_neighbours"]) == (2.5, 20)
    assert (r["ssfr"]["splat_radius"], r["ssfr"]["filter"], r["ssfr"]["cleanup_pass"]) == (0.7, 1, 0)
    # 0.5 of the lattice neighbours within the anisotropic radius 2.5 h = 5 spacings
    assert r["ssfr"]["depth_cull_neighbours"] == math.floor(0.5 * 4.18879 * 5.0 ** 3)
    plain = render_from_ini("", p)
    assert plain["ssfr"]["cleanup_pass"] == 1 and plain["ssfr"]["depth_cull_neighbours"] == 0
    assert plain["env"]["file"] is None and plain["view"] is None
