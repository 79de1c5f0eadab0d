"""The reference's params object: PRESETS / defaultParams (src/scene.js:3-39), the
preset .ini keys that reach the simulation (src/settingsini.js:3-33, applied by
src/main.js:361-381), and its conversion to the C struct of include/p4a.h.

Params are plain dicts with the reference's JS key names (spacing, restDensity,
gravity, substeps, iterations, cfmEpsilonRel, sCorrK, sCorrDq, xsphC, omega,
sorAverage, surfaceTensionK, targetParticleCount, box, bodies, bodySize,
noBoundary, pour) so that code written against the reference reads the same.
"""
import ctypes as C
import math

import numpy as np

from . import _abi

# src/scene.js:3-9. The ini presets are parsed from the same keys the reference's
# presets/*.ini files carry (see PRESET_INI below).
PRESETS = {
    "small": {"ini": "presets/small.ini"},
    "medium": {"ini": "presets/medium.ini"},
    "large": {"ini": "presets/large.ini"},
    "extreme": {"particles": 1000000, "box": [3.0, 3.0, 3.0], "substeps": 4, "iterations": 4,
                "bodies": ["sphere:0.5", "torus:0.8", "box:1.4"]},
}


def default_params(preset="small"):
    """defaultParams(preset) (src/scene.js:11-39)."""
    p = PRESETS.get(preset, {})
    out = {
        "preset": preset, "spacing": 0.02, "restDensity": 1000, "gravity": 9.81,
        "substeps": 4, "iterations": 4, "cfmEpsilonRel": 0.01, "sCorrK": 0.1,
        "sCorrDq": 0.3, "xsphC": 0.05, "omega": 1.0, "sorAverage": False,
        "surfaceTensionK": 0, "targetParticleCount": 60000, "box": [1.5, 1.5, 1.0],
        "bodies": ["sphere:0.5", "torus:0.8", "box:1.4"], "bodySize": 0,
    }
    if "substeps" in p:
        out["substeps"] = p["substeps"]
    if "iterations" in p:
        out["iterations"] = p["iterations"]
    if "particles" in p:
        out["targetParticleCount"] = p["particles"]
    if "box" in p:
        out["box"] = list(p["box"])
    if "bodies" in p:
        out["bodies"] = list(p["bodies"])
    out.update(p.get("params", {}))
    return out


# ini key -> params key for the keys that reach Sim (src/settingsini.js:3-33 maps
# ini keys to URL keys; src/main.js:361-381 maps URL keys to params).
_INI_TO_PARAM = {
    "substeps": ("substeps", int), "iterations": ("iterations", int),
    "cfm": ("cfmEpsilonRel", float), "scorrk": ("sCorrK", float),
    "scorrdq": ("sCorrDq", float), "xsph": ("xsphC", float),
    "tension": ("surfaceTensionK", float), "gravity": ("gravity", float),
    "omega": ("omega", float), "particles": ("targetParticleCount", int),
    "spacing": ("spacing", float), "bodysize": ("bodySize", float),
}


def parse_ini(text):
    """parseIni (src/settingsini.js:45-55): key=value lines, # and ; comments."""
    kv = {}
    for raw in str(text).splitlines():
        line = raw.strip()
        if not line or line.startswith("#") or line.startswith(";"):
            continue
        eq = line.find("=")
        if eq <= 0:
            continue
        kv[line[:eq].strip().lower()] = line[eq + 1:].strip()
    return kv


def apply_ini(params, text):
    """Apply the simulation keys of a preset .ini to a params dict (the path
    iniToQuery -> URL query -> qNum of src/settingsini.js:59-93, src/main.js:361-390)."""
    kv = parse_ini(text)
    for k, (name, conv) in _INI_TO_PARAM.items():
        if k in kv:
            params[name] = conv(float(kv[k])) if conv is int else conv(kv[k])
    # soraverage is on the reference's unsupported list (src/settingsini.js:35-43):
    # a preset's value is skipped, as there
    if "box" in kv:
        vals = [float(x) for x in kv["box"].replace(",", " ").split()]
        if len(vals) >= 3 and all(math.isfinite(v) for v in vals):
            params["box"] = vals[:3]
    if "body" in kv:
        params["bodies"] = [b for b in kv["body"].split(",") if b]
    return params


# ini key -> (settings group, field, conversion) for the render settings that
# src/main.js:320-400 reads from the URL keys src/settingsini.js:3-33 maps the ini
# keys to; "ray" fields are also copied into the SSFR settings every frame
# (src/main.js:955-963).
_INI_TO_RENDER = {
    "meshres": ("mesh", "resolution", int), "meshiso": ("mesh", "iso", float),
    "fieldsmooth": ("mesh", "field_passes", int), "normalsmooth": ("mesh", "normal_passes", int),
    "raysurface": ("ray", "use_surface", int),
    "anisoratio": ("aniso", "ratio", float), "anisolambda": ("aniso", "lambda", float),
    "anisonbrs": ("aniso", "min_neighbours", int), "anisolonely": ("aniso", "lonely", float),
    "anisoradius": ("aniso", "radius_scale", float), "anisostretch": ("aniso", "stretch", float),
    "anisoks": ("aniso", "ks", float),
    "ior": ("ray", "ior", float), "absorption": ("ray", "absorption", float),
    "thicksteps": ("ray", "thickness_steps", int), "groundreflection": ("ray", "ground_reflection", float),
    "roughness": ("ray", "roughness", float), "sunintensity": ("ray", "sun_intensity", float),
    "sunelev": ("ray", "sun_elevation", float), "sunazim": ("ray", "sun_azimuth", float),
    "exposure": ("ray", "exposure", float),
    "ssfrradius": ("ssfr", "splat_radius", float), "ssfrscale": ("ssfr", "render_scale", float),
    "ssfrfilter": ("ssfr", "filter", int), "ssfriters": ("ssfr", "filter_iterations", int),
    "ssfrsigma": ("ssfr", "filter_sigma", float), "ssfrdelta": ("ssfr", "narrow_delta", float),
    "ssfrmu": ("ssfr", "narrow_mu", float), "ssfrthickr": ("ssfr", "thickness_radius", float),
    "ssfrthick": ("ssfr", "thickness_scale", float), "ssfrthickblur": ("ssfr", "thickness_filter_size", int),
    "ssfrrange": ("ssfr", "bilateral_range", float),
}
_RAY_TO_SSFR = ("ior", "absorption", "transmit", "roughness", "sun_intensity", "sun_elevation", "sun_azimuth",
                "exposure", "ground_reflection")
_VIEWS = {0: "particles", 1: "mesh", 2: "mesh", 3: "ray", 4: "ssfr"}


def render_from_ini(text, params):
    """The render settings of a preset .ini for a scene with `params` (its spacing
    sets the SSFR depth cull): {"mesh", "aniso", "ssfr", "ray"} parameter dicts for
    p4a_mesh / p4a_aniso / p4a_ssfr / p4a_ray from the library's defaults with the
    preset's keys applied as the reference's viewer applies them, "env" (the
    panorama file name the preset names, its intensity and its yaw in radians) and
    "view". The ray pass's iso is the mesh's; floorplane sets both passes' floor;
    ssfrdepthcull is a fraction of the neighbours within the anisotropic radius
    (src/main.js:965-970)."""
    kv = parse_ini(text)
    out = {"mesh": default_mesh(), "aniso": default_aniso(), "ssfr": default_ssfr(), "ray": default_ray()}
    for k, (group, name, conv) in _INI_TO_RENDER.items():
        if k in kv:
            try:
                out[group][name] = conv(float(kv[k]))
            except ValueError:
                pass  # not a number: ignored here (the reference's Number() would give NaN)
    if "transmit" in kv:
        t = [float(x) for x in kv["transmit"].replace(",", " ").split()]
        if len(t) >= 3 and all(math.isfinite(x) for x in t):
            out["ray"]["transmit"] = t[:3]
    out["ssfr"]["cleanup_pass"] = 0 if kv.get("ssfrcleanup") == "0" else 1  # on unless "0"
    out["ray"]["iso"] = out["mesh"]["iso"]
    for k in _RAY_TO_SSFR:
        out["ssfr"][k] = out["ray"][k]
    env = {"file": None, "intensity": 1.0, "yaw": 0.0}
    if kv.get("cubemap"):
        name = kv["cubemap"].strip('"').replace("\\", "/").split("/")[-1]
        env["file"] = name or None
    if "cubemapintensity" in kv:
        env["intensity"] = float(kv["cubemapintensity"])
    if "cubemapyaw" in kv:
        env["yaw"] = float(kv["cubemapyaw"]) * math.pi / 180
    for group in ("ssfr", "ray"):
        out[group]["env_intensity"], out[group]["env_yaw"] = env["intensity"], env["yaw"]
        if "floorplane" in kv:
            out[group]["floor_plane"] = 0 if kv["floorplane"] == "0" else 1
    out["env"] = env
    frac = float(kv.get("ssfrdepthcull", 0.0))  # depthCullFraction, 0 by default
    h = 2 * params.get("spacing", 0.02)
    full = 4.18879 * (out["aniso"]["radius_scale"] * h / max(params.get("spacing", 0.02), 1e-6)) ** 3
    out["ssfr"]["depth_cull_neighbours"] = math.floor(frac * full) if frac > 0 else 0
    view = kv.get("display")
    out["view"] = _VIEWS.get(int(view), None) if view is not None and view.strip().lstrip("-").isdigit() else None
    return out


def _spec(s):
    bits = s.split(":")
    shape = bits[0]

    def num(i, dflt):
        try:
            v = float(bits[i]) if len(bits) > i else dflt
        except ValueError:
            v = float("nan")
        return v if (v == v and v != 0) else dflt   # Number(x) || dflt
    return _abi.SHAPES.get(shape, 2), num(1, 0.5), num(2, 0.75)


class CParams:
    """Owns a p4a_params struct (and its bodies array) built from a params dict."""

    def __init__(self, p):
        bodies = [_spec(b) for b in p.get("bodies", [])]
        self._bodies = (_abi.BodySpec * max(1, len(bodies)))()
        for i, (shape, dens, sy) in enumerate(bodies):
            self._bodies[i].shape, self._bodies[i].density, self._bodies[i].start_y = shape, dens, sy
        s = _abi.Params()
        s.spacing = p.get("spacing", 0.02)
        s.rest_density = p.get("restDensity", 1000)
        s.gravity = p.get("gravity", 9.81)
        s.substeps = int(p.get("substeps", 4))
        s.iterations = int(p.get("iterations", 4))
        s.cfm_epsilon_rel = p.get("cfmEpsilonRel", 0.01)
        s.s_corr_k = p.get("sCorrK", 0.1)
        s.s_corr_dq = p.get("sCorrDq", 0.3)
        s.xsph_c = p.get("xsphC", 0.05)
        s.omega = p.get("omega", 1.0)
        s.sor_average = 1 if p.get("sorAverage") else 0
        s.surface_tension_k = p.get("surfaceTensionK", 0)
        s.target_particle_count = int(p.get("targetParticleCount", 60000))
        box = p.get("box", [1.5, 1.5, 1.0])
        for k in range(3):
            s.box[k] = box[k]
        s.n_bodies = len(bodies)
        s.bodies = C.cast(self._bodies, C.POINTER(_abi.BodySpec))
        s.body_size = p.get("bodySize", 0)
        s.no_boundary = 1 if p.get("noBoundary") else 0
        s.pour = 0 if p.get("pour") is False else 1
        s.cfm_epsilon_abs = p.get("cfmEpsilonAbs", 0.0)
        self.struct = s

    def ref(self):
        return C.byref(self.struct)


def default_aniso():
    """SurfaceMesh defaults (src/mesh.js:81-89); min_extent 0 (anisoLimitToField off)."""
    return {"ratio": 4.0, "ks": 1.0, "stretch": 2.0, "lonely": 1.0, "min_neighbours": 25,
            "lambda": 0.9, "radius_scale": 2.0, "min_extent": 0.0}


def aniso_struct(a):
    s = _abi.AnisoParams()
    s.ratio, s.ks, s.stretch, s.lonely = a["ratio"], a["ks"], a["stretch"], a["lonely"]
    s.min_neighbours = int(a["min_neighbours"])
    s.lambda_, s.radius_scale, s.min_extent = a["lambda"], a["radius_scale"], a["min_extent"]
    return s


def default_mesh():
    """SurfaceMesh / UI defaults (src/main.js:320-327, src/mesh.js:17): resolution 128,
    iso 0.4, no field passes, 2 normal passes, 3 M triangles; blur along x as the
    reference executes it (blur_axes 0)."""
    return {"resolution": 128, "iso": 0.4, "field_passes": 0, "normal_passes": 2,
            "max_triangles": 3_000_000, "blur_axes": 0}


def mesh_struct(m):
    s = _abi.MeshParams()
    s.resolution, s.iso = int(m["resolution"]), float(m["iso"])
    s.field_passes, s.normal_passes = int(m["field_passes"]), int(m["normal_passes"])
    s.max_triangles, s.blur_axes = int(m["max_triangles"]), int(m["blur_axes"])
    return s


SSFR_MATRICES = ("view", "proj", "inv_view_proj", "inv_view")


def default_ssfr():
    """FluidSSFR's defaults (src/ssfr.js:9-47), an identity camera and a 640 x 480
    target; set the camera with camera.frame_matrices()."""
    from ._lib import lib
    s = _abi.SsfrParams()
    lib().p4a_default_ssfr_params(C.byref(s))
    out = {}
    for name, ctype in _abi.SsfrParams._fields_:
        v = getattr(s, name)
        out[name] = list(v) if hasattr(ctype, "_length_") else v
    return out


def default_ray():
    """RayMarch's defaults (src/ray.js:16-29), iso 0.4, the mesh surface as the
    surface (raySurface 1), an identity camera and a 640 x 480 target."""
    from ._lib import lib
    s = _abi.RayParams()
    lib().p4a_default_ray_params(C.byref(s))
    out = {}
    for name, ctype in _abi.RayParams._fields_:
        v = getattr(s, name)
        out[name] = list(v) if hasattr(ctype, "_length_") else v
    return out


def ray_struct(d):
    return _fill(_abi.RayParams(), d)


def ssfr_struct(d):
    return _fill(_abi.SsfrParams(), d)


def _fill(s, d):
    for name, ctype in type(s)._fields_:
        if name not in d:
            continue
        v = d[name]
        if hasattr(ctype, "_length_"):
            arr = getattr(s, name)
            vals = list(np.asarray(v, dtype=np.float64).ravel())
            if len(vals) != ctype._length_:
                raise ValueError(f"{name}: {len(vals)} values, expected {ctype._length_}")
            for k, x in enumerate(vals):
                arr[k] = x
        elif ctype in (C.c_int32,):
            setattr(s, name, int(v))
        else:
            setattr(s, name, float(v))
    return s
