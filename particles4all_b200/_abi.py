"""ctypes mirror of the C structs and constants declared in include/p4a.h."""
import ctypes as C

P4A_OK, P4A_ERR_ARG, P4A_ERR_OOM, P4A_ERR_CUDA = 0, 1, 2, 3
P4A_ERR_TIMEOUT, P4A_ERR_CAPACITY, P4A_ERR_STATE, P4A_ERR_NODEV = 4, 5, 6, 7

SHAPES = {"sphere": 0, "torus": 1, "box": 2}

BUF = dict(
    pos=0, vel=1, pred=2, body=3, rest=4, density=5, lambda_=6, corr=7, normal=8,
    cellStart=9, bpos=10, bpsi=11, bcellStart=12, bodyCentre=13, bodyRef=14,
    bodyRot=15, bodyInfo=16, statsOut=17, smoothPos=18, aniso=19, meshField=20, meshNField=21,
    meshVerts=22,
)
# element dtype / components of each buffer (numpy dtype string, components)
BUF_LAYOUT = {
    0: ("f4", 4), 1: ("f4", 4), 2: ("f4", 4), 3: ("u4", 4), 4: ("f4", 4),
    5: ("f4", 1), 6: ("f4", 1), 7: ("f4", 4), 8: ("f4", 4), 9: ("u4", 1),
    10: ("f4", 4), 11: ("f4", 1), 12: ("u4", 1), 13: ("f4", 4), 14: ("f4", 4),
    15: ("f4", 4), 16: ("f4", 4), 17: ("u4", 1), 18: ("f4", 4), 19: ("f4", 4),
    20: ("f4", 1), 21: ("f4", 1), 22: ("u4", 2),
}
A, B, LIVE = 0, 1, -1


class BodySpec(C.Structure):
    _fields_ = [("shape", C.c_int32), ("density", C.c_double), ("start_y", C.c_double)]


class Params(C.Structure):
    _fields_ = [
        ("spacing", C.c_double), ("rest_density", C.c_double), ("gravity", C.c_double),
        ("substeps", C.c_int32), ("iterations", C.c_int32),
        ("cfm_epsilon_rel", C.c_double), ("s_corr_k", C.c_double), ("s_corr_dq", C.c_double),
        ("xsph_c", C.c_double), ("omega", C.c_double), ("sor_average", C.c_int32),
        ("surface_tension_k", C.c_double), ("target_particle_count", C.c_int32),
        ("box", C.c_double * 3), ("n_bodies", C.c_int32), ("bodies", C.POINTER(BodySpec)),
        ("body_size", C.c_double), ("no_boundary", C.c_int32), ("pour", C.c_int32),
        ("cfm_epsilon_abs", C.c_double),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("pos", C.c_void_p), ("vel", C.c_void_p), ("phase", C.c_void_p),
        ("rest", C.c_void_p), ("n_bodies", C.c_int32), ("body_density", C.c_void_p),
        ("body_centre", C.c_void_p), ("mass", C.c_double), ("denom_rest", C.c_double),
        ("pour_budget", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("n_fluid", C.c_int32), ("n_body_parts", C.c_int32),
        ("n_bodies", C.c_int32), ("n_boundary", C.c_int32), ("cap", C.c_int32),
        ("pour_budget", C.c_int32), ("grid_dim", C.c_int32 * 3), ("n_cells", C.c_int32),
        ("parity", C.c_int32), ("pred_parity", C.c_int32), ("gen", C.c_int32),
        ("last_substeps", C.c_int32), ("h", C.c_double), ("mass", C.c_double),
        ("denom_rest", C.c_double), ("sim_time", C.c_double), ("last_advanced", C.c_double),
        ("time_bank", C.c_double), ("body_scale", C.c_double), ("cov_scale", C.c_double),
        ("held_body", C.c_int32), ("aniso_gen", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("avg_rho", C.c_double), ("max_rho", C.c_double), ("max_speed", C.c_double),
        ("ke", C.c_double), ("raw", C.c_uint32 * 4), ("valid", C.c_int32),
    ]


class AnisoParams(C.Structure):
    _fields_ = [
        ("ratio", C.c_double), ("ks", C.c_double), ("stretch", C.c_double),
        ("lonely", C.c_double), ("min_neighbours", C.c_int32), ("lambda_", C.c_double),
        ("radius_scale", C.c_double), ("min_extent", C.c_double),
    ]


class MeshParams(C.Structure):
    _fields_ = [("resolution", C.c_int32), ("iso", C.c_double), ("field_passes", C.c_int32),
                ("normal_passes", C.c_int32), ("max_triangles", C.c_int64), ("blur_axes", C.c_int32)]


class MeshInfo(C.Structure):
    _fields_ = [("vert_dim", C.c_int32 * 3), ("origin", C.c_double * 3), ("voxel", C.c_double),
                ("triangles", C.c_int64), ("mesh_gen", C.c_int32)]


class SsfrParams(C.Structure):
    _fields_ = [
        ("view", C.c_float * 16), ("proj", C.c_float * 16), ("inv_view_proj", C.c_float * 16),
        ("inv_view", C.c_float * 16), ("eye", C.c_float * 3), ("width", C.c_int32), ("height", C.c_int32),
        ("render_scale", C.c_double), ("splat_radius", C.c_double), ("thickness_radius", C.c_double),
        ("thickness_scale", C.c_double), ("thickness_filter_size", C.c_int32), ("thickness_half_res", C.c_int32),
        ("filter", C.c_int32), ("filter_iterations", C.c_int32), ("cleanup_pass", C.c_int32),
        ("cleanup_radius", C.c_int32), ("filter_max_radius", C.c_int32), ("depth_cull_neighbours", C.c_int32),
        ("filter_sigma", C.c_double), ("narrow_delta", C.c_double), ("narrow_mu", C.c_double),
        ("bilateral_range", C.c_double), ("ior", C.c_double), ("absorption", C.c_double),
        ("transmit", C.c_double * 3), ("roughness", C.c_double), ("sun_intensity", C.c_double),
        ("sun_elevation", C.c_double), ("sun_azimuth", C.c_double), ("exposure", C.c_double),
        ("ground_reflection", C.c_double), ("floor_plane", C.c_int32), ("debug", C.c_int32),
        ("env_intensity", C.c_double), ("env_yaw", C.c_double),
    ]


class SsfrInfo(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("map_w", C.c_int32), ("map_h", C.c_int32),
                ("thick_w", C.c_int32), ("thick_h", C.c_int32), ("ssfr_gen", C.c_int32)]


SSFR_BUF = {"eyeZ": 0, "rawZ": 1, "thick": 2, "image": 3, "bodyT": 4}


class RayParams(C.Structure):
    _fields_ = [
        ("proj", C.c_float * 16), ("inv_view_proj", C.c_float * 16), ("inv_view", C.c_float * 16),
        ("eye", C.c_float * 3), ("width", C.c_int32), ("height", C.c_int32), ("iso", C.c_double),
        ("ior", C.c_double), ("absorption", C.c_double), ("transmit", C.c_double * 3),
        ("thickness_steps", C.c_int32), ("floor_plane", C.c_int32), ("ground_reflection", C.c_double),
        ("skin_width", C.c_double), ("roughness", C.c_double), ("sun_intensity", C.c_double),
        ("sun_elevation", C.c_double), ("sun_azimuth", C.c_double), ("exposure", C.c_double),
        ("debug", C.c_int32), ("use_surface", C.c_int32), ("view", C.c_float * 16),
        ("env_intensity", C.c_double), ("env_yaw", C.c_double),
    ]


class Grid(C.Structure):
    _fields_ = [("box_min", C.c_float * 3), ("h", C.c_float), ("dim", C.c_int32 * 3)]


class Hose(C.Structure):
    _fields_ = [("nozzle", C.c_float * 3), ("spacing", C.c_float), ("jitter", C.c_float), ("speed", C.c_float),
                ("per_step", C.c_int32), ("seed", C.c_uint32), ("count", C.c_int32)]


class SceneCounts(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("n_fluid", C.c_int32), ("n_body", C.c_int32),
        ("n_bodies", C.c_int32), ("n_boundary", C.c_int32), ("mass", C.c_double),
        ("denom_rest", C.c_double), ("h", C.c_double),
    ]


class PhaseTime(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("ms", C.c_double), ("launches", C.c_int64)]


class BatchConfig(C.Structure):
    _fields_ = [("max_particles", C.c_int64), ("max_cells", C.c_int64), ("max_boundary", C.c_int64),
                ("max_scenes", C.c_int32), ("max_bodies", C.c_int32), ("max_body_parts", C.c_int64)]


class BatchUsage(C.Structure):
    _fields_ = [("free_particles", C.c_int64), ("free_cells", C.c_int64), ("free_boundary", C.c_int64),
                ("free_body_parts", C.c_int64), ("free_scenes", C.c_int32), ("free_bodies", C.c_int32),
                ("live_scenes", C.c_int32), ("device_bytes", C.c_int64)]


class BatchIO(C.Structure):
    _fields_ = [("scene_id", C.c_int32), ("pos_in", C.c_void_p), ("vel_in", C.c_void_p),
                ("pos_out", C.c_void_p), ("vel_out", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("arenas", BatchConfig), ("builder_threads", C.c_int32), ("max_frames_in_flight", C.c_int32),
                ("admit_timeout", C.c_double), ("max_pending_creates", C.c_int32), ("use_graphs", C.c_int32),
                ("plain", C.c_int32), ("upload_bytes", C.c_int64), ("readback_bytes", C.c_int64),
                ("frame_lanes", C.c_int32), ("lane_min_particles", C.c_int64)]


REQ_CREATE, REQ_STEP, REQ_DESTROY = 1, 2, 3
REQ_NAMES = {1: "create", 2: "step", 3: "destroy"}


class Completion(C.Structure):
    _fields_ = [("request", C.c_int64), ("kind", C.c_int32), ("scene", C.c_int32), ("status", C.c_int32),
                ("substeps", C.c_int32), ("particles", C.c_int64), ("submitted", C.c_double),
                ("started", C.c_double), ("finished", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("creates", C.c_int64), ("admitted", C.c_int64), ("rejected", C.c_int64),
                ("destroyed", C.c_int64), ("steps", C.c_int64), ("frames", C.c_int64),
                ("live_scenes", C.c_int32), ("queued_creates", C.c_int32), ("max_queued_creates", C.c_int32),
                ("building", C.c_int32), ("particle_substeps", C.c_double), ("step_p50_ms", C.c_double),
                ("step_p99_ms", C.c_double), ("step_mean_ms", C.c_double), ("step_max_ms", C.c_double),
                ("admit_p50_ms", C.c_double), ("admit_p99_ms", C.c_double), ("mean_frame_scenes", C.c_double),
                ("gpu_seconds", C.c_double), ("first_submit", C.c_double), ("last_finish", C.c_double),
                ("kernel_launches", C.c_int64)]


def info_dict(info):
    d = {k: getattr(info, k) for k, _ in Info._fields_}
    d["grid_dim"] = list(info.grid_dim)
    return d
