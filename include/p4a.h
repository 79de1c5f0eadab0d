/*
 * p4a.h — C ABI of the B200-native Particles4All simulation step.
 *
 * This is the drop-in boundary for the reference's `class Sim` (src/sim.js:9-814):
 * scene setup (`reset`), the substep loop (`step`), the interactive calls
 * (`appendFluid`, `applyRayImpulse`, `holdBody`, `releaseBody`, `resizeBox`) and
 * the device buffers the renderers read (`buf.*`, `livePos/liveVel/liveBody`).
 * The anisotropic-kernel pass that src/mesh.js:207-261 dispatches on the
 * simulation's buffers is exposed as p4a_aniso().
 *
 * Conventions
 *  - Every call returns an int status (P4A_OK == 0). The reference has no
 *    exceptions (device errors are asynchronous, src/main.js:217); here the
 *    last error text of a handle is available from p4a_last_error().
 *  - Plain pointers and sizes only. "device pointer" means CUDA global memory on
 *    the handle's device; "host pointer" means ordinary (pageable or pinned)
 *    host memory.
 *  - A handle owns all its device memory. Pointers returned by p4a_buffer()
 *    stay valid until the next p4a_reset / p4a_reset_scene / p4a_resize_box /
 *    p4a_append_fluid beyond capacity / p4a_destroy; `gen` in p4a_info
 *    increments whenever that happens (src/sim.js:73, 740).
 *  - Calls on one handle are not re-entrant. All device work of a handle is
 *    issued on one CUDA stream (p4a_set_stream), in call order.
 *  - Particle arrays are float4 / uint4 per particle, in cell-sorted order,
 *    ping-ponged between an A and a B copy selected by `parity`, exactly as
 *    the reference lays them out (src/sim.js:98-101, 811-813).
 */
#ifndef P4A_H
#define P4A_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P4A_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
  P4A_OK = 0,
  P4A_ERR_ARG = 1,       /* invalid argument                                   */
  P4A_ERR_OOM = 2,       /* device or pinned host allocation failed            */
  P4A_ERR_CUDA = 3,      /* a CUDA runtime call failed                         */
  P4A_ERR_TIMEOUT = 4,   /* a bounded device-side wait gave up                 */
  P4A_ERR_CAPACITY = 5,  /* a size is beyond the handle's or entry's capacity  */
  P4A_ERR_STATE = 6,     /* call not valid in the current state (e.g. no reset)*/
  P4A_ERR_NODEV = 7      /* no CUDA device / extension unavailable             */
};

/* ---- body shapes (src/scene.js:137-157) -------------------------------- */
enum { P4A_SHAPE_SPHERE = 0, P4A_SHAPE_TORUS = 1, P4A_SHAPE_BOX = 2 };

/* One entry of params.bodies: "shape:density:startY" (src/scene.js:167-171). */
typedef struct p4a_body_spec {
  int32_t shape;     /* P4A_SHAPE_*                                            */
  double density;    /* body density / fluid density, default 0.5              */
  double start_y;    /* centre height as a fraction of box[1], default 0.75   */
} p4a_body_spec;

/*
 * Scene and solver parameters: the reference's `params` object
 * (defaultParams, src/scene.js:11-39, plus the keys main.js sets:
 * noBoundary src/main.js:380, pour src/sim.js:94). JS numbers are doubles, so
 * the real-valued fields are double; the library rounds them to float where
 * the reference's uniform upload does (src/sim.js:371-413).
 */
typedef struct p4a_params {
  double spacing;                /* d, default 0.02                                 */
  double rest_density;           /* rho0, default 1000                              */
  double gravity;                /* default 9.81                                    */
  int32_t substeps;              /* default 4                                       */
  int32_t iterations;            /* Jacobi iterations k, default 4                  */
  double cfm_epsilon_rel;        /* default 0.01 (cfmEps = rel * denomRest)         */
  double s_corr_k;               /* default 0.1                                     */
  double s_corr_dq;              /* default 0.3                                     */
  double xsph_c;                 /* default 0.05                                    */
  double omega;                  /* default 1.0                                     */
  int32_t sor_average;           /* default 0                                       */
  double surface_tension_k;      /* default 0 (tension off)                         */
  int32_t target_particle_count; /* default 60000                                   */
  double box[3];                 /* default {1.5, 1.5, 1.0}                         */
  int32_t n_bodies;              /* entries used in `bodies`                        */
  const p4a_body_spec* bodies;   /* may be NULL when n_bodies == 0                  */
  double body_size;              /* 0 = 0.12 * min(box)                             */
  int32_t no_boundary;           /* 1 = skip the boundary samples in the solver     */
  int32_t pour;                  /* 1 = reserve capacity nFluid for appendFluid     */
  /* Extension, no counterpart in the reference: when > 0 it replaces
   * cfm_epsilon_rel * denomRest as the absolute CFM epsilon.                 */
  double cfm_epsilon_abs;
} p4a_params;

/*
 * An explicit initial scene (what buildScene returns, src/scene.js:313-314),
 * for scenes that are not the reference's own fluid block + bodies. Arrays are
 * HOST pointers. phase[4*i] is the 1-based body id (0 = fluid); bodies must
 * have at least one particle each. When mass <= 0 the mass is calibrated from
 * the fluid particles as src/scene.js:277-288 does; when denom_rest <= 0 it is
 * computed as src/scene.js:289-311 does.
 */
typedef struct p4a_scene_desc {
  int32_t n;                 /* particles                                          */
  const float* pos;          /* float4[n]                                          */
  const float* vel;          /* float4[n], may be NULL (zero)                      */
  const uint32_t* phase;     /* uint4[n],  may be NULL (all fluid)                 */
  const float* rest;         /* float4[n], may be NULL (zero)                      */
  int32_t n_bodies;
  const double* body_density;  /* [n_bodies]                                       */
  const double* body_centre;   /* [3*n_bodies] initial centre of mass              */
  double mass;
  double denom_rest;
  int32_t pour_budget;       /* extra capacity reserved for p4a_append_fluid       */
} p4a_scene_desc;

/* Read-only fields the reference's callers read from a Sim (src/sim.js). */
typedef struct p4a_info {
  int32_t n, n_fluid, n_body_parts, n_bodies, n_boundary;
  int32_t cap, pour_budget;
  int32_t grid_dim[3];
  int32_t n_cells;
  int32_t parity, pred_parity;
  int32_t gen;
  int32_t last_substeps;
  double h, mass, denom_rest;
  double sim_time, last_advanced, time_bank;
  double body_scale, cov_scale;
  int32_t held_body;
  int32_t aniso_gen;
} p4a_info;

/* Sim.stats after the fixed-point readback (src/sim.js:619-633). */
typedef struct p4a_stats {
  double avg_rho, max_rho, max_speed, ke;
  uint32_t raw[4];    /* statsOut[0..3] as the device wrote them */
  int32_t valid;      /* 0 until the first step completed         */
} p4a_stats;

/* Anisotropic kernel parameters (SurfaceMesh fields, src/mesh.js:81-89, and
 * the uniform packing at src/mesh.js:221-242). */
typedef struct p4a_aniso_params {
  double ratio;           /* anisoRatio  k_r, default 4.0          */
  double ks;              /* anisoKs,         default 1.0          */
  double stretch;         /* anisoStretch,    default 2.0          */
  double lonely;          /* anisoLonely  k_n,default 1.0          */
  int32_t min_neighbours; /* anisoMinNeighbours N_eps, default 25  */
  double lambda;          /* anisoLambda,     default 0.9          */
  double radius_scale;    /* anisoRadiusScale,default 2.0          */
  double min_extent;      /* F[16]: 1.25*voxel/h, or 0             */
} p4a_aniso_params;

/* Buffer ids for p4a_buffer / p4a_read / p4a_write (src/sim.js:98-161). */
enum {
  P4A_BUF_POS = 0,        /* float4[cap], A/B      */
  P4A_BUF_VEL = 1,        /* float4[cap], A/B      */
  P4A_BUF_PRED = 2,       /* float4[cap], A/B      */
  P4A_BUF_BODY = 3,       /* uint4[cap],  A/B      */
  P4A_BUF_REST = 4,       /* float4[cap], A/B      */
  P4A_BUF_DENSITY = 5,    /* float[cap]            */
  P4A_BUF_LAMBDA = 6,     /* float[cap]            */
  P4A_BUF_CORR = 7,       /* float4[cap]           */
  P4A_BUF_NORMAL = 8,     /* float4[cap]           */
  P4A_BUF_CELL_START = 9, /* uint32[nCells+2]      */
  P4A_BUF_BPOS = 10,      /* float4[max(1,nb)]     */
  P4A_BUF_BPSI = 11,      /* float[max(1,nb)]      */
  P4A_BUF_BCELL_START = 12, /* uint32[nCells+2]    */
  P4A_BUF_BODY_CENTRE = 13, /* float4[max(1,B)]    */
  P4A_BUF_BODY_REF = 14,    /* float4[max(1,B)]    */
  P4A_BUF_BODY_ROT = 15,    /* float4[3*max(1,B)], row-major rows */
  P4A_BUF_BODY_INFO = 16,   /* float4[max(1,B)], .x = 1/density   */
  P4A_BUF_STATS_OUT = 17,   /* uint32[8]           */
  P4A_BUF_SMOOTH_POS = 18,  /* float4[n] (aniso)   */
  P4A_BUF_ANISO_G = 19,     /* float4[2n] (aniso)  */
  P4A_BUF_MESH_FIELD = 20,  /* float[vertDim xyz] (mesh): density field   */
  P4A_BUF_MESH_NFIELD = 21, /* float[vertDim xyz] (mesh): normal field    */
  P4A_BUF_MESH_VERTS = 22,  /* uint2[3 * stored triangles] (mesh)         */
  P4A_BUF_COUNT = 23
};
/* `which` selector for A/B buffers. */
enum { P4A_A = 0, P4A_B = 1, P4A_LIVE = -1 };

/* ---- library ----------------------------------------------------------- */
int p4a_abi_version(void);
const char* p4a_status_string(int status);
/* defaultParams(preset) (src/scene.js:11-39). `preset` is "small", "medium",
 * "large" or "extreme" (src/scene.js:3-9); NULL or unknown = "small". The
 * bodies array points at static storage of the library. */
int p4a_default_params(const char* preset, p4a_params* out);
/* Number of devices and whether the sm_100a kernels can run on `device`. */
int p4a_device_check(int device);

/* ---- lifetime (new Sim(device), src/sim.js:10-18) ----------------------- */
typedef struct p4a_sim p4a_sim;
int p4a_create(int device, p4a_sim** out);
int p4a_destroy(p4a_sim* sim);
const char* p4a_last_error(const p4a_sim* sim);
/* Use `stream` (a cudaStream_t, NULL = the handle's own stream) for all work. */
int p4a_set_stream(p4a_sim* sim, void* stream);
int p4a_synchronize(p4a_sim* sim);

/* ---- Sim.reset(params) (src/sim.js:66-221) ------------------------------ */
int p4a_reset(p4a_sim* sim, const p4a_params* params);
/* reset() on an explicit scene instead of buildScene(params); the remaining
 * steps of src/sim.js:75-221 (grid, boundary, buffers, scales, prime) are the
 * same. params.spacing, rest_density, box and solver fields are used. */
int p4a_reset_scene(p4a_sim* sim, const p4a_params* params, const p4a_scene_desc* scene);

/* ---- Sim.step(frameDt) (src/sim.js:415-656) ----------------------------- */
int p4a_step(p4a_sim* sim, double frame_dt, int32_t* substeps_out);

/* ---- interactive API --------------------------------------------------- */
/* Sim.appendFluid(pos, vel) (src/sim.js:774-809): pos3/vel3 are HOST float3
 * arrays of `count` entries; appends min(count, cap - n), stored in *added. */
int p4a_append_fluid(p4a_sim* sim, const float* pos3, const float* vel3, int32_t count,
                     int32_t* added);
/* The layered hose of pourStep (src/main.js:106-160) at a fixed rate, emitted on
 * the device: the first min(count, cap - n) slots of one layer appended at index n
 * with the appendFluid semantics (src/sim.js:774-809: live pos/vel and the pred
 * parity written, density rho0, zero lambda/corr/normal/body/rest), computed by a
 * kernel from its emission index, so nothing crosses from the host and the call
 * does not wait. Layer slot q: row iy = q / k, column iz = q % k with
 * k = ceil(sqrt(per_step)); position nozzle + ((0, iy - c, iz - c) * spacing) + j,
 * c = (k - 1) / 2, velocity (speed, 0, 0); j per axis uniform in
 * [-jitter, jitter) from Philox4x32-10 keyed by (seed, emission, q). The host
 * restatement is particles4all_b200.configs.Hose. */
typedef struct p4a_hose {
  float nozzle[3];
  float spacing;
  float jitter;
  float speed;
  int32_t per_step;  /* slots of a full layer; sets the lattice side k          */
  uint32_t seed;
  int32_t count;     /* slots of this emission, 0..per_step (the first ones of  */
                     /* the layer); -1 = per_step. Capped by cap - n as well.   */
} p4a_hose;
int p4a_hose_emit(p4a_sim* sim, const p4a_hose* hose, int64_t emission, int32_t* added);
/* Sim.applyRayImpulse(origin, dir, impulse, radius, speedLimit) (src/sim.js:658-676). */
int p4a_apply_ray_impulse(p4a_sim* sim, const double origin[3], const double dir[3],
                          const double impulse[3], double radius, double speed_limit);
/* Sim.holdBody(body1Based, target, rate, limit) / releaseBody (src/sim.js:678-685). */
int p4a_hold_body(p4a_sim* sim, int32_t body_1based, const double target[3], double rate,
                  double limit);
int p4a_release_body(p4a_sim* sim);
/* Sim.resizeBox(newBox) (src/sim.js:687-772). */
int p4a_resize_box(p4a_sim* sim, const double box[3]);

/* ---- fields and buffers ------------------------------------------------ */
int p4a_get_info(const p4a_sim* sim, p4a_info* out);
/* Device pointer and byte size of a buffer. `which` = P4A_A, P4A_B or
 * P4A_LIVE (the `parity` copy, as livePos/liveVel/liveBody, src/sim.js:811-813);
 * ignored for single buffers. */
int p4a_buffer(p4a_sim* sim, int32_t id, int32_t which, void** dptr, size_t* bytes);
/* Synchronous copies between a buffer and host memory (the reference's
 * copyBufferToBuffer + mapAsync readback, src/main.js:841-852). */
int p4a_read(p4a_sim* sim, int32_t id, int32_t which, void* host, size_t offset, size_t bytes);
int p4a_write(p4a_sim* sim, int32_t id, int32_t which, const void* host, size_t offset,
              size_t bytes);
/* Asynchronous readback (the reference's copyBufferToBuffer + mapAsync without
 * the wait, src/main.js:841-852): the copy into `host` (pinned memory, so that it
 * overlaps) runs on the sim's copy stream, after the work queued so far, while
 * the caller queues more. Later calls that change that buffer are ordered after
 * the copy on the device (no host wait); calls that free or reallocate buffers
 * (reset, resize_box, destroy, set_stream) wait for it. `host` holds the data once
 * p4a_read_wait (or p4a_synchronize) returns. */
int p4a_read_async(p4a_sim* sim, int32_t id, int32_t which, void* host, size_t offset, size_t bytes);
int p4a_read_wait(p4a_sim* sim);
/* Sim.stats (src/sim.js:619-633). wait = 0: latest completed readback, as the
 * reference's async mapAsync; wait = 1: block until the last step's stats. */
int p4a_get_stats(p4a_sim* sim, int32_t wait, p4a_stats* out);
/* Sim.bodyPose (src/sim.js:635-655): centre3[3*i], rot9[9*i] column-major. */
int p4a_body_pose(p4a_sim* sim, int32_t wait, float* centre3, float* rot9, int32_t max_bodies);

/* ---- anisotropic kernel (src/aniso_wgsl.js:3-158, src/mesh.js:207-261) -- */
/* Runs on the live pos and the current cellStart; results in
 * P4A_BUF_SMOOTH_POS (float4[n], .w = 0) and P4A_BUF_ANISO_G (float4[2n]:
 * (G00,G10,G20,G11), (G21,G22,det G,n)). */
int p4a_aniso(p4a_sim* sim, const p4a_aniso_params* params);
int p4a_default_aniso_params(p4a_aniso_params* out);

/* ---- GPU timing (the reference's GpuTimer, src/gputimer.js; phase marks
 * src/sim.js:460-599) --------------------------------------------------- */
/* With profiling on, every kernel the handle launches is bracketed by CUDA
 * events on its stream; p4a_profile_read synchronizes and returns, per kernel
 * name, the accumulated device milliseconds and launch count since the last
 * p4a_profile_reset. */
typedef struct p4a_phase_time {
  char name[24];
  double ms;
  int64_t launches;
} p4a_phase_time;
int p4a_profile_enable(p4a_sim* sim, int32_t on);
int p4a_profile_reset(p4a_sim* sim);
int p4a_profile_read(p4a_sim* sim, p4a_phase_time* out, int32_t max_entries, int32_t* count);
/* Extension, no counterpart in the reference: kernels launched by this
 * library in this process (all handles and operator entries). */
uint64_t p4a_kernel_launches(void);

/* ---- surface mesh (src/mesh.js:99-340, src/mesh_wgsl.js:23-238) --------- */
/*
 * SurfaceMesh.generate on the simulation's live buffers: a density field on the
 * vertices of a voxel grid over the box (configure([0,0,0], box, resolution)),
 * `field_passes` blur passes of it, a normal field of `normal_passes` further
 * passes, and marching tetrahedra (six per voxel) writing triangles as packed
 * vertices: uint2 {x | y << 16, z | octahedral normal << 16}, positions in
 * 1/65535 of the grid, 3 per triangle. Triangles are stored in voxel order (the
 * reference's order is its atomic counter's); at most max_triangles are stored and
 * *triangles (may be NULL; then the call does not wait) receives the total, as
 * the reference's counter does.
 * blur_axes = 0 blurs every pass along x: the reference writes each pass's axis into
 * one uniform with queue.writeBuffer while encoding, and the last write of a frame
 * (generate's final setParams, axis x) is what all of its passes read. 1 cycles
 * x, y, z per pass as the pass structure intends.
 */
typedef struct p4a_mesh_params {
  int32_t resolution;     /* voxels along the longest box side (meshRes), default 128   */
  double iso;             /* meshIso, default 0.4                                       */
  int32_t field_passes;   /* fieldSmooth, default 0                                     */
  int32_t normal_passes;  /* normalSmoothPasses, default 2                              */
  int64_t max_triangles;  /* maxTriangles, default 3,000,000                            */
  int32_t blur_axes;      /* 0 = as the reference executes (x), 1 = x, y, z             */
} p4a_mesh_params;
typedef struct p4a_mesh_info {
  int32_t vert_dim[3];
  double origin[3];
  double voxel;
  int64_t triangles;      /* total of the last p4a_mesh that was waited for             */
  int32_t mesh_gen;       /* increments when the mesh buffers are reallocated           */
} p4a_mesh_info;
int p4a_default_mesh_params(p4a_mesh_params* out);
int p4a_mesh(p4a_sim* s, const p4a_mesh_params* mp, int64_t* triangles);
int p4a_mesh_get_info(p4a_sim* s, p4a_mesh_info* out);

/* ---- environment map (src/env.js:149-242) ------------------------------- */
/*
 * Environment.load / clear: `rgb` is an equirectangular panorama, float RGB,
 * `height` rows of `width` pixels, top row first (a decoded .hdr or image; the
 * Python package's hdr.load_hdr decodes Radiance .hdr files). It must be 2:1
 * (width within 2 * height +- 2). The library resamples it on the host into a cube
 * map of face size min(2048, max(16, width / 4)), rgba16float, as the reference
 * does, and keeps it on the device; p4a_ssfr and p4a_ray then take the sky, the
 * floor's far colour and reflections from it (times env_intensity, turned by
 * env_yaw). rgb = NULL clears it. The reference's viewer also turns the floor plane
 * off when a panorama loads, unless it was set explicitly: set floor_plane in the
 * render parameters to match.
 */
int p4a_set_environment(p4a_sim* s, const float* rgb, int32_t width, int32_t height);
/* The cube map's face size (0 when none) and, when `host` is not NULL, its
 * 6 * size * size texels of 4 halves each (face, row, column order), `bytes` at most. */
int p4a_environment_read(p4a_sim* s, int32_t* face_size, void* host, size_t bytes);

/* ---- screen-space fluid rendering (src/ssfr.js:7-356) ------------------- */
/*
 * FluidSSFR.render on the simulation's live buffers into headless device images:
 * ellipsoid depth splats of the anisotropic pass's smoothPos / G (p4a_aniso must
 * have run on the current particles), additive thickness splats, a separable
 * Gaussian blur of the thickness, the depth filter passes, a body-depth trace,
 * and the composite (refraction with absorption, Fresnel reflection, GGX sun
 * highlight, sky / floor / rigid-body background, tone map) into an RGBA8 image
 * of width x height. Field names follow FluidSSFR's members; matrices are
 * column-major float[16] as the reference's Float32Array matrices (view, proj,
 * invViewProj, invView of src/render.js:203-258). `bodies` is the rigid-body
 * renderer's packed buffer (6 float4 per body: centre + shape code, half extents,
 * three rotation rows, colour; src/ssfr_composite_wgsl.js:67-84), or NULL with
 * body_count 0. With an environment map set (p4a_set_environment), hasEnvMap = 1.
 * Depth ties keep the lower particle index (the first drawn); the thickness is
 * summed in fixed point, so every buffer is the same bits on every run.
 */
typedef struct p4a_ssfr_params {
  float view[16], proj[16], inv_view_proj[16], inv_view[16];
  float eye[3];
  int32_t width, height;          /* target size in pixels                          */
  double render_scale;            /* renderScale, 1.0 (maps: round(width x scale)) */
  double splat_radius;            /* splatRadius, 1.0                              */
  double thickness_radius;        /* thicknessRadius, 0.62 (x spacing)             */
  double thickness_scale;         /* thicknessScale, 3.0                           */
  int32_t thickness_filter_size;  /* thicknessFilterSize, 8 (<= 128)               */
  int32_t thickness_half_res;     /* thicknessHalfRes, 1                           */
  int32_t filter;                 /* 0 Gaussian, 1 bilateral, 2 narrow range (2)   */
  int32_t filter_iterations;      /* filterIterations, 2                           */
  int32_t cleanup_pass;           /* cleanupPass, 1                                */
  int32_t cleanup_radius;         /* cleanupRadius, 4                              */
  int32_t filter_max_radius;      /* filterMaxRadius, 32                           */
  int32_t depth_cull_neighbours;  /* depthCullNeighbours, 0                        */
  double filter_sigma;            /* filterSigma, 0.7                              */
  double narrow_delta;            /* narrowDelta, 10.0                             */
  double narrow_mu;               /* narrowMu, 1.0                                 */
  double bilateral_range;         /* bilateralRange, 2.0                           */
  double ior;                     /* 1.333                                         */
  double absorption;              /* 1.0                                           */
  double transmit[3];             /* 0.35, 0.62, 0.78                              */
  double roughness;               /* 0.055                                         */
  double sun_intensity;           /* 3.0                                           */
  double sun_elevation;           /* 38 degrees                                    */
  double sun_azimuth;             /* 40 degrees                                    */
  double exposure;                /* 1.0                                           */
  double ground_reflection;       /* 0.0                                           */
  int32_t floor_plane;            /* 1                                             */
  int32_t debug;                  /* 0 shaded, 1 normals, 2 depth, 3 thickness,
                                     4 unfiltered depth, 5 body depth              */
  double env_intensity;           /* environment map intensity, 1.0 (env.intensity) */
  double env_yaw;                 /* environment map yaw in radians, 0 (env.yaw)   */
} p4a_ssfr_params;
typedef struct p4a_ssfr_info {
  int32_t width, height;          /* image                                         */
  int32_t map_w, map_h;           /* depth maps (render scale)                     */
  int32_t thick_w, thick_h;       /* thickness map                                 */
  int32_t ssfr_gen;               /* increments when the buffers are reallocated   */
} p4a_ssfr_info;
enum { P4A_SSFR_EYEZ = 0, P4A_SSFR_RAWZ = 1, P4A_SSFR_THICK = 2, P4A_SSFR_IMAGE = 3, P4A_SSFR_BODYT = 4 };
int p4a_default_ssfr_params(p4a_ssfr_params* out);
int p4a_ssfr(p4a_sim* s, const p4a_ssfr_params* sp, const float* bodies, int32_t body_count);
int p4a_ssfr_get_info(p4a_sim* s, p4a_ssfr_info* out);
/* Device pointer and size of an SSFR buffer (float maps; the image is RGBA8). */
int p4a_ssfr_buffer(p4a_sim* s, int32_t which, void** dptr, size_t* bytes);
/* Copies the first `bytes` of an SSFR buffer to host memory (waits for the stream). */
int p4a_ssfr_read(p4a_sim* s, int32_t which, void* host, size_t bytes);

/* ---- ray-marched surface (src/ray.js:30-97, src/ray_wgsl.js:1-549) ------- */
/*
 * RayMarch.draw on the last p4a_mesh (call p4a_mesh first): the surface is the
 * mesh's triangles drawn into eye-depth and normal maps (SurfaceMesh.drawSurface,
 * use_surface = 1, the reference's default), or the iso crossing of the trilinear
 * density field found by walking the voxel grid (cubic fit, bracketed regula falsi;
 * use_surface = 0). Either way it is shaded with Fresnel reflection, absorption
 * along the refracted ray's optical depth through the field, the GGX sun
 * highlight, sky / floor and rigid bodies (`bodies` as for p4a_ssfr). The image is
 * RGBA8, width x height. With an environment map set, hasEnvMap = 1.
 */
typedef struct p4a_ray_params {
  float proj[16], inv_view_proj[16], inv_view[16];
  float eye[3];
  int32_t width, height;
  double iso;                 /* the field's iso level (meshIso), 0.4             */
  double ior;                 /* 1.333                                           */
  double absorption;          /* 1.0                                             */
  double transmit[3];         /* 0.35, 0.62, 0.78                                */
  int32_t thickness_steps;    /* thicknessSteps, 48                              */
  int32_t floor_plane;        /* 1                                               */
  double ground_reflection;   /* 0.0                                             */
  double skin_width;          /* skinWidth, 0.05                                 */
  double roughness;           /* 0.055                                           */
  double sun_intensity;       /* 3.0                                             */
  double sun_elevation;       /* 38 degrees                                      */
  double sun_azimuth;         /* 40 degrees                                      */
  double exposure;            /* 1.0                                             */
  int32_t debug;              /* 0 shaded, 1 normals, 2 distance, 3 thickness,
                                 4 reflection side, 5 slope, 6 reflection        */
  int32_t use_surface;        /* raySurface: 1 (default) the mesh's triangles drawn
                                 into eye-depth and normal maps give the surface;
                                 0 the field is marched                          */
  float view[16];             /* view matrix, for the mesh surface pass          */
  double env_intensity;       /* environment map intensity, 1.0                  */
  double env_yaw;             /* environment map yaw in radians, 0               */
} p4a_ray_params;
int p4a_default_ray_params(p4a_ray_params* out);
int p4a_ray(p4a_sim* s, const p4a_ray_params* rp, const float* bodies, int32_t body_count);
/* The last p4a_ray image (RGBA8): device pointer, or a host copy (waits). */
int p4a_ray_buffer(p4a_sim* s, void** dptr, size_t* bytes, int32_t* width, int32_t* height);
int p4a_ray_read(p4a_sim* s, void* host, size_t bytes);

/* ---- batched multi-scene stepping -------------------------------------- */
/*
 * Extension, no counterpart in the reference (which steps one scene per Sim).
 * Many independent scenes live in shared device arenas and are stepped together:
 * every pass of a substep is ONE launch over all listed scenes, whose blocks pull
 * (scene, tile) work items; the cell-key sort is one counting sort over the
 * scenes' disjoint key ranges. Each scene keeps its own parameters, time bank,
 * parity, iteration count and tension setting, and its results are bit-identical
 * to stepping it alone with p4a_step.
 */
typedef struct p4a_batch p4a_batch;
typedef struct p4a_batch_config {
  int64_t max_particles;   /* particle arena: sum of scene capacities        */
  int64_t max_cells;       /* cell arena: sum of scene cells (+ tile padding)*/
  int64_t max_boundary;    /* boundary-sample arena                          */
  int32_t max_scenes;
  int32_t max_bodies;      /* body arena: sum over scenes of (bodies + 1)    */
  int64_t max_body_parts;  /* body-particle list arena                       */
} p4a_batch_config;
typedef struct p4a_batch_usage {
  int64_t free_particles, free_cells, free_boundary, free_body_parts;
  int32_t free_scenes, free_bodies;
  int32_t live_scenes;
  int64_t device_bytes;    /* bytes the batch holds on the device            */
} p4a_batch_usage;
int p4a_batch_create(int device, const p4a_batch_config* cfg, p4a_batch** out);
/* Device bytes p4a_batch_create would allocate for cfg (its arenas; the per-frame
 * work lists, a few bytes per work item, come on top). Needs no device. */
int p4a_batch_footprint(const p4a_batch_config* cfg, int64_t* bytes);
int p4a_batch_destroy(p4a_batch* b);
const char* p4a_batch_last_error(const p4a_batch* b);
int p4a_batch_set_stream(p4a_batch* b, void* stream);
/* Admit a scene (reset() of the reference on an explicit scene / on params).
 * P4A_ERR_CAPACITY when an arena has no room: nothing is allocated then. */
int p4a_batch_add_scene(p4a_batch* b, const p4a_params* params, const p4a_scene_desc* scene,
                        int32_t* scene_id);
int p4a_batch_add_preset(p4a_batch* b, const p4a_params* params, int32_t* scene_id);
int p4a_batch_remove_scene(p4a_batch* b, int32_t scene_id);
/* Advance each listed scene by frame_dt (its own time bank and substeps). */
int p4a_batch_step(p4a_batch* b, const int32_t* scene_ids, int32_t count, double frame_dt);
int p4a_batch_synchronize(p4a_batch* b);
int p4a_batch_usage_get(const p4a_batch* b, p4a_batch_usage* out);
/* Per-scene views, as p4a_get_info / p4a_read / p4a_get_stats (which = P4A_LIVE,
 * P4A_A or P4A_B; the stats wait for the scene's last step). */
int p4a_batch_scene_info(p4a_batch* b, int32_t scene_id, p4a_info* out);
int p4a_batch_read(p4a_batch* b, int32_t scene_id, int32_t id, int32_t which, void* host,
                   size_t offset, size_t bytes);
int p4a_batch_write(p4a_batch* b, int32_t scene_id, int32_t id, int32_t which, const void* host,
                    size_t offset, size_t bytes);
int p4a_batch_stats(p4a_batch* b, int32_t scene_id, p4a_stats* out);
/* Asynchronous per-scene copies on the batch's stream, ordered after the frames
 * queued before them and before the ones queued after; the host memory (pinned
 * for an asynchronous copy) stays in use until p4a_batch_synchronize. The
 * cellStart buffer is not available here (p4a_batch_read converts its arena
 * indices). */
int p4a_batch_read_async(p4a_batch* b, int32_t scene_id, int32_t id, int32_t which, void* host,
                         size_t offset, size_t bytes);
int p4a_batch_write_async(p4a_batch* b, int32_t scene_id, int32_t id, int32_t which,
                          const void* host, size_t offset, size_t bytes);
/* One frame of the listed scenes with host I/O overlapped: every non-NULL pos_in /
 * vel_in (n x float4, n = the scene's particle count) is written into the scene's
 * live buffer, the scenes are stepped by frame_dt, and every non-NULL pos_out /
 * vel_out receives the live buffer after the step. The results are those of
 * write_async, p4a_batch_step and read_async in that order, bit for bit; here the
 * scenes are stepped as `groups` consecutive frames of about equal particle counts
 * (0: with two or more frame lanes one group per 750 k particles, at most 8; with
 * one lane two from 3 M particles up, else one), with the host-to-device copies of later
 * groups and the device-to-host copies of earlier ones on two copy streams of
 * their own, so that they overlap the frames of the other groups; with frame lanes
 * (p4a_batch_set_lanes) group g runs on lane g mod lanes, at the same time as the
 * groups on the other lanes. The copies of the first group's inputs and the last group's
 * outputs stay exposed. The copies are ordered after all
 * work queued on the batch's stream before the call and before all work queued
 * after it; host memory (pinned, for overlap) stays in use until
 * p4a_batch_synchronize. No counterpart in the reference, which steps one scene
 * and hands its live buffers to the renderer on the device (livePos / liveVel,
 * src/sim.js:811-812). */
typedef struct p4a_batch_io {
  int32_t scene_id;
  const void* pos_in;
  const void* vel_in;
  void* pos_out;
  void* vel_out;
} p4a_batch_io;
int p4a_batch_step_io(p4a_batch* b, const p4a_batch_io* io, int32_t count, double frame_dt,
                      int32_t groups);
/* Capture each distinct frame schedule as a CUDA graph and replay it (default on). */
int p4a_batch_use_graphs(p4a_batch* b, int32_t on);
/* Frame lanes of p4a_batch_step and the serving loop: with lanes = L > 1 (1-4,
 * default 2) a frame of at least min_particles particles (default 1,000,000) over
 * two or more scenes runs as L parts of about equal particle counts at once, each on
 * a stream of its own (the batch's stream waits for all), so that one part's launch
 * tails overlap the others' work; lanes = 1 runs every frame whole. Scenes are
 * independent: every scene gets the same bits either way. Frames stay whole while
 * profiling is on. No counterpart in the reference. */
int p4a_batch_set_lanes(p4a_batch* b, int32_t lanes, int64_t min_particles);
/* Per-kernel timing of batched frames, as p4a_profile_* for a Sim (the
 * counterpart of the reference's GpuTimer phases, src/gputimer.js): with it on,
 * every launch of a frame is bracketed by events (event-record nodes inside a
 * replayed graph), and p4a_profile_read-style totals per kernel name ("lambda",
 * "delta", ...) accumulate since the last reset. */
int p4a_batch_profile_enable(p4a_batch* b, int32_t on);
int p4a_batch_profile_reset(p4a_batch* b);
int p4a_batch_profile_read(p4a_batch* b, p4a_phase_time* out, int32_t max_entries, int32_t* count);

/* ---- serving loop (no counterpart in the reference) --------------------- */
/*
 * A request loop over one batch (continuous batching). Clients on any thread
 * submit create, step and destroy requests; an engine thread builds created
 * scenes on host worker threads, admits them as scene slots and arena space
 * free up (admission by free device memory), and packs every live scene that
 * has a pending step into the next batched frame while the previous frame is
 * still running on the GPU. Scene state stays resident on the device between
 * requests. Each request ends in exactly one p4a_completion, read with
 * p4a_server_poll. A step may ask for the scene's live positions and/or
 * velocities (float4[n], cell-sorted, as p4a_read of P4A_BUF_POS/VEL); the
 * output buffers must stay valid until the step's completion has been polled.
 * Per scene, steps run in submission order, one per frame.
 * plain = 1 serves the same requests with one plain Sim per scene, stepped one
 * after another (the comparison for the batched form).
 */
typedef struct p4a_server p4a_server;
typedef struct p4a_server_config {
  p4a_batch_config arenas;     /* batch arena sizes (ignored by plain = 1)          */
  int32_t builder_threads;     /* host threads building scenes, default 4           */
  int32_t max_frames_in_flight;/* frames on the GPU ahead of completion, default 2  */
  double admit_timeout;        /* seconds a create may wait for room; 0 = forever   */
  int32_t max_pending_creates; /* creates waiting beyond this are rejected; 0 = no cap */
  int32_t use_graphs;          /* replay captured frames, default 1                 */
  int32_t plain;               /* 1 = plain per-scene stepping                      */
  int64_t upload_bytes;        /* pinned staging for scene uploads, default 1 GiB   */
  int64_t readback_bytes;      /* pinned staging for step readbacks, default 1 GiB  */
  int32_t frame_lanes;         /* p4a_batch_set_lanes of the batched frames, 1-4,   */
                               /* default 2 (0 = 1)                                  */
  int64_t lane_min_particles;  /* frames split from this size on, default 1,000,000 */
} p4a_server_config;
enum { P4A_REQ_CREATE = 1, P4A_REQ_STEP = 2, P4A_REQ_DESTROY = 3 };
typedef struct p4a_completion {
  int64_t request;     /* id returned by the submit call                           */
  int32_t kind;        /* P4A_REQ_*                                                */
  int32_t scene;       /* scene handle                                             */
  int32_t status;      /* P4A_OK; P4A_ERR_CAPACITY = create rejected (no room in  */
                       /* time) or readback staging too small; P4A_ERR_STATE =    */
                       /* scene gone or server stopping; P4A_ERR_CUDA            */
  int32_t substeps;    /* STEP: substeps run                                       */
  int64_t particles;   /* the scene's particle count                               */
  double submitted;    /* server clock (s) at submission                           */
  double started;      /* when its work was issued to the GPU                      */
  double finished;     /* when the engine saw it complete                          */
} p4a_completion;
typedef struct p4a_server_stats {
  int64_t creates, admitted, rejected, destroyed, steps, frames;
  int32_t live_scenes, queued_creates, max_queued_creates, building;
  double particle_substeps;    /* of completed steps                               */
  double step_p50_ms, step_p99_ms, step_mean_ms, step_max_ms;  /* submit -> finish  */
  double admit_p50_ms, admit_p99_ms;  /* create submit -> admitted                 */
  double mean_frame_scenes;    /* scenes per stepping frame                        */
  double gpu_seconds;          /* device time of all frames (CUDA events)          */
  double first_submit, last_finish;   /* server clock                              */
  int64_t kernel_launches;     /* frames' kernels (graph replays count each node)  */
} p4a_server_stats;
int p4a_server_default_config(p4a_server_config* cfg);
int p4a_server_create(int device, const p4a_server_config* cfg, p4a_server** out);
/* Stops the engine: work on the GPU finishes, queued requests complete with
 * P4A_ERR_STATE, and every completion not yet polled is dropped. */
int p4a_server_destroy(p4a_server* s);
const char* p4a_server_last_error(const p4a_server* s);
double p4a_server_clock(const p4a_server* s);
/* Create a scene from params (scene = NULL: the reference's buildScene) or from
 * an explicit scene (copied before the call returns). *scene is the handle
 * steps and destroys refer to; the create's completion says if it was admitted. */
int p4a_server_create_scene(p4a_server* s, const p4a_params* params, const p4a_scene_desc* scene,
                            int32_t* scene_id, int64_t* request);
int p4a_server_step(p4a_server* s, int32_t scene_id, double frame_dt, float* pos_out,
                    float* vel_out, size_t out_bytes, int64_t* request);
int p4a_server_destroy_scene(p4a_server* s, int32_t scene_id, int64_t* request);
/* Up to max completions; waits up to wait_seconds for the first one. */
int p4a_server_poll(p4a_server* s, p4a_completion* out, int32_t max, int32_t* count,
                    double wait_seconds);
int p4a_server_get_stats(p4a_server* s, p4a_server_stats* out);

/* ---- launch-shape tuning (no counterpart in the reference) -------------- */
/*
 * The neighbour kernels run in one of several launch shapes (threads per
 * block x minimum resident blocks per SM); the arithmetic per particle is the
 * same in every shape, so the choice changes speed only. A table per kernel
 * maps a launch's particle count (the scene's for plain steps, the frame's
 * total for batched ones) to a shape: the first bucket whose max_particles is
 * >= the count, else variant 0. The table is process-wide.
 */
enum { P4A_KERNEL_LAMBDA = 0, P4A_KERNEL_DELTA = 1, P4A_KERNEL_NORMALS = 2, P4A_KERNEL_ANISO = 3 };
/* The batched launches (p4a_batch_step) of lambda, delta and xsph+normals have
 * tables of their own, keyed by the frame's total particles; while one is empty
 * the batched launch uses its plain kernel's table. Same shapes as the plain
 * kernel (p4a_kernel_shapes). */
enum { P4A_KERNEL_LAMBDA_BATCHED = 4, P4A_KERNEL_DELTA_BATCHED = 5, P4A_KERNEL_NORMALS_BATCHED = 6 };
int p4a_kernel_shapes(int32_t kernel, int32_t* threads, int32_t* min_blocks, int32_t max,
                      int32_t* count);
int p4a_tune_set(int32_t kernel, int64_t max_particles, int32_t variant);
int p4a_tune_clear(int32_t kernel);   /* -1 = every kernel */
int p4a_tune_get(int32_t kernel, int64_t particles, int32_t* variant);

/* ---- operator entry: predict + grid pass as one call ------------------- */
/*
 * The predict pass and the 'grid' pass of Sim.step (src/wgsl.js:56-70,
 * 352-475; schedule src/sim.js:473-489) on caller-owned DEVICE buffers:
 * v = vel + dt*(0,-gravity,0), pred = pos + dt*v, then a counting sort of the
 * particles by cell key (cellIndex(cellOf(pred)), src/wgsl.js:43-49). The sort
 * is stable: particles of one cell keep their input order.
 *   pos, vel            float4[n] in
 *   body, rest          uint4/float4[n] in, may be NULL (then *_out ignored)
 *   pos_out ... rest_out  outputs in sorted order (vel_out = (v,0), pred_out = (pred,1))
 *   cell_start          uint32[n_cells+1] out: exclusive scan of cell counts, [n_cells] = n
 *   slot_out            uint32[n] out (may be NULL): sorted position of input i
 *   workspace           device scratch of p4a_grid_sort_workspace_size() bytes
 */
typedef struct p4a_grid {
  float box_min[3];
  float h;
  int32_t dim[3];
} p4a_grid;
size_t p4a_grid_sort_workspace_size(int32_t n, int32_t n_cells);
/*   status              uint32 in DEVICE memory, or NULL. The scan's lookback
 *                       waits on its predecessor tiles with a bounded spin; when
 *                       one gives up, the outputs are invalid (every access still
 *                       stays in bounds). With status != NULL the call returns once
 *                       the work is queued and the error word is copied into
 *                       *status on `stream` (0 = complete, nonzero = a wait gave
 *                       up); with status == NULL the call waits for `stream` and
 *                       returns P4A_ERR_TIMEOUT when a wait gave up.
 * Returns P4A_ERR_ARG for a NULL grid, n < 0, a dim < 1 or h <= 0, and
 * P4A_ERR_CAPACITY when dim[0]*dim[1]*dim[2] exceeds 2^31 - 1 or the workspace is
 * too small; these checks run before any device work. */
int p4a_grid_sort(const p4a_grid* grid, int32_t n, float dt, float gravity,
                  const float* pos, const float* vel, const uint32_t* body, const float* rest,
                  float* pos_out, float* vel_out, float* pred_out, uint32_t* body_out,
                  float* rest_out, uint32_t* cell_start, uint32_t* slot_out, void* workspace,
                  size_t workspace_bytes, uint32_t* status, void* stream);
/* Test hook for the two grid-sort operators only (p4a_grid_sort and
 * p4a_grid_sort_noalloc; the simulation's own steps are unaffected): the number
 * of polls before the scan's lookback gives up (0 = the default, about 2^22
 * polls, a quarter of a second), and, when skip_first_tile is 1, the scan's tile
 * tickets start at 1, so tile 0 is never scanned and tile 1 waits on a flag that
 * nothing sets until its limit runs out. Process-wide; restore with (0, 0). */
int p4a_test_scan_wait(uint32_t spin_limit, int32_t skip_first_tile);

/* ---- operator entry without allocation ---------------------------------- */
/*
 * No counterpart in the reference. The same operation as p4a_grid_sort for
 * callers that cannot allocate device memory: a host that owns every device
 * allocation through its own arena (a renderer or plugin host with a fixed
 * budget), or a real-time frame loop in which a cudaMalloc, which may synchronise
 * the device, would stall the frame. The caller still passes every input and
 * output buffer; the scratch comes from one fixed device array inside the
 * library (about 8.4 MB, held by every GPU that loads the library until exit).
 *   - n <= P4A_NOALLOC_MAX_PARTICLES and dim[0]*dim[1]*dim[2] <=
 *     P4A_NOALLOC_MAX_CELLS, else P4A_ERR_CAPACITY with no device work (each
 *     dim is checked before it is multiplied in, so huge dims cannot wrap).
 *   - `status` as for p4a_grid_sort: a device word that receives the scan's
 *     error word on `stream`, or NULL to wait and get P4A_ERR_TIMEOUT.
 *   - Allocates nothing. The first call on a device looks up the array's
 *     address (once per device); make that first call before any stream capture.
 *     The address is kept until the process exits: a cudaDeviceReset after the
 *     first call on that device is not supported.
 *   - The array is shared by all calls: the parts that must start at zero (the
 *     histogram and tile states the call's cell count uses, the ticket and the
 *     error word) are cleared on `stream` at the start of each call, and calls
 *     whose work overlaps on the GPU race on it.
 */
#define P4A_NOALLOC_MAX_PARTICLES 524288
#define P4A_NOALLOC_MAX_CELLS 524288
int p4a_grid_sort_noalloc(const p4a_grid* grid, int32_t n, float dt, float gravity,
                          const float* pos, const float* vel, const uint32_t* body,
                          const float* rest, float* pos_out, float* vel_out, float* pred_out,
                          uint32_t* body_out, float* rest_out, uint32_t* cell_start,
                          uint32_t* slot_out, uint32_t* status, void* stream);

/* ---- host-side scene builder (src/scene.js:159-315) --------------------- */
/* buildScene(params) into caller-provided host arrays; call once with NULL
 * arrays to get the counts. pos/vel/rest float4[n], phase uint4[n]. */
typedef struct p4a_scene_counts {
  int32_t n, n_fluid, n_body, n_bodies, n_boundary;
  double mass, denom_rest, h;
} p4a_scene_counts;
int p4a_build_scene(const p4a_params* params, p4a_scene_counts* counts, float* pos, float* vel,
                    float* rest, uint32_t* phase, double* body_centre, double* body_density);

#ifdef __cplusplus
}
#endif
#endif /* P4A_H */
