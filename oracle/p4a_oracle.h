/*
 * p4a_oracle.h — CPU oracle for the Particles4All simulation step.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE. Only the tests, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this library, and only as what the
 * product's results are compared against or as the timed CPU baseline. The
 * product path (libp4a.so) never calls it.
 *
 * PARITY UNPINNED: the reference (a browser WebGPU demo, JS + WGSL) cannot be
 * executed in this environment (no JS runtime, no WebGPU/graphics stack) and
 * ships no tests, golden vectors or fixtures. This oracle is a restatement of
 * the reference's passes in their exact schedule; it is checked against
 * known-answer cases derived by hand from the reference source and against the
 * reference's own in-app verify checks (src/main.js:853-937), not against
 * reference outputs.
 *
 * Arithmetic contract (shared with the CUDA kernels, which must match it bit
 * for bit): float32 everywhere the reference's WGSL is f32; float64 where the
 * reference's JS is (scene setup, time bank, uniform packing). No contraction
 * except explicit fused multiply-adds in exactly two forms:
 *   dot3(a,b) = fma(a.z,b.z, fma(a.y,b.y, a.x*b.x))
 *   acc += s*v   ->  acc = fma(s, v, acc)   (only where a pass accumulates)
 * Cube roots use a fixed 5-step Newton iteration (cbrt_newton). Sorting is
 * stable (ties by pre-sort index), which is one of the orders the reference's
 * atomic scatter can produce (src/wgsl.js:436).
 */
#ifndef P4A_ORACLE_H
#define P4A_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#include "../include/p4a.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

orc_sim* orc_create(void);
void orc_destroy(orc_sim* s);
void orc_set_threads(int threads);
int orc_get_threads(void);

/* scene.js restatement: buildScene(params) (src/scene.js:159-315). */
int orc_build_scene(const p4a_params* p, p4a_scene_counts* counts, float* pos, float* vel,
                    float* rest, uint32_t* phase, double* body_centre, double* body_density);
/* boundaryParticles(p, d, h) (src/scene.js:76-135): pts float3[*count], psi float[*count]. */
int orc_boundary(const p4a_params* p, double d, double h, int32_t* count, double* pts,
                 float* psi);

/* Sim.reset(params) / reset on an explicit scene (src/sim.js:66-221). */
int orc_reset(orc_sim* s, const p4a_params* p);
int orc_reset_scene(orc_sim* s, const p4a_params* p, const p4a_scene_desc* sc);
/* Sim.step(frameDt) (src/sim.js:415-656). */
int orc_step(orc_sim* s, double frame_dt, int32_t* substeps_out);
int orc_append_fluid(orc_sim* s, const float* pos3, const float* vel3, int32_t count,
                     int32_t* added);
int orc_apply_ray_impulse(orc_sim* s, const double origin[3], const double dir[3],
                          const double impulse[3], double radius, double speed_limit);
int orc_hold_body(orc_sim* s, int32_t body_1based, const double target[3], double rate,
                  double limit);
int orc_release_body(orc_sim* s);
int orc_resize_box(orc_sim* s, const double box[3]);
int orc_aniso(orc_sim* s, const p4a_aniso_params* ap);
/* SurfaceMesh.configure + generate (src/mesh.js:99-352): triangles in voxel order. */
int orc_mesh(orc_sim* s, const p4a_mesh_params* mp, int64_t* triangles);
/* FluidSSFR.render (src/ssfr.js:173-356) on the anisotropic pass's output. */
int orc_ssfr(orc_sim* s, const p4a_ssfr_params* sp, const float* bodies, int32_t body_count);
int orc_ssfr_buffer(orc_sim* s, int32_t which, void** ptr, size_t* bytes);
/* RayMarch.draw (src/ray.js:30-97) on the density field of the last orc_mesh. */
int orc_ray(orc_sim* s, const p4a_ray_params* rp, const float* bodies, int32_t body_count);
int orc_ray_image(orc_sim* s, void** ptr, size_t* bytes);
int orc_set_environment(orc_sim* s, const float* rgb, int32_t width, int32_t height);
int orc_environment(orc_sim* s, const void** ptr, int32_t* size);
/* The render passes' exp and log (Cody-Waite + Taylor; atanh series). */
float orc_expf(float x);
float orc_logf(float x);
int orc_get_info(const orc_sim* s, p4a_info* out);
int orc_stats(const orc_sim* s, p4a_stats* out);
/* Host pointer + bytes of a buffer (same ids / which as p4a_buffer). */
int orc_buffer(orc_sim* s, int32_t id, int32_t which, void** ptr, size_t* bytes);

/* predict + grid pass on host arrays (the operator p4a_grid_sort restates). */
int orc_grid_sort(const p4a_grid* grid, int32_t n, float dt, float gravity, const float* pos,
                  const float* vel, const uint32_t* body, const float* rest, float* pos_out,
                  float* vel_out, float* pred_out, uint32_t* body_out, float* rest_out,
                  uint32_t* cell_start, uint32_t* slot_out);

/* The cube root used by the rigid-body resolve (fixed Newton iteration). */
float orc_cbrt_newton(float x);

#ifdef __cplusplus
}
#endif
#endif
