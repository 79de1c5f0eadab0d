// p4a_internal.h — device parameter block, buffer sets and kernel launchers shared
// by the CUDA translation units of libp4a.
//
// Arithmetic contract (identical to the CPU oracle, so that results match bit
// for bit): compiled with --fmad=false; the only fused multiply-adds are the
// explicit fmaf() calls in dot3() and in accumulations "acc += s*v"; division and
// square root are IEEE round-to-nearest; floats convert to ints with the
// saturating cvt forms (__float2int_rz / _rn, __float2uint_rz).
//
// Every pass runs in one of two forms with the same device code:
//   plain    one scene; the SimParams block is a kernel parameter and block b
//            handles the b-th tile of 256 particles (the reference's workgroup);
//   batched  many scenes in one launch; block b reads a (scene slot, item) pair
//            from a work list and loads that scene's SimParams into shared memory.
// Scenes of a batch live side by side in shared arenas: particle range
// [pOff, pOff + cap), cell range [cOff, cOff + nCells + 2), body range
// [bOff, bOff + nBodies + 1). Cell keys carry cOff, so one counting sort orders all
// scenes at once, and cellStart entries are arena particle indices.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/p4a.h"

namespace p4a {

// The reference's 192-byte uniform (src/wgsl.js:4-40), float32/int32 fields in
// the reference's order, followed by the scene's place in the arenas and the
// per-substep schedule values the passes need.
struct SimParams {
  float boxMin[3]; float dt;
  float boxMax[3]; float h;
  int32_t gridDim[3]; float h2;
  float clampMin[3]; float poly6;
  float clampMax[3]; float spikyGrad;
  float gravity, mass, rho0, invRho0;
  float cfmEps, sCorrK, sCorrWq, xsphC;
  uint32_t n, nCells, nBoundary, nBodyParts;
  uint32_t nBodies; float bodyScale, covScale, omega;
  uint32_t sorAverage; float invDt, volume, tension;
  float cohes, cohesTerm;
  // arena placement and schedule (not in the reference's uniform)
  uint32_t pOff;    // first particle of the scene in the particle arrays
  uint32_t pEnd;    // pOff + n
  uint32_t cOff;    // first cell of the scene in the cell arrays
  uint32_t bOff;    // first body of the scene in the body arrays
  uint32_t parity;  // live parity before this substep's sort
  uint32_t iters;   // Jacobi iterations (>= 1)
  uint32_t subs;    // substeps of the current frame (stats after the last)
  uint32_t slot;    // stats slot (statsOut + 8 * slot) and displacement slot
  // neighbour masks reused across Jacobi iterations (kernels_solve.cu)
  float skinH2;     // (h + skin)^2: radius of the reused candidate masks
  float skinHalf;   // reuse while the displacement bound stays <= this
  float volSpiky;   // volume * spikyGrad rounded to float: the first product of
                    // lambda's fluid gradient term, formed once per substep
};

// Jacobi iterations whose displacement bounds are tracked per substep; later
// iterations rebuild their masks.
constexpr int kDispSlots = 16;
// Skin of the reused masks, in units of h.
constexpr double kSkin = 0.03;

// Anisotropic-kernel uniform (src/aniso_wgsl.js:4-21, packed by src/mesh.js:227-241).
struct AnisoParams {
  uint32_t count; float lambda, invSupport, support;
  float boxMin[3]; float radius;
  int32_t gridDim[3]; int32_t cells;
  float kr, kn, ks, stretch;
  float minExtent; int32_t neps;
  // Row trimming (not in the reference's loop; it only skips candidates whose
  // r^2 >= radius^2 for certain): dispCount > 0 when every particle is known to
  // lie within the sum of disp[0 .. dispCount) of the position its cell was
  // binned by (the last substep's iterations since its sort); 0 turns it off.
  const float* disp;
  int32_t dispCount;
};

// Mesh uniform (src/mesh_wgsl.js:3-21, packed by src/mesh.js:137-153).
struct MeshParams {
  int32_t vertDim[3]; float voxel;
  float gridOrigin[3]; float iso;
  float boxMin[3]; float invSupport;
  int32_t simGridDim[3]; float support2;
  float poly6, mass, rho0;
  uint32_t maxTris, skipBodies;
};

// Screen-space fluid rendering (kernels_ssfr.cu). Matrices column-major.
// The splat uniform of src/ssfr_wgsl.js:2-14 (+ proj * view, which the depth
// fragment applies as one matrix) for one splat pass.
struct SsfrSplat {
  float view[16], proj[16], ivp[16], pv[16];
  float vw, vh, kernelScale, quadRadius, thickRadius, maxNeighbours;
  uint32_t skipBodies, count;
};
constexpr int kSsfrMaxBlur = 64;
struct SsfrBlur {  // src/ssfr_wgsl.js:156 + the pass's Gaussian weights
  int dirX, dirY, size, pad;
  float w[2 * kSsfrMaxBlur + 1];
};
struct SsfrFilter {  // src/ssfr_wgsl.js:186-199
  int dirX, dirY, maxRadius, mode;
  float sigmaWorld, proj11, viewH, delta, mu, rangeSigma;
  int clean, cleanRadius;
};
// An environment cube map on the device (src/env.js): six faces of size x size
// rgba16float texels, face-major then row-major; size 0 = no map. The render passes
// sample it at level 0 in the direction rotated by the yaw (cos, sin), times the
// intensity.
struct EnvMap {
  const ushort4* texels;
  int32_t size;
  float intensity, yawCos, yawSin;
};
// Environment.load's host part (src/env.js:180-236): the face size for a panorama
// `width` wide, and the panorama rgb[h][w][3] resampled into 6 * size * size
// rgba16float texels (alpha 1).
int env_face_size(int width);
void build_env_cube(const float* rgb, int w, int h, int size, uint16_t* out);
uint16_t env_half(float v);

struct SsfrComp {  // src/ssfr_composite_wgsl.js:2-26
  float ivp[16], iv[16];
  float eye[3], boxMin[3], boxMax[3], absorb[3], sunDir[3];
  float proj00, proj11, ior, sunIntensity, roughness, exposure, groundReflection, thicknessScale;
  int32_t bodyCount, floorPlane, debug;
  float mapScaleX, mapScaleY;
  int32_t width, height, mapW, mapH, thickW, thickH;
  EnvMap env;
};
struct SsfrFrame {
  SsfrSplat depth, thick;
  SsfrBlur blur[2];
  SsfrFilter filter[3];
  int filterSlot[64];
  int filterPasses;
  SsfrComp comp;
  int mapW, mapH, thickW, thickH;
  const float4* smoothPos;
  const float4* g;
  const uint4* phase;
  const float4* bodies;
  unsigned long long* depthKey;  // [mapW * mapH]
  unsigned long long* thickAcc;  // [thickW * thickH]
  float* eyeZ[2];                // [mapW * mapH] ping-pong
  float* raw;                    // [mapW * mapH] unfiltered eye-space z
  float* thickMap;               // [thickW * thickH]
  float* thickTmp;
  float* bodyT;                  // [mapW * mapH]
  uchar4* image;                 // [width * height] RGBA8
};
void launch_ssfr(const SsfrFrame& f, cudaStream_t st);

// Ray-march uniform (src/ray_wgsl.js:2-30, packed by src/ray.js:32-78; no
// environment map, no rasterised-mesh surface), plus the image size and the
// cosines of debug view 5's angle thresholds.
struct RayParams {
  float ivp[16], iv[16];
  float eye[3], gridOrigin[3], boxMin[3], boxMax[3], absorb[3], sunDir[3];
  float voxel, iso, ior, skin, sunIntensity, roughness, exposure, groundReflection, proj00, proj11;
  int32_t vertDim[3], thickSteps, bodyCount, floorPlane, debug;
  int32_t width, height;
  float cosDeg[4];
  int32_t useSurface;
  float view[16], vp[16];  // view, proj * view (mesh surface pass)
  EnvMap env;
};
// The mesh surface pass (src/mesh.js:380-396, src/mesh_wgsl.js:240-321 vs + fsSurf):
// the first min(*total, cap) triangles of verts into surfZ (eye-space z, -1e4 where
// empty) and surfN (normal, w = 1 where covered), key as the depth-test scratch.
void launch_surface(const RayParams& R, const uint2* verts, const uint32_t* total, uint32_t cap,
                    const float gridOrigin[3], const int32_t vertDim[3], float voxel,
                    unsigned long long* key, float* surfZ, float4* surfN, cudaStream_t st);
void launch_ray(const RayParams& R, const float* field, const float4* bodies, const float* surfZ,
                const float4* surfN, uchar4* image, cudaStream_t st);

// Device error word bits (set by kernels, read by the host at sync points).
enum : uint32_t { ERR_SCAN_TIMEOUT = 1u, ERR_BODY_OVERFLOW = 2u };

// Device buffers of a scene, or of the arenas of a batch (same layout).
constexpr uint32_t kListCap = 96;  // neighbour-list entries per particle (nbList)

struct DevScene {
  float4* pos[2];
  float4* vel[2];
  float4* pred[2];
  uint4* body[2];
  float4* rest[2];
  float* lambda;
  float* density;
  float4* corr;
  float4* normal;
  uint32_t* cellCount;  // all zero between substeps
  uint32_t* cellStart;
  uint32_t* key;
  uint32_t* rank;
  uint32_t* unordered;
  unsigned long long* scanState;  // epoch-tagged tile states
  uint32_t* scanTicket;
  float4* bpos;
  float* bpsi;
  uint32_t* bcellStart;
  int32_t* bodyAccum;   // 4 per body
  int32_t* bodyCov;     // 9 per body
  float4* bodyCentre;
  float4* bodyRef;
  float4* bodyRot;      // 3 rows per body
  float4* bodyInfo;
  uint32_t* bodyStart;  // per scene: nBodies + 1 prefix entries of its body list
  uint32_t* bodyFill;   // append cursors, zeroed by the key pass
  uint32_t* bodyList;   // arena positions of each body's particles
  uint32_t* statsOut;   // 8 per stats slot
  uint32_t* errorWord;
  float4* smoothPos;
  float4* anisoG;
  uint32_t* nbList;     // [kListCap][cap] neighbour lists (neighbours.cuh), shared by a pair of passes
  uint32_t* nbCount;    // [cap] list length, or kListOverflow
  uint32_t* nbCell;     // [cap] cell index lambda's list was built in
  float* disp;          // [slots][kDispSlots] max |dp| of each iteration of the substep
  float* cellDisp;      // [kDispSlots][cellStride] per sort cell: max |p - nbRef| of its particles
                        // after each iteration
  uint32_t cellStride;  // cells per cellDisp slot
  float4* nbRef;        // [cap] positions at the start of the substep's iterations
  float4* predLam;      // [cap] (position, lambda) written by lambda for the delta of the same iteration
  float4* velRho;       // [cap] (velFromPos, density) of the substep's last iteration, the two
                        // values xsph reads of each neighbour in one gather
  float4* normRho;      // [cap] (normal, density) written by xsph+normals for tension
  uint32_t cap;         // particle capacity (stride of nbList)
  uint32_t* slotOut;    // optional: sorted position of each input particle
};

// A batched launch is persistent: its blocks pull work items (scene slot, tile or
// body) from the launch's segment of the frame's item list through a pull cursor,
// until the segment is exhausted. Counts and offsets live in device memory, so a
// captured frame replays for any set of scenes with the same launch sequence.
struct WorkSeg {
  uint32_t off, count;  // items [off, off + count) of the frame's list
};
struct BatchWork {
  const SimParams* params;  // this substep's table, indexed by scene slot
  const uint2* items;       // the frame's item list
  const WorkSeg* seg;       // this launch's segment
  uint32_t* cursor;         // this launch's pull cursor, zero when the frame starts
};

constexpr int kBlock = 256;          // particles per block (the reference's workgroup)
constexpr int kScanItems = 8;        // cells per scan thread
constexpr int kScanTile = kBlock * kScanItems;
// Polls of a predecessor tile's state before the scan's lookback gives up and sets
// ERR_SCAN_TIMEOUT (each poll sleeps ~64 ns, so about a quarter of a second).
constexpr uint32_t kScanSpinLimit = 1u << 22;

inline int groups(long long n, int per = kBlock) {
  long long g = (n + per - 1) / per;
  return (int)(g < 1 ? 1 : g);
}
inline int scan_tiles(int nCells) { return groups(nCells, kScanTile); }

// ---- plain launchers (one scene; P.parity = live parity before the sort) ----
void launch_key_count(const SimParams& P, const DevScene& d, cudaStream_t st);
void launch_scan(uint32_t* cellCount, uint32_t* cellStart, int nCells,
                 unsigned long long* state, uint32_t* ticket, uint32_t epoch, uint32_t* err,
                 cudaStream_t st, uint32_t spinLimit = kScanSpinLimit);
void launch_fill(const SimParams& P, const DevScene& d, cudaStream_t st);
void launch_reorder(const SimParams& P, const DevScene& d, cudaStream_t st);
// Kernels with tuned launch shapes (threads per block x minimum blocks per SM; the
// per-particle arithmetic is the same in every shape). `variant` < 0 looks the
// shape up in the tuning table by the launch's particle count.
enum TunedKernel { TK_LAMBDA = 0, TK_DELTA = 1, TK_NORMALS = 2, TK_ANISO = 3, TK_COUNT = 4 };
constexpr int kVariants = 6;
struct LaunchShape {
  int threads, minBlocks;
};
extern const LaunchShape kShapes[TK_COUNT][kVariants];
int tuned_variant(int kernel, int64_t particles);
// Tables 4..6 hold the batched launches of lambda, delta and xsph+normals (tuned on
// batched frames: their register budget differs from the plain launches'); a
// batched launch falls back to the plain table while its own is empty.
constexpr int kTunedTables = 7;
int tuned_variant_batched(int kernel, int64_t particles);

void launch_lambda(const SimParams& P, const DevScene& d, int it, cudaStream_t st, int variant = -1);
void launch_delta(const SimParams& P, const DevScene& d, int it, cudaStream_t st, int variant = -1);
void launch_body_seed(const SimParams& P, const DevScene& d, cudaStream_t st);
void launch_body_match(const SimParams& P, const DevScene& d, int it, cudaStream_t st);
void launch_xsph_finalize(const SimParams& P, const DevScene& d, int substep, cudaStream_t st);
void launch_xsph_normals(const SimParams& P, const DevScene& d, cudaStream_t st, int variant = -1);
void launch_tension_finalize(const SimParams& P, const DevScene& d, int substep, cudaStream_t st);

// ---- batched launchers (items: tiles of 256 particles, scan tiles, or bodies) ----
// `maxItems` bounds the launch's item count: the grid is min(maxItems, the blocks
// resident on the device at once); pass a large value for a launch whose count is
// only known on the device (a replayed graph).
void launch_key_count_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
// the batched scan in three launches over the same tile items (kernels_grid.cu)
void launch_scan_sums_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
void launch_scan_offsets_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
void launch_scan_apply_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
void launch_fill_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
void launch_reorder_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
void launch_lambda_b(const BatchWork& w, int maxItems, const DevScene& d, int it, cudaStream_t st, int variant);
void launch_delta_b(const BatchWork& w, int maxItems, const DevScene& d, int it, cudaStream_t st, int variant);
void launch_body_seed_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st);
void launch_body_match_b(const BatchWork& w, int maxItems, const DevScene& d, int it, cudaStream_t st);
void launch_xsph_finalize_b(const BatchWork& w, int maxItems, const DevScene& d, int substep, cudaStream_t st);
void launch_xsph_normals_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st, int variant);
void launch_tension_finalize_b(const BatchWork& w, int maxItems, const DevScene& d, int substep,
                               cudaStream_t st);
// Zeroes the stats slots (P.slot) of the scenes listed in w's segment.
void launch_zero_stats_b(const BatchWork& w, uint32_t* stats, cudaStream_t st);

// Blocks of `kernel` (launched with `block` threads) resident on the current
// device at once, cached per device and kernel; the grid of a persistent launch.
int resident_grid(const void* kernel, int block);
inline int persistent_grid(const void* kernel, int block, int maxItems) {
  const int r = resident_grid(kernel, block);
  return maxItems < r ? (maxItems < 1 ? 1 : maxItems) : r;
}

// The grid pass as an operator on caller buffers (p4a_grid_sort and
// p4a_grid_sort_noalloc): input parity 0 = (pos, vel, body, rest), output parity 1
// = (*_out); key/rank/unordered hold n entries; cellCount, state, ticket and err
// must be zero on entry. Returns the launch status.
cudaError_t run_grid_sort(const p4a_grid& g, int32_t n, float dt, float gravity, const float* pos,
                          const float* vel, const uint32_t* body, const float* rest, float* posOut,
                          float* velOut, float* predOut, uint32_t* bodyOut, float* restOut,
                          uint32_t* cellStart, uint32_t* slotOut, uint32_t* key, uint32_t* rank,
                          uint32_t* unordered, uint32_t* cellCount, unsigned long long* state,
                          uint32_t* ticket, uint32_t* err, cudaStream_t st,
                          uint32_t spinLimit = kScanSpinLimit);

// The operator entries' shared checks and tail (p4a_grid_sort, p4a_grid_sort_noalloc).
// grid_sort_check: argument checks and the cell count, P4A_ERR_CAPACITY when it
// exceeds maxCells (computed without overflow). grid_sort_launch: runs the sort on
// zeroed scratch, then either queues a copy of the error word into `status`
// (device memory) or, when status is NULL, waits for the stream and returns
// P4A_ERR_TIMEOUT if the scan's bounded wait gave up.
extern std::atomic<uint32_t> g_op_spin_limit;
extern std::atomic<int32_t> g_op_skip_first_tile;
int grid_sort_check(const p4a_grid* g, int32_t n, long long maxCells, long long* cells);
int grid_sort_launch(const p4a_grid& g, int32_t n, float dt, float gravity, const float* pos, const float* vel,
                     const uint32_t* body, const float* rest, float* posOut, float* velOut, float* predOut,
                     uint32_t* bodyOut, float* restOut, uint32_t* cellStart, uint32_t* slotOut, uint32_t* key,
                     uint32_t* rank, uint32_t* unordered, uint32_t* cellCount, unsigned long long* state,
                     uint32_t* ticket, uint32_t* err, uint32_t* status, cudaStream_t st);

// Adds to the process-wide count of kernels launched by the library.
void count_launches(uint64_t n);

// ---- plain-only passes ----
void launch_body_drag(const DevScene& d, float4* vel, const uint4* body, uint32_t held,
                      uint32_t heldCount, uint32_t heldStart, const float goal[3], float rate,
                      float blend, float limit, cudaStream_t st);
void launch_impulse(uint32_t n, const float4* pos, float4* vel, const float origin[3],
                    const float dir[3], const float impulse[3], float radius, float speedLimit,
                    cudaStream_t st);
void launch_resize(uint32_t n, float4* pos, const float oldSize[3], const float newSize[3],
                   const float clampMin[3], const float clampMax[3], cudaStream_t st);
void launch_aniso(const AnisoParams& A, const float4* pos, const uint32_t* cellStart,
                  float4* smoothPos, float4* g, cudaStream_t st, int variant = -1);
// One hose layer appended at index `first` (kernels_hose.cu).
struct HoseEmit {
  float nozzle[3];
  float spacing, centre, jitter, speed, rho0;
  uint32_t k, count, first, seed;
  uint64_t emission;
};
void launch_hose_emit(const HoseEmit& H, const DevScene& d, int parity, int predParity, cudaStream_t st);


// ---- surface mesh (kernels_mesh.cu) ----
void launch_mesh_field(const MeshParams& M, const float4* pos, const float* rho, const uint32_t* cs,
                       const uint4* body, uint32_t n, float* field, cudaStream_t st);
cudaError_t launch_mesh_blur(const MeshParams& M, const float* src, float* dst, int axis, int passes,
                             cudaStream_t st);
void launch_mesh_count(const MeshParams& M, const float* field, uint32_t* counts, uint32_t nvox, cudaStream_t st);
void launch_mesh_emit(const MeshParams& M, const float* field, const float* nfield, const uint32_t* offsets,
                      uint32_t nvox, uint2* verts, cudaStream_t st);

}  // namespace p4a
