// p4a_internal.h — device parameter block, float contract helpers and kernel
// launchers shared by the CUDA translation units of libp4a.
//
// Arithmetic contract (identical to the CPU oracle, so that results match bit
// for bit): compiled with --fmad=false; the only fused multiply-adds are the
// explicit fmaf() calls in dot3() and in accumulations "acc += s*v"; division and
// square root are IEEE round-to-nearest; floats convert to ints with the
// saturating cvt forms (__float2int_rz / _rn, __float2uint_rz).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/p4a.h"

namespace p4a {

// The reference's 192-byte uniform (src/wgsl.js:4-40), float32/int32 fields in
// the reference's order. Passed to kernels by value (constant bank).
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
};

// Anisotropic-kernel uniform (src/aniso_wgsl.js:4-21, packed by src/mesh.js:227-241).
struct AnisoParams {
  uint32_t count; float lambda, invSupport, support;
  float boxMin[3]; float radius;
  int32_t gridDim[3]; int32_t cells;
  float kr, kn, ks, stretch;
  float minExtent; int32_t neps;
};

// Device error word bits (set by kernels, read by the host at sync points).
enum : uint32_t { ERR_SCAN_TIMEOUT = 1u, ERR_BODY_OVERFLOW = 2u };

// Buffers of one scene on the device.
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
  uint32_t* cellCount;  // [nCells+1], all zero between substeps
  uint32_t* cellStart;  // [nCells+2]
  uint32_t* key;        // [cap]
  uint32_t* rank;       // [cap]
  uint32_t* unordered;  // [cap]
  unsigned long long* scanState;  // [scan tiles], epoch-tagged
  uint32_t* scanTicket;           // [1]
  float4* bpos;
  float* bpsi;
  uint32_t* bcellStart;
  int32_t* bodyAccum;   // [4*B]
  int32_t* bodyCov;     // [9*B]
  float4* bodyCentre;
  float4* bodyRef;
  float4* bodyRot;      // [3*B] rows
  float4* bodyInfo;
  uint32_t* bodyStart;  // [B+1] prefix of body particle counts
  uint32_t* bodyFill;   // [B] append cursors, zeroed by the key pass
  uint32_t* bodyList;   // [nBodyParts] sorted positions of each body's particles
  uint32_t* statsOut;   // [8]
  uint32_t* errorWord;  // [1]
  float4* smoothPos;
  float4* anisoG;
  uint64_t* nbMask;     // [9][cap] per-row neighbour masks shared by a pair of passes
  uint32_t* nbLong;     // [cap] rows with more than 64 candidates
  uint32_t cap;         // particle capacity (stride of nbMask)
};

constexpr int kBlock = 256;          // particles per block (the reference's workgroup)
constexpr int kScanItems = 8;        // cells per scan thread
constexpr int kScanTile = kBlock * kScanItems;

inline int groups(long long n, int per = kBlock) {
  long long g = (n + per - 1) / per;
  return (int)(g < 1 ? 1 : g);
}
inline int scan_tiles(int nCells) { return groups(nCells, kScanTile); }

// ---- launchers (stream = the scene's stream) ------------------------------
// grid pass: predict + counting sort (kernels_grid.cu)
void launch_key_count(const SimParams& P, const float4* pos, const float4* vel, uint32_t* key,
                      uint32_t* rank, uint32_t* cellCount, uint32_t* bodyFill, uint32_t nBodies,
                      cudaStream_t st);
void launch_scan(uint32_t* cellCount, uint32_t* cellStart, int nCells,
                 unsigned long long* state, uint32_t* ticket, uint32_t epoch, uint32_t* err,
                 cudaStream_t st);
void launch_fill(uint32_t n, const uint32_t* key, const uint32_t* rank, const uint32_t* cellStart,
                 uint32_t* unordered, cudaStream_t st);
void launch_reorder(const SimParams& P, const uint32_t* key, const uint32_t* cellStart,
                    const uint32_t* unordered, const float4* pos, const float4* vel,
                    const uint4* body, const float4* rest, float4* posOut, float4* velOut,
                    float4* predOut, uint4* bodyOut, float4* restOut, uint32_t* slotOut,
                    const uint32_t* bodyStart, uint32_t* bodyFill, uint32_t* bodyList,
                    cudaStream_t st);
// solver (kernels_solve.cu)
void launch_lambda(const SimParams& P, const DevScene& d, const float4* pred, cudaStream_t st);
void launch_delta(const SimParams& P, const DevScene& d, const float4* pred, float4* predOut,
                  const float4* posLive, float4* velScratch, cudaStream_t st);
// finish (kernels_finish.cu)
void launch_xsph_finalize(const SimParams& P, const DevScene& d, const float4* pred,
                          const float4* velIn, float4* posOut, float4* velOut, float4* predCopy,
                          bool stats, cudaStream_t st);
void launch_xsph_normals(const SimParams& P, const DevScene& d, const float4* pred,
                         const float4* velIn, cudaStream_t st);
void launch_tension_finalize(const SimParams& P, const DevScene& d, const float4* pred,
                             const float4* velIn, float4* posOut, float4* velOut,
                             float4* predCopy, bool stats, cudaStream_t st);
// bodies (kernels_body.cu)
void launch_body_seed(const SimParams& P, const DevScene& d, const float4* pred, cudaStream_t st);
void launch_body_match(const SimParams& P, const DevScene& d, float4* pred, const float4* rest,
                       const float4* posLive, float4* velScratch, cudaStream_t st);
void launch_body_drag(const DevScene& d, float4* vel, const uint4* body, uint32_t held,
                      uint32_t heldCount, uint32_t heldStart, const float goal[3], float rate,
                      float blend, float limit, cudaStream_t st);
// interactive passes and the anisotropic kernel (kernels_misc.cu)
void launch_impulse(uint32_t n, const float4* pos, float4* vel, const float origin[3],
                    const float dir[3], const float impulse[3], float radius, float speedLimit,
                    cudaStream_t st);
void launch_resize(uint32_t n, float4* pos, const float oldSize[3], const float newSize[3],
                   const float clampMin[3], const float clampMax[3], cudaStream_t st);
void launch_aniso(const AnisoParams& A, const float4* pos, const uint32_t* cellStart,
                  float4* smoothPos, float4* g, cudaStream_t st);

}  // namespace p4a
