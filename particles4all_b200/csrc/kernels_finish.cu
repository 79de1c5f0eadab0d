// kernels_finish.cu — the 'finish' pass of a substep and the stats pass.
//   xsph       src/wgsl.js:85-123   (reads velFromPos velocities of neighbours)
//   normals    src/wgsl.js:250-288  (same neighbour walk as xsph: fused with it)
//   tension    src/wgsl.js:290-335
//   finalize   src/wgsl.js:337-350  (vel += corr; pos = pred), fused into the
//              last neighbour pass of the substep; the odd-k pred copy of
//              src/sim.js:568-573 is fused there too
//   stats      src/wgsl.js:785-832, fused into the last substep's finalize with
//              the reference's 256-particle workgroup trees, so the fixed-point
//              totals are the same bits
// With L = P.parity ^ 1 the live copy after the sort, the final positions are in
// pred[L ^ (iters & 1)]; the velFromPos velocities are in the non-live copy
// vel[L ^ 1], so the final velocity can be written to vel[L] while neighbours still
// read the other one. Each pass builds its neighbour list with radius h
// (neighbours.cuh) and walks it; xsph+normals stores the list for the tension pass,
// which walks the same positions.
#include <cuda_runtime.h>

#include "neighbours.cuh"
#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "pass_common.cuh"

namespace p4a {

// One 256-thread block's stats tree (src/wgsl.js:803-830): same pairings as the
// reference's shared-memory tree (shuffles reproduce them below 32).
__device__ __forceinline__ void block_stats(const SimParams& P, bool act, float dens, F3 v,
                                            uint32_t* __restrict__ out) {
  __shared__ float sR[kBlock], sM[kBlock], sV[kBlock], sK[kBlock];
  const int t = threadIdx.x;
  float rho = 0.0f, mrho = 0.0f, mv = 0.0f, ke = 0.0f;
  if (act) {
    rho = dens * P.invRho0;
    mrho = rho;
    const float v2 = dot3(v, v);
    mv = sqrtf(v2);
    ke = 0.5f * P.mass * v2;
  }
  sR[t] = rho; sM[t] = mrho; sV[t] = mv; sK[t] = ke;
  __syncthreads();
#pragma unroll
  for (int off = 128; off >= 32; off >>= 1) {
    if (t < off) {
      sR[t] = sR[t] + sR[t + off];
      sM[t] = fmaxf(sM[t], sM[t + off]);
      sV[t] = fmaxf(sV[t], sV[t + off]);
      sK[t] = sK[t] + sK[t + off];
    }
    __syncthreads();
  }
  if (t < 32) {
    float a = sR[t], b = sM[t], c = sV[t], e = sK[t];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a = a + __shfl_down_sync(0xffffffffu, a, off);
      b = fmaxf(b, __shfl_down_sync(0xffffffffu, b, off));
      c = fmaxf(c, __shfl_down_sync(0xffffffffu, c, off));
      e = e + __shfl_down_sync(0xffffffffu, e, off);
    }
    if (t == 0) {
      atomicAdd(&out[0], __float2uint_rz(a * 1024.0f));
      atomicMax(&out[1], __float2uint_rz(b * 1024.0f));
      atomicMax(&out[2], __float2uint_rz(c * 1024.0f));
      atomicAdd(&out[3], __float2uint_rz(e * 1024.0f));
    }
  }
}

// The neighbour list of the finishing passes (positions after the last Jacobi
// iteration): lambda's list when the displacement bound still covers it (its
// boundary samples are skipped by the walk: these passes have no boundary terms),
// else a new list with radius h, stored in nbList.
__device__ __forceinline__ uint32_t finish_list(const SimParams& P, const DevScene& d, const RowWalk& w,
                                                uint32_t i, F3 pi, const float4* __restrict__ pred,
                                                const uint32_t* __restrict__ cs) {
  const uint32_t c = __ldg(&d.nbCount[i]);
  if (list_reusable(P, d, (int)P.iters, i, w, cell_index(P, w.c), c)) return c;
  return build_list<false>(P, w, i, pi, pred, cs, nullptr, nullptr, d.nbList, d.cap, P.h2);
}

// xsph (+ finalize) of scene-local particle li for scenes without surface
// tension; returns its density and final velocity for the stats (zero past the
// scene's end).
__device__ __forceinline__ void xsph_finalize_particle(const SimParams& P, const DevScene& d, uint32_t li,
                                                       float& rhoi, F3& vf) {
  vf = {0.f, 0.f, 0.f};
  rhoi = 0.0f;
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int L = (int)P.parity ^ 1;
  const float4* __restrict__ pred = d.pred[L ^ ((int)P.iters & 1)];
  const float4* __restrict__ velIn = d.vel[L ^ 1];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const float4 p4 = __ldg(&pred[i]);
  const F3 pi = xyz(p4), vi = xyz(__ldg(&velIn[i]));
  const RowWalk w(P, pi);
  const uint32_t cap = d.cap;
  const uint32_t count = finish_list(P, d, w, i, pi, pred, cs);
  F3 acc = {0.f, 0.f, 0.f};
  // g = (velFromPos, density) of neighbour j
  auto fluid = [&](uint32_t, float4 q, float4 g) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2) return;  // in the skin of a reused list only
    const float t = P.h2 - r2;
    const float f = P.mass * (P.poly6 * t * t * t) / fmaxf(g.w, 0.5f * P.rho0);
    acc = fma3(f, sub3(xyz(g), vi), acc);
  };
  walk_neighbours2<true>(P, w, i, pi, pred, d.velRho, cs, d.nbList, cap, count, fluid);
  const F3 corr = mul3(acc, P.xsphC);
  vf = add3(vi, corr);
  d.vel[L][i] = make_float4(vf.x, vf.y, vf.z, 0.0f);
  d.pos[L][i] = p4;
  if ((P.iters & 1u) != 0u) d.pred[L][i] = p4;
  rhoi = __ldg(&d.density[i]);
}

// Block form: 256-particle tile `tile`, with the stats tree after the last substep.
// All threads reach the tree, so there is no early return.
__device__ __forceinline__ void xsph_finalize_body(const SimParams& P, const DevScene& d, uint32_t tile,
                                                   int substep) {
  const uint32_t li = tile * kBlock + threadIdx.x;
  float rhoi;
  F3 vf;
  xsph_finalize_particle(P, d, li, rhoi, vf);
  if (substep == (int)P.subs - 1) block_stats(P, li < P.n, rhoi, vf, d.statsOut + 8 * P.slot);
}

// xsph + normals (tension scenes): corr = xsphC * acc, normal = h * nacc.
template <int TB>
__device__ __forceinline__ void xsph_normals_body(const SimParams& P, const DevScene& d, uint32_t li) {
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int L = (int)P.parity ^ 1;
  const float4* __restrict__ pred = d.pred[L ^ ((int)P.iters & 1)];
  const float4* __restrict__ velIn = d.vel[L ^ 1];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const uint32_t cap = d.cap;
  const F3 pi = xyz(__ldg(&pred[i])), vi = xyz(__ldg(&velIn[i]));
  const RowWalk w(P, pi);
  const uint32_t count = finish_list(P, d, w, i, pi, pred, cs);
  d.nbCount[i] = count;
  F3 acc = {0.f, 0.f, 0.f}, nacc = {0.f, 0.f, 0.f};
  // g = (velFromPos, density) of neighbour j
  auto fluid = [&](uint32_t, float4 q, float4 g) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2) return;  // in the skin of a reused list only
    const float dj = fmaxf(g.w, 0.5f * P.rho0);
    const float t = P.h2 - r2;  // r2 < h2 here: poly6 without its range test
    const float f = P.mass * (P.poly6 * t * t * t) / dj;
    acc = fma3(f, sub3(xyz(g), vi), acc);
    if (r2 < 1.0e-12f) return;
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float coef = (P.mass / dj) * (P.spikyGrad * hr * hr / rr);
    nacc = fma3(coef, rij, nacc);
  };
  walk_neighbours2(P, w, i, pi, pred, d.velRho, cs, d.nbList, cap, count, fluid);
  d.corr[i] = make_float4(P.xsphC * acc.x, P.xsphC * acc.y, P.xsphC * acc.z, 0.0f);
  const F3 nrm = {P.h * nacc.x, P.h * nacc.y, P.h * nacc.z};
  d.normal[i] = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
  d.normRho[i] = make_float4(nrm.x, nrm.y, nrm.z, __ldg(&d.density[i]));  // for tension's gathers
}

// tension + finalize of scene-local particle li; density and final velocity out
// for the stats.
__device__ __forceinline__ void tension_finalize_particle(const SimParams& P, const DevScene& d, uint32_t li,
                                                          float& rhoi, F3& vf) {
  vf = {0.f, 0.f, 0.f};
  rhoi = 0.0f;
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int L = (int)P.parity ^ 1;
  const float4* __restrict__ pred = d.pred[L ^ ((int)P.iters & 1)];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const uint32_t cap = d.cap;
  const float4 p4 = __ldg(&pred[i]);
  const F3 pi = xyz(p4), ni = xyz(__ldg(&d.normal[i]));
  const float rho = __ldg(&d.density[i]);
  const RowWalk w(P, pi);
  const uint32_t count = __ldg(&d.nbCount[i]);  // xsph+normals' list for these positions
  F3 acc = {0.f, 0.f, 0.f};
  // g = (normal, density) of neighbour j
  auto fluid = [&](uint32_t, float4 q, float4 g) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2 || r2 < 1.0e-12f) return;
    const float rr = sqrtf(r2);
    const float hrr = P.h - rr;
    const float k = hrr * hrr * hrr * rr * rr * rr;
    float cw = P.cohes * (2.0f * k - P.cohesTerm);
    if (2.0f * rr > P.h) cw = P.cohes * k;
    const float sCoh = -P.tension * P.mass * cw / rr;
    const F3 fCoh = mul3(rij, sCoh);
    const F3 fCurv = mul3(sub3(ni, xyz(g)), -P.tension);
    const float wgt = 2.0f * P.rho0 / (rho + g.w);
    acc = fma3(wgt, add3(fCoh, fCurv), acc);
  };
  walk_neighbours2<true>(P, w, i, pi, pred, d.normRho, cs, d.nbList, cap, count, fluid);
  const float4 c0 = d.corr[i];
  const F3 cf = {fmaf(P.dt, acc.x, c0.x), fmaf(P.dt, acc.y, c0.y), fmaf(P.dt, acc.z, c0.z)};
  d.corr[i] = make_float4(cf.x, cf.y, cf.z, 0.0f);
  const F3 vi = xyz(__ldg(&d.vel[L ^ 1][i]));
  vf = add3(vi, cf);
  d.vel[L][i] = make_float4(vf.x, vf.y, vf.z, 0.0f);
  d.pos[L][i] = p4;
  if ((P.iters & 1u) != 0u) d.pred[L][i] = p4;
  rhoi = rho;
}

__device__ __forceinline__ void tension_finalize_body(const SimParams& P, const DevScene& d,
                                                      uint32_t tile, int substep) {
  const uint32_t li = tile * kBlock + threadIdx.x;
  float rhoi;
  F3 vf;
  tension_finalize_particle(P, d, li, rhoi, vf);
  if (substep == (int)P.subs - 1) block_stats(P, li < P.n, rhoi, vf, d.statsOut + 8 * P.slot);
}

__global__ void __launch_bounds__(kBlock, 5) k_xsph_finalize(const __grid_constant__ SimParams P,
                                                             const __grid_constant__ DevScene d,
                                                             int substep) {
  xsph_finalize_body(P, d, blockIdx.x, substep);
}
__global__ void __launch_bounds__(kBlock, 5) k_xsph_finalize_b(const __grid_constant__ BatchWork w,
                                                               const __grid_constant__ DevScene d,
                                                               int substep) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { xsph_finalize_body(P, d, t, substep); });
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_xsph_normals(const __grid_constant__ SimParams P,
                                                         const __grid_constant__ DevScene d, int) {
  xsph_normals_body<TB>(P, d, blockIdx.x * TB + threadIdx.x);
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_xsph_normals_b(const __grid_constant__ BatchWork w,
                                                           const __grid_constant__ DevScene d, int) {
  for_each_slice(w, [&](const SimParams& P, uint32_t li) { xsph_normals_body<TB>(P, d, li); });
}
using PlainFn = void (*)(SimParams, DevScene, int);
using BatchFn = void (*)(BatchWork, DevScene, int);
static const PlainFn kNormalsP[kVariants] = {k_xsph_normals<256, 4>, k_xsph_normals<256, 5>,
                                             k_xsph_normals<256, 3>, k_xsph_normals<128, 8>,
                                             k_xsph_normals<128, 10>, k_xsph_normals<128, 6>};
static const BatchFn kNormalsB[kVariants] = {k_xsph_normals_b<256, 4>, k_xsph_normals_b<256, 5>,
                                             k_xsph_normals_b<256, 3>, k_xsph_normals_b<128, 8>,
                                             k_xsph_normals_b<128, 10>, k_xsph_normals_b<128, 6>};
__global__ void __launch_bounds__(kBlock, 5) k_tension_finalize(const __grid_constant__ SimParams P,
                                                                const __grid_constant__ DevScene d,
                                                                int substep) {
  tension_finalize_body(P, d, blockIdx.x, substep);
}
__global__ void __launch_bounds__(kBlock, 5) k_tension_finalize_b(const __grid_constant__ BatchWork w,
                                                                  const __grid_constant__ DevScene d,
                                                                  int substep) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { tension_finalize_body(P, d, t, substep); });
}

void launch_xsph_finalize(const SimParams& P, const DevScene& d, int substep, cudaStream_t st) {
  k_xsph_finalize<<<groups(P.n), kBlock, 0, st>>>(P, d, substep);
}
void launch_xsph_normals(const SimParams& P, const DevScene& d, cudaStream_t st, int variant) {
  const int v = variant >= 0 && variant < kVariants ? variant : tuned_variant(TK_NORMALS, P.n);
  const int tb = kShapes[TK_NORMALS][v].threads;
  kNormalsP[v]<<<groups(P.n, tb), tb, 0, st>>>(P, d, 0);
}
void launch_tension_finalize(const SimParams& P, const DevScene& d, int substep, cudaStream_t st) {
  k_tension_finalize<<<groups(P.n), kBlock, 0, st>>>(P, d, substep);
}
void launch_xsph_finalize_b(const BatchWork& w, int maxItems, const DevScene& d, int substep, cudaStream_t st) {
  k_xsph_finalize_b<<<persistent_grid((const void*)k_xsph_finalize_b, kBlock, maxItems), kBlock, 0, st>>>(w, d, substep);
}
void launch_xsph_normals_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st, int variant) {
  const int v = variant >= 0 && variant < kVariants ? variant : tuned_variant(TK_NORMALS, (int64_t)maxItems * kBlock);
  const int tb = kShapes[TK_NORMALS][v].threads;
  kNormalsB[v]<<<persistent_grid((const void*)kNormalsB[v], tb, maxItems), tb, 0, st>>>(w, d, 0);
}
void launch_tension_finalize_b(const BatchWork& w, int maxItems, const DevScene& d, int substep,
                               cudaStream_t st) {
  k_tension_finalize_b<<<persistent_grid((const void*)k_tension_finalize_b, kBlock, maxItems), kBlock, 0, st>>>(w, d, substep);
}

}  // namespace p4a
