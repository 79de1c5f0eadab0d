// kernels_solve.cu — the PBF Jacobi iteration: lambda (src/wgsl.js:477-543) and
// delta (src/wgsl.js:545-612). Gather-only: each thread owns one particle and visits
// the neighbours of the 3x3 row ranges around cellOf(current pred), using the
// cellStart of the substep's sort (the reference's stale-cell semantics), fluid then
// boundary samples per row, j ascending: the reference's accumulation order, so the
// sums are bit-identical to it under the float contract. No float atomics.
//
// Buffers follow the substep's parity L = P.parity ^ 1 (the live copy after the
// sort): iteration `it` reads pred[L ^ (it & 1)] and delta writes the other copy.
// lambda builds the per-row neighbour masks (neighbours.cuh) and stores them; delta
// runs on the same positions, so it reuses them and skips the candidate tests.
// The masks are built with the radius h + skin and also serve later iterations of
// the substep: every delta (and the rigid projection) records the largest
// displacement of its iteration, and an iteration reuses the masks of the last
// rebuild while the summed displacements since then stay within skin / 2 (so every
// pair now within h was within h + skin then) and the particle is still in the cell
// it was in then (so its candidate rows are the same). Phase 2 tests r^2 < h^2 on
// every masked candidate, so the visited neighbours and their order are exactly the
// reference's either way.
// The last delta of a substep also writes velFromPos (src/wgsl.js:72-83) for every
// particle into the non-live velocity copy; body particles are overwritten by the
// rigid projection that follows.
#include <cuda_runtime.h>

#include "neighbours.cuh"
#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "pass_common.cuh"

namespace p4a {

template <int TB>
__device__ __forceinline__ void lambda_body(const SimParams& P, const DevScene& d, uint32_t li, int it) {
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int L = (int)P.parity ^ 1;
  const float4* __restrict__ pred = d.pred[L ^ (it & 1)];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const uint32_t* __restrict__ bcs = d.bcellStart + P.cOff;
  const uint32_t cap = d.cap;
  const F3 pi = xyz(__ldg(&pred[i]));
  const RowWalk w(P, pi);
  const RowStage<TB, true> st;
  // reuse the masks of the last rebuild while the displacement bound allows
  const uint32_t cell = cell_index(P, w.c);
  bool reuse = false;
  if (it > 0 && it < kDispSlots) {
    const float* disp = d.disp + (size_t)P.slot * kDispSlots;
    int ref = 0;
    float D = 0.0f;
    for (int t = 0; t < it; t++) {
      D += __ldg(&disp[t]);
      if (D * 1.00001f > P.skinHalf) {  // iteration t + 1 rebuilt
        ref = t + 1;
        D = 0.0f;
      }
    }
    reuse = ref < it && __ldg(&d.nbCell[i]) == cell;
  }
  uint32_t todo = 0u, longRows = 0u;
#pragma unroll
  for (int r = 0; r < kRows; r++) st.set(r, 0ull, 0u, 0u);
  if (reuse) {
    longRows = __ldg(&d.nbLong[i]);
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      const int rb = w.row_base(P, r);
      if (rb < 0) continue;
      const uint64_t mr = __ldg(&d.nbMask[(size_t)r * cap + i]);
      const uint32_t bm = __ldg(&d.nbBMask[(size_t)r * cap + i]);
      const bool lg = (longRows >> r) & 1u, lgb = (longRows >> (16 + r)) & 1u;
      st.set(r, lg ? 0ull : mr, __ldg(&cs[rb + w.x0]), lgb ? 0u : bm);
      todo |= (uint32_t)(mr != 0ull || lg || bm != 0u || lgb) << r;
    }
  } else {
    // phase 1: fluid and boundary masks of every row, radius h + skin (stored)
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      const int rb = w.row_base(P, r);
      if (rb < 0) continue;
      bool lg;
      uint32_t b;
      const uint64_t mr = row_mask(P, w, rb, pi, pred, cs, lg, b, P.skinH2);
      uint32_t bm = 0u;
      bool lgb = false;
      if (P.nBoundary > 0u) {
        const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
        if (be > bb) bm = boundary_mask(P, bb, be, pi, d.bpos, lgb, P.skinH2);
      }
      d.nbMask[(size_t)r * cap + i] = mr;
      d.nbBMask[(size_t)r * cap + i] = bm;
      st.set(r, lg ? 0ull : mr, b, lgb ? 0u : bm);
      longRows |= ((uint32_t)lg << r) | ((uint32_t)lgb << (16 + r));
      todo |= (uint32_t)(mr != 0ull || lg || bm != 0u || lgb) << r;
    }
    d.nbLong[i] = longRows;
    d.nbCell[i] = cell;
  }
  // phase 2
  float rho = P.mass * poly6(P, 0.0f);
  F3 gradSum = {0.f, 0.f, 0.f};
  float sumGrad2 = 0.0f;
  auto fluid = [&](uint32_t j) -> bool {
    if (j == i) return false;
    const F3 rij = sub3(pi, xyz(__ldg(&pred[j])));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2) return false;  // in the skin of the mask only
    rho = fmaf(P.mass, poly6(P, r2), rho);
    if (r2 > 1.0e-12f) {
      const float rr = sqrtf(r2);
      const float hr = P.h - rr;
      const float s = P.volume * P.spikyGrad * hr * hr / rr;
      const F3 g = mul3(rij, s);
      gradSum = add3(gradSum, g);
      sumGrad2 = sumGrad2 + dot3(g, g);
    }
    return true;
  };
  // one boundary sample k (1e-12 <= r^2 < h^2 is tested here or by the caller)
  auto sample = [&](uint32_t k) -> bool {
    const F3 rij = sub3(pi, xyz(__ldg(&d.bpos[k])));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2) return false;
    const float psi = __ldg(&d.bpsi[k]);
    rho = fmaf(psi, poly6(P, r2), rho);
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float s = psi * P.invRho0 * P.spikyGrad * hr * hr / rr;
    gradSum = fma3(s, rij, gradSum);
    return true;
  };
  walk_rows(
      st, todo, longRows & 0x1ffu, longRows >> 16, fluid,
      [&](int r, uint32_t k) { return sample(__ldg(&bcs[w.row_base(P, r) + w.x0]) + k); },
      [&](int r) { long_row(P, w, w.row_base(P, r), pi, pred, cs, fluid); },
      [&](int r) {
        const int rb = w.row_base(P, r);
        const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
        for (uint32_t k = bb; k < be; k++) {
          const F3 rij = sub3(pi, xyz(__ldg(&d.bpos[k])));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
          sample(k);
        }
      },
      [&](int r, uint64_t em, uint32_t ebm) { st.set(r, em, 0u, ebm); });  // the row's stage is free now
  // exact masks for delta, all rows at once (rows that were not walked hold zero)
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    d.nbMaskX[(size_t)r * cap + i] = st.mask[r * TB];
    d.nbBMaskX[(size_t)r * cap + i] = st.bmask[r * TB];
  }
  d.density[i] = rho;
  const float C = rho * P.invRho0 - 1.0f;
  if (C > 0.0f) {
    const float den = dot3(gradSum, gradSum) + sumGrad2 + P.cfmEps + 1.0e-12f;
    d.lambda[i] = -C / den;
  } else {
    d.lambda[i] = 0.0f;
  }
}

template <int TB>
__device__ __forceinline__ void delta_body(const SimParams& P, const DevScene& d, uint32_t li, int it) {
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int L = (int)P.parity ^ 1;
  const float4* __restrict__ pred = d.pred[L ^ (it & 1)];
  float4* __restrict__ predOut = d.pred[L ^ ((it + 1) & 1)];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const uint32_t* __restrict__ bcs = d.bcellStart + P.cOff;
  const float* __restrict__ lambda = d.lambda;
  const uint32_t cap = d.cap;
  const F3 pi = xyz(__ldg(&pred[i]));
  const float li_ = __ldg(&lambda[i]);
  const RowWalk w(P, pi);
  const uint32_t longRows = __ldg(&d.nbLong[i]);
  const RowStage<TB, true> st;
  uint32_t todo = 0u;
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    const int rb = w.row_base(P, r);
    if (rb < 0) continue;
    const uint64_t mr = __ldg(&d.nbMaskX[(size_t)r * cap + i]);  // lambda's exact masks
    const uint32_t bm = __ldg(&d.nbBMaskX[(size_t)r * cap + i]);
    const bool lg = (longRows >> r) & 1u, lgb = (longRows >> (16 + r)) & 1u;
    st.set(r, lg ? 0ull : mr, __ldg(&cs[rb + w.x0]), lgb ? 0u : bm);
    todo |= (uint32_t)(mr != 0ull || lg || bm != 0u || lgb) << r;
  }
  F3 dsum = {0.f, 0.f, 0.f}, dB = {0.f, 0.f, 0.f};
  float nc = 1.0f;
  auto fluid = [&](uint32_t j) -> bool {
    const F3 rij = sub3(pi, xyz(__ldg(&pred[j])));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2 || r2 < 1.0e-12f || j == i) return false;
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float s = P.spikyGrad * hr * hr / rr;
    const float t = P.h2 - r2;
    const float ratio = P.poly6 * t * t * t * P.sCorrWq;
    const float r2r = ratio * ratio;
    const float sc = -P.sCorrK * r2r * r2r;
    const float coef = (li_ + __ldg(&lambda[j]) + sc) * s;
    dsum = fma3(coef, rij, dsum);
    nc += 1.0f;
    return true;
  };
  auto sample = [&](uint32_t k) -> bool {
    const F3 rij = sub3(pi, xyz(__ldg(&d.bpos[k])));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2) return false;
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float coef = (li_ * __ldg(&d.bpsi[k])) * (P.spikyGrad * hr * hr / rr);
    dB = fma3(coef, rij, dB);
    return true;
  };
  walk_rows(
      st, todo, longRows & 0x1ffu, longRows >> 16, fluid,
      [&](int r, uint32_t k) { return sample(__ldg(&bcs[w.row_base(P, r) + w.x0]) + k); },
      [&](int r) { long_row(P, w, w.row_base(P, r), pi, pred, cs, fluid); },
      [&](int r) {
        const int rb = w.row_base(P, r);
        const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
        for (uint32_t k = bb; k < be; k++) {
          const F3 rij = sub3(pi, xyz(__ldg(&d.bpos[k])));
          const float r2 = dot3(rij, rij);
          if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
          sample(k);
        }
      },
      [](int, uint64_t, uint32_t) {});
  const F3 dd = {fmaf(dB.x, P.invRho0, dsum.x * P.volume), fmaf(dB.y, P.invRho0, dsum.y * P.volume),
                 fmaf(dB.z, P.invRho0, dsum.z * P.volume)};
  float scale = P.omega;
  if (P.sorAverage == 1u) scale = P.omega / fmaxf(nc, 1.0f);
  F3 o = fma3(scale, dd, pi);
  o.x = fminf(fmaxf(o.x, P.clampMin[0]), P.clampMax[0]);
  o.y = fminf(fmaxf(o.y, P.clampMin[1]), P.clampMax[1]);
  o.z = fminf(fmaxf(o.z, P.clampMin[2]), P.clampMax[2]);
  predOut[i] = make_float4(o.x, o.y, o.z, 1.0f);
  if (it < kDispSlots) record_displacement(d, P, it, sub3(o, pi));
  if (it == (int)P.iters - 1) {  // velFromPos into the non-live velocity copy
    const float4 p0 = __ldg(&d.pos[L][i]);
    d.vel[L ^ 1][i] = make_float4((o.x - p0.x) * P.invDt, (o.y - p0.y) * P.invDt,
                                  (o.z - p0.z) * P.invDt, 0.0f);
  }
}

// Plain: block b handles particles [b * TB, (b + 1) * TB). Batched: warps pull
// 32-particle slices of the segment's tiles.
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_lambda(const __grid_constant__ SimParams P,
                                                   const __grid_constant__ DevScene d, int it) {
  lambda_body<TB>(P, d, blockIdx.x * TB + threadIdx.x, it);
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_lambda_b(const __grid_constant__ BatchWork w,
                                                     const __grid_constant__ DevScene d, int it) {
  for_each_slice(w, [&](const SimParams& P, uint32_t li) { lambda_body<TB>(P, d, li, it); });
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_delta(const __grid_constant__ SimParams P,
                                                  const __grid_constant__ DevScene d, int it) {
  delta_body<TB>(P, d, blockIdx.x * TB + threadIdx.x, it);
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_delta_b(const __grid_constant__ BatchWork w,
                                                    const __grid_constant__ DevScene d, int it) {
  for_each_slice(w, [&](const SimParams& P, uint32_t li) { delta_body<TB>(P, d, li, it); });
}

using PlainFn = void (*)(SimParams, DevScene, int);
using BatchFn = void (*)(BatchWork, DevScene, int);
#define P4A_SHAPES(K, suffix)                                                                        \
  {K##suffix<256, 4>, K##suffix<256, 5>, K##suffix<256, 3>, K##suffix<128, 8>, K##suffix<128, 10>, \
   K##suffix<128, 6>}
#define P4A_SHAPES_D(K, suffix)                                                                      \
  {K##suffix<256, 5>, K##suffix<256, 4>, K##suffix<256, 6>, K##suffix<128, 10>, K##suffix<128, 8>, \
   K##suffix<128, 12>}
static const PlainFn kLambdaP[kVariants] = P4A_SHAPES(k_lambda, );
static const BatchFn kLambdaB[kVariants] = P4A_SHAPES(k_lambda, _b);
static const PlainFn kDeltaP[kVariants] = P4A_SHAPES_D(k_delta, );
static const BatchFn kDeltaB[kVariants] = P4A_SHAPES_D(k_delta, _b);

static int pick(int kernel, int variant, int64_t n) {
  return variant >= 0 && variant < kVariants ? variant : tuned_variant(kernel, n);
}

void launch_lambda(const SimParams& P, const DevScene& d, int it, cudaStream_t st, int variant) {
  const int v = pick(TK_LAMBDA, variant, P.n), tb = kShapes[TK_LAMBDA][v].threads;
  kLambdaP[v]<<<groups(P.n, tb), tb, 0, st>>>(P, d, it);
}
void launch_delta(const SimParams& P, const DevScene& d, int it, cudaStream_t st, int variant) {
  const int v = pick(TK_DELTA, variant, P.n), tb = kShapes[TK_DELTA][v].threads;
  kDeltaP[v]<<<groups(P.n, tb), tb, 0, st>>>(P, d, it);
}
void launch_lambda_b(const BatchWork& w, int maxItems, const DevScene& d, int it, cudaStream_t st, int variant) {
  const int v = pick(TK_LAMBDA, variant, (int64_t)maxItems * kBlock), tb = kShapes[TK_LAMBDA][v].threads;
  kLambdaB[v]<<<persistent_grid((const void*)kLambdaB[v], tb, maxItems), tb, 0, st>>>(w, d, it);
}
void launch_delta_b(const BatchWork& w, int maxItems, const DevScene& d, int it, cudaStream_t st, int variant) {
  const int v = pick(TK_DELTA, variant, (int64_t)maxItems * kBlock), tb = kShapes[TK_DELTA][v].threads;
  kDeltaB[v]<<<persistent_grid((const void*)kDeltaB[v], tb, maxItems), tb, 0, st>>>(w, d, it);
}

}  // namespace p4a
