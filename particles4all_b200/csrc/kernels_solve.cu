// kernels_solve.cu — the PBF Jacobi iteration: lambda (src/wgsl.js:477-543) and
// delta (src/wgsl.js:545-612). Gather-only: each thread owns one particle and visits
// the neighbours of the 3x3 row ranges around cellOf(current pred), using the
// cellStart of the substep's sort (the reference's stale-cell semantics), fluid then
// boundary samples per row, j ascending: the reference's accumulation order, so the
// sums are bit-identical to it under the float contract. No float atomics.
//
// Buffers follow the substep's parity L = P.parity ^ 1 (the live copy after the
// sort): iteration `it` reads pred[L ^ (it & 1)] and delta writes the other copy.
// lambda builds each particle's neighbour list (neighbours.cuh) with the radius
// h + skin and stores it; delta runs on the same positions and walks the same
// list. The list also serves later iterations of the substep: every delta (and
// the rigid projection) records the largest displacement of its iteration and the
// largest displacement from the substep's start positions, and a particle reuses
// its list while those bound every particle's movement since the list was built
// by skin / 2 (so every pair now within h was within h + skin then) and it is
// still in the cell it was in then (so its candidate rows are the same); see
// list_reusable. Every pass re-tests r^2 < h^2 on each listed candidate, so the
// visited neighbours and their order are exactly the reference's either way.
// The last delta of a substep also writes velFromPos (src/wgsl.js:72-83) for every
// particle into the non-live velocity copy; body particles are overwritten by the
// rigid projection that follows.
#include <cuda_runtime.h>

#include "neighbours.cuh"
#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "pass_common.cuh"

namespace p4a {

// Called by all 32 lanes of a warp. PF: whether the list walk runs the two-deep
// prefetch pipeline (measured faster in the batched launches, slower in the plain
// ones, whose register budget it squeezes; delta's walk always prefetches). (lanes past the scene's end only take part in the
// warp's list builds).
template <bool PF>
__device__ __forceinline__ void lambda_body(const SimParams& P, const DevScene& d, uint32_t li, int it) {
  const bool act = li < P.n;
  const uint32_t i = P.pOff + (act ? li : 0u);
  const int L = (int)P.parity ^ 1;
  const float4* __restrict__ pred = d.pred[L ^ (it & 1)];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const uint32_t* __restrict__ bcs = d.bcellStart + P.cOff;
  const uint32_t cap = d.cap;
  const F3 pi = xyz(__ldg(&pred[i]));
  const RowWalk w(P, pi);
  // reuse the stored list while the displacement bounds allow
  const uint32_t cell = cell_index(P, w.c);
  if (it == 0 && act) d.nbRef[i] = make_float4(pi.x, pi.y, pi.z, 0.0f);  // the substep's start positions
  uint32_t count = it > 0 && act ? __ldg(&d.nbCount[i]) : kListOverflow;
  const bool need = act && !list_reusable(P, d, it, i, w, cell, count);
  count = build_lists_warp<true>(P, need, w, i, pi, pred, cs, bcs, d.bpos, d.nbList, cap, P.skinH2, count);
  if (need) {
    if (count != kListOverflow) count |= (uint32_t)it << kBuildShift;
    d.nbCount[i] = count;
    d.nbCell[i] = cell;
  }
  if (!act) return;
  float rho = P.mass * poly6(P, 0.0f);
  F3 gradSum = {0.f, 0.f, 0.f};
  float sumGrad2 = 0.0f;
  auto fluid = [&](uint32_t, float4 q) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2) return;  // in the skin of the list only
    const float t = P.h2 - r2;
    rho = fmaf(P.mass, P.poly6 * t * t * t, rho);  // poly6 within h
    if (r2 > 1.0e-12f) {
      const float rr = sqrtf(r2);
      const float hr = P.h - rr;
      const float s = P.volSpiky * hr * hr / rr;
      const F3 g = mul3(rij, s);
      gradSum = add3(gradSum, g);
      sumGrad2 = sumGrad2 + dot3(g, g);
    }
  };
  auto bound = [&](uint32_t k, float4 q) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2 || r2 < 1.0e-12f) return;
    const float psi = __ldg(&d.bpsi[k]);
    const float t = P.h2 - r2;
    rho = fmaf(psi, P.poly6 * t * t * t, rho);
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float s = psi * P.invRho0 * P.spikyGrad * hr * hr / rr;
    gradSum = fma3(s, rij, gradSum);
  };
  if (count != kListOverflow) {
    if constexpr (PF) {
      walk_list<true>(d.nbList, cap, i, count, pred, d.bpos, [&](uint32_t k, float4 q, bool isB) {
        if (isB) {
          bound(k, q);
        } else {
          fluid(k, q);
        }
      });
    } else {
      // The same terms on one path, fluid or boundary selected per lane: faster
      // than the branches above in the plain launches (5-9 % per launch where
      // warps mix wall and interior particles), slower in the pipelined walk of
      // the batched ones, whose registers it squeezes.
      walk_list<false, kFetchBound>(d.nbList, cap, i, count, pred, d.bpos, [&](uint32_t k, float4 q, bool isB) {
        const F3 rij = sub3(pi, xyz(q));
        const float r2 = dot3(rij, rij);
        if (r2 >= P.h2 || (isB && r2 < 1.0e-12f)) return;
        const float psi = isB ? __ldg(&d.bpsi[k]) : 0.0f;
        const float t = P.h2 - r2;
        rho = fmaf(isB ? psi : P.mass, P.poly6 * t * t * t, rho);
        if (isB || r2 > 1.0e-12f) {
          const float rr = sqrtf(r2);
          const float hr = P.h - rr;
          const float c0 = isB ? psi * P.invRho0 * P.spikyGrad : P.volSpiky;
          const float s = c0 * hr * hr / rr;
          const F3 g = mul3(rij, s);
          const F3 gf = add3(gradSum, g), gb = fma3(s, rij, gradSum);
          gradSum = isB ? gb : gf;
          const float sg = sumGrad2 + dot3(g, g);
          sumGrad2 = isB ? sumGrad2 : sg;
        }
      });
    }
  } else {
    walk_direct<true>(P, w, pi, i, pred, cs, bcs, d.bpos, fluid, bound);
  }
  d.density[i] = rho;
  const float C = rho * P.invRho0 - 1.0f;
  float lam = 0.0f;
  if (C > 0.0f) {
    const float den = dot3(gradSum, gradSum) + sumGrad2 + P.cfmEps + 1.0e-12f;
    lam = -C / den;
  }
  d.lambda[i] = lam;
  // delta reads position and lambda of a neighbour with one 16-byte gather
  d.predLam[i] = make_float4(pi.x, pi.y, pi.z, lam);
}

__device__ __forceinline__ void delta_body(const SimParams& P, const DevScene& d, uint32_t li, int it) {
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int L = (int)P.parity ^ 1;
  float4* __restrict__ predOut = d.pred[L ^ ((it + 1) & 1)];
  const uint32_t* __restrict__ cs = d.cellStart + P.cOff;
  const uint32_t* __restrict__ bcs = d.bcellStart + P.cOff;
  // lambda's (position, lambda) of this iteration: the positions of pred[L ^ (it & 1)]
  const float4* __restrict__ pl = d.predLam;
  const uint32_t cap = d.cap;
  const float4 self = __ldg(&pl[i]);
  const F3 pi = xyz(self);
  const float li_ = self.w;
  const uint32_t count = __ldg(&d.nbCount[i]);  // lambda's list for these positions
  F3 dsum = {0.f, 0.f, 0.f}, dB = {0.f, 0.f, 0.f};
  float nc = 1.0f;
  auto fluid = [&](uint32_t, float4 q) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2 || r2 < 1.0e-12f) return;
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float s = P.spikyGrad * hr * hr / rr;
    const float t = P.h2 - r2;
    const float ratio = P.poly6 * t * t * t * P.sCorrWq;
    const float r2r = ratio * ratio;
    const float sc = -P.sCorrK * r2r * r2r;
    const float coef = (li_ + q.w + sc) * s;
    dsum = fma3(coef, rij, dsum);
    nc += 1.0f;
  };
  auto bound = [&](uint32_t k, float4 q) {
    const F3 rij = sub3(pi, xyz(q));
    const float r2 = dot3(rij, rij);
    if (r2 >= P.h2 || r2 < 1.0e-12f) return;
    const float rr = sqrtf(r2);
    const float hr = P.h - rr;
    const float coef = (li_ * __ldg(&d.bpsi[k])) * (P.spikyGrad * hr * hr / rr);
    dB = fma3(coef, rij, dB);
  };
  if (count != kListOverflow) {
    walk_list<true, kFetchBound>(d.nbList, cap, i, count, pl, d.bpos, [&](uint32_t k, float4 q, bool isB) {
      if (isB) {
        bound(k, q);
      } else {
        fluid(k, q);
      }
    });
  } else {
    const RowWalk w(P, pi);
    walk_direct<true>(P, w, pi, i, pl, cs, bcs, d.bpos, fluid, bound);
  }
  const F3 dd = {fmaf(dB.x, P.invRho0, dsum.x * P.volume), fmaf(dB.y, P.invRho0, dsum.y * P.volume),
                 fmaf(dB.z, P.invRho0, dsum.z * P.volume)};
  float scale = P.omega;
  if (P.sorAverage == 1u) scale = P.omega / fmaxf(nc, 1.0f);
  F3 o = fma3(scale, dd, pi);
  o.x = fminf(fmaxf(o.x, P.clampMin[0]), P.clampMax[0]);
  o.y = fminf(fmaxf(o.y, P.clampMin[1]), P.clampMax[1]);
  o.z = fminf(fmaxf(o.z, P.clampMin[2]), P.clampMax[2]);
  predOut[i] = make_float4(o.x, o.y, o.z, 1.0f);
  if (it < kDispSlots) {
    record_displacement(d, P, it, sub3(o, pi));
    record_cell_displacement(d, P, it, o, xyz(__ldg(&d.nbRef[i])));
  }
  if (it == (int)P.iters - 1) {  // velFromPos into the non-live velocity copy
    const float4 p0 = __ldg(&d.pos[L][i]);
    const F3 v = {(o.x - p0.x) * P.invDt, (o.y - p0.y) * P.invDt, (o.z - p0.z) * P.invDt};
    d.vel[L ^ 1][i] = make_float4(v.x, v.y, v.z, 0.0f);
    d.velRho[i] = make_float4(v.x, v.y, v.z, __ldg(&d.density[i]));
  }
}

// Plain: block b handles particles [b * TB, (b + 1) * TB). Batched: warps pull
// 32-particle slices of the segment's tiles.
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_lambda(const __grid_constant__ SimParams P,
                                                   const __grid_constant__ DevScene d, int it) {
  lambda_body<false>(P, d, blockIdx.x * TB + threadIdx.x, it);
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_lambda_b(const __grid_constant__ BatchWork w,
                                                     const __grid_constant__ DevScene d, int it) {
  for_each_slice(w, [&](const SimParams& P, uint32_t li) { lambda_body<true>(P, d, li, it); });
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_delta(const __grid_constant__ SimParams P,
                                                  const __grid_constant__ DevScene d, int it) {
  delta_body(P, d, blockIdx.x * TB + threadIdx.x, it);
}
template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_delta_b(const __grid_constant__ BatchWork w,
                                                    const __grid_constant__ DevScene d, int it) {
  for_each_slice(w, [&](const SimParams& P, uint32_t li) { delta_body(P, d, li, it); });
}

using PlainFn = void (*)(SimParams, DevScene, int);
using BatchFn = void (*)(BatchWork, DevScene, int);
#define P4A_SHAPES(K, suffix)                                                                        \
  {K##suffix<256, 4>, K##suffix<256, 5>, K##suffix<256, 6>, K##suffix<128, 8>, K##suffix<128, 10>, \
   K##suffix<128, 12>}
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
