// kernels_solve.cu — the PBF Jacobi iteration: lambda (src/wgsl.js:477-543) and
// delta (src/wgsl.js:545-612). Gather-only: each thread owns one particle and visits
// the neighbours of the 3x3 row ranges around cellOf(current pred), using the
// cellStart of the substep's sort (the reference's stale-cell semantics), fluid then
// boundary samples per row, j ascending: the reference's accumulation order, so the
// sums are bit-identical to it under the float contract. No float atomics.
//
// lambda builds the per-row neighbour masks (neighbours.cuh) and stores them; delta
// runs on the same positions, so it reuses them and skips the candidate tests.
// The last delta of a substep also writes velFromPos (src/wgsl.js:72-83) for every
// particle into the scratch velocity buffer; body particles are overwritten by the
// rigid projection that follows.
#include <cuda_runtime.h>

#include "neighbours.cuh"
#include "p4a_internal.h"
#include "p4a_math.cuh"

namespace p4a {

__global__ void __launch_bounds__(kBlock, 4) k_lambda(
    const __grid_constant__ SimParams P, const float4* __restrict__ pred,
    float* __restrict__ lambda, float* __restrict__ density, const uint32_t* __restrict__ cs,
    const float4* __restrict__ bpos, const float* __restrict__ bpsi,
    const uint32_t* __restrict__ bcs, uint64_t* __restrict__ masks, uint32_t* __restrict__ longs,
    uint32_t cap) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= P.n) return;
  const F3 pi = xyz(__ldg(&pred[i]));
  const RowWalk w(P, pi);
  uint32_t longRows = 0u;

  float rho = P.mass * poly6(P, 0.0f);
  F3 gradSum = {0.f, 0.f, 0.f};
  float sumGrad2 = 0.0f;
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    const int rb = w.row_base(P, r);
    if (rb < 0) continue;
    bool lg;
    const uint64_t mr = row_mask(P, w, rb, pi, pred, cs, lg);
    masks[(size_t)r * cap + i] = mr;
    if (lg) longRows |= 1u << r;
    visit_row(P, w, rb, pi, mr, lg, pred, cs, [&](uint32_t j) {
      if (j == i) return;
      const F3 rij = sub3(pi, xyz(__ldg(&pred[j])));
      const float r2 = dot3(rij, rij);
      rho = fmaf(P.mass, poly6(P, r2), rho);
      if (r2 > 1.0e-12f) {
        const float rr = sqrtf(r2);
        const float hr = P.h - rr;
        const float s = P.volume * P.spikyGrad * hr * hr / rr;
        const F3 g = mul3(rij, s);
        gradSum = add3(gradSum, g);
        sumGrad2 = sumGrad2 + dot3(g, g);
      }
    });
    if (P.nBoundary > 0u) {
      const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
      for (uint32_t k = bb; k < be; k++) {
        const F3 rij = sub3(pi, xyz(__ldg(&bpos[k])));
        const float r2 = dot3(rij, rij);
        if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
        const float psi = __ldg(&bpsi[k]);
        rho = fmaf(psi, poly6(P, r2), rho);
        const float rr = sqrtf(r2);
        const float hr = P.h - rr;
        const float s = psi * P.invRho0 * P.spikyGrad * hr * hr / rr;
        gradSum = fma3(s, rij, gradSum);
      }
    }
  }
  longs[i] = longRows;
  density[i] = rho;
  const float C = rho * P.invRho0 - 1.0f;
  if (C > 0.0f) {
    const float den = dot3(gradSum, gradSum) + sumGrad2 + P.cfmEps + 1.0e-12f;
    lambda[i] = -C / den;
  } else {
    lambda[i] = 0.0f;
  }
}

__global__ void __launch_bounds__(kBlock, 5) k_delta(
    const __grid_constant__ SimParams P, const float4* __restrict__ pred,
    float4* __restrict__ predOut, const float* __restrict__ lambda,
    const uint32_t* __restrict__ cs, const float4* __restrict__ bpos,
    const float* __restrict__ bpsi, const uint32_t* __restrict__ bcs,
    const uint64_t* __restrict__ masks, const uint32_t* __restrict__ longs, uint32_t cap,
    const float4* __restrict__ posLive, float4* __restrict__ velScratch) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= P.n) return;
  const F3 pi = xyz(__ldg(&pred[i]));
  const float li = __ldg(&lambda[i]);
  const RowWalk w(P, pi);
  const uint32_t longRows = __ldg(&longs[i]);
  F3 d = {0.f, 0.f, 0.f}, dB = {0.f, 0.f, 0.f};
  float nc = 1.0f;
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    const int rb = w.row_base(P, r);
    if (rb < 0) continue;
    const uint64_t mr = __ldg(&masks[(size_t)r * cap + i]);
    visit_row(P, w, rb, pi, mr, (longRows >> r) & 1u, pred, cs, [&](uint32_t j) {
      const F3 rij = sub3(pi, xyz(__ldg(&pred[j])));
      const float r2 = dot3(rij, rij);
      if (r2 < 1.0e-12f || j == i) return;
      const float rr = sqrtf(r2);
      const float hr = P.h - rr;
      const float s = P.spikyGrad * hr * hr / rr;
      const float t = P.h2 - r2;
      const float ratio = P.poly6 * t * t * t * P.sCorrWq;
      const float r2r = ratio * ratio;
      const float sc = -P.sCorrK * r2r * r2r;
      const float coef = (li + __ldg(&lambda[j]) + sc) * s;
      d = fma3(coef, rij, d);
      nc += 1.0f;
    });
    if (P.nBoundary > 0u) {
      const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
      for (uint32_t k = bb; k < be; k++) {
        const F3 rij = sub3(pi, xyz(__ldg(&bpos[k])));
        const float r2 = dot3(rij, rij);
        if (r2 >= P.h2 || r2 < 1.0e-12f) continue;
        const float rr = sqrtf(r2);
        const float hr = P.h - rr;
        const float coef = (li * __ldg(&bpsi[k])) * (P.spikyGrad * hr * hr / rr);
        dB = fma3(coef, rij, dB);
      }
    }
  }
  const F3 dd = {fmaf(dB.x, P.invRho0, d.x * P.volume), fmaf(dB.y, P.invRho0, d.y * P.volume),
                 fmaf(dB.z, P.invRho0, d.z * P.volume)};
  float scale = P.omega;
  if (P.sorAverage == 1u) scale = P.omega / fmaxf(nc, 1.0f);
  F3 o = fma3(scale, dd, pi);
  o.x = fminf(fmaxf(o.x, P.clampMin[0]), P.clampMax[0]);
  o.y = fminf(fmaxf(o.y, P.clampMin[1]), P.clampMax[1]);
  o.z = fminf(fmaxf(o.z, P.clampMin[2]), P.clampMax[2]);
  predOut[i] = make_float4(o.x, o.y, o.z, 1.0f);
  if (velScratch) {
    const float4 p0 = __ldg(&posLive[i]);
    velScratch[i] = make_float4((o.x - p0.x) * P.invDt, (o.y - p0.y) * P.invDt,
                                (o.z - p0.z) * P.invDt, 0.0f);
  }
}

void launch_lambda(const SimParams& P, const DevScene& d, const float4* pred, cudaStream_t st) {
  k_lambda<<<groups(P.n), kBlock, 0, st>>>(P, pred, d.lambda, d.density, d.cellStart, d.bpos,
                                           d.bpsi, d.bcellStart, d.nbMask, d.nbLong, d.cap);
}

void launch_delta(const SimParams& P, const DevScene& d, const float4* pred, float4* predOut,
                  const float4* posLive, float4* velScratch, cudaStream_t st) {
  k_delta<<<groups(P.n), kBlock, 0, st>>>(P, pred, predOut, d.lambda, d.cellStart, d.bpos,
                                          d.bpsi, d.bcellStart, d.nbMask, d.nbLong, d.cap,
                                          posLive, velScratch);
}

}  // namespace p4a
