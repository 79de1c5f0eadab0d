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
// The velFromPos velocities live in a scratch buffer (the non-live vel copy), so
// the final velocity can be written to the live copy while neighbours still read
// the scratch one. xsph+normals builds the neighbour masks (neighbours.cuh) and
// stores them for the tension pass, which walks the same positions.
#include <cuda_runtime.h>

#include "neighbours.cuh"
#include "p4a_internal.h"
#include "p4a_math.cuh"

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
    float a = sR[t], b = sM[t], c = sV[t], d = sK[t];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a = a + __shfl_down_sync(0xffffffffu, a, off);
      b = fmaxf(b, __shfl_down_sync(0xffffffffu, b, off));
      c = fmaxf(c, __shfl_down_sync(0xffffffffu, c, off));
      d = d + __shfl_down_sync(0xffffffffu, d, off);
    }
    if (t == 0) {
      atomicAdd(&out[0], __float2uint_rz(a * 1024.0f));
      atomicMax(&out[1], __float2uint_rz(b * 1024.0f));
      atomicMax(&out[2], __float2uint_rz(c * 1024.0f));
      atomicAdd(&out[3], __float2uint_rz(d * 1024.0f));
    }
  }
}

// xsph (+ finalize) for scenes without surface tension.
__global__ void __launch_bounds__(kBlock, 5) k_xsph_finalize(
    const __grid_constant__ SimParams P, const float4* __restrict__ pred,
    const float4* __restrict__ velIn, const float* __restrict__ density,
    const uint32_t* __restrict__ cs, float4* __restrict__ posOut, float4* __restrict__ velOut,
    float4* __restrict__ predCopy, uint32_t* __restrict__ statsOut) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  const bool act = i < P.n;
  F3 vf = {0.f, 0.f, 0.f};
  float rhoi = 0.0f;
  if (act) {
    const float4 p4 = __ldg(&pred[i]);
    const F3 pi = xyz(p4), vi = xyz(__ldg(&velIn[i]));
    const RowWalk w(P, pi);
    uint32_t longRows = 0u;
    F3 acc = {0.f, 0.f, 0.f};
#pragma unroll
    for (int r = 0; r < kRows; r++) {
      const int rb = w.row_base(P, r);
      if (rb < 0) continue;
      bool lg;
      const uint64_t mr = row_mask(P, w, rb, pi, pred, cs, lg);
      visit_row(P, w, rb, pi, mr, lg, pred, cs, [&](uint32_t j) {
        if (j == i) return;
        const F3 rij = sub3(pi, xyz(__ldg(&pred[j])));
        const float r2 = dot3(rij, rij);
        const float f = P.mass * poly6(P, r2) / fmaxf(__ldg(&density[j]), 0.5f * P.rho0);
        acc = fma3(f, sub3(xyz(__ldg(&velIn[j])), vi), acc);
      });
    }
    const F3 corr = mul3(acc, P.xsphC);
    vf = add3(vi, corr);
    velOut[i] = make_float4(vf.x, vf.y, vf.z, 0.0f);
    posOut[i] = p4;
    if (predCopy) predCopy[i] = p4;
    rhoi = __ldg(&density[i]);
  }
  if (statsOut) block_stats(P, act, rhoi, vf, statsOut);
}

// xsph + normals (tension scenes): corr = xsphC * acc, normal = h * nacc.
__global__ void __launch_bounds__(kBlock, 4) k_xsph_normals(
    const __grid_constant__ SimParams P, const float4* __restrict__ pred,
    const float4* __restrict__ velIn, const float* __restrict__ density,
    const uint32_t* __restrict__ cs, float4* __restrict__ corrOut, float4* __restrict__ normalOut,
    uint64_t* __restrict__ masks, uint32_t* __restrict__ longs, uint32_t cap) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= P.n) return;
  const F3 pi = xyz(__ldg(&pred[i])), vi = xyz(__ldg(&velIn[i]));
  const RowWalk w(P, pi);
  uint32_t longRows = 0u;
  F3 acc = {0.f, 0.f, 0.f}, nacc = {0.f, 0.f, 0.f};
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
      const float dj = fmaxf(__ldg(&density[j]), 0.5f * P.rho0);
      const float f = P.mass * poly6(P, r2) / dj;
      acc = fma3(f, sub3(xyz(__ldg(&velIn[j])), vi), acc);
      if (r2 < 1.0e-12f) return;
      const float rr = sqrtf(r2);
      const float hr = P.h - rr;
      const float coef = (P.mass / dj) * (P.spikyGrad * hr * hr / rr);
      nacc = fma3(coef, rij, nacc);
    });
  }
  longs[i] = longRows;
  corrOut[i] = make_float4(P.xsphC * acc.x, P.xsphC * acc.y, P.xsphC * acc.z, 0.0f);
  normalOut[i] = make_float4(P.h * nacc.x, P.h * nacc.y, P.h * nacc.z, 0.0f);
}

// tension + finalize.
__global__ void __launch_bounds__(kBlock, 5) k_tension_finalize(
    const __grid_constant__ SimParams P, const float4* __restrict__ pred,
    const float4* __restrict__ velIn, const float* __restrict__ density,
    const float4* __restrict__ normal, float4* __restrict__ corr, const uint32_t* __restrict__ cs,
    float4* __restrict__ posOut, float4* __restrict__ velOut, float4* __restrict__ predCopy,
    uint32_t* __restrict__ statsOut, const uint64_t* __restrict__ masks,
    const uint32_t* __restrict__ longs, uint32_t cap) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  const bool act = i < P.n;
  F3 vf = {0.f, 0.f, 0.f};
  float rhoi = 0.0f;
  if (act) {
    const float4 p4 = __ldg(&pred[i]);
    const F3 pi = xyz(p4), ni = xyz(__ldg(&normal[i]));
    rhoi = __ldg(&density[i]);
    const RowWalk w(P, pi);
    const uint32_t longRows = __ldg(&longs[i]);
    F3 acc = {0.f, 0.f, 0.f};
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
        const float hrr = P.h - rr;
        const float k = hrr * hrr * hrr * rr * rr * rr;
        float cw = P.cohes * (2.0f * k - P.cohesTerm);
        if (2.0f * rr > P.h) cw = P.cohes * k;
        const float sCoh = -P.tension * P.mass * cw / rr;
        const F3 fCoh = mul3(rij, sCoh);
        const F3 fCurv = mul3(sub3(ni, xyz(__ldg(&normal[j]))), -P.tension);
        const float wgt = 2.0f * P.rho0 / (rhoi + __ldg(&density[j]));
        acc = fma3(wgt, add3(fCoh, fCurv), acc);
      });
    }
    const float4 c0 = corr[i];
    const F3 cf = {fmaf(P.dt, acc.x, c0.x), fmaf(P.dt, acc.y, c0.y), fmaf(P.dt, acc.z, c0.z)};
    corr[i] = make_float4(cf.x, cf.y, cf.z, 0.0f);
    const F3 vi = xyz(__ldg(&velIn[i]));
    vf = add3(vi, cf);
    velOut[i] = make_float4(vf.x, vf.y, vf.z, 0.0f);
    posOut[i] = p4;
    if (predCopy) predCopy[i] = p4;
  }
  if (statsOut) block_stats(P, act, rhoi, vf, statsOut);
}

void launch_xsph_finalize(const SimParams& P, const DevScene& d, const float4* pred,
                          const float4* velIn, float4* posOut, float4* velOut, float4* predCopy,
                          bool stats, cudaStream_t st) {
  k_xsph_finalize<<<groups(P.n), kBlock, 0, st>>>(P, pred, velIn, d.density, d.cellStart, posOut,
                                                  velOut, predCopy, stats ? d.statsOut : nullptr);
}

void launch_xsph_normals(const SimParams& P, const DevScene& d, const float4* pred,
                         const float4* velIn, cudaStream_t st) {
  k_xsph_normals<<<groups(P.n), kBlock, 0, st>>>(P, pred, velIn, d.density, d.cellStart, d.corr,
                                                 d.normal, d.nbMask, d.nbLong, d.cap);
}

void launch_tension_finalize(const SimParams& P, const DevScene& d, const float4* pred,
                             const float4* velIn, float4* posOut, float4* velOut,
                             float4* predCopy, bool stats, cudaStream_t st) {
  k_tension_finalize<<<groups(P.n), kBlock, 0, st>>>(P, pred, velIn, d.density, d.normal, d.corr,
                                                     d.cellStart, posOut, velOut, predCopy,
                                                     stats ? d.statsOut : nullptr, d.nbMask,
                                                     d.nbLong, d.cap);
}

}  // namespace p4a
