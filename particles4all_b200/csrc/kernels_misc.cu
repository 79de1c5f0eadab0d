// kernels_misc.cu — the interactive passes and the anisotropic kernel.
//   impulse  src/wgsl.js:216-248 (Sim.applyRayImpulse, src/sim.js:658-676)
//   resize   src/wgsl.js:125-157 (Sim.resizeBox, src/sim.js:687-772)
//   aniso    src/aniso_wgsl.js:3-158 (dispatched by src/mesh.js:207-261): weighted
//            covariance over radius R, Laplacian-smoothed centre, 6-sweep cyclic
//            Jacobi eigen-decomposition, clamped/stretched extents, and the
//            smoothstep blend between the isotropic and the anisotropic G.
#include <cuda_runtime.h>

#include "p4a_internal.h"
#include "p4a_math.cuh"

namespace p4a {

__global__ void __launch_bounds__(kBlock) k_impulse(uint32_t n, const float4* __restrict__ pos,
                                                    float4* __restrict__ vel, F3 o, F3 dr, F3 im,
                                                    float R, float sl) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const F3 toP = sub3(xyz(pos[i]), o);
  const float along = dot3(toP, dr);
  if (along <= 0.0f) return;
  const F3 radial = sub3(toP, mul3(dr, along));
  const float d2 = dot3(radial, radial);
  if (d2 >= R * R) return;
  const float x = 1.0f - sqrtf(d2) / R;
  const F3 v = xyz(vel[i]);
  const float oldSpeed = length3(v);
  F3 nv = add3(v, mul3(im, x * x));
  const float ns = length3(nv);
  const float allowed = fmaxf(oldSpeed, sl);
  if (ns > allowed) nv = mul3(nv, allowed / ns);
  vel[i] = make_float4(nv.x, nv.y, nv.z, 0.0f);
}

__global__ void __launch_bounds__(kBlock) k_resize(uint32_t n, float4* __restrict__ pos, F3 oldS,
                                                   F3 newS, F3 cMin, F3 cMax) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  float4 p4 = pos[i];
  float p[3] = {p4.x, p4.y, p4.z};
  const float os[3] = {oldS.x, oldS.y, oldS.z}, ns[3] = {newS.x, newS.y, newS.z};
  const float lo[3] = {cMin.x, cMin.y, cMin.z}, hi[3] = {cMax.x, cMax.y, cMax.z};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (ns[a] < os[a]) {
      const float t = fminf(fmaxf((p[a] - 0.0f) / os[a], 0.0f), 1.0f);
      p[a] = 0.0f + t * ns[a];
    }
    p[a] = fminf(fmaxf(p[a], lo[a]), hi[a]);
  }
  pos[i] = make_float4(p[0], p[1], p[2], p4.w);
}

__device__ __forceinline__ void store_g(float4* __restrict__ g, uint32_t i, const M3& G, float last) {
  g[i * 2 + 0] = make_float4(elc(G, 0, 0), elc(G, 1, 0), elc(G, 2, 0), elc(G, 1, 1));
  g[i * 2 + 1] = make_float4(elc(G, 2, 1), elc(G, 2, 2), det3(G), last);
}

// Distance along one axis from coordinate `r` to cell k of n (size `support`),
// with cell 0 open to -inf and cell n - 1 open to +inf.
__device__ __forceinline__ float open_gap(int k, int n, float r, float support) {
  const float below = k > 0 ? (float)k * support - r : 0.0f;
  const float above = k < n - 1 ? r - (float)(k + 1) * support : 0.0f;
  return fmaxf(fmaxf(below, above), 0.0f);
}

__device__ __forceinline__ void aniso_body(const AnisoParams& A, const float4* __restrict__ pos,
                                           const uint32_t* __restrict__ cs, float4* __restrict__ smoothPos,
                                           float4* __restrict__ g, uint32_t i) {
  if (i >= A.count) return;
  const F3 xi = xyz(__ldg(&pos[i]));
  I3 c;
  c.x = min(max(__float2int_rz(floorf((xi.x - A.boxMin[0]) * A.invSupport)), 0), A.gridDim[0] - 1);
  c.y = min(max(__float2int_rz(floorf((xi.y - A.boxMin[1]) * A.invSupport)), 0), A.gridDim[1] - 1);
  c.z = min(max(__float2int_rz(floorf((xi.z - A.boxMin[2]) * A.invSupport)), 0), A.gridDim[2] - 1);
  const int x0 = max(c.x - A.cells, 0), x1 = min(c.x + A.cells, A.gridDim[0] - 1);
  const float r2max = A.radius * A.radius;
  const float invR = 1.0f / A.radius;
  const F3 rel = {xi.x - A.boxMin[0], xi.y - A.boxMin[1], xi.z - A.boxMin[2]};
  // Row trimming: a candidate binned into cell X lies within `moved` of X's box
  // (the first and last cell of an axis taken as reaching to -inf / +inf, since
  // the sort clamps positions beyond the grid into them), so a cell whose box is
  // at least radius + moved + slack away holds none with r^2 < radius^2. Per row
  // only the x cells closer than that are walked: a sub-range of the row's
  // candidates in the same order, so the sums are the reference loop's.
  float lim2 = -1.0f;
  if (A.dispCount > 0) {
    float moved = 0.0f;
    for (int t = 0; t < A.dispCount; t++) moved += __ldg(&A.disp[t]);
    const float lim = A.radius + moved * 1.001f + 1.0e-3f * A.support;
    lim2 = lim * lim;
  }
  F3 sd = {0.f, 0.f, 0.f};
  M3 m2 = {{{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}};
  float wsum = 0.0f;
  int nn = 0;
  for (int dz = -A.cells; dz <= A.cells; dz++) {
    const int z = c.z + dz;
    if (z < 0 || z >= A.gridDim[2]) continue;
    const float dzMin = fmaxf(fmaxf((float)z * A.support - rel.z, rel.z - (float)(z + 1) * A.support), 0.0f);
    const float dz2 = dzMin * dzMin;
    if (dz2 >= r2max) continue;
    for (int dy = -A.cells; dy <= A.cells; dy++) {
      const int y = c.y + dy;
      if (y < 0 || y >= A.gridDim[1]) continue;
      const float dyMin = fmaxf(fmaxf((float)y * A.support - rel.y, rel.y - (float)(y + 1) * A.support), 0.0f);
      if (dz2 + dyMin * dyMin >= r2max) continue;
      const uint32_t rowBase = (uint32_t)((z * A.gridDim[1] + y) * A.gridDim[0]);
      int xa = x0, xb = x1;
      if (lim2 > 0.0f) {  // false for a NaN bound: no trimming
        const float gz = open_gap(z, A.gridDim[2], rel.z, A.support), gy = open_gap(y, A.gridDim[1], rel.y, A.support);
        const float half2 = lim2 - (gz * gz + gy * gy);
        if (half2 <= 0.0f) continue;  // no candidate of the row is within the radius
        const float half = sqrtf(half2);
        // clamped into [x0, x1], so an infinite bound walks the whole row
        xa = max(x0, min(x1, __float2int_rd((rel.x - half) * A.invSupport)));
        xb = min(x1, max(x0, __float2int_rd((rel.x + half) * A.invSupport)));
      }
      const uint32_t jb = __ldg(&cs[rowBase + xa]), je = min(__ldg(&cs[rowBase + xb + 1]), A.count);
      // one candidate of the row in the reference's order; four loads are issued
      // ahead of their tests, so the row's gathers overlap (the sums keep their order)
      auto cand = [&](float4 q) {
        const F3 d = sub3(xyz(q), xi);
        const float r2 = dot3(d, d);
        if (r2 >= r2max) return;
        const float t = sqrtf(r2) * invR;
        const float w = 1.0f - t * t * t;
        sd = fma3(w, d, sd);
        m2.c[0] = fma3(d.x * w, d, m2.c[0]);
        m2.c[1] = fma3(d.y * w, d, m2.c[1]);
        m2.c[2] = fma3(d.z * w, d, m2.c[2]);
        wsum = wsum + w;
        nn = nn + 1;
      };
      uint32_t j = jb;
      for (; j + 4 <= je; j += 4) {
        const float4 q0 = __ldg(&pos[j]), q1 = __ldg(&pos[j + 1]);
        const float4 q2 = __ldg(&pos[j + 2]), q3 = __ldg(&pos[j + 3]);
        cand(q0);
        cand(q1);
        cand(q2);
        cand(q3);
      }
      for (; j < je; j++) cand(__ldg(&pos[j]));
    }
  }
  if (wsum <= 0.0f) {
    smoothPos[i] = make_float4(xi.x, xi.y, xi.z, 0.0f);
    store_g(g, i, scale3(ident3(), A.kn / A.support), 0.0f);
    return;
  }
  const F3 dbar = {sd.x / wsum, sd.y / wsum, sd.z / wsum};
  smoothPos[i] = make_float4(xi.x + dbar.x * A.lambda, xi.y + dbar.y * A.lambda,
                             xi.z + dbar.z * A.lambda, 0.0f);
  M3 cov;
  const float db[3] = {dbar.x, dbar.y, dbar.z};
#pragma unroll
  for (int k = 0; k < 3; k++)
    cov.c[k] = {m2.c[k].x / wsum - dbar.x * db[k], m2.c[k].y / wsum - dbar.y * db[k],
                m2.c[k].z / wsum - dbar.z * db[k]};
  // jacobi (src/aniso_wgsl.js:30-55)
  M3 a = cov, v = ident3();
  for (int sweep = 0; sweep < 6; sweep++) {
#pragma unroll
    for (int pI = 0; pI < 2; pI++) {
#pragma unroll
      for (int qI = pI + 1; qI < 3; qI++) {
        const float apq = elc(a, qI, pI);
        if (fabsf(apq) < 1.0e-12f) continue;
        const float theta = (elc(a, qI, qI) - elc(a, pI, pI)) / (2.0f * apq);
        const float sgn = theta > 0.0f ? 1.0f : (theta < 0.0f ? -1.0f : 0.0f);
        float t = sgn / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
        if (theta == 0.0f) t = 1.0f;
        const float cth = 1.0f / sqrtf(t * t + 1.0f);
        const float sn = t * cth;
        M3 r = ident3();
        el(r, pI, pI) = cth; el(r, qI, qI) = cth;
        el(r, qI, pI) = sn; el(r, pI, qI) = -sn;
        a = matmul(matmul(transpose3(r), a), r);
        v = matmul(v, r);
      }
    }
  }
  const F3 sig = {elc(a, 0, 0), elc(a, 1, 1), elc(a, 2, 2)};
  const float s1 = fmaxf(sig.x, fmaxf(sig.y, sig.z));
  const float sl = s1 / A.kr;
  F3 ext = {A.ks * fmaxf(sig.x, sl), A.ks * fmaxf(sig.y, sl), A.ks * fmaxf(sig.z, sl)};
  const float den = fmaxf(1.0f, fmaxf(ext.x, fmaxf(ext.y, ext.z)) / A.stretch);
  ext = {ext.x / den, ext.y / den, ext.z / den};
  ext = {fmaxf(ext.x, A.minExtent), fmaxf(ext.y, A.minExtent), fmaxf(ext.z, A.minExtent)};
  const F3 inv = {1.0f / (A.support * ext.x), 1.0f / (A.support * ext.y), 1.0f / (A.support * ext.z)};
  const M3 D = {{{inv.x, 0.f, 0.f}, {0.f, inv.y, 0.f}, {0.f, 0.f, inv.z}}};
  const M3 Gan = matmul(matmul(v, D), transpose3(v));
  const M3 Giso = scale3(ident3(), A.kn / A.support);
  const float lo = (float)A.neps * 0.4f, hi = (float)A.neps * 1.6f;
  float tt = ((float)nn - lo) / (hi - lo);
  tt = fminf(fmaxf(tt, 0.0f), 1.0f);
  const float w = tt * tt * (3.0f - 2.0f * tt);
  M3 G;
#pragma unroll
  for (int k = 0; k < 3; k++)
    G.c[k] = {Giso.c[k].x * (1.0f - w) + Gan.c[k].x * w, Giso.c[k].y * (1.0f - w) + Gan.c[k].y * w,
              Giso.c[k].z * (1.0f - w) + Gan.c[k].z * w};
  store_g(g, i, G, (float)nn);
}

void launch_impulse(uint32_t n, const float4* pos, float4* vel, const float origin[3],
                    const float dir[3], const float impulse[3], float radius, float speedLimit,
                    cudaStream_t st) {
  k_impulse<<<groups(n), kBlock, 0, st>>>(n, pos, vel, F3{origin[0], origin[1], origin[2]},
                                          F3{dir[0], dir[1], dir[2]},
                                          F3{impulse[0], impulse[1], impulse[2]}, radius, speedLimit);
}

void launch_resize(uint32_t n, float4* pos, const float oldSize[3], const float newSize[3],
                   const float clampMin[3], const float clampMax[3], cudaStream_t st) {
  k_resize<<<groups(n), kBlock, 0, st>>>(n, pos, F3{oldSize[0], oldSize[1], oldSize[2]},
                                         F3{newSize[0], newSize[1], newSize[2]},
                                         F3{clampMin[0], clampMin[1], clampMin[2]},
                                         F3{clampMax[0], clampMax[1], clampMax[2]});
}

template <int TB, int MB>
__global__ void __launch_bounds__(TB, MB) k_aniso(const __grid_constant__ AnisoParams A,
                                                  const float4* __restrict__ pos,
                                                  const uint32_t* __restrict__ cs,
                                                  float4* __restrict__ smoothPos, float4* __restrict__ g) {
  aniso_body(A, pos, cs, smoothPos, g, blockIdx.x * TB + threadIdx.x);
}
using AnisoFn = void (*)(AnisoParams, const float4*, const uint32_t*, float4*, float4*);
static const AnisoFn kAniso[kVariants] = {k_aniso<128, 10>, k_aniso<128, 8>, k_aniso<128, 12>,
                                          k_aniso<256, 5>,  k_aniso<256, 4>, k_aniso<64, 20>};

void launch_aniso(const AnisoParams& A, const float4* pos, const uint32_t* cellStart,
                  float4* smoothPos, float4* g, cudaStream_t st, int variant) {
  const int v = variant >= 0 && variant < kVariants ? variant : tuned_variant(TK_ANISO, A.count);
  const int tb = kShapes[TK_ANISO][v].threads;
  kAniso[v]<<<groups(A.count, tb), tb, 0, st>>>(A, pos, cellStart, smoothPos, g);
}

}  // namespace p4a
