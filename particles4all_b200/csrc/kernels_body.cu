// kernels_body.cu — rigid shape matching (src/wgsl.js:159-214, 614-783; schedule
// src/sim.js:496-563) as one CTA per body over that body's particle list:
//   body_seed   the 'bodies' pass after the sort: bodyClear, bodyCompact,
//               bodyCentre, bodySeed (with the binding swap of src/sim.js:346,
//               so bodyRef = bodyCentre + mean offset) and bodyRefLoad
//   body_match  the per-iteration chain bodyClear, bodyCentre, bodySeed, bodyCov,
//               bodyResolve, bodyProject
// The sums are the reference's fixed-point i32 values (round half to even of
// (pred - centre) * bodyScale and of p_r q_c * covScale), added with wrap-around
// in a warp-shuffle tree: integer addition is associative, so the totals are the
// bits the reference's atomics produce in any order. The resolve runs on one
// thread with the reference's float order.
// The per-body particle lists are rebuilt by the reorder of every sort
// (bodyList[bodyStart[b] + k]), replacing the reference's global atomic compaction.
// A work item is a body: plain launches use block b = body b of the one scene,
// batched launches read (scene slot, body) pairs; body arrays are indexed at
// P.bOff + b.
#include <cuda_runtime.h>

#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "pass_common.cuh"

namespace p4a {

constexpr int kBodyBlock = 256;

__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum N u32 lanes over the block; result valid in s_out[0..N) after the call.
template <int N>
__device__ __forceinline__ void block_sum_u32(uint32_t (&v)[N], uint32_t* s_scratch,
                                              uint32_t* s_out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; k++) {
    const uint32_t w = warp_sum_u32(v[k]);
    if (lane == 0) s_scratch[warp * N + k] = w;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    uint32_t t = 0;
    for (int w = 0; w < kBodyBlock / 32; w++) t += s_scratch[w * N + threadIdx.x];
    s_out[threadIdx.x] = t;
  }
  __syncthreads();
}

// acc = sum round((pred - centre) * bodyScale) over the body (bodyCentre pass).
__device__ __forceinline__ void centre_sums(const SimParams& P, const float4* __restrict__ pred,
                                            const uint32_t* __restrict__ list, uint32_t count,
                                            F3 centre, uint32_t* s_scratch, uint32_t* s_acc) {
  uint32_t a[3] = {0u, 0u, 0u};
  for (uint32_t t = threadIdx.x; t < count; t += kBodyBlock) {
    const uint32_t i = list[t];
    const F3 d = mul3(sub3(xyz(pred[i]), centre), P.bodyScale);
    a[0] += (uint32_t)round_i32(d.x);
    a[1] += (uint32_t)round_i32(d.y);
    a[2] += (uint32_t)round_i32(d.z);
  }
  block_sum_u32<3>(a, s_scratch, s_acc);
}

__device__ __forceinline__ void body_seed_body(const SimParams& P, const DevScene& d, uint32_t b) {
  __shared__ uint32_t s_scratch[(kBodyBlock / 32) * 9];
  __shared__ uint32_t s_acc[9];
  const uint32_t gb = P.bOff + b;
  const float4* __restrict__ pred = d.pred[(int)P.parity ^ 1];
  const uint32_t start = d.bodyStart[gb], count = d.bodyStart[gb + 1] - start;
  const F3 centre = xyz(d.bodyCentre[gb]);
  centre_sums(P, pred, d.bodyList + start, count, centre, s_scratch, s_acc);
  if (threadIdx.x == 0) {
    const int32_t ax = (int32_t)s_acc[0], ay = (int32_t)s_acc[1], az = (int32_t)s_acc[2];
    d.bodyAccum[gb * 4 + 0] = ax; d.bodyAccum[gb * 4 + 1] = ay; d.bodyAccum[gb * 4 + 2] = az;
    d.bodyAccum[gb * 4 + 3] = (int32_t)count;
#pragma unroll
    for (int k = 0; k < 9; k++) d.bodyCov[gb * 9 + k] = 0;
    const float cnt = (float)(int32_t)count;
    if (cnt > 0.0f) {
      const float den = P.bodyScale * cnt;
      d.bodyRef[gb] = make_float4(centre.x + (float)ax / den, centre.y + (float)ay / den,
                                  centre.z + (float)az / den, 0.0f);
    }
    d.bodyCentre[gb] = d.bodyRef[gb];
  }
}

// mat3x3fInverse (src/wgsl.js:749-760), transposed: columns r0/d, r1/d, r2/d.
__device__ __forceinline__ M3 inverse_transposed(const M3& m) {
  const F3 a = m.c[0], b = m.c[1], c = m.c[2];
  const F3 r0 = cross3(b, c), r1 = cross3(c, a), r2 = cross3(a, b);
  const float det = dot3(a, r0);
  const float invd = fabsf(det) > 1.0e-20f ? 1.0f / det : 0.0f;
  return {{mul3(r0, invd), mul3(r1, invd), mul3(r2, invd)}};
}

__device__ __forceinline__ void body_match_body(const SimParams& P, const DevScene& d, uint32_t b, int it) {
  __shared__ uint32_t s_scratch[(kBodyBlock / 32) * 9];
  __shared__ uint32_t s_acc[9];
  __shared__ float s_ref[3];
  __shared__ float s_pose[12];  // centre xyz, rows of R
  const int L = (int)P.parity ^ 1;
  float4* __restrict__ pred = d.pred[L ^ ((it + 1) & 1)];
  const float4* __restrict__ rest = d.rest[L];
  const uint32_t gb = P.bOff + b;
  const uint32_t start = d.bodyStart[gb], count = d.bodyStart[gb + 1] - start;
  const uint32_t* list = d.bodyList + start;
  const F3 centre = xyz(d.bodyCentre[gb]);
  // bodyClear + bodyCentre
  centre_sums(P, pred, list, count, centre, s_scratch, s_acc);
  const int32_t ax = (int32_t)s_acc[0], ay = (int32_t)s_acc[1], az = (int32_t)s_acc[2];
  const float cnt = (float)(int32_t)count;
  // bodySeed: bodyRef = bodyCentre + mean offset
  if (threadIdx.x == 0) {
    F3 r = xyz(d.bodyRef[gb]);
    if (cnt > 0.0f) {
      const float den = P.bodyScale * cnt;
      r = {centre.x + (float)ax / den, centre.y + (float)ay / den, centre.z + (float)az / den};
      d.bodyRef[gb] = make_float4(r.x, r.y, r.z, 0.0f);
    }
    s_ref[0] = r.x; s_ref[1] = r.y; s_ref[2] = r.z;
  }
  __syncthreads();
  // bodyCov: A = sum round((pred - ref)_r * rest_c * covScale), column-major
  const F3 ref = {s_ref[0], s_ref[1], s_ref[2]};
  uint32_t cv[9] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  for (uint32_t t = threadIdx.x; t < count; t += kBodyBlock) {
    const uint32_t i = list[t];
    const F3 p = sub3(xyz(pred[i]), ref);
    const F3 q = xyz(__ldg(&rest[i]));
    cv[0] += (uint32_t)round_i32(p.x * q.x * P.covScale);
    cv[1] += (uint32_t)round_i32(p.y * q.x * P.covScale);
    cv[2] += (uint32_t)round_i32(p.z * q.x * P.covScale);
    cv[3] += (uint32_t)round_i32(p.x * q.y * P.covScale);
    cv[4] += (uint32_t)round_i32(p.y * q.y * P.covScale);
    cv[5] += (uint32_t)round_i32(p.z * q.y * P.covScale);
    cv[6] += (uint32_t)round_i32(p.x * q.z * P.covScale);
    cv[7] += (uint32_t)round_i32(p.y * q.z * P.covScale);
    cv[8] += (uint32_t)round_i32(p.z * q.z * P.covScale);
  }
  block_sum_u32<9>(cv, s_scratch, s_acc);
  // bodyResolve on one thread
  if (threadIdx.x == 0) {
    d.bodyAccum[gb * 4 + 0] = ax; d.bodyAccum[gb * 4 + 1] = ay; d.bodyAccum[gb * 4 + 2] = az;
    d.bodyAccum[gb * 4 + 3] = (int32_t)count;
    int32_t c9[9];
#pragma unroll
    for (int k = 0; k < 9; k++) { c9[k] = (int32_t)s_acc[k]; d.bodyCov[gb * 9 + k] = c9[k]; }
    F3 cen = centre;
    float rows[9];
    bool wrote = false;
    if (cnt > 0.0f) {
      const float den = P.bodyScale * cnt;
      F3 delta = {(float)ax / den, (float)ay / den, (float)az / den};
      const float invRatio = d.bodyInfo[gb].x;
      if (invRatio > 0.0f) delta = mul3(delta, invRatio);
      cen = {centre.x + delta.x, centre.y + delta.y, centre.z + delta.z};
      d.bodyCentre[gb] = make_float4(cen.x, cen.y, cen.z, 0.0f);
      M3 A = {{{(float)c9[0], (float)c9[1], (float)c9[2]},
               {(float)c9[3], (float)c9[4], (float)c9[5]},
               {(float)c9[6], (float)c9[7], (float)c9[8]}}};
      A = scale3(A, 1.0f / P.covScale);
      float det = det3(A);
      if (fabsf(det) < 1.0e-12f) { A = ident3(); det = 1.0f; }
      const float s = cbrt_newton(fabsf(det));
      if (s > 1.0e-6f) A = scale3(A, 1.0f / s);
      M3 R = A;
      for (int k = 0; k < 8; k++) {
        const M3 inv = inverse_transposed(R);
        M3 next;
#pragma unroll
        for (int c = 0; c < 3; c++) next.c[c] = mul3(add3(R.c[c], inv.c[c]), 0.5f);
        const F3 d0 = sub3(next.c[0], R.c[0]), d1 = sub3(next.c[1], R.c[1]),
                 d2 = sub3(next.c[2], R.c[2]);
        R = next;
        if (dot3(d0, d0) + dot3(d1, d1) + dot3(d2, d2) < 1.0e-12f) break;
      }
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const F3 row = row3(R, r);
        d.bodyRot[gb * 3 + r] = make_float4(row.x, row.y, row.z, 0.0f);
        rows[r * 3 + 0] = row.x; rows[r * 3 + 1] = row.y; rows[r * 3 + 2] = row.z;
      }
      wrote = true;
    }
    if (!wrote) {
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const float4 row = d.bodyRot[gb * 3 + r];
        rows[r * 3 + 0] = row.x; rows[r * 3 + 1] = row.y; rows[r * 3 + 2] = row.z;
      }
    }
    s_pose[0] = cen.x; s_pose[1] = cen.y; s_pose[2] = cen.z;
#pragma unroll
    for (int k = 0; k < 9; k++) s_pose[3 + k] = rows[k];
  }
  __syncthreads();
  // bodyProject (+ velFromPos of the body particles on the last iteration)
  const bool last = it == (int)P.iters - 1;
  const F3 cen = {s_pose[0], s_pose[1], s_pose[2]};
  const F3 r0 = {s_pose[3], s_pose[4], s_pose[5]}, r1 = {s_pose[6], s_pose[7], s_pose[8]},
           r2 = {s_pose[9], s_pose[10], s_pose[11]};
  for (uint32_t t = threadIdx.x; t < count; t += kBodyBlock) {
    const uint32_t i = list[t];
    const F3 q = xyz(__ldg(&rest[i]));
    const F3 p = {dot3(r0, q), dot3(r1, q), dot3(r2, q)};
    const F3 o = add3(cen, p);
    pred[i] = make_float4(o.x, o.y, o.z, 1.0f);
    // the projection moves the particle from this iteration's input position
    if (it < kDispSlots) {
      record_displacement(d, P, it, sub3(o, xyz(__ldg(&d.pred[L ^ (it & 1)][i]))));
      record_cell_displacement(d, P, it, o, xyz(__ldg(&d.nbRef[i])));
    }
    if (last) {
      const float4 p0 = __ldg(&d.pos[L][i]);
      const F3 v = {(o.x - p0.x) * P.invDt, (o.y - p0.y) * P.invDt, (o.z - p0.z) * P.invDt};
      d.vel[L ^ 1][i] = make_float4(v.x, v.y, v.z, 0.0f);
      d.velRho[i] = make_float4(v.x, v.y, v.z, __ldg(&d.density[i]));
    }
  }
}

__global__ void __launch_bounds__(kBodyBlock) k_body_seed(const __grid_constant__ SimParams P,
                                                          const __grid_constant__ DevScene d) {
  body_seed_body(P, d, blockIdx.x);
}
__global__ void __launch_bounds__(kBodyBlock) k_body_seed_b(const __grid_constant__ BatchWork w,
                                                            const __grid_constant__ DevScene d) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { body_seed_body(P, d, t); });
}
__global__ void __launch_bounds__(kBodyBlock) k_body_match(const __grid_constant__ SimParams P,
                                                           const __grid_constant__ DevScene d, int it) {
  body_match_body(P, d, blockIdx.x, it);
}
__global__ void __launch_bounds__(kBodyBlock) k_body_match_b(const __grid_constant__ BatchWork w,
                                                             const __grid_constant__ DevScene d,
                                                             int it) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { body_match_body(P, d, t, it); });
}

// bodyDrag (src/wgsl.js:187-214) over the held body's particle list.
__global__ void __launch_bounds__(kBlock) k_body_drag(float4* __restrict__ vel,
                                                      const uint4* __restrict__ body,
                                                      const uint32_t* __restrict__ list,
                                                      uint32_t count, uint32_t held,
                                                      const float4* __restrict__ bodyCentre,
                                                      float gx, float gy, float gz, float rate,
                                                      float blend, float limit) {
  const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= count) return;
  const uint32_t i = list[t];
  if (body[i].x != held) return;
  const float4 c = bodyCentre[held - 1u];
  F3 vWant = {(gx - c.x) * rate, (gy - c.y) * rate, (gz - c.z) * rate};
  const float sp = length3(vWant);
  if (sp > limit) vWant = mul3(vWant, limit / sp);
  const float4 v4 = vel[i];
  const F3 v = xyz(v4);
  const F3 dv = mul3(sub3(vWant, v), blend);
  vel[i] = make_float4(v.x + dv.x, v.y + dv.y, v.z + dv.z, v4.w);
}

void launch_body_seed(const SimParams& P, const DevScene& d, cudaStream_t st) {
  if (P.nBodies == 0) return;
  k_body_seed<<<P.nBodies, kBodyBlock, 0, st>>>(P, d);
}
void launch_body_match(const SimParams& P, const DevScene& d, int it, cudaStream_t st) {
  if (P.nBodies == 0) return;
  k_body_match<<<P.nBodies, kBodyBlock, 0, st>>>(P, d, it);
}
void launch_body_seed_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_body_seed_b<<<persistent_grid((const void*)k_body_seed_b, kBodyBlock, maxItems), kBodyBlock, 0, st>>>(w, d);
}
void launch_body_match_b(const BatchWork& w, int maxItems, const DevScene& d, int it, cudaStream_t st) {
  k_body_match_b<<<persistent_grid((const void*)k_body_match_b, kBodyBlock, maxItems), kBodyBlock, 0, st>>>(w, d, it);
}

void launch_body_drag(const DevScene& d, float4* vel, const uint4* body, uint32_t held,
                      uint32_t heldCount, uint32_t heldStart, const float goal[3], float rate,
                      float blend, float limit, cudaStream_t st) {
  if (heldCount == 0) return;
  k_body_drag<<<groups(heldCount), kBlock, 0, st>>>(vel, body, d.bodyList + heldStart, heldCount,
                                                    held, d.bodyCentre, goal[0], goal[1], goal[2],
                                                    rate, blend, limit);
}

}  // namespace p4a
