// p4a_math.cuh — device helpers for the float arithmetic contract (see
// p4a_internal.h): explicit fmaf only in dot3 and accumulations, IEEE division and
// square root, saturating float->int conversions. Compiled with --fmad=false.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "p4a_internal.h"

namespace p4a {

struct F3 { float x, y, z; };

__device__ __forceinline__ F3 xyz(const float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 add3(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 mul3(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
// dot(a, b) of WGSL under the contract: fma(a.z,b.z, fma(a.y,b.y, a.x*b.x)).
__device__ __forceinline__ float dot3(F3 a, F3 b) {
  return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x));
}
// acc += s * v under the contract.
__device__ __forceinline__ F3 fma3(float s, F3 v, F3 acc) {
  return {fmaf(s, v.x, acc.x), fmaf(s, v.y, acc.y), fmaf(s, v.z, acc.z)};
}
__device__ __forceinline__ F3 cross3(F3 b, F3 c) {
  return {b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
}
__device__ __forceinline__ float length3(F3 a) { return sqrtf(dot3(a, a)); }

// i32(round(x)) of WGSL: round half to even, saturating, NaN -> 0.
__device__ __forceinline__ int32_t round_i32(float x) { return __float2int_rn(x); }

struct I3 { int x, y, z; };

// cellOf (src/wgsl.js:43-46): clamp(vec3i(floor((p - boxMin) / h)), 0, gridDim-1).
__device__ __forceinline__ I3 cell_of(const SimParams& P, F3 p) {
  I3 c;
  c.x = __float2int_rz(floorf((p.x - P.boxMin[0]) / P.h));
  c.y = __float2int_rz(floorf((p.y - P.boxMin[1]) / P.h));
  c.z = __float2int_rz(floorf((p.z - P.boxMin[2]) / P.h));
  c.x = min(max(c.x, 0), P.gridDim[0] - 1);
  c.y = min(max(c.y, 0), P.gridDim[1] - 1);
  c.z = min(max(c.z, 0), P.gridDim[2] - 1);
  return c;
}
// cellIndex (src/wgsl.js:47-49).
__device__ __forceinline__ uint32_t cell_index(const SimParams& P, I3 c) {
  return (uint32_t)((c.z * P.gridDim[1] + c.y) * P.gridDim[0] + c.x);
}
// poly6 (src/wgsl.js:50-53).
__device__ __forceinline__ float poly6(const SimParams& P, float r2) {
  const float t = P.h2 - r2;
  return r2 < P.h2 ? P.poly6 * t * t * t : 0.0f;
}

// The predict pass (src/wgsl.js:56-70) for one particle: v and pred.
__device__ __forceinline__ void predict_one(const SimParams& P, float4 pos, float4 vel, F3& v, F3& pr) {
  const float gx = P.dt * 0.0f, gy = P.dt * -P.gravity, gz = P.dt * 0.0f;
  v = {vel.x + gx, vel.y + gy, vel.z + gz};
  pr = {pos.x + P.dt * v.x, pos.y + P.dt * v.y, pos.z + P.dt * v.z};
}

// Cube root by a fixed 5-step Newton iteration on the mantissa (x > 0, normal):
// the rigid-body resolve's pow(|det|, 1/3) (src/wgsl.js:730). IEEE basic ops
// only, so host and device give the same bits.
__device__ __forceinline__ float cbrt_newton(float x) {
  if (!(x > 0.0f) || isinf(x)) return x;
  const uint32_t bits = __float_as_uint(x);
  int e = (int)((bits >> 23) & 0xffu);
  if (e == 0) return 0.0f;
  e -= 127;
  const int q = (e + 300) / 3 - 100;
  const int r = e - 3 * q;
  float t = __uint_as_float((bits & 0x7fffffu) | 0x3f800000u);
  if (r >= 1) t = t * 2.0f;
  if (r >= 2) t = t * 2.0f;
  float y = 0.75f + 0.1666667f * t;
#pragma unroll
  for (int it = 0; it < 5; it++) y = (2.0f * y + t / (y * y)) * 0.33333334f;
  return y * __uint_as_float((uint32_t)(q + 127) << 23);
}

// Column-major 3x3 (c[k] is column k), as WGSL's mat3x3f.
struct M3 { F3 c[3]; };
__device__ __forceinline__ float& el(M3& a, int c, int r) { return (&a.c[c].x)[r]; }
__device__ __forceinline__ float elc(const M3& a, int c, int r) { return (&a.c[c].x)[r]; }
__device__ __forceinline__ M3 ident3() { return {{{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}}}; }
__device__ __forceinline__ float det3(const M3& a) { return dot3(a.c[0], cross3(a.c[1], a.c[2])); }
__device__ __forceinline__ F3 row3(const M3& a, int r) { return {elc(a, 0, r), elc(a, 1, r), elc(a, 2, r)}; }
__device__ __forceinline__ M3 matmul(const M3& A, const M3& B) {
  M3 o;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int r = 0; r < 3; r++) el(o, c, r) = dot3(row3(A, r), B.c[c]);
  return o;
}
__device__ __forceinline__ M3 transpose3(const M3& a) {
  M3 o;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int r = 0; r < 3; r++) el(o, c, r) = elc(a, r, c);
  return o;
}
__device__ __forceinline__ M3 scale3(const M3& a, float s) {
  return {{mul3(a.c[0], s), mul3(a.c[1], s), mul3(a.c[2], s)}};
}

// The largest |dp| of iteration `it` of the scene (max over the lanes that call
// together, one atomic per group): the bound that decides whether the next
// iteration may reuse the neighbour masks.
__device__ __forceinline__ void record_displacement(const DevScene& d, const SimParams& P, int it, F3 dp) {
  const float len = sqrtf(dot3(dp, dp));
  const unsigned am = __activemask();
  const uint32_t m = __reduce_max_sync(am, __float_as_uint(len));  // non-negative floats order as ints
  if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1))
    atomicMax(reinterpret_cast<unsigned int*>(d.disp + (size_t)P.slot * kDispSlots + it), m);
}
// The particle's displacement from its substep start position `ref` into the slot of
// iteration `it` of its sort cell (the cell of `ref`, which is the position the
// sort binned it by); lanes with the same cell combine into one atomic.
__device__ __forceinline__ void record_cell_displacement(const DevScene& d, const SimParams& P, int it, F3 p,
                                                         F3 ref) {
  const F3 dp = sub3(p, ref);
  const float len = sqrtf(dot3(dp, dp));
  const uint32_t c = P.cOff + cell_index(P, cell_of(P, ref));
  const unsigned am = __activemask();
  const unsigned peers = __match_any_sync(am, c);
  const uint32_t m = __reduce_max_sync(peers, __float_as_uint(len));
  if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1))
    atomicMax(reinterpret_cast<unsigned int*>(d.cellDisp + (size_t)it * d.cellStride + c), m);
}

}  // namespace p4a
