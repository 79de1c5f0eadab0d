// render_common.cuh — vector and shading helpers shared by the screen-space fluid
// rendering (kernels_ssfr.cu) and the ray march (kernels_ray.cu): the sky, floor,
// rigid-body SDF trace, body shading, reflections, Fresnel, GGX and tone map that
// src/ssfr_composite_wgsl.js and src/ray_wgsl.js both define (their preludes are
// the same functions). Shading functions take the pass's uniform U, which has
// sunDir[3], boxMin[3], floorPlane, groundReflection, bodyCount, exposure and env.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fmath.h"
#include "p4a_internal.h"
#include "p4a_math.cuh"

namespace p4a {
namespace render {

struct V4 {
  float x, y, z, w;
};
__device__ __forceinline__ F3 f3(const float* a) { return {a[0], a[1], a[2]}; }

__device__ __forceinline__ V4 mat_vec4(const float* m, V4 v) {
  V4 o;
  o.x = fmaf(m[12], v.w, fmaf(m[8], v.z, fmaf(m[4], v.y, m[0] * v.x)));
  o.y = fmaf(m[13], v.w, fmaf(m[9], v.z, fmaf(m[5], v.y, m[1] * v.x)));
  o.z = fmaf(m[14], v.w, fmaf(m[10], v.z, fmaf(m[6], v.y, m[2] * v.x)));
  o.w = fmaf(m[15], v.w, fmaf(m[11], v.z, fmaf(m[7], v.y, m[3] * v.x)));
  return o;
}
// 3x3 column-major c[col][row]
struct Mat3 {
  float c[3][3];
};
__device__ __forceinline__ F3 mat3_vec(const Mat3& m, F3 v) {
  return {fmaf(m.c[2][0], v.z, fmaf(m.c[1][0], v.y, m.c[0][0] * v.x)),
          fmaf(m.c[2][1], v.z, fmaf(m.c[1][1], v.y, m.c[0][1] * v.x)),
          fmaf(m.c[2][2], v.z, fmaf(m.c[1][2], v.y, m.c[0][2] * v.x))};
}
__device__ __forceinline__ Mat3 mat3_mul(const Mat3& a, const Mat3& b) {
  Mat3 o;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int r = 0; r < 3; r++)
      o.c[c][r] = fmaf(a.c[2][r], b.c[c][2], fmaf(a.c[1][r], b.c[c][1], a.c[0][r] * b.c[c][0]));
  return o;
}
__device__ __forceinline__ float len3(F3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ F3 normalize3(F3 a) {
  const float l = sqrtf(dot3(a, a));
  return {a.x / l, a.y / l, a.z / l};
}
__device__ __forceinline__ F3 lerp3(F3 a, F3 b, float t) {  // WGSL mix: a * (1 - t) + b * t
  const float u = 1.0f - t;
  return {a.x * u + b.x * t, a.y * u + b.y * t, a.z * u + b.z * t};
}
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float smooth(float e0, float e1, float x) {
  const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ F3 reflect3(F3 i, F3 n) {  // i - 2 dot(n, i) n
  const float d = 2.0f * dot3(n, i);
  return {i.x - d * n.x, i.y - d * n.y, i.z - d * n.z};
}
__device__ __forceinline__ F3 refract3(F3 i, F3 n, float eta) {
  const float ni = dot3(n, i);
  const float k = 1.0f - eta * eta * (1.0f - ni * ni);
  if (k < 0.0f) return {0.f, 0.f, 0.f};
  const float a = eta * ni + sqrtf(k);
  return {eta * i.x - a * n.x, eta * i.y - a * n.y, eta * i.z - a * n.z};
}

__device__ __forceinline__ float fract1(float x) { return x - floorf(x); }
__device__ __forceinline__ float fetch_z(const float* __restrict__ z, int x, int y, int w, int h) {
  if (x < 0 || y < 0 || x >= w || y >= h) return -1.0e4f;
  return __ldg(&z[(size_t)y * w + x]);
}

__device__ __forceinline__ F3 bd(const float4* __restrict__ b, int k) {
  const float4 v = __ldg(&b[k]);
  return {v.x, v.y, v.z};
}
__device__ __forceinline__ float body_dist(const float4* __restrict__ bdata, int i, F3 p) {
  const int b = i * 6;
  const float4 c4 = __ldg(&bdata[b]);
  const F3 centre = {c4.x, c4.y, c4.z};
  const int shape = (int)(c4.w + 0.5f);
  const F3 h = bd(bdata, b + 1);
  const F3 d0 = sub3(p, centre);
  const F3 q = {dot3(bd(bdata, b + 2), d0), dot3(bd(bdata, b + 3), d0), dot3(bd(bdata, b + 4), d0)};
  if (shape == 1) return len3(q) - h.x;
  if (shape == 2) {
    const float tx = sqrtf(fmaf(q.z, q.z, q.x * q.x)) - h.x, ty = q.y;
    return sqrtf(fmaf(ty, ty, tx * tx)) - h.y;
  }
  const F3 d = {fabsf(q.x) - h.x, fabsf(q.y) - h.y, fabsf(q.z) - h.z};
  const F3 dm = {fmaxf(d.x, 0.0f), fmaxf(d.y, 0.0f), fmaxf(d.z, 0.0f)};
  return len3(dm) + fminf(fmaxf(d.x, fmaxf(d.y, d.z)), 0.0f);
}
struct BodyTrace {
  float t;
  F3 nrm, col;
};
template <class U>
__device__ __forceinline__ BodyTrace trace_bodies(const U& C, const float4* __restrict__ bdata, F3 ro,
                                                  F3 rd, float tMax) {
  BodyTrace o;
  o.t = -1.0f;
  o.nrm = {0.0f, 1.0f, 0.0f};
  o.col = {0.8f, 0.8f, 0.8f};
  if (C.bodyCount == 0) return o;
  float t = 1.0e-4f;
  for (int it = 0; it < 128; it++) {
    const F3 p = {ro.x + rd.x * t, ro.y + rd.y * t, ro.z + rd.z * t};
    float dist = 1.0e30f;
    int id = -1;
    for (int i = 0; i < C.bodyCount; i++) {
      const float d = body_dist(bdata, i, p);
      if (d < dist) {
        dist = d;
        id = i;
      }
    }
    if (dist < 5.0e-5f) {
      const float e = 2.0e-4f;
      o.nrm = normalize3({body_dist(bdata, id, {p.x + e, p.y, p.z}) - body_dist(bdata, id, {p.x - e, p.y, p.z}),
                          body_dist(bdata, id, {p.x, p.y + e, p.z}) - body_dist(bdata, id, {p.x, p.y - e, p.z}),
                          body_dist(bdata, id, {p.x, p.y, p.z + e}) - body_dist(bdata, id, {p.x, p.y, p.z - e})});
      o.col = bd(bdata, id * 6 + 5);
      o.t = t;
      return o;
    }
    t += fmaxf(dist, 1.0e-4f);
    if (t > tMax) break;
  }
  return o;
}

// rgba16float texel channel to float (exact).
__device__ __forceinline__ float half_bits(unsigned short b) { return __half2float(__ushort_as_half(b)); }
// The cube map at level 0 in direction d: face by the largest component (x, then
// y, then z on ties), the face's (s, t) in [0, 1], bilinear within the face with
// its edge texels clamped, as textureSampleLevel with a linear, clamp-to-edge
// sampler defines it.
__device__ __forceinline__ F3 cube_sample(const EnvMap& E, F3 d) {
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int face;
  float ma, sc, tc;
  if (ax >= ay && ax >= az) {
    face = d.x >= 0.0f ? 0 : 1;
    ma = ax;
    sc = d.x >= 0.0f ? -d.z : d.z;
    tc = -d.y;
  } else if (ay >= az) {
    face = d.y >= 0.0f ? 2 : 3;
    ma = ay;
    sc = d.x;
    tc = d.y >= 0.0f ? d.z : -d.z;
  } else {
    face = d.z >= 0.0f ? 4 : 5;
    ma = az;
    sc = d.z >= 0.0f ? d.x : -d.x;
    tc = -d.y;
  }
  const float n = (float)E.size;
  // a NaN or zero direction lands on texel (0, 0) of its face
  const float u = fminf(fmaxf(0.5f * (sc / ma + 1.0f) * n - 0.5f, -1.0f), n);
  const float v = fminf(fmaxf(0.5f * (tc / ma + 1.0f) * n - 0.5f, -1.0f), n);
  const float fu = floorf(u), fv = floorf(v);
  const float tx = u - fu, ty = v - fv;
  const int x0 = min(max((int)fu, 0), E.size - 1), x1 = min(max((int)fu + 1, 0), E.size - 1);
  const int y0 = min(max((int)fv, 0), E.size - 1), y1 = min(max((int)fv + 1, 0), E.size - 1);
  const ushort4* __restrict__ f = E.texels + (size_t)face * E.size * E.size;
  const ushort4 a = __ldg(&f[y0 * E.size + x0]), b = __ldg(&f[y0 * E.size + x1]);
  const ushort4 c = __ldg(&f[y1 * E.size + x0]), e = __ldg(&f[y1 * E.size + x1]);
  const F3 top = lerp3({half_bits(a.x), half_bits(a.y), half_bits(a.z)}, {half_bits(b.x), half_bits(b.y), half_bits(b.z)},
                       tx);
  const F3 bot = lerp3({half_bits(c.x), half_bits(c.y), half_bits(c.z)}, {half_bits(e.x), half_bits(e.y), half_bits(e.z)},
                       tx);
  return lerp3(top, bot, ty);
}
// envSample (src/ray_wgsl.js:46-50, src/ssfr_composite_wgsl.js:38-42).
__device__ __forceinline__ F3 env_sample(const EnvMap& E, F3 d) {
  const F3 r = {E.yawCos * d.x + E.yawSin * d.z, d.y, -E.yawSin * d.x + E.yawCos * d.z};
  const F3 c = cube_sample(E, r);
  return {c.x * E.intensity, c.y * E.intensity, c.z * E.intensity};
}

template <class U>
__device__ __forceinline__ F3 sky_color(const U& C, F3 d) {
  if (C.env.size > 0) return env_sample(C.env, d);
  const float h = clampf(d.y, 0.0f, 1.0f);
  const F3 haze = {0.62f, 0.74f, 0.90f}, zenith = {0.09f, 0.28f, 0.72f}, mid = {0.25f, 0.48f, 0.85f};
  F3 c = lerp3(haze, mid, smooth(0.0f, 0.16f, h));
  c = lerp3(c, zenith, smooth(0.10f, 0.85f, h));
  const float s = fmaxf(dot3(d, f3(C.sunDir)), 0.0f);
  const float p1 = fm_pow(s, 3000.0f), p2 = fm_pow(s, 24.0f);
  c = {c.x + 1.00f * p1 * 14.0f, c.y + 0.96f * p1 * 14.0f, c.z + 0.88f * p1 * 14.0f};
  c = {c.x + 1.00f * p2 * 0.20f, c.y + 0.92f * p2 * 0.20f, c.z + 0.78f * p2 * 0.20f};
  return c;
}
__device__ __forceinline__ F3 floor_color(F3 p) {
  const F3 base = {0.30f, 0.305f, 0.315f};
  const float gx = fabsf(fract1(p.x) - 0.5f), gz = fabsf(fract1(p.z) - 0.5f);
  const float line = 1.0f - smooth(0.0f, 0.015f, fminf(gx, gz));
  F3 c = lerp3(base, {0.50f, 0.51f, 0.52f}, line * 0.8f);
  const float fs = floorf(p.x) + floorf(p.z);
  const float chk = fs - 2.0f * floorf(fs * 0.5f);
  const float m = lerpf(0.88f, 1.10f, chk);
  return {c.x * m, c.y * m, c.z * m};
}
template <class U>
__device__ __forceinline__ F3 background(const U& C, F3 o, F3 d) {
  if (C.floorPlane != 0 && d.y < -1.0e-4f) {
    const float t = (C.boxMin[1] - o.y) / d.y;
    if (t > 0.0f) {
      const F3 p = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
      const float fade = 1.0f - fm_exp(-0.02f * t);
      const F3 far = C.env.size > 0 ? env_sample(C.env, d) : F3{0.62f, 0.74f, 0.90f};
      return lerp3(floor_color(p), far, fade);
    }
  }
  return sky_color(C, d);
}
template <class U>
__device__ __forceinline__ F3 shade_body(const U& C, F3 n, F3 base, F3 rd, F3 env) {
  const float ndl = fmaxf(dot3(n, f3(C.sunDir)), 0.0f);
  const F3 h = normalize3(sub3(f3(C.sunDir), rd));
  const float spec = fm_pow(fmaxf(dot3(n, h), 0.0f), 60.0f);
  const float fres = fm_pow(1.0f - fmaxf(dot3({-rd.x, -rd.y, -rd.z}, n), 0.0f), 4.0f);
  const float k = 0.22f + 0.78f * ndl;
  return {base.x * k + 0.7f * spec + env.x * fres * 0.25f, base.y * k + 0.7f * spec + env.y * fres * 0.25f,
          base.z * k + 0.7f * spec + env.z * fres * 0.25f};
}
template <class U>
__device__ __forceinline__ F3 env_reflect(const U& C, F3 d) {
  if (C.env.size > 0) return env_sample(C.env, d);
  if (d.y >= 0.0f) return sky_color(C, d);
  const float k = clampf(-d.y * 4.0f, 0.0f, 1.0f);
  return lerp3({0.62f, 0.74f, 0.90f}, {0.32f, 0.325f, 0.335f}, k);
}
template <class U>
__device__ __forceinline__ F3 water_reflect(const U& C, F3 d, F3 n) {
  const F3 physical = env_reflect(C, d);
  if (d.y >= 0.0f || C.groundReflection >= 1.0f) return physical;
  const float top = smooth(0.819152f, 0.939693f, n.y);
  const float below = smooth(0.0f, 0.10f, -d.y);
  const float suppress = (1.0f - clampf(C.groundReflection, 0.0f, 1.0f)) * top * below;
  const float xzl = fmaxf(sqrtf(fmaf(d.z, d.z, d.x * d.x)), 1.0e-4f);
  const F3 hd = {d.x / xzl, 0.0f, d.z / xzl};
  return lerp3(physical, sky_color(C, hd), suppress);
}
template <class U>
__device__ __forceinline__ F3 scene_color(const U& C, const float4* __restrict__ bdata, F3 o, F3 d) {
  const BodyTrace b = trace_bodies(C, bdata, o, d, 60.0f);
  if (b.t < 0.0f) return background(C, o, d);
  const F3 p = {o.x + d.x * b.t, o.y + d.y * b.t, o.z + d.z * b.t};
  const F3 po = {p.x + b.nrm.x * 1.0e-4f, p.y + b.nrm.y * 1.0e-4f, p.z + b.nrm.z * 1.0e-4f};
  return shade_body(C, b.nrm, b.col, d, background(C, po, reflect3(d, b.nrm)));
}
__device__ __forceinline__ float fresnel_full(float cosI, float n1, float n2) {
  const float eta = n1 / n2;
  const float sinT2 = eta * eta * (1.0f - cosI * cosI);
  if (sinT2 >= 1.0f) return 1.0f;
  const float cosT = sqrtf(1.0f - sinT2);
  const float rs = (n1 * cosI - n2 * cosT) / (n1 * cosI + n2 * cosT);
  const float rp = (n1 * cosT - n2 * cosI) / (n1 * cosT + n2 * cosI);
  return clampf(0.5f * (rs * rs + rp * rp), 0.0f, 1.0f);
}
__device__ __forceinline__ float ggx_spec(F3 n, F3 v, F3 l, float rough) {
  const float a = fmaxf(rough * rough, 1.0e-4f);
  const F3 h = normalize3(add3(l, v));
  const float ndh = fmaxf(dot3(n, h), 0.0f);
  const float ndl = fmaxf(dot3(n, l), 0.0f);
  const float ndv = fmaxf(dot3(n, v), 0.0f);
  const float a2 = a * a;
  const float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
  const float ndf = a2 / fmaxf(3.14159265f * d * d, 1.0e-7f);
  const float k = a * 0.5f;
  const float gl = ndl / fmaxf(ndl * (1.0f - k) + k, 1.0e-5f);
  const float gv = ndv / fmaxf(ndv * (1.0f - k) + k, 1.0e-5f);
  return ndf * gl * gv * ndl / fmaxf(4.0f * ndl * ndv, 1.0e-4f);
}
template <class U>
__device__ __forceinline__ F3 view_pos(const U& C, float nx, float ny, float z) {
  return {-nx * z / C.proj00, -ny * z / C.proj11, z};
}
template <class U>
__device__ __forceinline__ F3 tonemap(const U& C, F3 c) {
  F3 col = {c.x * C.exposure, c.y * C.exposure, c.z * C.exposure};
  const float m = 1.0f + fmaxf(fmaxf(col.x, col.y), col.z) * 0.35f;
  col = {col.x / m, col.y / m, col.z / m};
  const float g = (float)(1.0 / 2.2);  // the shader's constant expression, rounded once
  return {fm_pow(col.x, g), fm_pow(col.y, g), fm_pow(col.z, g)};
}
__device__ __forceinline__ uchar4 to_unorm8(F3 c) {
  auto u = [](float v) -> unsigned char {
    const float x = clampf(v, 0.0f, 1.0f) * 255.0f + 0.5f;
    return (unsigned char)(int)floorf(x);
  };
  return make_uchar4(u(c.x), u(c.y), u(c.z), 255);
}


}  // namespace render
}  // namespace p4a
