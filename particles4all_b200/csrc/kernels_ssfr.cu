// kernels_ssfr.cu — screen-space fluid rendering (src/ssfr.js:173-356,
// src/ssfr_wgsl.js:1-338, src/ssfr_composite_wgsl.js:1-333) as CUDA passes that
// write headless image buffers.
//
// The reference rasterises one quad per particle (a triangle strip of 4 vertices,
// instanced) and shades the covered pixels. Here the vertex shader's quad is
// computed per particle and the pixels whose centres fall inside it
// (x0 <= px + 0.5 < x1, same for y: the top-left rule for an axis-aligned
// rectangle) get the fragment shader's work:
//   depth      ray / ellipsoid hit; the depth test (compare 'less', cleared to
//              1.0) keeps the nearest fragment, the first drawn on equal depth:
//              a 64-bit atomicMin of (depth bits, instance); a resolve pass
//              recomputes the winner's eye-space z;
//   thickness  ray / sphere chord, blended additively: accumulated in 2^-32
//              fixed point with 64-bit atomics (order-independent sums, the same
//              bits on every run), converted to float once;
// then the full-screen passes: separable Gaussian blur of the thickness, the
// depth filter (narrow-range, bilateral or Gaussian; separable passes and the 2D
// clean-up pass), the body-depth trace and the composite (refraction through the
// thickness with absorption, Fresnel reflection, GGX sun highlight, sky / floor /
// rigid-body background, tone map) into an RGBA8 image.
//
// Matrices are column-major float[16] (WGSL mat4x4f); M * v is evaluated as a
// nested fmaf over the columns, WGSL dot() as fma(a.z,b.z, fma(a.y,b.y, a.x*b.x)),
// every other expression as written with IEEE operations; exp/log/pow are the
// host/device functions of fmath.h. Storage is float32 throughout (the reference
// stores thickness as r16float).
#include <cuda_runtime.h>

#include "fmath.h"
#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "render_common.cuh"

namespace p4a {

namespace {

using namespace render;


// kernelG (src/ssfr_wgsl.js:19-25): the symmetric G from the packed aniso output.
__device__ __forceinline__ Mat3 kernel_g(const float4* __restrict__ g, uint32_t i) {
  const float4 a = __ldg(&g[i * 2u]), b = __ldg(&g[i * 2u + 1u]);
  Mat3 m;
  m.c[0][0] = a.x; m.c[0][1] = a.y; m.c[0][2] = a.z;
  m.c[1][0] = a.y; m.c[1][1] = a.w; m.c[1][2] = b.x;
  m.c[2][0] = a.z; m.c[2][1] = b.x; m.c[2][2] = b.y;
  return m;
}
// kernelInverse (src/ssfr_wgsl.js:27-39)
__device__ __forceinline__ Mat3 kernel_inverse(const float4* __restrict__ g, uint32_t i) {
  const Mat3 m = kernel_g(g, i);
  const float a = m.c[0][0], b = m.c[1][0], c = m.c[2][0];
  const float d = m.c[0][1], e = m.c[1][1], f = m.c[2][1];
  const float gg = m.c[0][2], h = m.c[1][2], k = m.c[2][2];
  const float A = e * k - f * h;
  const float B = f * gg - d * k;
  const float C = d * h - e * gg;
  const float det = a * A + b * B + c * C;
  const float inv = 1.0f / (fabsf(det) < 1.0e-20f ? 1.0e-20f : det);
  Mat3 o;
  o.c[0][0] = A * inv; o.c[0][1] = B * inv; o.c[0][2] = C * inv;
  o.c[1][0] = (c * h - b * k) * inv; o.c[1][1] = (a * k - c * gg) * inv; o.c[1][2] = (b * gg - a * h) * inv;
  o.c[2][0] = (b * f - c * e) * inv; o.c[2][1] = (c * d - a * f) * inv; o.c[2][2] = (a * e - b * d) * inv;
  return o;
}

// The vertex shader (src/ssfr_wgsl.js:48-83): the covered pixel rectangle
// [x0, x1) x [y0, y1) of particle ii, or false when the quad is culled or clipped.
struct Quad {
  int x0, x1, y0, y1;
};
__device__ __forceinline__ bool splat_quad(const SsfrSplat& S, const float4* __restrict__ smoothPos,
                                           const float4* __restrict__ g, const uint4* __restrict__ phase,
                                           uint32_t ii, Quad& q) {
  const float4 c4 = __ldg(&smoothPos[ii]);
  if (S.skipBodies != 0u && __ldg(&phase[ii]).x != 0u) return false;
  if (S.maxNeighbours > 0.0f && __ldg(&g[ii * 2u + 1u]).w > S.maxNeighbours) return false;
  const V4 ec = mat_vec4(S.view, {c4.x, c4.y, c4.z, 1.0f});
  const float zeye = fmaxf(-ec.z, 1.0e-4f);
  const V4 clip = mat_vec4(S.proj, ec);
  F3 e;
  if (S.quadRadius > 0.0f) {
    e = {S.quadRadius, S.quadRadius, S.quadRadius};
  } else {
    Mat3 v3;
#pragma unroll
    for (int cc = 0; cc < 3; cc++)
#pragma unroll
      for (int r = 0; r < 3; r++) v3.c[cc][r] = S.view[cc * 4 + r];
    Mat3 ki = kernel_inverse(g, ii);
#pragma unroll
    for (int cc = 0; cc < 3; cc++)
#pragma unroll
      for (int r = 0; r < 3; r++) ki.c[cc][r] = ki.c[cc][r] * S.kernelScale;
    const Mat3 M = mat3_mul(v3, ki);
    e = {len3({M.c[0][0], M.c[1][0], M.c[2][0]}), len3({M.c[0][1], M.c[1][1], M.c[2][1]}),
         len3({M.c[0][2], M.c[1][2], M.c[2][2]})};
  }
  const float znear = fmaxf(zeye - e.z, 1.0e-4f);
  const float hx = S.proj[0] * e.x / znear, hy = S.proj[5] * e.y / znear;
  // clipping: all four corners share clip.z and clip.w (WebGPU keeps 0 <= z <= w)
  if (!(clip.w > 0.0f) || clip.z < 0.0f || clip.z > clip.w) return false;
  // corners clip.xy +- hsize * clip.w, to framebuffer coordinates
  const float lx = clip.x - hx * clip.w, rx = clip.x + hx * clip.w;
  const float ty = clip.y + hy * clip.w, by = clip.y - hy * clip.w;
  const float fx0 = (lx / clip.w * 0.5f + 0.5f) * S.vw, fx1 = (rx / clip.w * 0.5f + 0.5f) * S.vw;
  const float fy0 = (0.5f - ty / clip.w * 0.5f) * S.vh, fy1 = (0.5f - by / clip.w * 0.5f) * S.vh;
  // pixels px with fx0 <= px + 0.5 < fx1
  const float a0 = fmaxf(ceilf(fx0 - 0.5f), 0.0f), a1 = fminf(ceilf(fx1 - 0.5f), S.vw);
  const float b0 = fmaxf(ceilf(fy0 - 0.5f), 0.0f), b1 = fminf(ceilf(fy1 - 0.5f), S.vh);
  if (!(a0 < a1) || !(b0 < b1)) return false;
  q.x0 = (int)a0; q.x1 = (int)a1; q.y0 = (int)b0; q.y1 = (int)b1;
  return true;
}

// fragmentRay (src/ssfr_wgsl.js:110-119)
__device__ __forceinline__ void fragment_ray(const float* ivp, float vw, float vh, float fx, float fy, F3& ro,
                                             F3& rd) {
  const float nx = fx / vw * 2.0f - 1.0f, ny = 1.0f - fy / vh * 2.0f;
  const V4 nh = mat_vec4(ivp, {nx, ny, -1.0f, 1.0f});
  const V4 fh = mat_vec4(ivp, {nx, ny, 1.0f, 1.0f});
  ro = {nh.x / nh.w, nh.y / nh.w, nh.z / nh.w};
  rd = normalize3(sub3({fh.x / fh.w, fh.y / fh.w, fh.z / fh.w}, ro));
}
__device__ __forceinline__ void ndc_ray(const float* ivp, float nx, float ny, F3& ro, F3& rd) {
  const V4 nh = mat_vec4(ivp, {nx, ny, -1.0f, 1.0f});
  const V4 fh = mat_vec4(ivp, {nx, ny, 1.0f, 1.0f});
  ro = {nh.x / nh.w, nh.y / nh.w, nh.z / nh.w};
  rd = normalize3(sub3({fh.x / fh.w, fh.y / fh.w, fh.z / fh.w}, ro));
}

// The depth fragment (src/ssfr_wgsl.js:85-108, 122-139): false on a miss; else the
// depth the test compares and the eye-space z.
__device__ __forceinline__ bool depth_fragment(const SsfrSplat& S, const float4* __restrict__ smoothPos,
                                               const float4* __restrict__ g, uint32_t ii, int px, int py,
                                               float& depth, float& eyeZ) {
  const float4 c4 = __ldg(&smoothPos[ii]);
  const F3 centre = {c4.x, c4.y, c4.z};
  F3 ro, rd;
  fragment_ray(S.ivp, S.vw, S.vh, (float)px + 0.5f, (float)py + 0.5f, ro, rd);
  Mat3 G = kernel_g(g, ii);
  const float sc = 1.0f / S.kernelScale;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int r = 0; r < 3; r++) G.c[c][r] = G.c[c][r] * sc;
  const F3 oc = sub3(ro, centre);
  const F3 ga = mat3_vec(G, rd), gb = mat3_vec(G, oc);
  const float A = dot3(ga, ga);
  const float B = 2.0f * dot3(ga, gb);
  const float C = dot3(gb, gb) - 1.0f;
  const float disc = B * B - 4.0f * A * C;
  if (disc <= 0.0f || A <= 0.0f) return false;
  const float sq = sqrtf(disc);
  const float t = (-B - sq) / (2.0f * A);
  if (!(t > 0.0f)) return false;
  const F3 p = {ro.x + rd.x * t, ro.y + rd.y * t, ro.z + rd.z * t};
  const V4 ve = mat_vec4(S.view, {p.x, p.y, p.z, 1.0f});
  const V4 cl = mat_vec4(S.pv, {p.x, p.y, p.z, 1.0f});  // (proj * view) * p, as the shader groups it
  depth = clampf(cl.z / cl.w, 0.0f, 1.0f);
  eyeZ = ve.z;
  return true;
}

__global__ void k_ssfr_depth(const __grid_constant__ SsfrSplat S, const float4* __restrict__ smoothPos,
                             const float4* __restrict__ g, const uint4* __restrict__ phase,
                             unsigned long long* __restrict__ key, int width) {
  const uint32_t ii = blockIdx.x * blockDim.x + threadIdx.x;
  if (ii >= S.count) return;
  Quad q;
  if (!splat_quad(S, smoothPos, g, phase, ii, q)) return;
  for (int py = q.y0; py < q.y1; py++)
    for (int px = q.x0; px < q.x1; px++) {
      float depth, ez;
      if (!depth_fragment(S, smoothPos, g, ii, px, py, depth, ez)) continue;
      if (!(depth < 1.0f)) continue;  // 'less' against the cleared 1.0
      const unsigned long long k = ((unsigned long long)__float_as_uint(depth) << 32) | ii;
      atomicMin(&key[(size_t)py * width + px], k);
    }
}

__global__ void k_ssfr_depth_resolve(const __grid_constant__ SsfrSplat S, const float4* __restrict__ smoothPos,
                                     const float4* __restrict__ g, const unsigned long long* __restrict__ key,
                                     float* __restrict__ eyeZ, float* __restrict__ raw, int width, int height) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
  if (px >= width || py >= height) return;
  const size_t o = (size_t)py * width + px;
  const unsigned long long k = key[o];
  float z = -1.0e4f;
  if (k != ~0ull) {
    float depth;
    depth_fragment(S, smoothPos, g, (uint32_t)(k & 0xffffffffu), px, py, depth, z);
  }
  eyeZ[o] = z;
  raw[o] = z;
}

// thickFS (src/ssfr_wgsl.js:142-153)
__global__ void k_ssfr_thick(const __grid_constant__ SsfrSplat S, const float4* __restrict__ smoothPos,
                             const float4* __restrict__ g, const uint4* __restrict__ phase,
                             unsigned long long* __restrict__ acc, int width) {
  const uint32_t ii = blockIdx.x * blockDim.x + threadIdx.x;
  if (ii >= S.count) return;
  Quad q;
  if (!splat_quad(S, smoothPos, g, phase, ii, q)) return;
  const float4 c4 = __ldg(&smoothPos[ii]);
  const F3 centre = {c4.x, c4.y, c4.z};
  const float r2 = S.thickRadius * S.thickRadius;
  for (int py = q.y0; py < q.y1; py++)
    for (int px = q.x0; px < q.x1; px++) {
      F3 ro, rd;
      fragment_ray(S.ivp, S.vw, S.vh, (float)px + 0.5f, (float)py + 0.5f, ro, rd);
      const F3 oc = sub3(ro, centre);
      const float b = dot3(oc, rd);
      const float c = dot3(oc, oc) - r2;
      const float disc = b * b - c;
      if (disc <= 0.0f) continue;
      const float chord = 2.0f * sqrtf(disc);
      atomicAdd(&acc[(size_t)py * width + px], (unsigned long long)__float2ull_rn(chord * 4294967296.0f));
    }
}

__global__ void k_ssfr_thick_resolve(const unsigned long long* __restrict__ acc, float* __restrict__ thick, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  thick[i] = (float)((double)acc[i] * (1.0 / 4294967296.0));
}

// thickFilterWGSL (src/ssfr_wgsl.js:155-183): one separable pass, weights from
// the host (exp(-i^2 / 2 sigma^2) for i = -size..size).
__global__ void k_ssfr_thick_blur(const __grid_constant__ SsfrBlur B, const float* __restrict__ src,
                                  float* __restrict__ dst, int width, int height) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
  if (px >= width || py >= height) return;
  float sum = 0.0f, wsum = 0.0f;
  for (int i = -B.size; i <= B.size; i++) {
    const int x = min(max(px + B.dirX * i, 0), width - 1), y = min(max(py + B.dirY * i, 0), height - 1);
    const float w = B.w[i + B.size];
    sum = sum + __ldg(&src[(size_t)y * width + x]) * w;
    wsum = wsum + w;
  }
  dst[(size_t)py * width + px] = sum / wsum;
}

// filterWGSL (src/ssfr_wgsl.js:185-338)
__device__ __forceinline__ void narrow_range(float& z, float& w, float& wOther, float& upper, float& lower,
                                             float lowerClamp, float threshold) {
  if (z > upper) {
    w = 0.0f;
    wOther = 0.0f;
  } else if (z < lower) {
    z = lowerClamp;
  } else {
    upper = fmaxf(upper, z + threshold);
    lower = fminf(lower, z - threshold);
  }
}

__global__ void k_ssfr_filter(const __grid_constant__ SsfrFilter F, const float* __restrict__ eyeZ,
                              float* __restrict__ out, int width, int height) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
  if (px >= width || py >= height) return;
  const float zi = __ldg(&eyeZ[(size_t)py * width + px]);
  if (zi < -1.0e3f) {
    out[(size_t)py * width + px] = zi;
    return;
  }
  const float sigma = fmaxf(F.sigmaWorld * F.viewH * F.proj11 / (2.0f * fabsf(zi)), 0.5f);
  int R = (int)fminf(3.0f * sigma, (float)F.maxRadius);
  if (F.clean != 0) R = F.cleanRadius;
  float s = sigma;
  if (F.clean != 0) s = fmaxf((float)R / 3.0f, 1.0e-3f);
  const float inv2s2 = 1.0f / (2.0f * s * s);
  float upperP = zi + F.delta, lowerP = zi - F.delta;
  float upperM = zi + F.delta, lowerM = zi - F.delta;
  const float lowerClamp = zi - F.mu;
  float sum = zi, wsum = 1.0f;
  if (F.clean != 0) {
    float upper = zi + F.delta, lower = zi - F.delta;
    for (int dy = 1; dy <= R; dy++) {
      for (int dx = 1; dx <= R; dx++) {
        const float gw = fm_exp(-(float)(dx * dx + dy * dy) * inv2s2);
        float za = fetch_z(eyeZ, px + dx, py + dy, width, height);
        float zb = fetch_z(eyeZ, px + dx, py - dy, width, height);
        float zc = fetch_z(eyeZ, px - dx, py + dy, width, height);
        float zd = fetch_z(eyeZ, px - dx, py - dy, width, height);
        float wa = gw, wb = gw, wc = gw, wd = gw;
        narrow_range(za, wa, wd, upper, lower, lowerClamp, F.delta);
        narrow_range(zb, wb, wc, upper, lower, lowerClamp, F.delta);
        narrow_range(zc, wc, wb, upper, lower, lowerClamp, F.delta);
        narrow_range(zd, wd, wa, upper, lower, lowerClamp, F.delta);
        sum = sum + za * wa + zb * wb + zc * wc + zd * wd;
        wsum = wsum + wa + wb + wc + wd;
      }
    }
    for (int t = 1; t <= R; t++) {
      const float gw = fm_exp(-(float)(t * t) * inv2s2);
      float zv[4] = {fetch_z(eyeZ, px + t, py, width, height), fetch_z(eyeZ, px - t, py, width, height),
                     fetch_z(eyeZ, px, py + t, width, height), fetch_z(eyeZ, px, py - t, width, height)};
      float wv[4] = {gw, gw, gw, gw};
      narrow_range(zv[0], wv[0], wv[1], upper, lower, lowerClamp, F.delta);
      narrow_range(zv[1], wv[1], wv[0], upper, lower, lowerClamp, F.delta);
      narrow_range(zv[2], wv[2], wv[3], upper, lower, lowerClamp, F.delta);
      narrow_range(zv[3], wv[3], wv[2], upper, lower, lowerClamp, F.delta);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        sum = sum + zv[k] * wv[k];
        wsum = wsum + wv[k];
      }
    }
  } else {
    for (int t = 1; t <= R; t++) {
      float zj = fetch_z(eyeZ, px + F.dirX * t, py + F.dirY * t, width, height);
      float zk = fetch_z(eyeZ, px - F.dirX * t, py - F.dirY * t, width, height);
      const float gw = fm_exp(-(float)(t * t) * inv2s2);
      float wj = gw, wk = gw;
      if (F.mode == 2) {
        narrow_range(zj, wj, wk, upperP, lowerP, lowerClamp, F.delta);
        narrow_range(zk, wk, wj, upperM, lowerM, lowerClamp, F.delta);
        sum = sum + zj * wj + zk * wk;
        wsum = wsum + wj + wk;
      } else {
        if (!(zj < -1.0e3f)) {
          float w = gw;
          if (F.mode == 1) {
            const float dz = zj - zi;
            w = w * fm_exp(-dz * dz / (2.0f * F.rangeSigma * F.rangeSigma));
          }
          sum = sum + w * zj;
          wsum = wsum + w;
        }
        if (!(zk < -1.0e3f)) {
          float w = gw;
          if (F.mode == 1) {
            const float dz = zk - zi;
            w = w * fm_exp(-dz * dz / (2.0f * F.rangeSigma * F.rangeSigma));
          }
          sum = sum + w * zk;
          wsum = wsum + w;
        }
      }
    }
  }
  out[(size_t)py * width + px] = sum / wsum;
}

// bodyDepthFS (src/ssfr_composite_wgsl.js:190-201) on the map grid
__global__ void k_ssfr_body_t(const __grid_constant__ SsfrComp C, const float4* __restrict__ bdata,
                              float* __restrict__ bodyT, int width, int height) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
  if (px >= width || py >= height) return;
  const float nx = ((float)px + 0.5f) / (float)width * 2.0f - 1.0f;
  const float ny = 1.0f - ((float)py + 0.5f) / (float)height * 2.0f;
  float t = 1.0e30f;
  if (C.bodyCount > 0) {
    F3 ro, rd;
    ndc_ray(C.ivp, nx, ny, ro, rd);
    const BodyTrace b = trace_bodies(C, bdata, ro, rd, 60.0f);
    if (b.t >= 0.0f) t = b.t;
  }
  bodyT[(size_t)py * width + px] = t;
}

// compositeFS (src/ssfr_composite_wgsl.js:203-333) on the target grid
__global__ void k_ssfr_composite(const __grid_constant__ SsfrComp C, const float4* __restrict__ bdata,
                                 const float* __restrict__ eyeZ, const float* __restrict__ rawZ,
                                 const float* __restrict__ thickMap, const float* __restrict__ bodyT,
                                 uchar4* __restrict__ image) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= C.width || y >= C.height) return;
  const float fx = (float)x + 0.5f, fy = (float)y + 0.5f;
  const float nx = fx / (float)C.width * 2.0f - 1.0f, ny = 1.0f - fy / (float)C.height * 2.0f;
  const float u = nx * 0.5f + 0.5f, v = 0.5f - ny * 0.5f;
  const int ipx = (int)(fx * C.mapScaleX), ipy = (int)(fy * C.mapScaleY);
  const int lw = C.mapW, lh = C.mapH;
  const float z = __ldg(&eyeZ[(size_t)ipy * lw + ipx]);
  // bilinear sample of the thickness map (clamp to edge), texel centres at (i + 0.5) / size
  float thick;
  {
    const float tu = u * (float)C.thickW - 0.5f, tv = v * (float)C.thickH - 0.5f;
    const float fu = floorf(tu), fv = floorf(tv);
    const float au = tu - fu, av = tv - fv;
    const int i0 = min(max((int)fu, 0), C.thickW - 1), i1 = min(max((int)fu + 1, 0), C.thickW - 1);
    const int j0 = min(max((int)fv, 0), C.thickH - 1), j1 = min(max((int)fv + 1, 0), C.thickH - 1);
    const float t00 = __ldg(&thickMap[(size_t)j0 * C.thickW + i0]), t10 = __ldg(&thickMap[(size_t)j0 * C.thickW + i1]);
    const float t01 = __ldg(&thickMap[(size_t)j1 * C.thickW + i0]), t11 = __ldg(&thickMap[(size_t)j1 * C.thickW + i1]);
    const float top = t00 * (1.0f - au) + t10 * au, bot = t01 * (1.0f - au) + t11 * au;
    thick = (top * (1.0f - av) + bot * av) * C.thicknessScale;
  }
  F3 ro, rd;
  ndc_ray(C.ivp, nx, ny, ro, rd);
  uchar4 out;
  if (C.debug == 3) {
    out = to_unorm8({thick, thick * 0.25f, 0.0f});
  } else if (C.debug == 2 || C.debug == 4) {
    const float d = C.debug == 4 ? __ldg(&rawZ[(size_t)ipy * lw + ipx]) : z;
    float s = 0.0f;
    if (!(d < -1.0e3f)) s = clampf(-d / 4.0f, 0.0f, 1.0f);
    out = to_unorm8({1.0f - s, 1.0f - s, 1.0f - s});
  } else {
    const float tBody = __ldg(&bodyT[(size_t)ipy * lw + ipx]);
    if (C.debug == 5) {
      out = tBody > 1.0e29f ? to_unorm8({0.0f, 0.0f, 0.6f}) : to_unorm8({fract1(tBody), fract1(tBody * 0.1f), 0.0f});
    } else {
      const F3 p0 = view_pos(C, nx, ny, z);
      const V4 pw = mat_vec4(C.iv, {p0.x, p0.y, p0.z, 1.0f});
      const F3 p = {pw.x, pw.y, pw.z};
      const bool bodyInFront = tBody < len3(sub3(p, ro));
      if (z < -1.0e3f || bodyInFront) {
        out = to_unorm8(tonemap(C, scene_color(C, bdata, ro, rd)));
      } else {
        const float pxs = 2.0f / (float)lw, pys = 2.0f / (float)lh;
        const float zxp = fetch_z(eyeZ, ipx + 1, ipy, lw, lh), zxm = fetch_z(eyeZ, ipx - 1, ipy, lw, lh);
        const float zyp = fetch_z(eyeZ, ipx, ipy - 1, lw, lh), zym = fetch_z(eyeZ, ipx, ipy + 1, lw, lh);
        const F3 dxr = sub3(view_pos(C, nx + pxs, ny, zxp), p0);
        const F3 dxl = sub3(p0, view_pos(C, nx - pxs, ny, zxm));
        const F3 dyt = sub3(view_pos(C, nx, ny + pys, zyp), p0);
        const F3 dyb = sub3(p0, view_pos(C, nx, ny - pys, zym));
        const F3 dpx = fabsf(dxr.z) < fabsf(dxl.z) ? dxr : dxl;
        const F3 dpy = fabsf(dyt.z) < fabsf(dyb.z) ? dyt : dyb;
        const F3 nView = normalize3(cross3(dpx, dpy));
        Mat3 iv3;
#pragma unroll
        for (int cc = 0; cc < 3; cc++)
#pragma unroll
          for (int r = 0; r < 3; r++) iv3.c[cc][r] = C.iv[cc * 4 + r];
        F3 n = normalize3(mat3_vec(iv3, nView));
        if (n.x != n.x || n.y != n.y || n.z != n.z) n = {-rd.x, -rd.y, -rd.z};
        if (dot3(n, rd) > 0.0f) n = {-n.x, -n.y, -n.z};
        if (C.debug == 1) {
          out = to_unorm8({n.x * 0.5f + 0.5f, n.y * 0.5f + 0.5f, n.z * 0.5f + 0.5f});
        } else {
          const F3 mrd = {-rd.x, -rd.y, -rd.z};
          const float kS = fresnel_full(fmaxf(dot3(mrd, n), 0.0f), 1.0f, C.ior);
          const F3 refl = water_reflect(C, reflect3(rd, n), n);
          F3 refrDir = refract3(rd, n, 1.0f / C.ior);
          if (dot3(refrDir, refrDir) < 1.0e-8f) refrDir = reflect3(rd, n);
          const F3 ro2 = {p.x + refrDir.x * 1.0e-3f, p.y + refrDir.y * 1.0e-3f, p.z + refrDir.z * 1.0e-3f};
          const BodyTrace st = trace_bodies(C, bdata, ro2, refrDir, 60.0f);
          F3 hitCol;
          if (st.t >= 0.0f) {
            const F3 sp = {ro2.x + refrDir.x * st.t, ro2.y + refrDir.y * st.t, ro2.z + refrDir.z * st.t};
            (void)sp;
            hitCol = shade_body(C, st.nrm, st.col, refrDir, env_reflect(C, reflect3(refrDir, st.nrm)));
            thick = fminf(thick, st.t);
          } else {
            hitCol = background(C, ro2, refrDir);
          }
          const F3 trans = {hitCol.x * fm_exp(-C.absorb[0] * thick), hitCol.y * fm_exp(-C.absorb[1] * thick),
                            hitCol.z * fm_exp(-C.absorb[2] * thick)};
          F3 col = lerp3(trans, refl, kS);
          const float gs = ggx_spec(n, mrd, f3(C.sunDir), C.roughness);
          col = {col.x + 1.0f * C.sunIntensity * gs * kS, col.y + 0.97f * C.sunIntensity * gs * kS,
                 col.z + 0.90f * C.sunIntensity * gs * kS};
          out = to_unorm8(tonemap(C, col));
        }
      }
    }
  }
  image[(size_t)y * C.width + x] = out;
}

}  // namespace

void launch_ssfr(const SsfrFrame& f, cudaStream_t st) {
  const int tpb = 128;
  const int64_t mapN = (int64_t)f.mapW * f.mapH, thN = (int64_t)f.thickW * f.thickH;
  cudaMemsetAsync(f.depthKey, 0xff, (size_t)mapN * 8, st);
  cudaMemsetAsync(f.thickAcc, 0, (size_t)thN * 8, st);
  const dim3 mapGrid((f.mapW + tpb - 1) / tpb, f.mapH), thGrid((f.thickW + tpb - 1) / tpb, f.thickH);
  count_launches(1);
  k_ssfr_body_t<<<mapGrid, tpb, 0, st>>>(f.comp, f.bodies, f.bodyT, f.mapW, f.mapH);
  if (f.depth.count > 0) {
    count_launches(1);
    k_ssfr_depth<<<(f.depth.count + tpb - 1) / tpb, tpb, 0, st>>>(f.depth, f.smoothPos, f.g, f.phase, f.depthKey,
                                                                  f.mapW);
    count_launches(1);
    k_ssfr_thick<<<(f.thick.count + tpb - 1) / tpb, tpb, 0, st>>>(f.thick, f.smoothPos, f.g, f.phase, f.thickAcc,
                                                                  f.thickW);
  }
  count_launches(1);
  k_ssfr_depth_resolve<<<mapGrid, tpb, 0, st>>>(f.depth, f.smoothPos, f.g, f.depthKey, f.eyeZ[0], f.raw, f.mapW,
                                               f.mapH);
  count_launches(1);
  k_ssfr_thick_resolve<<<(int)((thN + 255) / 256), 256, 0, st>>>(f.thickAcc, f.thickMap, (int)thN);
  if (f.blur[0].size > 0) {
    count_launches(1);
    k_ssfr_thick_blur<<<thGrid, tpb, 0, st>>>(f.blur[0], f.thickMap, f.thickTmp, f.thickW, f.thickH);
    count_launches(1);
    k_ssfr_thick_blur<<<thGrid, tpb, 0, st>>>(f.blur[1], f.thickTmp, f.thickMap, f.thickW, f.thickH);
  }
  int src = 0;
  for (int p = 0; p < f.filterPasses; p++) {
    count_launches(1);
    k_ssfr_filter<<<mapGrid, tpb, 0, st>>>(f.filter[f.filterSlot[p]], f.eyeZ[src], f.eyeZ[1 - src], f.mapW, f.mapH);
    src = 1 - src;
  }
  const dim3 tgtGrid((f.comp.width + tpb - 1) / tpb, f.comp.height);
  count_launches(1);
  k_ssfr_composite<<<tgtGrid, tpb, 0, st>>>(f.comp, f.bodies, f.eyeZ[src], f.raw, f.thickMap, f.bodyT, f.image);
}

}  // namespace p4a
