// kernels_ray.cu — the ray-marched fluid surface (src/ray.js:30-97,
// src/ray_wgsl.js:1-549) as a CUDA pass writing a headless RGBA8 image. One thread
// per pixel: the eye ray is clipped to the density field's volume, walked cell by
// cell through the voxel grid (3D DDA), and in each cell the trilinear field along
// the segment is fitted with a cubic whose iso crossing is bracketed at the cubic's
// turning points and refined by 12 regula-falsi steps; rigid bodies are traced as
// signed distance fields; the surface is shaded with Fresnel reflection, refraction
// through an optical depth integrated along the refracted ray, and a GGX sun
// highlight, then tone-mapped. With useSurface (the reference's default) the
// surface comes instead from the mesh's triangles drawn into an eye-depth map and a
// normal map (the surface pass below: a triangle per thread, pixel centres inside
// the triangle or on its edges, depth test 'less' as an atomicMin of (depth bits,
// triangle), perspective-correct world position and normal in a resolve pass;
// triangles are clipped to 0 <= z <= w first, their visible part drawn as a fan).
// The field is the one p4a_mesh produced (SurfaceMesh.generateField + smoothField).
// Float contract as in kernels_ssfr.cu; acos in debug view 5 is replaced by the
// equivalent comparison of |n.y| against the cosines of the thresholds.
#include <cuda_runtime.h>

#include <algorithm>

#include "fmath.h"
#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "render_common.cuh"

namespace p4a {

namespace {

using namespace render;

struct Cell {
  float d000, d100, d010, d110, d001, d101, d011, d111;
};

__device__ __forceinline__ float fget(const RayParams& R, const float* __restrict__ field, int x, int y, int z) {
  x = min(max(x, 0), R.vertDim[0] - 1);
  y = min(max(y, 0), R.vertDim[1] - 1);
  z = min(max(z, 0), R.vertDim[2] - 1);
  return __ldg(&field[((size_t)z * R.vertDim[1] + y) * R.vertDim[0] + x]);
}
__device__ __forceinline__ Cell cell_at(const RayParams& R, const float* __restrict__ field, int cx, int cy, int cz) {
  Cell k;
  k.d000 = fget(R, field, cx, cy, cz);
  k.d100 = fget(R, field, cx + 1, cy, cz);
  k.d010 = fget(R, field, cx, cy + 1, cz);
  k.d110 = fget(R, field, cx + 1, cy + 1, cz);
  k.d001 = fget(R, field, cx, cy, cz + 1);
  k.d101 = fget(R, field, cx + 1, cy, cz + 1);
  k.d011 = fget(R, field, cx, cy + 1, cz + 1);
  k.d111 = fget(R, field, cx + 1, cy + 1, cz + 1);
  return k;
}
__device__ __forceinline__ float tri_local(const Cell& k, F3 u) {
  const float x00 = lerpf(k.d000, k.d100, u.x), x10 = lerpf(k.d010, k.d110, u.x);
  const float x01 = lerpf(k.d001, k.d101, u.x), x11 = lerpf(k.d011, k.d111, u.x);
  return lerpf(lerpf(x00, x10, u.y), lerpf(x01, x11, u.y), u.z);
}
__device__ __forceinline__ float tri_at(const RayParams& R, const float* __restrict__ field, F3 g) {
  const int cx = (int)floorf(g.x), cy = (int)floorf(g.y), cz = (int)floorf(g.z);
  const F3 u = {clampf(g.x - (float)cx, 0.0f, 1.0f), clampf(g.y - (float)cy, 0.0f, 1.0f),
                clampf(g.z - (float)cz, 0.0f, 1.0f)};
  return tri_local(cell_at(R, field, cx, cy, cz), u);
}
__device__ __forceinline__ F3 smooth_normal(const RayParams& R, const float* __restrict__ field, F3 g) {
  return {tri_at(R, field, {g.x + 1.0f, g.y, g.z}) - tri_at(R, field, {g.x - 1.0f, g.y, g.z}),
          tri_at(R, field, {g.x, g.y + 1.0f, g.z}) - tri_at(R, field, {g.x, g.y - 1.0f, g.z}),
          tri_at(R, field, {g.x, g.y, g.z + 1.0f}) - tri_at(R, field, {g.x, g.y, g.z - 1.0f})};
}
__device__ __forceinline__ F3 grad_local(const Cell& k, F3 u) {
  const float ox = 1.0f - u.x, oy = 1.0f - u.y, oz = 1.0f - u.z;
  const float gx = (k.d100 - k.d000) * oy * oz + (k.d110 - k.d010) * u.y * oz + (k.d101 - k.d001) * oy * u.z +
                   (k.d111 - k.d011) * u.y * u.z;
  const float gy = (k.d010 - k.d000) * ox * oz + (k.d110 - k.d100) * u.x * oz + (k.d011 - k.d001) * ox * u.z +
                   (k.d111 - k.d101) * u.x * u.z;
  const float gz = (k.d001 - k.d000) * ox * oy + (k.d101 - k.d100) * u.x * oy + (k.d011 - k.d010) * ox * u.y +
                   (k.d111 - k.d110) * u.x * u.y;
  return {gx, gy, gz};
}
struct Cubic {
  float A, B, C, D;
};
__device__ __forceinline__ Cubic cubic_of(const Cell& k, F3 u0, F3 du) {
  const float third = (float)(1.0 / 3.0), twoThirds = (float)(2.0 / 3.0);
  const float f0 = tri_local(k, u0);
  const float f1 = tri_local(k, {u0.x + du.x * third, u0.y + du.y * third, u0.z + du.z * third});
  const float f2 = tri_local(k, {u0.x + du.x * twoThirds, u0.y + du.y * twoThirds, u0.z + du.z * twoThirds});
  const float f3v = tri_local(k, {u0.x + du.x, u0.y + du.y, u0.z + du.z});
  const float g1 = f1 - f0, g2 = f2 - f0, g3 = f3v - f0;
  Cubic c;
  c.A = 4.5f * (3.0f * g1 - 3.0f * g2 + g3);
  c.B = -(27.0f * g1 - 9.0f * g3 + 8.0f * c.A) / 6.0f;
  c.C = g3 - c.A - c.B;
  c.D = f0;
  return c;
}
__device__ __forceinline__ float cubic_at(const Cubic& c, float t) { return ((c.A * t + c.B) * t + c.C) * t + c.D; }
__device__ __forceinline__ float solve_monotone(const Cubic& c, float iso, float lo, float hi, float vlo, float vhi) {
  float t = lo;
  for (int i = 0; i < 12; i++) {
    t = lo + (hi - lo) * (-vlo) / fmaxf(vhi - vlo, 1.0e-9f);
    t = clampf(t, lo, hi);
    const float v = cubic_at(c, t) - iso;
    if (v * vlo > 0.0f) {
      lo = t;
      vlo = v;
    } else {
      hi = t;
      vhi = v;
    }
  }
  return t;
}
__device__ __forceinline__ float segment_crossing(const Cell& k, F3 u0, F3 du, float iso) {
  const Cubic c = cubic_of(k, u0, du);
  float e0 = 2.0f, e1 = 2.0f;
  const float a = 3.0f * c.A, b = 2.0f * c.B, cc = c.C;
  if (fabsf(a) > 1.0e-12f) {
    const float disc = b * b - 4.0f * a * cc;
    if (disc > 0.0f) {
      const float sq = sqrtf(disc);
      const float r0 = (-b - sq) / (2.0f * a), r1 = (-b + sq) / (2.0f * a);
      e0 = fminf(r0, r1);
      e1 = fmaxf(r0, r1);
    }
  } else if (fabsf(b) > 1.0e-12f) {
    e0 = -cc / b;
  }
  float bounds[4] = {0.0f, 1.0f, 1.0f, 1.0f};
  int n = 1;
  if (e0 > 0.0f && e0 < 1.0f) bounds[n++] = e0;
  if (e1 > 0.0f && e1 < 1.0f && e1 > e0) bounds[n++] = e1;
  bounds[n++] = 1.0f;
  float lo = bounds[0];
  float vlo = cubic_at(c, lo) - iso;
  for (int i = 1; i < n; i++) {
    const float hi = bounds[i];
    const float vhi = cubic_at(c, hi) - iso;
    if ((vlo <= 0.0f && vhi >= 0.0f) || (vlo >= 0.0f && vhi <= 0.0f)) return solve_monotone(c, iso, lo, hi, vlo, vhi);
    lo = hi;
    vlo = vhi;
  }
  return -1.0f;
}
struct Slab {
  bool hit;
  float t0, t1;
};
__device__ __forceinline__ Slab box_hit(F3 o, F3 d, F3 lo, F3 hi) {
  const F3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  const F3 a = {(lo.x - o.x) * inv.x, (lo.y - o.y) * inv.y, (lo.z - o.z) * inv.z};
  const F3 b = {(hi.x - o.x) * inv.x, (hi.y - o.y) * inv.y, (hi.z - o.z) * inv.z};
  const F3 tmin = {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)};
  const F3 tmax = {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)};
  Slab s;
  s.t0 = fmaxf(fmaxf(tmin.x, tmin.y), tmin.z);
  s.t1 = fminf(fminf(tmax.x, tmax.y), tmax.z);
  s.hit = s.t1 > fmaxf(s.t0, 0.0f);
  return s;
}
__device__ __forceinline__ float body_scene_dist(const RayParams& R, const float4* __restrict__ bdata, F3 p) {
  float dist = 1.0e30f;
  for (int i = 0; i < R.bodyCount; i++) {
    const float d = body_dist(bdata, i, p);
    if (d < dist) dist = d;
  }
  return dist;
}
__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

struct March {
  float t;
  F3 pos, nrm;
};
__device__ __forceinline__ March march(const RayParams& R, const float* __restrict__ field,
                                       const float4* __restrict__ bdata, F3 ro, F3 rd, float tStart, float tEnd) {
  March out;
  out.t = -1.0f;
  out.pos = {0.f, 0.f, 0.f};
  out.nrm = {0.0f, 1.0f, 0.0f};
  const F3 go = f3(R.gridOrigin);
  const F3 g0 = {(ro.x - go.x) / R.voxel, (ro.y - go.y) / R.voxel, (ro.z - go.z) / R.voxel};
  const F3 gd = {rd.x / R.voxel, rd.y / R.voxel, rd.z / R.voxel};
  const F3 p0 = {g0.x + gd.x * tStart, g0.y + gd.y * tStart, g0.z + gd.z * tStart};
  int c[3] = {min(max((int)floorf(p0.x), 0), R.vertDim[0] - 2), min(max((int)floorf(p0.y), 0), R.vertDim[1] - 2),
              min(max((int)floorf(p0.z), 0), R.vertDim[2] - 2)};
  const int stp[3] = {(int)signf(gd.x), (int)signf(gd.y), (int)signf(gd.z)};
  const float gda[3] = {gd.x, gd.y, gd.z}, g0a[3] = {g0.x, g0.y, g0.z};
  float tMax[3], tDelta[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float invD = 1.0f / fmaxf(fabsf(gda[a]), 1.0e-12f);
    const float nextEdge = (float)c[a] + fmaxf((float)stp[a], 0.0f);
    tMax[a] = (nextEdge - g0a[a]) / gda[a];
    tDelta[a] = invD;
    if (gda[a] == 0.0f) {
      tMax[a] = 1.0e30f;
      tDelta[a] = 1.0e30f;
    }
  }
  float t = tStart;
  for (int i = 0; i < 4096; i++) {
    const float tNext = fminf(fminf(tMax[0], tMax[1]), tMax[2]);
    const float segEnd = fminf(tNext, tEnd);
    if (segEnd > t) {
      const Cell k = cell_at(R, field, c[0], c[1], c[2]);
      const F3 u0 = {g0.x + gd.x * t - (float)c[0], g0.y + gd.y * t - (float)c[1], g0.z + gd.z * t - (float)c[2]};
      const float span = segEnd - t;
      const F3 du = {gd.x * span, gd.y * span, gd.z * span};
      const float s = segment_crossing(k, u0, du, R.iso);
      if (s >= 0.0f) {
        const float tHit = t + s * (segEnd - t);
        const F3 p = {ro.x + rd.x * tHit, ro.y + rd.y * tHit, ro.z + rd.z * tHit};
        bool inside = false;
        if (R.bodyCount > 0) inside = body_scene_dist(R, bdata, p) < 0.0f;
        if (!inside) {
          out.t = tHit;
          out.pos = p;
          out.nrm = grad_local(k, {clampf(u0.x + du.x * s, 0.0f, 1.0f), clampf(u0.y + du.y * s, 0.0f, 1.0f),
                                   clampf(u0.z + du.z * s, 0.0f, 1.0f)});
          return out;
        }
      }
    }
    t = tNext;
    if (t >= tEnd) break;
    if (tMax[0] <= tMax[1] && tMax[0] <= tMax[2]) {
      c[0] += stp[0];
      tMax[0] += tDelta[0];
    } else if (tMax[1] <= tMax[2]) {
      c[1] += stp[1];
      tMax[1] += tDelta[1];
    } else {
      c[2] += stp[2];
      tMax[2] += tDelta[2];
    }
    if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] > R.vertDim[0] - 2 || c[1] > R.vertDim[1] - 2 ||
        c[2] > R.vertDim[2] - 2)
      break;
  }
  return out;
}
__device__ __forceinline__ float optical_depth(const RayParams& R, const float* __restrict__ field, F3 ro, F3 rd,
                                               float tMax) {
  const F3 lo = f3(R.gridOrigin);
  const F3 hi = {lo.x + R.voxel * (float)(R.vertDim[0] - 1), lo.y + R.voxel * (float)(R.vertDim[1] - 1),
                 lo.z + R.voxel * (float)(R.vertDim[2] - 1)};
  const Slab s = box_hit(ro, rd, lo, hi);
  if (!s.hit) return 0.0f;
  const float a = fmaxf(s.t0, 0.0f);
  const float b = fminf(fmaxf(s.t1, 0.0f), tMax);
  if (b <= a) return 0.0f;
  const float dt = (b - a) / (float)R.thickSteps;
  float acc = 0.0f;
  for (int i = 0; i < R.thickSteps; i++) {
    const float t = a + ((float)i + 0.5f) * dt;
    const F3 q = {(ro.x + rd.x * t - lo.x) / R.voxel, (ro.y + rd.y * t - lo.y) / R.voxel,
                  (ro.z + rd.z * t - lo.z) / R.voxel};
    acc += smooth(R.iso * 0.55f, R.iso * 1.45f, tri_at(R, field, q));
  }
  return acc * dt;
}

// ---- mesh surface pass ----
struct SurfGrid {
  float origin[3], voxel;
  int32_t dim[3];
};
// meshDrawWGSL vs (src/mesh_wgsl.js:268-286): a packed vertex to world position and
// unit normal.
__device__ __forceinline__ void unpack_vertex(const SurfGrid& G, uint2 v, F3& p, F3& n) {
  const float px = (float)(v.x & 0xFFFFu) / 65535.0f, py = (float)(v.x >> 16) / 65535.0f,
              pz = (float)(v.y & 0xFFFFu) / 65535.0f;
  p = {G.origin[0] + px * (float)(G.dim[0] - 1) * G.voxel, G.origin[1] + py * (float)(G.dim[1] - 1) * G.voxel,
       G.origin[2] + pz * (float)(G.dim[2] - 1) * G.voxel};
  const uint32_t oct = v.y >> 16;
  const float ex = (float)(oct & 0xFFu) / 255.0f * 2.0f - 1.0f, ey = (float)(oct >> 8) / 255.0f * 2.0f - 1.0f;
  F3 m = {ex, ey, 1.0f - fabsf(ex) - fabsf(ey)};
  if (m.z < 0.0f) {
    const float tx = (1.0f - fabsf(m.y)) * (m.x >= 0.0f ? 1.0f : -1.0f);
    const float ty = (1.0f - fabsf(m.x)) * (m.y >= 0.0f ? 1.0f : -1.0f);
    m = {tx, ty, m.z};
  }
  n = normalize3(m);
}
// A vertex of a triangle's visible part: clip coordinates, world position, normal.
struct SVert {
  V4 c;
  F3 p, n;
};
constexpr int kClipMax = 5;  // a triangle cut by the two depth planes keeps at most 5 vertices
__device__ __forceinline__ SVert lerp_vert(const SVert& A, const SVert& B, float t) {
  SVert o;
  o.c = {A.c.x + t * (B.c.x - A.c.x), A.c.y + t * (B.c.y - A.c.y), A.c.z + t * (B.c.z - A.c.z),
         A.c.w + t * (B.c.w - A.c.w)};
  o.p = {A.p.x + t * (B.p.x - A.p.x), A.p.y + t * (B.p.y - A.p.y), A.p.z + t * (B.p.z - A.p.z)};
  o.n = {A.n.x + t * (B.n.x - A.n.x), A.n.y + t * (B.n.y - A.n.y), A.n.z + t * (B.n.z - A.n.z)};
  return o;
}
// One Sutherland-Hodgman step: the part of polygon in[0..m) where the plane's
// distance (z for the near plane, w - z for the far one) is >= 0, at most `cap`
// vertices. Clip-space attributes are affine in clip space, so the cut vertices
// interpolate them linearly, as the rasteriser's clipper does.
template <bool Far>
__device__ __forceinline__ int clip_plane(const SVert* in, int m, SVert* out, int cap) {
  int k = 0;
  for (int a = 0; a < m; a++) {
    const SVert& A = in[a];
    const SVert& B = in[a + 1 < m ? a + 1 : 0];
    const float da = Far ? A.c.w - A.c.z : A.c.z, db = Far ? B.c.w - B.c.z : B.c.z;
    if (da >= 0.0f && k < cap) out[k++] = A;
    if ((da >= 0.0f) != (db >= 0.0f) && k < cap) out[k++] = lerp_vert(A, B, da / (da - db));
  }
  return k;
}
// Triangle t clipped to 0 <= z <= w: its visible part as a convex polygon P[0..m),
// drawn as the fan (P[0], P[s + 1], P[s + 2]), s < m - 2. Returns m (< 3: nothing).
__device__ __forceinline__ int clip_triangle(const RayParams& R, const SurfGrid& G, const uint2* __restrict__ verts,
                                             uint32_t t, SVert P[kClipMax]) {
  SVert a[3], b[kClipMax - 1];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    unpack_vertex(G, __ldg(&verts[3 * (size_t)t + k]), a[k].p, a[k].n);
    a[k].c = mat_vec4(R.vp, {a[k].p.x, a[k].p.y, a[k].p.z, 1.0f});
  }
  const int m = clip_plane<false>(a, 3, b, kClipMax - 1);
  return clip_plane<true>(b, m, P, kClipMax);
}
struct Tri {
  V4 clip[3];
  F3 p[3], n[3];
  float sx[3], sy[3], sz[3], area;
};
// Fan triangle s of polygon P in screen space; false when it has no area or a
// vertex at or behind the eye.
__device__ __forceinline__ bool fan_tri(const RayParams& R, const SVert* P, int s, Tri& T) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const SVert& v = P[k == 0 ? 0 : s + k];
    T.clip[k] = v.c;
    T.p[k] = v.p;
    T.n[k] = v.n;
    if (!(v.c.w > 0.0f)) return false;
    T.sx[k] = (v.c.x / v.c.w * 0.5f + 0.5f) * (float)R.width;
    T.sy[k] = (0.5f - v.c.y / v.c.w * 0.5f) * (float)R.height;
    T.sz[k] = v.c.z / v.c.w;
  }
  T.area = (T.sx[1] - T.sx[0]) * (T.sy[2] - T.sy[0]) - (T.sx[2] - T.sx[0]) * (T.sy[1] - T.sy[0]);
  return T.area != 0.0f;
}
// Screen-space barycentrics of the pixel centre (cx, cy), normalised so that the
// inside is b >= 0 for either winding; false outside.
__device__ __forceinline__ bool bary(const Tri& T, float cx, float cy, float b[3]) {
  float w0 = (T.sx[2] - T.sx[1]) * (cy - T.sy[1]) - (T.sy[2] - T.sy[1]) * (cx - T.sx[1]);
  float w1 = (T.sx[0] - T.sx[2]) * (cy - T.sy[2]) - (T.sy[0] - T.sy[2]) * (cx - T.sx[2]);
  float w2 = (T.sx[1] - T.sx[0]) * (cy - T.sy[0]) - (T.sy[1] - T.sy[0]) * (cx - T.sx[0]);
  float a = T.area;
  if (a < 0.0f) {
    w0 = -w0;
    w1 = -w1;
    w2 = -w2;
    a = -a;
  }
  if (w0 < 0.0f || w1 < 0.0f || w2 < 0.0f) return false;
  b[0] = w0 / a;
  b[1] = w1 / a;
  b[2] = w2 / a;
  return true;
}
__global__ void k_surf_raster(const __grid_constant__ RayParams R, const __grid_constant__ SurfGrid G,
                              const uint2* __restrict__ verts, const uint32_t* __restrict__ total, uint32_t cap,
                              unsigned long long* __restrict__ key) {
  const uint32_t count = min(__ldg(total), cap);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    SVert P[kClipMax];
    const int m = clip_triangle(R, G, verts, t, P);
    for (int s = 0; s + 2 < m; s++) {
      Tri T;
      if (!fan_tri(R, P, s, T)) continue;
      const float lo_x = fminf(T.sx[0], fminf(T.sx[1], T.sx[2])), hi_x = fmaxf(T.sx[0], fmaxf(T.sx[1], T.sx[2]));
      const float lo_y = fminf(T.sy[0], fminf(T.sy[1], T.sy[2])), hi_y = fmaxf(T.sy[0], fmaxf(T.sy[1], T.sy[2]));
      // clamped before the conversion, so that infinite or NaN bounds stay in range
      const int x0 = (int)fminf(fmaxf(ceilf(lo_x - 0.5f), 0.0f), (float)R.width);
      const int x1 = (int)fmaxf(fminf(floorf(hi_x - 0.5f), (float)R.width - 1.0f), -1.0f);
      const int y0 = (int)fminf(fmaxf(ceilf(lo_y - 0.5f), 0.0f), (float)R.height);
      const int y1 = (int)fmaxf(fminf(floorf(hi_y - 0.5f), (float)R.height - 1.0f), -1.0f);
      const unsigned long long id = (unsigned long long)(t * 4u + (uint32_t)s);
      for (int py = y0; py <= y1; py++)
        for (int px = x0; px <= x1; px++) {
          float b[3];
          if (!bary(T, (float)px + 0.5f, (float)py + 0.5f, b)) continue;
          // + 0 turns a -0 (a zero weight negated for the winding) into +0, so that the
          // bits of every depth >= 0 order as the values do
          const float depth = b[0] * T.sz[0] + b[1] * T.sz[1] + b[2] * T.sz[2] + 0.0f;
          if (!(depth < 1.0f)) continue;
          atomicMin(&key[(size_t)py * R.width + px], ((unsigned long long)__float_as_uint(depth) << 32) | id);
        }
    }
  }
}
__global__ void k_surf_resolve(const __grid_constant__ RayParams R, const __grid_constant__ SurfGrid G,
                               const uint2* __restrict__ verts, const unsigned long long* __restrict__ key,
                               float* __restrict__ surfZ, float4* __restrict__ surfN) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
  if (px >= R.width || py >= R.height) return;
  const size_t o = (size_t)py * R.width + px;
  const unsigned long long k = key[o];
  float z = -1.0e4f;
  float4 nn = make_float4(0.f, 0.f, 0.f, 0.f);
  if (k != ~0ull) {
    const uint32_t id = (uint32_t)(k & 0xffffffffu), s = id & 3u;
    SVert P[kClipMax];
    const int m = clip_triangle(R, G, verts, id >> 2, P);
    Tri T;
    float b[3];
    if ((int)s + 2 < m && fan_tri(R, P, (int)s, T) && bary(T, (float)px + 0.5f, (float)py + 0.5f, b)) {
      // perspective-correct interpolation of the world position and the normal
      const float q0 = b[0] / T.clip[0].w, q1 = b[1] / T.clip[1].w, q2 = b[2] / T.clip[2].w;
      const float qs = q0 + q1 + q2;
      const F3* p = T.p;
      const F3* n = T.n;
      const F3 wp = {(q0 * p[0].x + q1 * p[1].x + q2 * p[2].x) / qs, (q0 * p[0].y + q1 * p[1].y + q2 * p[2].y) / qs,
                     (q0 * p[0].z + q1 * p[1].z + q2 * p[2].z) / qs};
      const F3 wn = {(q0 * n[0].x + q1 * n[1].x + q2 * n[2].x) / qs, (q0 * n[0].y + q1 * n[1].y + q2 * n[2].y) / qs,
                     (q0 * n[0].z + q1 * n[1].z + q2 * n[2].z) / qs};
      z = mat_vec4(R.view, {wp.x, wp.y, wp.z, 1.0f}).z;  // fsSurf: (V.view * world).z
      const F3 un = normalize3(wn);
      nn = make_float4(un.x, un.y, un.z, 1.0f);
    }
  }
  surfZ[o] = z;
  surfN[o] = nn;
}

__global__ void k_ray(const __grid_constant__ RayParams R, const float* __restrict__ field,
                      const float4* __restrict__ bdata, const float* __restrict__ surfZ,
                      const float4* __restrict__ surfN, uchar4* __restrict__ image) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= R.width || y >= R.height) return;
  const float nx = ((float)x + 0.5f) / (float)R.width * 2.0f - 1.0f;
  const float ny = 1.0f - ((float)y + 0.5f) / (float)R.height * 2.0f;
  const V4 nh = mat_vec4(R.ivp, {nx, ny, -1.0f, 1.0f});
  const V4 fh = mat_vec4(R.ivp, {nx, ny, 1.0f, 1.0f});
  const F3 nearP = {nh.x / nh.w, nh.y / nh.w, nh.z / nh.w}, farP = {fh.x / fh.w, fh.y / fh.w, fh.z / fh.w};
  const F3 ro = f3(R.eye);
  const F3 rd = normalize3(sub3(farP, nearP));
  const F3 volLo = f3(R.gridOrigin);
  const F3 volHi = {volLo.x + R.voxel * (float)(R.vertDim[0] - 1), volLo.y + R.voxel * (float)(R.vertDim[1] - 1),
                    volLo.z + R.voxel * (float)(R.vertDim[2] - 1)};
  float tHit = -1.0f;
  F3 hit = {0.f, 0.f, 0.f};
  F3 meshN = {0.0f, 1.0f, 0.0f};
  if (R.useSurface != 0) {
    // meshSurfaceHit (src/ray_wgsl.js:397-412)
    const size_t o = (size_t)y * R.width + x;
    const float z = __ldg(&surfZ[o]);
    if (!(z < -1.0e3f)) {
      const F3 pv = {-nx * z / R.proj00, -ny * z / R.proj11, z};
      const V4 wv = mat_vec4(R.iv, {pv.x, pv.y, pv.z, 1.0f});
      const float4 n4 = __ldg(&surfN[o]);
      const F3 nv = {n4.x, n4.y, n4.z};
      if (!(dot3(nv, nv) < 1.0e-8f)) {
        hit = {wv.x, wv.y, wv.z};
        meshN = normalize3(nv);
        tHit = len3(sub3(hit, ro));
      }
    }
  } else {
    const Slab slab = box_hit(ro, rd, volLo, volHi);
    if (slab.hit) {
      const March m = march(R, field, bdata, ro, rd, fmaxf(slab.t0, 0.0f) + 1.0e-5f, slab.t1);
      tHit = m.t;
      hit = m.pos;
    }
  }
  float tMaxBody = 60.0f;
  if (tHit >= 0.0f) tMaxBody = tHit + R.skin;
  const BodyTrace bt = trace_bodies(R, bdata, ro, rd, tMaxBody);
  F3 col = {0.f, 0.f, 0.f};
  F3 n = {0.0f, 1.0f, 0.0f};
  float thick = 0.0f;
  if (bt.t >= 0.0f && (tHit < 0.0f || bt.t < tHit + R.skin)) {
    col = shade_body(R, bt.nrm, bt.col, rd, env_reflect(R, reflect3(rd, bt.nrm)));
  } else if (tHit < 0.0f) {
    col = background(R, ro, rd);
  } else {
    if (R.useSurface != 0) {
      n = meshN;
    } else {
      const F3 go = f3(R.gridOrigin);
      const F3 sn =
          smooth_normal(R, field, {(hit.x - go.x) / R.voxel, (hit.y - go.y) / R.voxel, (hit.z - go.z) / R.voxel});
      n = normalize3({-sn.x, -sn.y, -sn.z});
    }
    if (dot3(n, rd) > 0.0f) n = {-n.x, -n.y, -n.z};
    const F3 mrd = {-rd.x, -rd.y, -rd.z};
    const float kS = fresnel_full(fmaxf(dot3(mrd, n), 0.0f), 1.0f, R.ior);
    const F3 reflDir = reflect3(rd, n);
    F3 refrDir = refract3(rd, n, 1.0f / R.ior);
    if (dot3(refrDir, refrDir) < 1.0e-8f) refrDir = reflDir;
    const F3 refl = water_reflect(R, reflDir, n);
    const float off = R.voxel * 0.02f;
    const F3 ro2 = {hit.x + refrDir.x * off, hit.y + refrDir.y * off, hit.z + refrDir.z * off};
    const BodyTrace st = trace_bodies(R, bdata, ro2, refrDir, 60.0f);
    F3 trans;
    if (st.t >= 0.0f) {
      trans = shade_body(R, st.nrm, st.col, refrDir, env_reflect(R, reflect3(refrDir, st.nrm)));
    } else {
      trans = background(R, ro2, refrDir);
    }
    const float tSolid = st.t >= 0.0f ? st.t : 1.0e30f;
    thick = optical_depth(R, field, ro2, refrDir, tSolid);
    trans = {trans.x * fm_exp(-R.absorb[0] * thick), trans.y * fm_exp(-R.absorb[1] * thick),
             trans.z * fm_exp(-R.absorb[2] * thick)};
    col = lerp3(trans, refl, kS);
    const float gs = ggx_spec(n, mrd, f3(R.sunDir), R.roughness);
    col = {col.x + 1.0f * R.sunIntensity * gs * kS, col.y + 0.97f * R.sunIntensity * gs * kS,
           col.z + 0.90f * R.sunIntensity * gs * kS};
  }
  if (R.debug == 1) {
    col = tHit < 0.0f ? F3{0.f, 0.f, 0.f} : F3{n.x * 0.5f + 0.5f, n.y * 0.5f + 0.5f, n.z * 0.5f + 0.5f};
  } else if (R.debug == 2) {
    col = tHit < 0.0f ? F3{0.f, 0.f, 0.f} : F3{fract1(tHit), fract1(tHit * 0.1f), 0.0f};
  } else if (R.debug == 3) {
    col = {thick, thick * 0.25f, 0.0f};
  } else if (R.debug == 4) {
    F3 c4 = {0.1f, 0.3f, 1.0f};
    if (reflect3(rd, n).y < 0.0f) c4 = {1.0f, 0.1f, 0.1f};
    col = tHit < 0.0f ? F3{0.f, 0.f, 0.f} : c4;
  } else if (R.debug == 6) {
    col = tHit < 0.0f ? background(R, ro, rd) : water_reflect(R, reflect3(rd, n), n);
  } else if (R.debug == 5) {
    if (tHit < 0.0f) {
      col = {0.f, 0.f, 0.f};
    } else {
      // degrees(acos(|n.y|)) < 5 / 10 / 20 / 40  <=>  |n.y| > cos of the threshold
      const float a = clampf(fabsf(n.y), 0.0f, 1.0f);
      if (a > R.cosDeg[0]) col = {0.1f, 0.3f, 1.0f};
      else if (a > R.cosDeg[1]) col = {0.1f, 0.9f, 0.9f};
      else if (a > R.cosDeg[2]) col = {0.2f, 0.9f, 0.2f};
      else if (a > R.cosDeg[3]) col = {0.95f, 0.9f, 0.2f};
      else col = {1.0f, 0.15f, 0.1f};
    }
  }
  image[(size_t)y * R.width + x] = to_unorm8(tonemap(R, col));
}

}  // namespace

void launch_surface(const RayParams& R, const uint2* verts, const uint32_t* total, uint32_t cap,
                    const float gridOrigin[3], const int32_t vertDim[3], float voxel,
                    unsigned long long* key, float* surfZ, float4* surfN, cudaStream_t st) {
  SurfGrid G;
  for (int k = 0; k < 3; k++) {
    G.origin[k] = gridOrigin[k];
    G.dim[k] = vertDim[k];
  }
  G.voxel = voxel;
  cudaMemsetAsync(key, 0xff, (size_t)R.width * R.height * 8, st);
  const int tpb = 128;
  if (cap > 0) {
    const int grid = (int)std::min<uint32_t>((cap + tpb - 1) / tpb, 148u * 16u);
    count_launches(1);
    k_surf_raster<<<grid, tpb, 0, st>>>(R, G, verts, total, cap, key);
  }
  const dim3 rgrid((R.width + tpb - 1) / tpb, R.height);
  count_launches(1);
  k_surf_resolve<<<rgrid, tpb, 0, st>>>(R, G, verts, key, surfZ, surfN);
}

void launch_ray(const RayParams& R, const float* field, const float4* bodies, const float* surfZ,
                const float4* surfN, uchar4* image, cudaStream_t st) {
  const int tpb = 128;
  const dim3 grid((R.width + tpb - 1) / tpb, R.height);
  count_launches(1);
  k_ray<<<grid, tpb, 0, st>>>(R, field, bodies, surfZ, surfN, image);
}

}  // namespace p4a
