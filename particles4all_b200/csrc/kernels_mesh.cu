// kernels_mesh.cu — the surface mesh of the simulation (src/mesh_wgsl.js:23-238,
// driven by src/mesh.js:99-340): a density field on the vertices of a voxel grid
// gathered from the particles, 3-tap blur passes, and marching tetrahedra (six
// tetrahedra per voxel) emitting triangles as packed vertices (16-bit grid
// position, octahedral normal).
//
// The reference appends triangles through an atomic counter, so its triangle order
// is whatever the atomics produce. Here a count pass, the decoupled-lookback scan of
// kernels_grid.cu and an emit pass write them in voxel order (tetrahedra and quad
// halves in the reference's order within a voxel): the same triangles, in one
// fixed order, and the total is the count the reference's counter reaches.
#include <cuda_runtime.h>

#include "p4a_internal.h"
#include "p4a_math.cuh"

namespace p4a {

__device__ __forceinline__ I3 grid_vertex(const MeshParams& M, uint32_t idx, const int32_t dim[3]) {
  I3 v;
  v.x = (int)(idx % (uint32_t)dim[0]);
  v.y = (int)((idx / (uint32_t)dim[0]) % (uint32_t)dim[1]);
  v.z = (int)(idx / ((uint32_t)dim[0] * (uint32_t)dim[1]));
  return v;
}

// meshDensity (src/mesh_wgsl.js:23-69)
__global__ void __launch_bounds__(kBlock) k_mesh_field(const __grid_constant__ MeshParams M,
                                                       const float4* __restrict__ pos,
                                                       const float* __restrict__ rho,
                                                       const uint32_t* __restrict__ cs,
                                                       const uint4* __restrict__ body, uint32_t n,
                                                       float* __restrict__ field) {
  const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
  const uint32_t total = (uint32_t)M.vertDim[0] * (uint32_t)M.vertDim[1] * (uint32_t)M.vertDim[2];
  if (idx >= total) return;
  const I3 v = grid_vertex(M, idx, M.vertDim);
  const F3 p = {M.gridOrigin[0] + M.voxel * (float)v.x, M.gridOrigin[1] + M.voxel * (float)v.y,
                M.gridOrigin[2] + M.voxel * (float)v.z};
  I3 c;
  c.x = min(max(__float2int_rz(floorf((p.x - M.boxMin[0]) * M.invSupport)), 0), M.simGridDim[0] - 1);
  c.y = min(max(__float2int_rz(floorf((p.y - M.boxMin[1]) * M.invSupport)), 0), M.simGridDim[1] - 1);
  c.z = min(max(__float2int_rz(floorf((p.z - M.boxMin[2]) * M.invSupport)), 0), M.simGridDim[2] - 1);
  const int x0 = max(c.x - 1, 0), x1 = min(c.x + 1, M.simGridDim[0] - 1);
  const float rhoMin = 0.5f * M.rho0;
  float acc = 0.0f;
  for (int dz = -1; dz <= 1; dz++) {
    const int z = c.z + dz;
    if (z < 0 || z >= M.simGridDim[2]) continue;
    for (int dy = -1; dy <= 1; dy++) {
      const int y = c.y + dy;
      if (y < 0 || y >= M.simGridDim[1]) continue;
      const uint32_t rowBase = (uint32_t)((z * M.simGridDim[1] + y) * M.simGridDim[0]);
      const uint32_t b = __ldg(&cs[rowBase + x0]), e = min(__ldg(&cs[rowBase + x1 + 1]), n);
      for (uint32_t j = b; j < e; j++) {
        if (M.skipBodies != 0u && __ldg(&body[j]).x != 0u) continue;
        const float vol = M.mass / fmaxf(__ldg(&rho[j]), rhoMin);
        const F3 r = sub3(p, xyz(__ldg(&pos[j])));
        const float r2 = dot3(r, r);
        if (r2 >= M.support2) continue;
        const float t = M.support2 - r2;
        acc = fmaf(((vol * M.poly6) * t) * t, t, acc);
      }
    }
  }
  field[idx] = acc;
}

// meshSmooth (src/mesh_wgsl.js:71-92) along one axis, `passes` times in a row: one
// warp per grid line, the line held in shared memory (two buffers of `len` floats
// per warp), clamped at the ends like the reference's S().
__global__ void __launch_bounds__(128) k_mesh_blur(const float* __restrict__ src, float* __restrict__ dst,
                                                   int dx, int dy, int dz, int axis, int passes, int lines) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int line = blockIdx.x * 4 + warp;
  if (line >= lines) return;  // whole warps
  const int len = axis == 0 ? dx : axis == 1 ? dy : dz;
  float* a = smem + (size_t)warp * 2 * len;
  float* b = a + len;
  size_t base, stride;
  if (axis == 0) {
    base = (size_t)line * dx;
    stride = 1;
  } else if (axis == 1) {
    base = (size_t)(line / dx) * dx * dy + (size_t)(line % dx);
    stride = (size_t)dx;
  } else {
    base = (size_t)line;
    stride = (size_t)dx * dy;
  }
  for (int k = lane; k < len; k += 32) a[k] = src[base + k * stride];
  __syncwarp();
  for (int p = 0; p < passes; p++) {
    for (int k = lane; k < len; k += 32) {
      const float l = a[max(k - 1, 0)], m = a[k], r = a[min(k + 1, len - 1)];
      b[k] = (0.25f * l + 0.5f * m) + 0.25f * r;
    }
    __syncwarp();
    float* t = a;
    a = b;
    b = t;
  }
  for (int k = lane; k < len; k += 32) dst[base + k * stride] = a[k];
}

// ---- marching tetrahedra (src/mesh_wgsl.js:94-238) ---------------------------

__device__ __forceinline__ float field_at(const float* __restrict__ f, const MeshParams& M, I3 v) {
  v.x = min(max(v.x, 0), M.vertDim[0] - 1);
  v.y = min(max(v.y, 0), M.vertDim[1] - 1);
  v.z = min(max(v.z, 0), M.vertDim[2] - 1);
  return __ldg(&f[(uint32_t)((v.z * M.vertDim[1] + v.y) * M.vertDim[0] + v.x)]);
}

__device__ __forceinline__ F3 grad_at(const float* __restrict__ nf, const MeshParams& M, I3 v) {
  return {field_at(nf, M, {v.x + 1, v.y, v.z}) - field_at(nf, M, {v.x - 1, v.y, v.z}),
          field_at(nf, M, {v.x, v.y + 1, v.z}) - field_at(nf, M, {v.x, v.y - 1, v.z}),
          field_at(nf, M, {v.x, v.y, v.z + 1}) - field_at(nf, M, {v.x, v.y, v.z - 1})};
}

struct Corner {
  float d;
  F3 p, g;
};

__device__ __forceinline__ uint32_t to_u32(float x) { return __float2uint_rz(x); }

__device__ __forceinline__ uint2 pack_vertex(const MeshParams& M, F3 pg, F3 nIn) {
  const F3 pn = {fminf(fmaxf(pg.x / (float)(M.vertDim[0] - 1), 0.0f), 1.0f),
                 fminf(fmaxf(pg.y / (float)(M.vertDim[1] - 1), 0.0f), 1.0f),
                 fminf(fmaxf(pg.z / (float)(M.vertDim[2] - 1), 0.0f), 1.0f)};
  const uint32_t qx = to_u32(pn.x * 65535.0f + 0.5f), qy = to_u32(pn.y * 65535.0f + 0.5f),
                 qz = to_u32(pn.z * 65535.0f + 0.5f);
  const float l1 = fmaxf((fabsf(nIn.x) + fabsf(nIn.y)) + fabsf(nIn.z), 1.0e-12f);
  const F3 nv = {nIn.x / l1, nIn.y / l1, nIn.z / l1};
  float ex = nv.x, ey = nv.y;
  if (nv.z < 0.0f) {
    ex = (1.0f - fabsf(nv.y)) * (nv.x >= 0.0f ? 1.0f : -1.0f);
    ey = (1.0f - fabsf(nv.x)) * (nv.y >= 0.0f ? 1.0f : -1.0f);
  }
  const uint32_t ox = to_u32(fminf(fmaxf(ex * 0.5f + 0.5f, 0.0f), 1.0f) * 255.0f + 0.5f);
  const uint32_t oy = to_u32(fminf(fmaxf(ey * 0.5f + 0.5f, 0.0f), 1.0f) * 255.0f + 0.5f);
  return make_uint2(qx | (qy << 16), qz | ((ox | (oy << 8)) << 16));
}

// mix(x, y, t) = x * (1 - t) + y * t
__device__ __forceinline__ F3 mix3(F3 x, F3 y, float t) {
  const float s = 1.0f - t;
  return {x.x * s + y.x * t, x.y * s + y.y * t, x.z * s + y.z * t};
}

__device__ __forceinline__ uint2 edge_vertex(const MeshParams& M, const Corner& a, const Corner& b) {
  const float t = (M.iso - a.d) / (b.d - a.d);
  const F3 p = mix3(a.p, b.p, t);
  const F3 g = mix3(a.g, b.g, t);
  return pack_vertex(M, p, {-g.x, -g.y, -g.z});
}

// Triangles of one tetrahedron (emitTet): 0, 1 (one corner in or out) or 2 (a quad).
__device__ __forceinline__ int tet_triangles(bool ia, bool ib, bool ic, bool id) {
  const int nin = (int)ia + (int)ib + (int)ic + (int)id;
  return nin == 0 || nin == 4 ? 0 : nin == 2 ? 2 : 1;
}

struct Emitter {
  uint2* __restrict__ verts;
  uint32_t at, limit;
  __device__ __forceinline__ void tri(uint2 a, uint2 b, uint2 c) {
    if (at < limit) {
      verts[(size_t)at * 3 + 0] = a;
      verts[(size_t)at * 3 + 1] = b;
      verts[(size_t)at * 3 + 2] = c;
    }
    at++;
  }
};

__device__ __forceinline__ void emit_tet(const MeshParams& M, Emitter& E, const Corner& a, const Corner& b,
                                         const Corner& c, const Corner& d) {
  const bool ia = a.d > M.iso, ib = b.d > M.iso, ic = c.d > M.iso, id = d.d > M.iso;
  const int nin = (int)ia + (int)ib + (int)ic + (int)id;
  if (nin == 0 || nin == 4) return;
  auto lone = [&](const Corner& l, const Corner& p1, const Corner& p2, const Corner& p3) {
    E.tri(edge_vertex(M, l, p1), edge_vertex(M, l, p2), edge_vertex(M, l, p3));
  };
  auto quad = [&](const Corner& qa, const Corner& qb, const Corner& qc, const Corner& qd) {
    const uint2 q0 = edge_vertex(M, qa, qc), q1 = edge_vertex(M, qa, qd);
    const uint2 q2 = edge_vertex(M, qb, qd), q3 = edge_vertex(M, qb, qc);
    E.tri(q0, q1, q2);
    E.tri(q0, q2, q3);
  };
  if (nin == 1 || nin == 3) {
    const bool look = nin == 1;
    if (ia == look) lone(a, b, c, d);
    else if (ib == look) lone(b, a, c, d);
    else if (ic == look) lone(c, a, b, d);
    else lone(d, a, b, c);
  } else {
    if (ia && ib) quad(a, b, c, d);
    else if (ia && ic) quad(a, c, b, d);
    else if (ia && id) quad(a, d, b, c);
    else if (ib && ic) quad(b, c, a, d);
    else if (ib && id) quad(b, d, a, c);
    else quad(c, d, a, b);
  }
}

// The six tetrahedra of a voxel, corners (0,1,3,7) (0,1,5,7) (0,2,3,7) (0,2,6,7)
// (0,4,5,7) (0,4,6,7); corner k = (k & 1, k >> 1 & 1, k >> 2 & 1).
__constant__ int kTets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

__device__ __forceinline__ I3 voxel_of(const MeshParams& M, uint32_t idx) {
  const int32_t nv[3] = {M.vertDim[0] - 1, M.vertDim[1] - 1, M.vertDim[2] - 1};
  return grid_vertex(M, idx, nv);
}

__global__ void __launch_bounds__(kBlock) k_mesh_count(const __grid_constant__ MeshParams M,
                                                       const float* __restrict__ field,
                                                       uint32_t* __restrict__ counts, uint32_t nvox) {
  const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
  if (idx >= nvox) return;
  const I3 v = voxel_of(M, idx);
  bool in[8];
  int mask = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    in[k] = field_at(field, M, {v.x + (k & 1), v.y + ((k >> 1) & 1), v.z + ((k >> 2) & 1)}) > M.iso;
    mask |= (int)in[k] << k;
  }
  uint32_t c = 0;
  if (mask != 0 && mask != 255) {
#pragma unroll
    for (int t = 0; t < 6; t++) c += (uint32_t)tet_triangles(in[kTets[t][0]], in[kTets[t][1]], in[kTets[t][2]], in[kTets[t][3]]);
  }
  counts[idx] = c;
}

__global__ void __launch_bounds__(kBlock) k_mesh_emit(const __grid_constant__ MeshParams M,
                                                      const float* __restrict__ field,
                                                      const float* __restrict__ nfield,
                                                      const uint32_t* __restrict__ offsets, uint32_t nvox,
                                                      uint2* __restrict__ verts) {
  const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
  if (idx >= nvox) return;
  const uint32_t first = offsets[idx];
  if (offsets[idx + 1] == first || first >= M.maxTris) return;
  const I3 v = voxel_of(M, idx);
  Corner cn[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const I3 w = {v.x + (k & 1), v.y + ((k >> 1) & 1), v.z + ((k >> 2) & 1)};
    cn[k].d = field_at(field, M, w);
    cn[k].p = {(float)w.x, (float)w.y, (float)w.z};
    cn[k].g = grad_at(nfield, M, w);
  }
  Emitter E{verts, first, M.maxTris};
#pragma unroll 1
  for (int t = 0; t < 6; t++)
    emit_tet(M, E, cn[kTets[t][0]], cn[kTets[t][1]], cn[kTets[t][2]], cn[kTets[t][3]]);
}

void launch_mesh_field(const MeshParams& M, const float4* pos, const float* rho, const uint32_t* cs,
                       const uint4* body, uint32_t n, float* field, cudaStream_t st) {
  const long long total = (long long)M.vertDim[0] * M.vertDim[1] * M.vertDim[2];
  k_mesh_field<<<groups(total), kBlock, 0, st>>>(M, pos, rho, cs, body, n, field);
}

cudaError_t launch_mesh_blur(const MeshParams& M, const float* src, float* dst, int axis, int passes,
                             cudaStream_t st) {
  const int dx = M.vertDim[0], dy = M.vertDim[1], dz = M.vertDim[2];
  const int len = axis == 0 ? dx : axis == 1 ? dy : dz;
  const int lines = (dx * dy * dz) / len;
  const size_t smem = (size_t)4 * 2 * len * sizeof(float);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_mesh_blur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_mesh_blur<<<(lines + 3) / 4, 128, smem, st>>>(src, dst, dx, dy, dz, axis, passes, lines);
  return cudaGetLastError();
}

void launch_mesh_count(const MeshParams& M, const float* field, uint32_t* counts, uint32_t nvox, cudaStream_t st) {
  k_mesh_count<<<groups(nvox), kBlock, 0, st>>>(M, field, counts, nvox);
}

void launch_mesh_emit(const MeshParams& M, const float* field, const float* nfield, const uint32_t* offsets,
                      uint32_t nvox, uint2* verts, cudaStream_t st) {
  k_mesh_emit<<<groups(nvox), kBlock, 0, st>>>(M, field, nfield, offsets, nvox, verts);
}

}  // namespace p4a
