// neighbours.cuh — the neighbour walk shared by the gather passes.
//
// The reference walks, for particle i, the 3x3 row ranges
// [cellStart[row+x0], cellStart[row+x1+1]) of the cell block around
// cellOf(pred_i) and tests every candidate j against r^2 < h^2 (src/wgsl.js:98-111).
// Here that walk is split in two phases:
//   1. a cheap test of every candidate that records, per row, a 64-bit mask of the
//      candidates within h (bit k <-> j = rowStart + k);
//   2. the pass's real work over the set bits in ascending order.
// Phase 2 therefore visits exactly the reference's neighbours in exactly its order
// (rows z->y, j ascending, the boundary samples of a row after its fluid
// particles), so sums are bit-identical, while the expensive in-range work no
// longer runs warp-wide on every candidate iteration. Two passes that walk the
// same positions (lambda then delta, xsph+normals then tension) share the masks:
// the first stores them, the second skips phase 1. Rows with more than 64
// candidates (never seen at rest density, where a row holds ~24) fall back to
// the reference's direct loop.
#pragma once
#include "p4a_math.cuh"

namespace p4a {

constexpr int kRows = 9;
constexpr uint32_t kMaskBits = 64;

// Row r = 3*(dz+1) + (dy+1), the reference's dz-outer, dy-inner order.
struct RowWalk {
  int x0, x1;
  I3 c;
  __device__ __forceinline__ RowWalk(const SimParams& P, F3 p) {
    c = cell_of(P, p);
    x0 = max(c.x - 1, 0);
    x1 = min(c.x + 1, P.gridDim[0] - 1);
  }
  // Row base index of row r, or -1 when the row is outside the grid.
  __device__ __forceinline__ int row_base(const SimParams& P, int r) const {
    const int z = c.z + r / 3 - 1, y = c.y + r % 3 - 1;
    if (z < 0 || z >= P.gridDim[2] || y < 0 || y >= P.gridDim[1]) return -1;
    return (z * P.gridDim[1] + y) * P.gridDim[0];
  }
};

// Phase 1 for one row (row base rb >= 0): the mask of candidates with r^2 < h^2;
// sets *isLong when the row has more than 64 candidates.
__device__ __forceinline__ uint64_t row_mask(const SimParams& P, const RowWalk& w, int rb, F3 pi,
                                             const float4* __restrict__ pred,
                                             const uint32_t* __restrict__ cs, bool& isLong) {
  uint64_t m = 0ull;
  const uint32_t b = __ldg(&cs[rb + w.x0]);
  const uint32_t e = min(__ldg(&cs[rb + w.x1 + 1]), P.pEnd);
  const uint32_t len = e > b ? e - b : 0u;
  isLong = len > kMaskBits;
  const uint32_t lim = min(len, kMaskBits);
  uint32_t k = 0;
  for (; k + 4 <= lim; k += 4) {
    const float4 q0 = __ldg(&pred[b + k]), q1 = __ldg(&pred[b + k + 1]);
    const float4 q2 = __ldg(&pred[b + k + 2]), q3 = __ldg(&pred[b + k + 3]);
    const F3 d0 = sub3(pi, xyz(q0)), d1 = sub3(pi, xyz(q1));
    const F3 d2 = sub3(pi, xyz(q2)), d3 = sub3(pi, xyz(q3));
    const uint32_t bits = (dot3(d0, d0) < P.h2 ? 1u : 0u) | (dot3(d1, d1) < P.h2 ? 2u : 0u) |
                          (dot3(d2, d2) < P.h2 ? 4u : 0u) | (dot3(d3, d3) < P.h2 ? 8u : 0u);
    m |= (uint64_t)bits << k;
  }
  for (; k < lim; k++) {
    const F3 d0 = sub3(pi, xyz(__ldg(&pred[b + k])));
    if (dot3(d0, d0) < P.h2) m |= 1ull << k;
  }
  return m;
}

// Phase 2 over one row: calls f(j) for the row's fluid neighbours in ascending j
// (from the mask, or by the direct loop for a long row). The caller handles the
// row's boundary samples after it.
template <class F>
__device__ __forceinline__ void visit_row(const SimParams& P, const RowWalk& w, int rb, F3 pi,
                                          uint64_t m, bool longRow,
                                          const float4* __restrict__ pred,
                                          const uint32_t* __restrict__ cs, F&& f) {
  const uint32_t b = __ldg(&cs[rb + w.x0]);
  if (!longRow) {
    while (m) {
      const int k = __ffsll((long long)m) - 1;
      m &= m - 1ull;
      f(b + (uint32_t)k);
    }
  } else {
    const uint32_t e = min(__ldg(&cs[rb + w.x1 + 1]), P.pEnd);
    for (uint32_t j = b; j < e; j++) {
      const F3 d = sub3(pi, xyz(__ldg(&pred[j])));
      if (dot3(d, d) < P.h2) f(j);
    }
  }
}

// The masks shared by a pair of passes are stored [row][particle] (row-major over
// the capacity), so each row's loads and stores are coalesced.

}  // namespace p4a
