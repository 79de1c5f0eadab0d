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
//
// Phase 2 is one loop over all nine rows (walk_rows), not a loop per row: each
// thread's row masks and row starts are staged in shared memory and every
// iteration handles exactly one neighbour of every lane that has one left. Lanes
// of a warp hold different numbers of neighbours per row, so a loop per row runs
// each row to its warp maximum (about half the lanes idle in the expensive body);
// the single loop runs to the warp maximum of the totals instead.
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

// Phase 1 for one row (row base rb >= 0): the mask of candidates with r^2 < r2lim
// (h^2, or (h + skin)^2 for masks that later iterations reuse); sets *isLong when the
// row has more than 64 candidates and *b to the row's start.
__device__ __forceinline__ uint64_t row_mask(const SimParams& P, const RowWalk& w, int rb, F3 pi,
                                             const float4* __restrict__ pred,
                                             const uint32_t* __restrict__ cs, bool& isLong,
                                             uint32_t& b, float r2lim) {
  uint64_t m = 0ull;
  b = __ldg(&cs[rb + w.x0]);
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
    const uint32_t bits = (dot3(d0, d0) < r2lim ? 1u : 0u) | (dot3(d1, d1) < r2lim ? 2u : 0u) |
                          (dot3(d2, d2) < r2lim ? 4u : 0u) | (dot3(d3, d3) < r2lim ? 8u : 0u);
    m |= (uint64_t)bits << k;
  }
  for (; k < lim; k++) {
    const F3 d0 = sub3(pi, xyz(__ldg(&pred[b + k])));
    if (dot3(d0, d0) < r2lim) m |= 1ull << k;
  }
  return m;
}

// The reference's direct loop over one row's fluid candidates (rows longer than 64).
template <class F>
__device__ __forceinline__ void long_row(const SimParams& P, const RowWalk& w, int rb, F3 pi,
                                         const float4* __restrict__ pred,
                                         const uint32_t* __restrict__ cs, F&& f) {
  const uint32_t b = __ldg(&cs[rb + w.x0]);
  const uint32_t e = min(__ldg(&cs[rb + w.x1 + 1]), P.pEnd);
  for (uint32_t j = b; j < e; j++) {
    const F3 d = sub3(pi, xyz(__ldg(&pred[j])));
    if (dot3(d, d) < P.h2) f(j);
  }
}

// Phase 1 for one row's boundary samples [bb, be): the mask of samples with
// 1e-12 <= r^2 < r2lim (the ones the reference's boundary terms use, when r2lim is
// h^2); sets *isLong when the row has more than 32 samples.
constexpr uint32_t kBMaskBits = 32;
__device__ __forceinline__ uint32_t boundary_mask(const SimParams& P, uint32_t bb, uint32_t be, F3 pi,
                                                  const float4* __restrict__ bpos, bool& isLong,
                                                  float r2lim) {
  const uint32_t len = be > bb ? be - bb : 0u;
  isLong = len > kBMaskBits;
  const uint32_t lim = min(len, kBMaskBits);
  uint32_t m = 0u;
  for (uint32_t k = 0; k < lim; k++) {
    const F3 d = sub3(pi, xyz(__ldg(&bpos[bb + k])));
    const float r2 = dot3(d, d);
    if (r2 < r2lim && r2 >= 1.0e-12f) m |= 1u << k;
  }
  return m;
}

// Per-thread row staging in shared memory for a block of TB threads: fluid mask,
// row start and (when the pass has boundary terms, B) boundary mask of each of the
// nine rows, in columns [r * TB + threadIdx.x].
template <int TB, bool B>
struct RowStage {
  uint64_t* mask;
  uint32_t* base;
  uint32_t* bmask;
  __device__ __forceinline__ RowStage() {
    __shared__ uint64_t sMask[kRows * TB];
    __shared__ uint32_t sBase[kRows * TB];
    mask = sMask + threadIdx.x;
    base = sBase + threadIdx.x;
    if constexpr (B) {
      __shared__ uint32_t sBMask[kRows * TB];
      bmask = sBMask + threadIdx.x;
    } else {
      bmask = nullptr;
    }
  }
  __device__ __forceinline__ void set(int r, uint64_t m, uint32_t b, uint32_t bm = 0u) const {
    mask[r * TB] = m;
    base[r * TB] = b;
    if constexpr (B) bmask[r * TB] = bm;
  }
};

// Phase 2 over all rows in order. Each row's events are its fluid neighbours (set
// bits, j ascending), then its boundary samples (set bits, k ascending): every loop
// iteration handles one event of every lane that has one left, with fluid(j) or
// bound(r, k) (k the sample's offset in the row's boundary range), which return
// whether the candidate was within h. A row longer than its mask runs longFluid(r)
// in place of its fluid bits, or longBound(r) in place of its boundary bits. When a
// row is done, rowDone(r, em, ebm) receives the masks of the candidates that were
// within h. `todo` has bit r set for every row with anything to visit; lr / lb are
// the long-row bits.
template <int TB, bool B, class FFluid, class FBound, class FLongF, class FLongB, class FDone>
__device__ __forceinline__ void walk_rows(const RowStage<TB, B>& st, uint32_t todo, uint32_t lr, uint32_t lb,
                                          FFluid&& fluid, FBound&& bound, FLongF&& longFluid,
                                          FLongB&& longBound, FDone&& rowDone) {
  int r = -1;
  uint64_t m = 0ull, em = 0ull;
  uint32_t mb = 0u, ebm = 0u, base = 0u;
  for (;;) {
    while ((m | (uint64_t)mb) == 0ull) {
      if (r >= 0) {
        if ((lb >> r) & 1u) longBound(r);
        rowDone(r, em, ebm);
        todo &= todo - 1u;  // r is the lowest pending row
      }
      if (todo == 0u) return;
      r = __ffs(todo) - 1;
      m = st.mask[r * TB];
      base = st.base[r * TB];
      if constexpr (B) mb = st.bmask[r * TB];
      em = 0ull;
      ebm = 0u;
      if ((lr >> r) & 1u) longFluid(r);  // a long row's fluid comes before its boundary samples
    }
    if (m != 0ull) {
      const int k = __ffsll((long long)m) - 1;
      m &= m - 1ull;
      if (fluid(base + (uint32_t)k)) em |= 1ull << k;
    } else {
      const int k = __ffs(mb) - 1;
      mb &= mb - 1u;
      if (bound(r, (uint32_t)k)) ebm |= 1u << k;
    }
  }
}

// Fluid-only form (passes without boundary terms); fluid(j) returns void.
template <int TB, class FFluid, class FLongF>
__device__ __forceinline__ void walk_fluid_rows(const RowStage<TB, false>& st, uint32_t todo, uint32_t lr,
                                                FFluid&& fluid, FLongF&& longFluid) {
  walk_rows(
      st, todo, lr, 0u, [&](uint32_t j) { fluid(j); return false; }, [](int, uint32_t) { return false; },
      longFluid, [](int) {}, [](int, uint64_t, uint32_t) {});
}

// The masks shared by a pair of passes are stored [row][particle] (row-major over
// the capacity), so each row's loads and stores are coalesced.

}  // namespace p4a
