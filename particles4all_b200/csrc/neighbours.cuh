// neighbours.cuh — the neighbour walk shared by the gather passes.
//
// The reference walks, for particle i, the 3x3 row ranges
// [cellStart[row+x0], cellStart[row+x1+1]) of the cell block around
// cellOf(pred_i) and tests every candidate j against r^2 < h^2 (src/wgsl.js:98-111),
// the boundary samples of a row after its fluid particles (src/wgsl.js:497-533).
// Here that walk is split in two phases:
//   1. build_list tests every candidate once and appends the ones within a radius
//      (h, or h + skin for lists that later Jacobi iterations reuse) to the
//      particle's neighbour list, in the reference's visiting order: rows z->y,
//      fluid j ascending, then the row's boundary samples (tagged kBoundTag);
//   2. walk_list runs the pass's real work over the list, one entry per loop
//      iteration, every entry re-tested against r^2 < h^2 with the current
//      positions by the pass itself.
// Phase 2 therefore visits exactly the reference's neighbours in exactly its
// order, so sums are bit-identical, while the expensive in-range work no longer
// runs warp-wide on every candidate, and the loop has no per-row bookkeeping:
// lanes of a warp hold different numbers of neighbours per row, so a walk that
// switches rows inside the loop pays the switch in almost every iteration.
// The list is stored [entry][particle] (entry k of particle i at k * cap + i), so
// the lanes of a warp read entry k of 32 consecutive particles with one
// coalesced load. The particle itself is never listed (it contributes to no
// pass). A particle with more than kListCap entries is marked kListOverflow and
// walked with the reference's direct loop instead.
#pragma once
#include "p4a_math.cuh"

namespace p4a {

constexpr int kRows = 9;
constexpr uint32_t kListOverflow = 0xffffffffu;  // count of a particle whose list did not fit
constexpr uint32_t kBoundTag = 0x80000000u;      // entry = kBoundTag | boundary sample index
constexpr uint32_t kHasBound = 0x40000000u;      // count flag: the list holds boundary samples
constexpr uint32_t kCountMask = 0x0000ffffu;
constexpr int kBuildShift = 16;                  // count bits 16-19: the iteration that built the list

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

// Phase 1: the list of particle i (scene-local cellStart cs / bcs, arena index i)
// with every candidate j != i of the nine rows within r^2 < r2lim, and, when B,
// every boundary sample of each row within r^2 < r2lim after the row's fluid
// candidates. Returns the entry count (| kHasBound when boundary samples were
// listed), or kListOverflow.
template <bool B>
__device__ __forceinline__ uint32_t build_list(const SimParams& P, const RowWalk& w, uint32_t i, F3 pi,
                                               const float4* __restrict__ pred,
                                               const uint32_t* __restrict__ cs,
                                               const uint32_t* __restrict__ bcs,
                                               const float4* __restrict__ bpos, uint32_t* __restrict__ list,
                                               uint32_t cap, float r2lim) {
  uint32_t c = 0, flags = 0u;
  uint32_t* __restrict__ out = list + i;  // entry c at list[c * cap + i]
  auto push = [&](uint32_t e) {
    if (c < kListCap) {
      *out = e;
      out += cap;
    }
    c++;
  };
#pragma unroll 1
  for (int r = 0; r < kRows; r++) {
    const int rb = w.row_base(P, r);
    if (rb < 0) continue;
    const uint32_t b = __ldg(&cs[rb + w.x0]);
    const uint32_t e = min(__ldg(&cs[rb + w.x1 + 1]), P.pEnd);
    uint32_t j = b;
    for (; j + 4 <= e; j += 4) {
      const float4 q0 = __ldg(&pred[j]), q1 = __ldg(&pred[j + 1]);
      const float4 q2 = __ldg(&pred[j + 2]), q3 = __ldg(&pred[j + 3]);
      const F3 d0 = sub3(pi, xyz(q0)), d1 = sub3(pi, xyz(q1));
      const F3 d2 = sub3(pi, xyz(q2)), d3 = sub3(pi, xyz(q3));
      const bool i0 = dot3(d0, d0) < r2lim, i1 = dot3(d1, d1) < r2lim;
      const bool i2 = dot3(d2, d2) < r2lim, i3 = dot3(d3, d3) < r2lim;
      if (i0 && j != i) push(j);
      if (i1 && j + 1 != i) push(j + 1);
      if (i2 && j + 2 != i) push(j + 2);
      if (i3 && j + 3 != i) push(j + 3);
    }
    for (; j < e; j++) {
      const F3 d0 = sub3(pi, xyz(__ldg(&pred[j])));
      if (dot3(d0, d0) < r2lim && j != i) push(j);
    }
    if constexpr (B) {
      if (P.nBoundary > 0u) {
        const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
        for (uint32_t k = bb; k < be; k++) {
          const F3 d0 = sub3(pi, xyz(__ldg(&bpos[k])));
          if (dot3(d0, d0) < r2lim) {
            push(kBoundTag | k);
            flags = kHasBound;
          }
        }
      }
    }
  }
  return c > kListCap ? kListOverflow : c | flags;
}

// build_list for one particle (iL, piL, its row walk wL) by all 32 lanes of a warp:
// lane k tests candidate base + k of each row, and a ballot orders the appends, so
// the list (entries, order, count, flags) is the one build_list writes.
template <bool B>
__device__ __forceinline__ uint32_t build_list_coop(const SimParams& P, const RowWalk& wL, uint32_t iL, F3 piL,
                                                    const float4* __restrict__ pred,
                                                    const uint32_t* __restrict__ cs,
                                                    const uint32_t* __restrict__ bcs,
                                                    const float4* __restrict__ bpos, uint32_t* __restrict__ list,
                                                    uint32_t cap, float r2lim) {
  const uint32_t lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
  uint32_t c = 0, flags = 0u;
#pragma unroll 1
  for (int r = 0; r < kRows; r++) {
    const int rb = wL.row_base(P, r);
    if (rb < 0) continue;
    const uint32_t b = __ldg(&cs[rb + wL.x0]);
    const uint32_t e = min(__ldg(&cs[rb + wL.x1 + 1]), P.pEnd);
    for (uint32_t base = b; base < e; base += 32u) {
      const uint32_t j = base + lane;
      bool in = false;
      if (j < e && j != iL) {
        const F3 dd = sub3(piL, xyz(__ldg(&pred[j])));
        in = dot3(dd, dd) < r2lim;
      }
      const uint32_t m = __ballot_sync(0xffffffffu, in);
      if (in) {
        const uint32_t pos = c + (uint32_t)__popc(m & below);
        if (pos < kListCap) list[(size_t)pos * cap + iL] = j;
      }
      c += (uint32_t)__popc(m);
    }
    if constexpr (B) {
      if (P.nBoundary > 0u) {
        const uint32_t bb = __ldg(&bcs[rb + wL.x0]), be = __ldg(&bcs[rb + wL.x1 + 1]);
        for (uint32_t base = bb; base < be; base += 32u) {
          const uint32_t k = base + lane;
          bool in = false;
          if (k < be) {
            const F3 dd = sub3(piL, xyz(__ldg(&bpos[k])));
            in = dot3(dd, dd) < r2lim;
          }
          const uint32_t m = __ballot_sync(0xffffffffu, in);
          if (in) {
            const uint32_t pos = c + (uint32_t)__popc(m & below);
            if (pos < kListCap) list[(size_t)pos * cap + iL] = kBoundTag | k;
          }
          if (m) flags = kHasBound;
          c += (uint32_t)__popc(m);
        }
      }
    }
  }
  return c > kListCap ? kListOverflow : c | flags;
}

// The lanes of a warp that `need` a new list get one; all 32 lanes must call.
// When few lanes need one, the whole warp builds each of their lists in turn
// (build_list_coop), instead of letting the warp wait while those lanes test
// their ~216 candidates one by one; when many do, each lane builds its own.
// Returns the lane's new count word, or `current` for lanes that need none.
constexpr int kCoopLanes = 12;
template <bool B>
__device__ __forceinline__ uint32_t build_lists_warp(const SimParams& P, bool need, const RowWalk& w, uint32_t i,
                                                     F3 pi, const float4* __restrict__ pred,
                                                     const uint32_t* __restrict__ cs,
                                                     const uint32_t* __restrict__ bcs,
                                                     const float4* __restrict__ bpos, uint32_t* __restrict__ list,
                                                     uint32_t cap, float r2lim, uint32_t current) {
  const unsigned needMask = __ballot_sync(0xffffffffu, need);
  if (needMask == 0u) return current;
  if (__popc(needMask) > kCoopLanes) return need ? build_list<B>(P, w, i, pi, pred, cs, bcs, bpos, list, cap, r2lim)
                                                 : current;
  const int lane = (int)(threadIdx.x & 31u);
  uint32_t out = current;
  for (unsigned m = needMask; m != 0u; m &= m - 1u) {
    const int L = __ffs(m) - 1;
    RowWalk wL = w;
    wL.c.x = __shfl_sync(0xffffffffu, w.c.x, L);
    wL.c.y = __shfl_sync(0xffffffffu, w.c.y, L);
    wL.c.z = __shfl_sync(0xffffffffu, w.c.z, L);
    wL.x0 = __shfl_sync(0xffffffffu, w.x0, L);
    wL.x1 = __shfl_sync(0xffffffffu, w.x1, L);
    const uint32_t iL = __shfl_sync(0xffffffffu, i, L);
    const F3 piL = {__shfl_sync(0xffffffffu, pi.x, L), __shfl_sync(0xffffffffu, pi.y, L),
                    __shfl_sync(0xffffffffu, pi.z, L)};
    const uint32_t cnt = build_list_coop<B>(P, wL, iL, piL, pred, cs, bcs, bpos, list, cap, r2lim);
    if (lane == L) out = cnt;
  }
  return out;
}

// Whether particle i, now in `cell`, may walk its stored list before iteration `it`
// of this substep (it = iters: the positions after the last iteration). The list
// was built at iteration b (its count word's bits 16-19) from the positions then,
// with radius h + skin, in the cell recorded in nbCell. It still holds every pair
// now within h when the particle is in the same cell (same candidate rows) and
// every candidate (the particles sorted into the block's cells) and the particle
// itself moved at most skin / 2 since iteration b, by either bound:
//  - S: the sum of the iterations' largest single-iteration displacements since b
//    over the whole scene (disp[t], recorded by every delta and rigid projection);
//  - V: per block cell, the largest displacement of the cell's particles from the
//    substep's start positions now, plus the same at iteration b (cellDisp[t] after
//    iteration t), since |p(now) - p(b)| <= |p(now) - ref| + |p(b) - ref|.
// V is local: a fast particle elsewhere in the scene does not force this list to
// be rebuilt.
__device__ __forceinline__ bool list_reusable(const SimParams& P, const DevScene& d, int it, uint32_t i,
                                              const RowWalk& w, uint32_t cell, uint32_t countWord) {
  if (it <= 0 || it >= kDispSlots || countWord == kListOverflow) return false;
  if (__ldg(&d.nbCell[i]) != cell) return false;
  const int b = (int)((countWord >> kBuildShift) & 0xfu);
  if (b >= it) return false;
  const float* disp = d.disp + (size_t)P.slot * kDispSlots;
  float S = 0.0f;
  for (int t = b; t < it; t++) S += __ldg(&disp[t]);
  if (S * 1.00001f <= P.skinHalf) return true;
  const float* vNow = d.cellDisp + (size_t)(it - 1) * d.cellStride + P.cOff;
  const float* vB = b > 0 ? d.cellDisp + (size_t)(b - 1) * d.cellStride + P.cOff : nullptr;
  // the particle's own sort cell (the cell of its start position) may lie outside
  // the block when it moved more than a cell since the sort
  const I3 a = cell_of(P, xyz(__ldg(&d.nbRef[i])));
  const uint32_t ac = cell_index(P, a);
  float V = __ldg(&vNow[ac]) + (vB ? __ldg(&vB[ac]) : 0.0f);
  // The 27 cells with every load independent of the others (a loop over rows with
  // a data-dependent skip issued them row by row, one memory latency per row): a
  // row outside the grid reads the particle's own row and counts as 0, and x is
  // clamped into the grid, which repeats x0 or x1 at an edge. The slots hold
  // displacement lengths, so neither changes the maximum.
  const int gx = P.gridDim[0], gy = P.gridDim[1], gz = P.gridDim[2];
  const int ownRow = (w.c.z * gy + w.c.y) * gx;
#pragma unroll
  for (int r = 0; r < kRows; r++) {
    const int z = w.c.z + r / 3 - 1, y = w.c.y + r % 3 - 1;
    const bool in = z >= 0 && z < gz && y >= 0 && y < gy;
    const int rb = in ? (z * gy + y) * gx : ownRow;
#pragma unroll
    for (int dx = -1; dx <= 1; dx++) {
      const int x = min(max(w.c.x + dx, 0), gx - 1);
      const float v = __ldg(&vNow[rb + x]) + (vB ? __ldg(&vB[rb + x]) : 0.0f);
      V = fmaxf(V, in ? v : 0.0f);
    }
  }
  return V * 1.00001f <= P.skinHalf;
}

// Phase 2 over a list of `count` entries: pair(idx, q, isBound) for every entry,
// with q = fsrc[idx] for a fluid entry and q = bsrc[idx] for a boundary sample
// (for a pass that skips boundary samples their calls carry an unused q). One callback for both kinds, so that a pass can treat them on one path with
// per-lane selects where that is cheaper than running both paths in turn for a
// warp whose lanes hold entries of both kinds. With PF the walk is
// software pipelined two entries deep: while entry k is processed, the gather of
// entry k+1 and the list load of entry k+2 are already in flight, so the latency
// of the dependent list-then-gather chain overlaps the arithmetic of the current
// pair. The gather address is chosen without a branch, in one of two forms (both
// give the same q; which is faster depends on the kernel's register budget):
// kFetchBound for a pass that reads boundary samples from bsrc, and kFetchAny that
// decides by bsrc != null at run time (a boundary entry of a pass without boundary
// samples loads the particle's own fsrc[i]).
enum FetchForm { kFetchAny, kFetchBound };
template <bool PF = true, FetchForm FORM = kFetchAny, class FPair>
__device__ __forceinline__ void walk_list(const uint32_t* __restrict__ list, uint32_t cap, uint32_t i,
                                          uint32_t count, const float4* __restrict__ fsrc,
                                          const float4* __restrict__ bsrc, FPair&& pair) {
  count &= kCountMask;
  if (count == 0u) return;
  auto fetch = [&](uint32_t e) {
    const bool b = (e & kBoundTag) != 0u;
    if constexpr (FORM == kFetchBound) {
      return __ldg((b ? bsrc : fsrc) + (e & ~kBoundTag));  // a fluid entry has no tag bit
    } else {
      const float4* src = b && bsrc ? bsrc : fsrc;
      const uint32_t idx = b ? (bsrc ? (e & ~kBoundTag) : i) : e;
      return __ldg(src + idx);
    }
  };
  auto visit = [&](uint32_t cur, float4 q) { pair(cur & ~kBoundTag, q, (cur & kBoundTag) != 0u); };
  const uint32_t* __restrict__ at = list + i;  // entry k of the particle at list[k * cap + i]
  uint32_t e0 = __ldg(at);
  if constexpr (PF) {
    float4 q0 = fetch(e0);
    at += cap;
    uint32_t e1 = count > 1u ? __ldg(at) : 0u;
    for (uint32_t k = 1; k <= count; k++) {
      const uint32_t cur = e0;
      const float4 qc = q0;
      if (k < count) {
        e0 = e1;
        q0 = fetch(e1);
        if (k + 1 < count) {
          at += cap;
          e1 = __ldg(at);
        }
      }
      visit(cur, qc);
    }
  } else {
    // one entry ahead; the loop runs while a next entry exists, the last entry is
    // visited after it
    for (uint32_t k = 1; k < count; k++) {
      const uint32_t cur = e0;
      at += cap;
      e0 = __ldg(at);
      visit(cur, fetch(cur));
    }
    visit(e0, fetch(e0));
  }
}

// The reference's direct loop (particles whose list overflowed): every candidate
// j != self of the nine rows with r^2 < h^2 (the particle itself contributes to
// no pass), then, when B, the row's boundary samples with 1e-12 <= r^2 < h^2. fsrc
// holds the candidate positions in .xyz (and whatever the pass keeps in .w).
template <bool B, class FFluid, class FBound>
__device__ __forceinline__ void walk_direct(const SimParams& P, const RowWalk& w, F3 pi, uint32_t self,
                                            const float4* __restrict__ fsrc, const uint32_t* __restrict__ cs,
                                            const uint32_t* __restrict__ bcs, const float4* __restrict__ bpos,
                                            FFluid&& fluid, FBound&& bound) {
#pragma unroll 1
  for (int r = 0; r < kRows; r++) {
    const int rb = w.row_base(P, r);
    if (rb < 0) continue;
    const uint32_t b = __ldg(&cs[rb + w.x0]);
    const uint32_t e = min(__ldg(&cs[rb + w.x1 + 1]), P.pEnd);
    for (uint32_t j = b; j < e; j++) {
      const float4 q = __ldg(&fsrc[j]);
      const F3 d = sub3(pi, xyz(q));
      if (dot3(d, d) < P.h2 && j != self) fluid(j, q);
    }
    if constexpr (B) {
      if (P.nBoundary > 0u) {
        const uint32_t bb = __ldg(&bcs[rb + w.x0]), be = __ldg(&bcs[rb + w.x1 + 1]);
        for (uint32_t k = bb; k < be; k++) {
          const float4 q = __ldg(&bpos[k]);
          const F3 d = sub3(pi, xyz(q));
          const float r2 = dot3(d, d);
          if (r2 < P.h2 && r2 >= 1.0e-12f) bound(k, q);
        }
      }
    }
  }
}

// Fluid-only passes (xsph, normals, tension): fluid(j, q, g) for every fluid
// neighbour entry of the list, q = pred[j] and g = gsrc[j] (the pass's packed
// per-neighbour values), both loaded in the walk's two-deep pipeline so that
// neither gather's latency is waited for in the pair's arithmetic; boundary
// entries of a reused list are skipped. An overflowed list walks the direct loop.
// PEEL: the loop runs only while a next entry exists and the last two entries are
// visited after it (no per-entry tests of what is left, the pair term inlined three
// times), measured faster in the block-form finalize passes and slower elsewhere.
template <bool PEEL = false, class FFluid>
__device__ __forceinline__ void walk_neighbours2(const SimParams& P, const RowWalk& w, uint32_t i, F3 pi,
                                                 const float4* __restrict__ pred,
                                                 const float4* __restrict__ gsrc,
                                                 const uint32_t* __restrict__ cs,
                                                 const uint32_t* __restrict__ list, uint32_t cap, uint32_t count,
                                                 FFluid&& fluid) {
  if (count == kListOverflow) {
    auto none = [](uint32_t, float4) {};
    walk_direct<false>(P, w, pi, i, pred, cs, nullptr, nullptr,
                       [&](uint32_t j, float4 q) { fluid(j, q, __ldg(&gsrc[j])); }, none);
    return;
  }
  count &= kCountMask;
  if (count == 0u) return;
  auto slot = [&](uint32_t e) { return (e & kBoundTag) != 0u ? i : e; };  // a boundary entry loads i
  const uint32_t* __restrict__ at = list + i;  // entry k of the particle at list[k * cap + i]
  uint32_t e0 = __ldg(at);
  float4 q0 = __ldg(pred + slot(e0)), g0 = __ldg(gsrc + slot(e0));
  if constexpr (PEEL) {
    uint32_t e1 = 0u;
    if (count > 1u) {
      at += cap;
      e1 = __ldg(at);
    }
    auto visit = [&](uint32_t cur, float4 qc, float4 gc) {
      if ((cur & kBoundTag) == 0u) fluid(cur, qc, gc);
    };
    for (uint32_t k = 1; k + 1 < count; k++) {
      const uint32_t cur = e0;
      const float4 qc = q0, gc = g0;
      e0 = e1;
      q0 = __ldg(pred + slot(e1));
      g0 = __ldg(gsrc + slot(e1));
      at += cap;
      e1 = __ldg(at);
      visit(cur, qc, gc);
    }
    if (count > 1u) {
      const uint32_t cur = e0;
      const float4 qc = q0, gc = g0;
      e0 = e1;
      q0 = __ldg(pred + slot(e1));
      g0 = __ldg(gsrc + slot(e1));
      visit(cur, qc, gc);
    }
    visit(e0, q0, g0);
    return;
  }
  at += cap;
  uint32_t e1 = count > 1u ? __ldg(at) : 0u;
  for (uint32_t k = 1; k <= count; k++) {
    const uint32_t cur = e0;
    const float4 qc = q0, gc = g0;
    if (k < count) {
      e0 = e1;
      q0 = __ldg(pred + slot(e1));
      g0 = __ldg(gsrc + slot(e1));
      if (k + 1 < count) {
        at += cap;
        e1 = __ldg(at);
      }
    }
    if ((cur & kBoundTag) == 0u) fluid(cur, qc, gc);
  }
}

}  // namespace p4a
