// pass_common.cuh — how the blocks of a batched launch find their work.
#pragma once
#include "p4a_internal.h"

namespace p4a {

// Batched form: the block pulls work items (scene slot, item) from its launch's
// segment, one per cursor increment, and calls f(P, item, k) for each, with P the
// item's SimParams in shared memory (reloaded only when the scene changes) and k
// the item's position in the segment. With AHEAD the next item is claimed while
// the current one runs, so the cursor's round trip is hidden. Items are claimed in
// increasing k and a block claims its next item only while working on one, so the
// smallest unfinished item is always being worked on: a block that waits on
// earlier items waits on blocks that finish. For items that wait on their
// predecessors (the scan's lookback) AHEAD is off: the next item is claimed only
// after the current one is done, so every claimed item is being worked on and no
// item waits on one that is claimed but not started (such waits chained up and
// made the batched scan ten times slower than its memory traffic).
// f may contain block barriers: every thread of the block makes every call.
template <bool AHEAD = true, class F>
__device__ __forceinline__ void for_each_item(const BatchWork& w, F&& f) {
  __shared__ __align__(16) SimParams sP;
  __shared__ uint32_t sNext[2], sSlot;
  const WorkSeg seg = *w.seg;
  if (threadIdx.x == 0) {
    sSlot = 0xffffffffu;
    sNext[0] = atomicAdd(w.cursor, 1u);
  }
  __syncthreads();
  for (int p = 0;; p ^= 1) {
    const uint32_t k = sNext[p];
    if (k >= seg.count) break;
    if (AHEAD && threadIdx.x == 0) sNext[p ^ 1] = atomicAdd(w.cursor, 1u);
    const uint2 it = w.items[seg.off + k];
    if (it.x != sSlot) {
      __syncthreads();  // every thread has compared against the old slot
      const uint32_t* src = reinterpret_cast<const uint32_t*>(w.params + it.x);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sP);
      for (int q = threadIdx.x; q < (int)(sizeof(SimParams) / 4); q += blockDim.x) dst[q] = src[q];
      if (threadIdx.x == 0) sSlot = it.x;
      __syncthreads();
    }
    f(static_cast<const SimParams&>(sP), it.y, k);
    if (!AHEAD && threadIdx.x == 0) sNext[p ^ 1] = atomicAdd(w.cursor, 1u);
    __syncthreads();  // the item is done with sP; sNext[p ^ 1] is visible
  }
}

// Warp-granular form for passes whose particles are independent: each warp pulls
// slices of 32 particles (item k = slice k % 8 of tile k / 8 of the segment) and
// calls f(P, li) with li the scene-local particle index of its lane. Warps never
// wait on one another, so a warp that finishes a slice early starts the next one
// instead of idling at a block barrier. Each warp keeps its own copy of the
// current scene's SimParams. f is called by all 32 lanes together.
constexpr int kSlices = kBlock / 32;
template <class F>
__device__ __forceinline__ void for_each_slice(const BatchWork& w, F&& f) {
  __shared__ __align__(16) SimParams sP[kSlices];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  SimParams& P = sP[warp];
  const WorkSeg seg = *w.seg;
  const uint32_t total = seg.count * (uint32_t)kSlices;
  uint32_t slot = 0xffffffffu, next = 0u;
  if (lane == 0) next = atomicAdd(w.cursor, 1u);
  next = __shfl_sync(0xffffffffu, next, 0);
  while (next < total) {
    const uint32_t k = next;
    if (lane == 0) next = atomicAdd(w.cursor, 1u);  // claim the next slice now
    const uint2 it = w.items[seg.off + k / kSlices];
    if (it.x != slot) {
      __syncwarp();
      const uint32_t* src = reinterpret_cast<const uint32_t*>(w.params + it.x);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&P);
      for (int q = lane; q < (int)(sizeof(SimParams) / 4); q += 32) dst[q] = src[q];
      __syncwarp();
      slot = it.x;
    }
    f(static_cast<const SimParams&>(P), it.y * (uint32_t)kBlock + (k % kSlices) * 32u + (uint32_t)lane);
    next = __shfl_sync(0xffffffffu, next, 0);
  }
}

}  // namespace p4a
