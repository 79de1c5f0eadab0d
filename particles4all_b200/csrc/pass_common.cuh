// pass_common.cuh — how the blocks of a batched launch find their work.
#pragma once
#include "p4a_internal.h"

namespace p4a {

// Batched form: the block pulls work items (scene slot, item) from its launch's
// segment, one per cursor increment, and calls f(P, item, k) for each, with P the
// item's SimParams in shared memory (reloaded only when the scene changes) and k
// the item's position in the segment. The next item is claimed while the current
// one runs, so the cursor's round trip is hidden. Items are claimed in increasing
// k and a block claims its next item only while working on one, so the smallest
// unfinished item is always being worked on: a block that waits on earlier items
// (the scan's lookback) waits on blocks that finish.
// f may contain block barriers: every thread of the block makes every call.
template <class F>
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
    if (threadIdx.x == 0) sNext[p ^ 1] = atomicAdd(w.cursor, 1u);
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
    __syncthreads();  // the item is done with sP; sNext[p ^ 1] is visible
  }
}

}  // namespace p4a
