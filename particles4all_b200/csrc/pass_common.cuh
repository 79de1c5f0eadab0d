// pass_common.cuh — how a block of a plain or batched launch finds its scene.
#pragma once
#include "p4a_internal.h"

namespace p4a {

// Batched form: loads the SimParams of this block's work item (scene slot, item)
// into shared memory and returns it; *item receives the tile or body index.
__device__ __forceinline__ const SimParams& batch_scene(const BatchWork& w, uint32_t& item) {
  __shared__ __align__(16) SimParams sP;
  const uint2 it = w.items[blockIdx.x];
  const uint32_t* src = reinterpret_cast<const uint32_t*>(w.params + it.x);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sP);
  for (int k = threadIdx.x; k < (int)(sizeof(SimParams) / 4); k += blockDim.x) dst[k] = __ldg(src + k);
  __syncthreads();
  item = it.y;
  return sP;
}

}  // namespace p4a
