// kernels_grid.cu — the predict pass and the 'grid' pass of Sim.step
// (src/wgsl.js:56-70, 352-475; schedule src/sim.js:473-492) as a stable counting
// sort on cell keys:
//   key_count  predict + cellOf + warp-aggregated atomic histogram; each particle
//              keeps the arrival rank its warp leader got for it
//   scan       single-pass decoupled-lookback exclusive scan of the histogram into
//              cellStart (and zeroes the histogram for the next substep)
//   fill       unordered[cellStart[key] + rank] = i   (a per-cell bucket list)
//   reorder    stable rank = #{ j in the particle's bucket : j < i }, then the
//              permutation of pos/vel/pred/body/rest into cell order
// The reference's scatterSlot takes slots in atomic order (src/wgsl.js:436), so its
// in-cell order is whatever the hardware produced; here it is the stable order
// (ties by pre-sort index), which is one of the orders the reference can produce
// and is the same on every run.
#include <cuda_runtime.h>

#include "p4a_internal.h"
#include "p4a_math.cuh"

namespace p4a {

__global__ void __launch_bounds__(kBlock) k_key_count(const __grid_constant__ SimParams P,
                                                      const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel,
                                                      uint32_t* __restrict__ key,
                                                      uint32_t* __restrict__ rank,
                                                      uint32_t* __restrict__ cellCount,
                                                      uint32_t* __restrict__ bodyFill,
                                                      uint32_t nBodies) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (bodyFill && i < nBodies) bodyFill[i] = 0u;
  const bool act = i < P.n;
  uint32_t k = 0xffffffffu;
  if (act) {
    F3 v, pr;
    predict_one(P, __ldg(&pos[i]), __ldg(&vel[i]), v, pr);
    k = cell_index(P, cell_of(P, pr));
  }
  const unsigned peers = __match_any_sync(0xffffffffu, k);
  if (act) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    const uint32_t lt = peers & ((1u << lane) - 1u);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&cellCount[k], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    key[i] = k;
    rank[i] = base + (uint32_t)__popc(lt);
  }
}

// Tile status word: epoch (30 bits) | flag (2 bits) | value (32 bits).
constexpr unsigned long long kFlagAgg = 1ull, kFlagPrefix = 2ull;
__device__ __forceinline__ unsigned long long pack_state(uint32_t epoch, unsigned long long flag, uint32_t v) {
  return ((unsigned long long)epoch << 34) | (flag << 32) | (unsigned long long)v;
}

__global__ void __launch_bounds__(kBlock) k_scan(uint32_t* __restrict__ cellCount,
                                                 uint32_t* __restrict__ cellStart, int nCells,
                                                 unsigned long long* __restrict__ state,
                                                 uint32_t* __restrict__ ticket, uint32_t epoch,
                                                 int nTiles, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ uint32_t s_warp[kBlock / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int tile = (int)s_tile;
  if (tile >= nTiles) {  // only after an earlier launch failed mid-way: never index past the state
    if (threadIdx.x == 0) atomicOr(err, ERR_SCAN_TIMEOUT);
    return;
  }
  const long long base = (long long)tile * kScanTile + (long long)tid * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    v[j] = idx < nCells ? cellCount[idx] : 0u;
    sum += v[j];
  }
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    if (idx < nCells) cellCount[idx] = 0u;
  }
  // block exclusive scan of the per-thread sums
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kBlock / 32 ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < kBlock / 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kBlock / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
    const uint32_t aggregate = __shfl_sync(0xffffffffu, wi, kBlock / 32 - 1);
    if (lane == 0) {
      uint32_t exclusive = 0;
      if (tile == 0) {
        atomicExch(&state[0], pack_state(epoch, kFlagPrefix, aggregate));
      } else {
        atomicExch(&state[tile], pack_state(epoch, kFlagAgg, aggregate));
        int j = tile - 1;
        uint32_t spins = 0;
        while (j >= 0) {
          const unsigned long long w64 = *((volatile unsigned long long*)&state[j]);
          const uint32_t we = (uint32_t)(w64 >> 34);
          const unsigned long long wf = (w64 >> 32) & 3ull;
          if (we != epoch || wf == 0ull) {
            if (++spins > (1u << 22)) {  // bounded wait: flag the error and stop looking
              atomicOr(err, ERR_SCAN_TIMEOUT);
              break;
            }
            __nanosleep(64);
            continue;
          }
          exclusive += (uint32_t)w64;
          if (wf == kFlagPrefix) break;
          j--;
        }
        atomicExch(&state[tile], pack_state(epoch, kFlagPrefix, exclusive + aggregate));
      }
      s_prefix = exclusive;
      if (tile == nTiles - 1) {
        cellStart[nCells] = exclusive + aggregate;
        *ticket = 0u;  // every tile has taken its ticket; reset for the next launch
      }
    }
  }
  __syncthreads();
  uint32_t run = s_prefix + s_warp[warp] + (incl - sum);
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    if (idx < nCells) cellStart[idx] = run;
    run += v[j];
  }
}

__global__ void __launch_bounds__(kBlock) k_fill(uint32_t n, const uint32_t* __restrict__ key,
                                                 const uint32_t* __restrict__ rank,
                                                 const uint32_t* __restrict__ cellStart,
                                                 uint32_t* __restrict__ unordered) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const uint32_t at = __ldg(&cellStart[key[i]]) + rank[i];
  if (at < n) unordered[at] = i;  // always true after a completed scan
}

__global__ void __launch_bounds__(kBlock) k_reorder(
    const __grid_constant__ SimParams P, const uint32_t* __restrict__ key,
    const uint32_t* __restrict__ cellStart, const uint32_t* __restrict__ unordered,
    const float4* __restrict__ pos, const float4* __restrict__ vel, const uint4* __restrict__ body,
    const float4* __restrict__ rest, float4* __restrict__ posOut, float4* __restrict__ velOut,
    float4* __restrict__ predOut, uint4* __restrict__ bodyOut, float4* __restrict__ restOut,
    uint32_t* __restrict__ slotOut, const uint32_t* __restrict__ bodyStart,
    uint32_t* __restrict__ bodyFill, uint32_t* __restrict__ bodyList) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= P.n) return;
  const uint32_t k = key[i];
  // min() keeps every access in bounds even if a scan gave up (error word set)
  const uint32_t e = min(__ldg(&cellStart[k + 1]), P.n), b = min(__ldg(&cellStart[k]), e);
  uint32_t r = 0;
  for (uint32_t m = b; m < e; m++) r += __ldg(&unordered[m]) < i ? 1u : 0u;
  const uint32_t s = min(b + r, P.n - 1u);
  const float4 p4 = __ldg(&pos[i]);
  F3 v, pr;
  predict_one(P, p4, __ldg(&vel[i]), v, pr);
  posOut[s] = p4;
  velOut[s] = make_float4(v.x, v.y, v.z, 0.0f);
  predOut[s] = make_float4(pr.x, pr.y, pr.z, 1.0f);
  if (body) {
    const uint4 bd = __ldg(&body[i]);
    bodyOut[s] = bd;
    if (bodyList && bd.x != 0u && bd.x <= P.nBodies) {
      const uint32_t slot = atomicAdd(&bodyFill[bd.x - 1u], 1u);
      const uint32_t at = bodyStart[bd.x - 1u] + slot;
      if (at < bodyStart[bd.x]) bodyList[at] = s;
    }
  }
  if (rest) restOut[s] = __ldg(&rest[i]);
  if (slotOut) slotOut[i] = s;
}

void launch_key_count(const SimParams& P, const float4* pos, const float4* vel, uint32_t* key,
                      uint32_t* rank, uint32_t* cellCount, uint32_t* bodyFill, uint32_t nBodies,
                      cudaStream_t st) {
  const long long work = (long long)P.n > (long long)nBodies ? P.n : nBodies;
  k_key_count<<<groups(work), kBlock, 0, st>>>(P, pos, vel, key, rank, cellCount, bodyFill, nBodies);
}

void launch_scan(uint32_t* cellCount, uint32_t* cellStart, int nCells, unsigned long long* state,
                 uint32_t* ticket, uint32_t epoch, uint32_t* err, cudaStream_t st) {
  const int tiles = scan_tiles(nCells);
  k_scan<<<tiles, kBlock, 0, st>>>(cellCount, cellStart, nCells, state, ticket, epoch, tiles, err);
}

void launch_fill(uint32_t n, const uint32_t* key, const uint32_t* rank, const uint32_t* cellStart,
                 uint32_t* unordered, cudaStream_t st) {
  k_fill<<<groups(n), kBlock, 0, st>>>(n, key, rank, cellStart, unordered);
}

void launch_reorder(const SimParams& P, const uint32_t* key, const uint32_t* cellStart,
                    const uint32_t* unordered, const float4* pos, const float4* vel,
                    const uint4* body, const float4* rest, float4* posOut, float4* velOut,
                    float4* predOut, uint4* bodyOut, float4* restOut, uint32_t* slotOut,
                    const uint32_t* bodyStart, uint32_t* bodyFill, uint32_t* bodyList,
                    cudaStream_t st) {
  k_reorder<<<groups(P.n), kBlock, 0, st>>>(P, key, cellStart, unordered, pos, vel, body, rest,
                                            posOut, velOut, predOut, bodyOut, restOut, slotOut,
                                            bodyStart, bodyFill, bodyList);
}

}  // namespace p4a
