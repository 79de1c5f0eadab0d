// kernels_grid.cu — the predict pass and the 'grid' pass of Sim.step
// (src/wgsl.js:56-70, 352-475; schedule src/sim.js:473-492) as a stable counting
// sort on cell keys:
//   key_count  predict + cellOf + warp-aggregated atomic histogram; each particle
//              keeps the arrival rank its warp leader got for it
//   scan       single-pass decoupled-lookback exclusive scan of the histogram into
//              cellStart (and zeroes the histogram for the next substep); the
//              batched form restarts the scan at every scene, seeded with the
//              scene's first particle index
//   fill       unordered[cellStart[key] + rank] = i   (a per-cell bucket list)
//   reorder    stable rank = #{ j in the particle's bucket : j < i }, then the
//              permutation of pos/vel/pred/body/rest into cell order
// The reference's scatterSlot takes slots in atomic order (src/wgsl.js:436), so its
// in-cell order is whatever the hardware produced; here it is the stable order
// (ties by pre-sort index), which is one of the orders the reference can produce
// and is the same on every run. The pass reads parity P.parity and writes the
// other parity.
#include <cuda_runtime.h>

#include "p4a_internal.h"
#include "p4a_math.cuh"
#include "pass_common.cuh"

namespace p4a {

__device__ __forceinline__ void key_count_body(const SimParams& P, const DevScene& d, uint32_t li) {
  if (d.bodyFill && li < P.nBodies) d.bodyFill[P.bOff + li] = 0u;
  if (d.disp && li < (uint32_t)kDispSlots) d.disp[P.slot * kDispSlots + li] = 0.0f;
  const bool act = li < P.n;
  const uint32_t i = P.pOff + li;
  uint32_t k = 0xffffffffu;
  if (act) {
    F3 v, pr;
    predict_one(P, __ldg(&d.pos[P.parity][i]), __ldg(&d.vel[P.parity][i]), v, pr);
    k = P.cOff + cell_index(P, cell_of(P, pr));
  }
  const unsigned peers = __match_any_sync(0xffffffffu, k);
  if (act) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    const uint32_t lt = peers & ((1u << lane) - 1u);
    uint32_t base = 0;
    if (lane == leader) {
      base = atomicAdd(&d.cellCount[k], (uint32_t)__popc(peers));
      // this substep's per-cell displacement slots start at zero for every occupied
      // cell (list reuse only: a slot left larger makes the bound looser, never wrong).
      // Done here by the warp leaders rather than in the scan: measured cheaper, the
      // stores hide among the key pass's loads (a clear in the batched scan cost
      // ~60 us per launch on the 96-scene mix and saved ~6 us here).
      if (d.cellDisp) {
        const uint32_t slots = min(P.iters, (uint32_t)kDispSlots);
        for (uint32_t t = 0; t < slots; t++) d.cellDisp[(size_t)t * d.cellStride + k] = 0.0f;
      }
    }
    base = __shfl_sync(peers, base, leader);
    d.key[i] = k;
    d.rank[i] = base + (uint32_t)__popc(lt);
  }
}

__device__ __forceinline__ void fill_body(const SimParams& P, const DevScene& d, uint32_t li) {
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const uint32_t at = __ldg(&d.cellStart[d.key[i]]) + d.rank[i];
  if (at < P.pEnd) d.unordered[at] = i;  // always true after a completed scan
}

__device__ __forceinline__ void reorder_body(const SimParams& P, const DevScene& d, uint32_t li) {
  if (li >= P.n) return;
  const uint32_t i = P.pOff + li;
  const int src = P.parity, dst = P.parity ^ 1;
  const uint32_t k = d.key[i];
  // min() keeps every access in bounds even if a scan gave up (error word set)
  const uint32_t e = min(__ldg(&d.cellStart[k + 1]), P.pEnd);
  const uint32_t b = min(__ldg(&d.cellStart[k]), e);
  uint32_t r = 0;
  for (uint32_t m = b; m < e; m++) r += __ldg(&d.unordered[m]) < i ? 1u : 0u;
  const uint32_t s = min(b + r, P.pEnd - 1u);
  const float4 p4 = __ldg(&d.pos[src][i]);
  F3 v, pr;
  predict_one(P, p4, __ldg(&d.vel[src][i]), v, pr);
  d.pos[dst][s] = p4;
  d.vel[dst][s] = make_float4(v.x, v.y, v.z, 0.0f);
  d.pred[dst][s] = make_float4(pr.x, pr.y, pr.z, 1.0f);
  if (d.body[src]) {
    const uint4 bd = __ldg(&d.body[src][i]);
    d.body[dst][s] = bd;
    if (d.bodyList && bd.x != 0u && bd.x <= P.nBodies) {
      const uint32_t gb = P.bOff + bd.x - 1u;
      const uint32_t slot = atomicAdd(&d.bodyFill[gb], 1u);
      const uint32_t at = d.bodyStart[gb] + slot;
      if (at < d.bodyStart[gb + 1]) d.bodyList[at] = s;
    }
  }
  if (d.rest[src]) d.rest[dst][s] = __ldg(&d.rest[src][i]);
  if (d.slotOut) d.slotOut[li] = s - P.pOff;
}

__global__ void __launch_bounds__(kBlock) k_key_count(const __grid_constant__ SimParams P,
                                                      const __grid_constant__ DevScene d) {
  key_count_body(P, d, blockIdx.x * kBlock + threadIdx.x);
}
// The batched streaming passes take whole 256-particle tiles per claim (one atomic
// per tile instead of one per 32-particle slice: their per-particle work is short,
// so a cursor shared by every warp would serialise them).
__global__ void __launch_bounds__(kBlock) k_key_count_b(const __grid_constant__ BatchWork w,
                                                        const __grid_constant__ DevScene d) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { key_count_body(P, d, t * kBlock + threadIdx.x); });
}
__global__ void __launch_bounds__(kBlock) k_fill(const __grid_constant__ SimParams P,
                                                 const __grid_constant__ DevScene d) {
  fill_body(P, d, blockIdx.x * kBlock + threadIdx.x);
}
__global__ void __launch_bounds__(kBlock) k_fill_b(const __grid_constant__ BatchWork w,
                                                   const __grid_constant__ DevScene d) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { fill_body(P, d, t * kBlock + threadIdx.x); });
}
__global__ void __launch_bounds__(kBlock) k_reorder(const __grid_constant__ SimParams P,
                                                    const __grid_constant__ DevScene d) {
  reorder_body(P, d, blockIdx.x * kBlock + threadIdx.x);
}
__global__ void __launch_bounds__(kBlock) k_reorder_b(const __grid_constant__ BatchWork w,
                                                      const __grid_constant__ DevScene d) {
  for_each_item(w, [&](const SimParams& P, uint32_t t, uint32_t) { reorder_body(P, d, t * kBlock + threadIdx.x); });
}

// Tile status word: epoch (30 bits) | flag (2 bits) | value (32 bits).
constexpr unsigned long long kFlagAgg = 1ull, kFlagPrefix = 2ull;

// A predecessor's status word, read at GPU scope every time (the word is published
// with an atomic at L2; a load that may be served from the SM's L1 could keep
// returning the stale word).
__device__ __forceinline__ unsigned long long load_state(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long pack_state(uint32_t epoch, unsigned long long flag, uint32_t v) {
  return ((unsigned long long)epoch << 34) | (flag << 32) | (unsigned long long)v;
}

// One scan tile: loads up to kScanTile counts at cells [base, base + kScanTile)
// clipped to `limit`, zeroes them, and writes the exclusive prefix seeded with
// the tile's predecessors (lookback down to tile `firstTile`, which is seeded with
// `seed`). Returns nothing; the last tile of a segment writes the segment total.
__device__ __forceinline__ void scan_tile(uint32_t* __restrict__ cellCount,
                                          uint32_t* __restrict__ cellStart, long long cellBase,
                                          long long limit, int tile, int firstTile, uint32_t seed,
                                          bool lastOfSegment, unsigned long long* __restrict__ state,
                                          uint32_t epoch, uint32_t* __restrict__ err, uint32_t spinLimit) {
  __shared__ uint32_t s_prefix;
  __shared__ uint32_t s_warp[kBlock / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long base = cellBase + (long long)tid * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    v[j] = idx < limit ? cellCount[idx] : 0u;
    sum += v[j];
  }
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    if (idx < limit) cellCount[idx] = 0u;
  }
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t wv = lane < kBlock / 32 ? s_warp[lane] : 0u;
    uint32_t wi = wv;
#pragma unroll
    for (int o = 1; o < kBlock / 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kBlock / 32) s_warp[lane] = wi - wv;  // exclusive warp offsets
    const uint32_t aggregate = __shfl_sync(0xffffffffu, wi, kBlock / 32 - 1);
    uint32_t exclusive = seed;
    if (tile == firstTile) {
      if (lane == 0) atomicExch(&state[tile], pack_state(epoch, kFlagPrefix, seed + aggregate));
    } else {
      if (lane == 0) atomicExch(&state[tile], pack_state(epoch, kFlagAgg, aggregate));
      // Warp-wide lookback: lane l reads the state of tile top - l, 32 predecessors
      // per step. The nearest tile with an inclusive prefix ends the walk; every
      // tile between it and this one must have published its aggregate first.
      // Tiles before the segment's first count as a prefix of 0 (the first tile
      // always publishes one, so the walk never passes it).
      exclusive = 0;
      int top = tile - 1;
      uint32_t spins = 0;
      while (true) {
        const int t = top - lane;
        bool ready = true, prefix = true;
        uint32_t value = 0;
        if (t >= firstTile) {
          const unsigned long long w64 = load_state(&state[t]);
          const unsigned long long wf = (w64 >> 32) & 3ull;
          ready = (uint32_t)(w64 >> 34) == epoch && wf != 0ull;
          prefix = ready && wf == kFlagPrefix;
          value = (uint32_t)w64;
        }
        const uint32_t prefixes = __ballot_sync(0xffffffffu, prefix);
        const uint32_t waiting = __ballot_sync(0xffffffffu, !ready);
        const int first = prefixes ? __ffs(prefixes) - 1 : 31;  // nearest prefix lane, or the window
        const uint32_t span = first == 31 ? 0xffffffffu : ((2u << first) - 1u);
        if (waiting & span) {
          if (++spins > spinLimit) {  // bounded wait: flag the error and stop looking
            if (lane == 0) atomicOr(err, ERR_SCAN_TIMEOUT);
            break;
          }
          __nanosleep(64);
          continue;
        }
        uint32_t part = lane <= first ? value : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        exclusive += part;
        if (prefixes) break;
        top -= 32;
      }
      if (lane == 0) atomicExch(&state[tile], pack_state(epoch, kFlagPrefix, exclusive + aggregate));
    }
    if (lane == 0) {
      s_prefix = exclusive;
      if (lastOfSegment) cellStart[limit] = exclusive + aggregate;
    }
  }
  __syncthreads();
  uint32_t run = s_prefix + s_warp[warp] + (incl - sum);
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    if (idx < limit) cellStart[idx] = run;
    run += v[j];
  }
}

__global__ void __launch_bounds__(kBlock) k_scan(uint32_t* __restrict__ cellCount,
                                                 uint32_t* __restrict__ cellStart, int nCells,
                                                 unsigned long long* __restrict__ state,
                                                 uint32_t* __restrict__ ticket, uint32_t epoch,
                                                 int nTiles, uint32_t* __restrict__ err, uint32_t spinLimit) {
  __shared__ uint32_t s_tile;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const int tile = (int)s_tile;
  if (tile >= nTiles) {  // only after an earlier launch failed mid-way: never index past the state
    if (threadIdx.x == 0) atomicOr(err, ERR_SCAN_TIMEOUT);
    return;
  }
  scan_tile(cellCount, cellStart, (long long)tile * kScanTile, nCells, tile, 0, 0u,
            tile == nTiles - 1, state, epoch, err, spinLimit);
  if (threadIdx.x == 0 && tile == nTiles - 1) *ticket = 0u;  // all tickets taken: reset
}

// Batched: a three-phase scan with no waiting, over items[g] = (scene slot, local
// tile) in scene order (every scene's tiles are scanned on their own, seeded with
// the scene's first particle index):
//   sums     each tile's cell total into tileSum[g];
//   offsets  the block that gets a scene's first tile scans that scene's tile sums
//            into tileOffset[g] = pOff + the sum of the scene's earlier tiles;
//   apply    each tile's exclusive scan from tileOffset[g]: cellStart, the cleared
//            histogram, and the scene's total from its last tile.
// tileSum and tileOffset share the scan-state array (two u32 per tile). The
// single-pass lookback of the plain scan serialised here: with thousands of tiles
// of ~100 scenes in flight, its waits chained (178 us for 9.2 M cells).
__device__ __forceinline__ uint32_t tile_counts(const uint32_t* __restrict__ cellCount, long long base,
                                                long long limit, uint32_t (&v)[kScanItems]) {
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const long long idx = base + j;
    v[j] = idx < limit ? cellCount[idx] : 0u;
    sum += v[j];
  }
  return sum;
}

// Block-wide exclusive scan of one value per thread; returns the thread's exclusive
// prefix and the block total in *total. Every thread of the block calls it.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t x, uint32_t* total) {
  __shared__ uint32_t s_w[kBlock / 32];
  __shared__ uint32_t s_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t wv = lane < kBlock / 32 ? s_w[lane] : 0u;
    uint32_t wi = wv;
#pragma unroll
    for (int o = 1; o < kBlock / 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kBlock / 32) s_w[lane] = wi - wv;
    if (lane == kBlock / 32 - 1) s_total = wi;
  }
  __syncthreads();
  const uint32_t r = s_w[warp] + (incl - x);
  *total = s_total;
  __syncthreads();  // s_w and s_total may be reused by the next call
  return r;
}

// Tile sums and offsets of the batched scan live at the scene's own tiles (its cell
// range starts on a tile boundary), so frames that run at once on different
// streams, with different scenes, never share a slot.
__device__ __forceinline__ size_t scene_tile0(const SimParams& P) { return (size_t)(P.cOff / kScanTile); }

__global__ void __launch_bounds__(kBlock) k_scan_sums_b(const __grid_constant__ BatchWork w,
                                                        const __grid_constant__ DevScene d) {
  uint32_t* tileSum = reinterpret_cast<uint32_t*>(d.scanState);
  for_each_item(w, [&](const SimParams& P, uint32_t lt, uint32_t) {
    const long long limit = (long long)P.cOff + P.nCells;
    const long long base = (long long)P.cOff + (long long)lt * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    const uint32_t sum = tile_counts(d.cellCount, base, limit, v);
    uint32_t total = 0;
    block_exclusive(sum, &total);
    if (threadIdx.x == 0) tileSum[2 * (scene_tile0(P) + lt)] = total;
  });
}

__global__ void __launch_bounds__(kBlock) k_scan_offsets_b(const __grid_constant__ BatchWork w,
                                                           const __grid_constant__ DevScene d) {
  uint32_t* st = reinterpret_cast<uint32_t*>(d.scanState);
  for_each_item(w, [&](const SimParams& P, uint32_t lt, uint32_t) {
    if (lt != 0u) return;  // the block that gets a scene's first tile scans the scene
    const uint32_t tiles = (uint32_t)((P.nCells + kScanTile - 1) / kScanTile);
    const size_t t0s = scene_tile0(P);
    uint32_t carry = P.pOff;
    for (uint32_t t0 = 0; t0 < tiles; t0 += kBlock) {
      const uint32_t t = t0 + threadIdx.x;
      const uint32_t x = t < tiles ? st[2 * (t0s + t)] : 0u;
      uint32_t total = 0;
      const uint32_t ex = block_exclusive(x, &total);
      if (t < tiles) st[2 * (t0s + t) + 1] = carry + ex;
      carry += total;
    }
  });
}

__global__ void __launch_bounds__(kBlock) k_scan_apply_b(const __grid_constant__ BatchWork w,
                                                         const __grid_constant__ DevScene d) {
  const uint32_t* st = reinterpret_cast<const uint32_t*>(d.scanState);
  for_each_item(w, [&](const SimParams& P, uint32_t lt, uint32_t) {
    const long long limit = (long long)P.cOff + P.nCells;
    const long long base = (long long)P.cOff + (long long)lt * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    const uint32_t sum = tile_counts(d.cellCount, base, limit, v);
#pragma unroll
    for (int j = 0; j < kScanItems; j++)
      if (base + j < limit) d.cellCount[base + j] = 0u;
    uint32_t total = 0;
    const uint32_t offset = st[2 * (scene_tile0(P) + lt) + 1];
    uint32_t run = offset + block_exclusive(sum, &total);
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
      if (base + j < limit) d.cellStart[base + j] = run;
      run += v[j];
    }
    if (threadIdx.x == 0 && (long long)(lt + 1) * kScanTile >= (long long)P.nCells) d.cellStart[limit] = offset + total;
  });
}

void launch_key_count(const SimParams& P, const DevScene& d, cudaStream_t st) {
  const long long work = (long long)P.n > (long long)P.nBodies ? P.n : P.nBodies;
  k_key_count<<<groups(work), kBlock, 0, st>>>(P, d);
}
void launch_scan(uint32_t* cellCount, uint32_t* cellStart, int nCells, unsigned long long* state,
                 uint32_t* ticket, uint32_t epoch, uint32_t* err, cudaStream_t st, uint32_t spinLimit) {
  const int tiles = scan_tiles(nCells);
  k_scan<<<tiles, kBlock, 0, st>>>(cellCount, cellStart, nCells, state, ticket, epoch, tiles, err, spinLimit);
}
void launch_fill(const SimParams& P, const DevScene& d, cudaStream_t st) {
  k_fill<<<groups(P.n), kBlock, 0, st>>>(P, d);
}
void launch_reorder(const SimParams& P, const DevScene& d, cudaStream_t st) {
  k_reorder<<<groups(P.n), kBlock, 0, st>>>(P, d);
}
cudaError_t run_grid_sort(const p4a_grid& g, int32_t n, float dt, float gravity, const float* pos,
                          const float* vel, const uint32_t* body, const float* rest, float* posOut,
                          float* velOut, float* predOut, uint32_t* bodyOut, float* restOut,
                          uint32_t* cellStart, uint32_t* slotOut, uint32_t* key, uint32_t* rank,
                          uint32_t* unordered, uint32_t* cellCount, unsigned long long* state,
                          uint32_t* ticket, uint32_t* err, cudaStream_t st, uint32_t spinLimit) {
  SimParams P{};
  for (int k = 0; k < 3; k++) {
    P.boxMin[k] = g.box_min[k];
    P.gridDim[k] = g.dim[k];
  }
  P.h = g.h;
  P.dt = dt;
  P.gravity = gravity;
  P.n = (uint32_t)n;
  P.pEnd = (uint32_t)n;
  const int nCells = g.dim[0] * g.dim[1] * g.dim[2];
  P.nCells = (uint32_t)nCells;
  DevScene d{};
  d.pos[0] = (float4*)pos; d.pos[1] = (float4*)posOut;
  d.vel[0] = (float4*)vel; d.vel[1] = (float4*)velOut;
  d.pred[1] = (float4*)predOut;
  d.body[0] = (uint4*)body; d.body[1] = (uint4*)bodyOut;
  d.rest[0] = (float4*)rest; d.rest[1] = (float4*)restOut;
  d.cellCount = cellCount;
  d.cellStart = cellStart;
  d.key = key;
  d.rank = rank;
  d.unordered = unordered;
  d.slotOut = slotOut;
  launch_key_count(P, d, st);
  launch_scan(cellCount, cellStart, nCells, state, ticket, 1u, err, st, spinLimit);
  launch_fill(P, d, st);
  launch_reorder(P, d, st);
  return cudaGetLastError();
}

void launch_key_count_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_key_count_b<<<persistent_grid((const void*)k_key_count_b, kBlock, maxItems), kBlock, 0, st>>>(w, d);
}
void launch_scan_sums_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_scan_sums_b<<<persistent_grid((const void*)k_scan_sums_b, kBlock, maxItems), kBlock, 0, st>>>(w, d);
}
void launch_scan_offsets_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_scan_offsets_b<<<persistent_grid((const void*)k_scan_offsets_b, kBlock, maxItems), kBlock, 0, st>>>(w, d);
}
void launch_scan_apply_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_scan_apply_b<<<persistent_grid((const void*)k_scan_apply_b, kBlock, maxItems), kBlock, 0, st>>>(w, d);
}
void launch_fill_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_fill_b<<<persistent_grid((const void*)k_fill_b, kBlock, maxItems), kBlock, 0, st>>>(w, d);
}
void launch_reorder_b(const BatchWork& w, int maxItems, const DevScene& d, cudaStream_t st) {
  k_reorder_b<<<persistent_grid((const void*)k_reorder_b, kBlock, maxItems), kBlock, 0, st>>>(w, d);
}

__global__ void __launch_bounds__(kBlock) k_zero_stats_b(const __grid_constant__ BatchWork w,
                                                         uint32_t* __restrict__ stats) {
  const WorkSeg seg = *w.seg;
  for (uint32_t t = blockIdx.x * kBlock + threadIdx.x; t < seg.count * 8u; t += gridDim.x * kBlock)
    stats[w.params[w.items[seg.off + t / 8u].x].slot * 8u + (t % 8u)] = 0u;
}
void launch_zero_stats_b(const BatchWork& w, uint32_t* stats, cudaStream_t st) {
  k_zero_stats_b<<<8, kBlock, 0, st>>>(w, stats);
}

}  // namespace p4a
