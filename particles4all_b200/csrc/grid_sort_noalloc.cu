// grid_sort_noalloc.cu — p4a_grid_sort_noalloc: the predict + grid-sort operator
// for callers that cannot allocate device memory.
//
// Who needs it: hosts that own every device allocation themselves (a renderer or
// plugin host with a fixed memory budget and its own arena) and real-time frame
// loops where a cudaMalloc, which may synchronise the device, would stall the
// frame. Such callers can pass their input and output buffers but cannot hand the
// operator a workspace, so the operator's scratch (cell keys, arrival ranks, the
// bucket lists, the cell histogram and the scan's tile states) lives in one
// file-scope device array instead. That array is part of the library image: every
// GPU that loads libp4a holds it until the process exits.
//
// The entry point calls no cudaMalloc, cudaFree or other allocating routine. On the
// first call on a device it looks up the array's device address with
// cudaGetSymbolAddress (once per device, under a lock); make that first call before
// any stream capture. The address is kept for the life of the process, so a
// cudaDeviceReset after the first call on that device is not supported (the
// library image may be loaded again at another address). The array is shared by
// every call: the parts that must start at zero (the histogram and scan tile states
// this call's cell count uses, the ticket and the error word) are cleared on the
// caller's stream at the start of each call, and calls whose work overlaps on the
// GPU (different streams, or different host threads without ordering) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/p4a.h"
#include "p4a_internal.h"

namespace p4a {
namespace {
constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kMaxN = P4A_NOALLOC_MAX_PARTICLES;
constexpr size_t kMaxCells = P4A_NOALLOC_MAX_CELLS;
constexpr size_t kMaxTiles = (kMaxCells + kScanTile - 1) / kScanTile;
// layout: key, rank, unordered | ticket, error word | cellCount | scan tile states
// (the ticket and error word sit right before the histogram, so one clear covers
// them and the histogram's first cells+1 entries)
constexpr size_t kOffRank = align256(kMaxN * 4);
constexpr size_t kOffUnordered = kOffRank + align256(kMaxN * 4);
constexpr size_t kOffTicket = kOffUnordered + align256(kMaxN * 4);
constexpr size_t kOffErr = kOffTicket + 4;
constexpr size_t kOffCount = kOffTicket + 256;
constexpr size_t kOffState = kOffCount + align256((kMaxCells + 1) * 4);
constexpr size_t kScratchBytes = kOffState + align256(kMaxTiles * 8);
}  // namespace
}  // namespace p4a

// The operator's scratch, one per device that loads the library.
static __device__ __align__(256) unsigned char g_noalloc_scratch[p4a::kScratchBytes];

namespace p4a {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return P4A_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return P4A_ERR_NODEV;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return P4A_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return P4A_OK;
}

}  // namespace
}  // namespace p4a

extern "C" int p4a_grid_sort_noalloc(const p4a_grid* grid, int32_t n, float dt, float gravity,
                                     const float* pos, const float* vel, const uint32_t* body,
                                     const float* rest, float* pos_out, float* vel_out,
                                     float* pred_out, uint32_t* body_out, float* rest_out,
                                     uint32_t* cell_start, uint32_t* slot_out, uint32_t* status,
                                     void* stream) {
  using namespace p4a;
  long long cells = 0;
  int rc = grid_sort_check(grid, n, (long long)kMaxCells, &cells);
  if (rc != P4A_OK) return rc;
  if ((size_t)n > kMaxN) return P4A_ERR_CAPACITY;
  if (n > 0 && (!pos || !vel || !pos_out || !vel_out || !pred_out)) return P4A_ERR_ARG;
  if ((body && !body_out) || (rest && !rest_out) || !cell_start) return P4A_ERR_ARG;
  void* base = nullptr;
  rc = scratch_address(&base);
  if (rc != P4A_OK) return rc;
  char* w = (char*)base;
  uint32_t* key = (uint32_t*)w;
  uint32_t* rank = (uint32_t*)(w + kOffRank);
  uint32_t* unordered = (uint32_t*)(w + kOffUnordered);
  uint32_t* ticket = (uint32_t*)(w + kOffTicket);
  uint32_t* errw = (uint32_t*)(w + kOffErr);
  uint32_t* cellCount = (uint32_t*)(w + kOffCount);
  unsigned long long* state = (unsigned long long*)(w + kOffState);
  cudaStream_t st = (cudaStream_t)stream;
  // ticket, error word, the histogram's cells + 1 entries and this call's tile
  // states start at zero on every call; nothing beyond what the call uses is cleared
  const size_t countBytes = (kOffCount - kOffTicket) + ((size_t)cells + 1) * 4;
  const size_t stateBytes = (size_t)scan_tiles((int)cells) * 8;
  if (cudaMemsetAsync(ticket, 0, countBytes, st) != cudaSuccess) return P4A_ERR_CUDA;
  if (cudaMemsetAsync(state, 0, stateBytes, st) != cudaSuccess) return P4A_ERR_CUDA;
  return grid_sort_launch(*grid, n, dt, gravity, pos, vel, body, rest, pos_out, vel_out, pred_out, body_out,
                          rest_out, cell_start, slot_out, key, rank, unordered, cellCount, state, ticket, errw,
                          status, st);
}
