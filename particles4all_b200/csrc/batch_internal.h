// batch_internal.h — the batched engine's host-side state, shared by the batch
// API (batch.cu) and the serving loop (server.cu).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/p4a.h"
#include "p4a_internal.h"
#include "scene.h"

namespace p4a {

constexpr int kMaxSubsteps = 64;  // per frame (the time bank caps at 8 x substeps)

// First-fit allocator of aligned ranges in [0, capacity).
class RangeAlloc {
 public:
  void init(int64_t cap) {
    free_.clear();
    cap_ = cap;
    if (cap > 0) free_[0] = cap;
  }
  int64_t alloc(int64_t size, int64_t align) {
    if (size <= 0) size = 1;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      const int64_t start = (it->first + align - 1) / align * align;
      const int64_t end = it->first + it->second;
      if (start + size > end) continue;
      const int64_t f0 = it->first;
      free_.erase(it);
      if (start > f0) free_[f0] = start - f0;
      if (end > start + size) free_[start + size] = end - (start + size);
      return start;
    }
    return -1;
  }
  void release(int64_t off, int64_t size) {
    if (size <= 0) size = 1;
    auto it = free_.emplace(off, size).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t free_total() const {
    int64_t t = 0;
    for (auto& kv : free_) t += kv.second;
    return t;
  }

 private:
  std::map<int64_t, int64_t> free_;
  int64_t cap_ = 0;
};

struct Range {
  int64_t off = -1, size = 0;
};

struct BScene {
  bool live = false;
  p4a_params params{};
  std::vector<p4a_body_spec> specs;
  double mass = 0, denomRest = 0, h = 0;
  int n = 0, nFluid = 0, cap = 0, nBodies = 0, nBodyParts = 0, nBoundary = 0;
  int gridDim[3] = {1, 1, 1};
  int nCells = 1;
  double bodyScale = 0, covScale = 0;
  Range part, cells, bodies, list, bound;
  int parity = 0;
  double timeBank = 0, simTime = 0, lastAdvanced = 0;
  int lastSubsteps = 0;
  int gen = 0;
  bool statsValid = false;
  bool primed = false;
  SimParams P{};
};

}  // namespace p4a

struct p4a_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  std::string err;
  p4a_batch_config cfg{};
  p4a::DevScene d{};
  std::vector<void*> allocs;
  size_t deviceBytes = 0;
  bool sizeOnly = false;  // balloc counts bytes instead of allocating (p4a_batch_footprint)
  p4a::RangeAlloc partA, cellA, boundA, bodyA, listA;
  std::vector<p4a::BScene> scenes;
  int64_t scanTilesCap = 0;
  // Frame lanes. A lane holds what its frames upload (params rows, items, segments,
  // through double-buffered pinned staging), their pull cursors, and the CUDA graphs
  // of the frame shapes (substeps and iterations per substep), captured with the
  // lane's table addresses. Lane 0 runs on the batch's stream, every other lane on a
  // stream of its own: p4a_batch_step splits a large frame into parts that run at
  // once, one per lane, so that the launch tails of one part overlap the others' work.
  struct Lane {
    cudaStream_t stream = nullptr;       // lane 0: the batch's stream
    p4a::SimParams* dParams = nullptr;   // [kMaxSubsteps][max_scenes], row k = the frame's k-th scene
    uint2* dItems = nullptr;
    int64_t itemsCap = 0;
    p4a::WorkSeg* dSegs = nullptr;       // one per launch of the frame
    uint32_t* dCursors = nullptr;        // pull cursors, one per launch
    int64_t launchCap = 0;
    unsigned char* staging[2] = {nullptr, nullptr};
    size_t stagingCap = 0;
    cudaEvent_t stagingDone[2] = {nullptr, nullptr};
    int stagingIdx = 0;
    std::map<std::vector<int>, cudaGraphExec_t> graphs;
  };
  static constexpr int kMaxLanes = 4;
  Lane lanes[kMaxLanes];
  Lane* lane = &lanes[0];          // the lane the next frame runs on
  int laneCount = 2;               // p4a_batch_set_lanes
  int64_t laneMinParticles = 1000000;
  cudaEvent_t laneFork = nullptr;
  cudaEvent_t laneJoin[kMaxLanes] = {};
  bool useGraphs = true;
  cudaStream_t upStream = nullptr;  // admissions' uploads (serving loop)
  // p4a_batch_step_io: a stream per copy direction and the events that order the
  // copies against the frames ([0] the call's start, [1 + 2g] group g written,
  // [2 + 2g] group g stepped, then the reads' end)
  cudaStream_t h2dStream = nullptr, d2hStream = nullptr;
  std::vector<cudaEvent_t> ioEvents;
  // per-kernel timing of frames (p4a_batch_profile_*): an event before every launch
  // of a frame and one after the last; in a graph these are event-record nodes,
  // pointed at a fresh set of events before each replay
  struct ProfNodes {
    cudaGraph_t graph = nullptr;            // kept: the exec's nodes belong to it
    std::vector<cudaGraphNode_t> nodes;     // event-record node of event index k
  };
  struct ProfPending {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kinds;  // launch kind of interval k (-1: nothing launched)
  };
  bool prof = false;
  std::map<std::vector<int>, ProfNodes> profNodes;  // by graph key
  std::vector<std::vector<cudaEvent_t>> profFree;
  std::vector<ProfPending> profPending;
  double profMs[16] = {};
  long long profLaunches[16] = {};
};


namespace p4a {

// Host part of an admission, computed without the device: the scene's counts,
// fixed-point scales and boundary samples, and the bytes to upload (values relative
// to the scene's own ranges; place_scene adds the arena offsets).
struct PreparedScene {
  BScene s;
  HostScene sc;
  HostBoundary hb;
  std::vector<int> bodyCounts;
  int nb1 = 1;
  // byte offsets of the pieces in the upload blob
  size_t oPos = 0, oVel = 0, oPhase = 0, oRest = 0, oBpos = 0, oBpsi = 0, oBcs = 0, oInfo = 0,
         oCentre = 0, oRot = 0, oBstart = 0, bytes = 0;
};

int bfail(p4a_batch* b, int code, const char* fmt, ...);
#define BTRY(b, call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return ::p4a::bfail((b), e_ == cudaErrorMemoryAllocation ? P4A_ERR_OOM : P4A_ERR_CUDA, \
                          "%s: %s", #call, cudaGetErrorString(e_));                      \
  } while (0)
// Fills ps from a built scene (no CUDA calls; safe on any thread). Returns a status.
int prepare_scene(const p4a_params& params, HostScene& sc, int pourBudget, PreparedScene& ps,
                  std::string& err);
// Writes the upload blob of ps into `blob` (ps.bytes bytes of host memory).
void write_blob(const PreparedScene& ps, unsigned char* blob);
// Takes a free slot and arena ranges for ps (P4A_ERR_CAPACITY when full: nothing is
// kept), adds the ranges' offsets to the blob and enqueues the clears and copies on
// `st`. The blob must stay valid until that work is done. The scene is not primed.
int place_scene(p4a_batch* b, PreparedScene& ps, unsigned char* blob, cudaStream_t st, int32_t* slot);
// The prime frame (src/sim.js:223-253) of placed scenes, one set of launches for all,
// on the batch's stream.
int prime_scenes(p4a_batch* b, const std::vector<int>& slots);
// One frame: each listed scene advances by its own frame_dt (time bank and substeps).
int step_frame(p4a_batch* b, const int32_t* ids, const double* frameDt, int32_t count);
// step_frame split across the batch's two frame lanes when the frame is large.
int step_scenes(p4a_batch* b, const int32_t* ids, const double* dts, int32_t count);
// Device pointer and byte size of a scene's view of buffer `id` (P4A_BUF_*), copy
// `which` (P4A_LIVE, P4A_A, P4A_B).
int scene_buffer(p4a_batch* b, const BScene& s, int32_t id, int32_t which, void** p, size_t* bytes);
// Returns a scene's arena ranges and slot; the caller guarantees no queued work uses them.
void release_scene(p4a_batch* b, BScene& s);

}  // namespace p4a
