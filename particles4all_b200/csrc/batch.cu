// batch.cu — batched multi-scene stepping (p4a_batch_*): many independent scenes in
// shared device arenas, every pass of a substep launched once for all of them.
//
// Layout: scene s owns the particle range [pOff, pOff + cap) of every particle
// array, the cell range [cOff, cOff + nCells + 2) (tile-aligned) of the cell arrays,
// the body range [bOff, bOff + nBodies + 1) of the body arrays, a bodyList range and
// a boundary-sample range. Cell keys carry cOff, so the counting sort of all listed
// scenes is one pass; the scan restarts at each scene, seeded with pOff, so
// cellStart holds arena particle indices and each scene's particles stay inside
// its range. Kernels pick their scene from a work list of (scene slot, item) pairs
// built on the host per frame and uploaded with the per-substep SimParams tables.
// Each distinct frame schedule is captured once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/p4a.h"
#include "p4a_internal.h"
#include "scene.h"

using namespace p4a;

namespace {

const double kPi = 3.14159265358979323846;
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
  SimParams P{};
};

// One launch of a frame schedule: a segment of the work-item buffer.
struct Seg {
  int64_t off = 0;
  int count = 0;
};

}  // namespace

struct p4a_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  std::string err;
  p4a_batch_config cfg{};
  DevScene d{};
  std::vector<void*> allocs;
  size_t deviceBytes = 0;
  RangeAlloc partA, cellA, boundA, bodyA, listA;
  std::vector<BScene> scenes;
  int64_t scanTilesCap = 0;
  // per-frame schedule upload (double-buffered pinned staging)
  SimParams* dParams = nullptr;  // [kMaxSubsteps][max_scenes]
  uint2* dItems = nullptr;
  int64_t itemsCap = 0;
  unsigned char* staging[2] = {nullptr, nullptr};
  size_t stagingCap = 0;
  cudaEvent_t stagingDone[2] = {nullptr, nullptr};
  int stagingIdx = 0;
  // CUDA graphs of frame schedules
  bool useGraphs = true;
  std::vector<int64_t> graphKey;
  cudaGraphExec_t graph = nullptr;
  uint64_t graphKernels = 0;  // kernels in the captured frame
};

namespace {

int bfail(p4a_batch* b, int code, const char* fmt, ...) {
  if (b) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    b->err = buf;
  }
  return code;
}

#define BTRY(b, call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return bfail((b), e_ == cudaErrorMemoryAllocation ? P4A_ERR_OOM : P4A_ERR_CUDA,    \
                   "%s: %s", #call, cudaGetErrorString(e_));                             \
  } while (0)

template <class T>
int balloc(p4a_batch* b, T** out, int64_t count) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(16, (size_t)count * sizeof(T));
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return bfail(b, P4A_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  if ((e = cudaMemset(p, 0, bytes)) != cudaSuccess) {
    cudaFree(p);
    return bfail(b, P4A_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
  }
  b->allocs.push_back(p);
  b->deviceBytes += bytes;
  *out = (T*)p;
  return P4A_OK;
}

// The uniform of one scene (src/sim.js:371-413) plus its arena placement.
void pack(BScene& s, double dt, int slot) {
  const p4a_params& p = s.params;
  SimParams& F = s.P;
  const double h = s.h, d = p.spacing;
  F.boxMin[0] = F.boxMin[1] = F.boxMin[2] = 0.0f;
  F.dt = (float)dt;
  for (int k = 0; k < 3; k++) F.boxMax[k] = (float)p.box[k];
  F.h = (float)h;
  for (int k = 0; k < 3; k++) F.gridDim[k] = s.gridDim[k];
  F.h2 = (float)(h * h);
  const double halfD = 0.5 * d;
  for (int k = 0; k < 3; k++) F.clampMin[k] = (float)halfD;
  const double poly6 = 315 / (64 * kPi * std::pow(h, 9));
  F.poly6 = (float)poly6;
  for (int k = 0; k < 3; k++) F.clampMax[k] = (float)(p.box[k] - halfD);
  F.spikyGrad = (float)(-45 / (kPi * std::pow(h, 6)));
  F.gravity = (float)p.gravity;
  F.mass = (float)s.mass;
  F.rho0 = (float)p.rest_density;
  F.invRho0 = (float)(1 / p.rest_density);
  F.cfmEps = (float)(p.cfm_epsilon_abs > 0 ? p.cfm_epsilon_abs
                                           : std::max(1e-9, p.cfm_epsilon_rel * s.denomRest));
  F.sCorrK = (float)(p.s_corr_k / (s.denomRest * std::max(1, p.iterations)));
  const double rq = p.s_corr_dq * h, tq = h * h - rq * rq;
  const double wq = poly6 * tq * tq * tq;
  F.sCorrWq = (float)(wq > 0 ? 1 / wq : 0);
  F.xsphC = (float)p.xsph_c;
  F.n = (uint32_t)s.n;
  F.nCells = (uint32_t)s.nCells;
  F.nBoundary = p.no_boundary ? 0u : (uint32_t)s.nBoundary;
  F.nBodyParts = (uint32_t)s.nBodyParts;
  F.nBodies = (uint32_t)s.nBodies;
  F.bodyScale = (float)s.bodyScale;
  F.covScale = (float)s.covScale;
  F.omega = (float)p.omega;
  F.sorAverage = p.sor_average ? 1u : 0u;
  F.invDt = (float)(dt > 0 ? 1 / dt : 0);
  F.volume = (float)(s.mass / p.rest_density);
  F.tension = (float)p.surface_tension_k;
  F.cohes = (float)(32 / (kPi * std::pow(h, 9)));
  F.cohesTerm = (float)(std::pow(h, 6) / 64);
  F.pOff = (uint32_t)s.part.off;
  F.pEnd = (uint32_t)(s.part.off + s.n);
  F.cOff = (uint32_t)s.cells.off;
  F.bOff = (uint32_t)s.bodies.off;
  F.parity = (uint32_t)s.parity;
  F.iters = (uint32_t)std::max(1, p.iterations);
  F.subs = 1;
  F.slot = (uint32_t)slot;
}

void release_scene(p4a_batch* b, BScene& s) {
  if (s.part.off >= 0) b->partA.release(s.part.off, s.part.size);
  if (s.cells.off >= 0) b->cellA.release(s.cells.off, s.cells.size);
  if (s.bodies.off >= 0) b->bodyA.release(s.bodies.off, s.bodies.size);
  if (s.list.off >= 0) b->listA.release(s.list.off, s.list.size);
  if (s.bound.off >= 0) b->boundA.release(s.bound.off, s.bound.size);
  s = BScene();
}

// A frame schedule: per substep the work-item segments of every launch.
struct Schedule {
  std::vector<uint2> items;
  struct Sub {
    Seg key, scan, part, seed, finishPlain, finishTension;
    std::vector<Seg> iter, bodyIter;
  };
  std::vector<Sub> subs;
  int maxIters = 0;
};

Seg push_tiles(std::vector<uint2>& v, uint32_t slot, int64_t tiles) {
  Seg s{(int64_t)v.size(), (int)tiles};
  for (int64_t t = 0; t < tiles; t++) v.push_back(make_uint2(slot, (uint32_t)t));
  return s;
}

void append_to(Seg& seg, std::vector<uint2>& v, uint32_t slot, int64_t count) {
  // Segments are built scene by scene; keep each launch's items contiguous.
  if (seg.count == 0) seg.off = (int64_t)v.size();
  for (int64_t t = 0; t < count; t++) v.push_back(make_uint2(slot, (uint32_t)t));
  seg.count += (int)count;
}

// Kernels one frame of the schedule launches.
uint64_t frame_kernels(const Schedule& sch) {
  uint64_t k = 0;
  for (const auto& u : sch.subs) {
    k += (u.key.count > 0) + (u.scan.count > 0) + 2 * (u.part.count > 0) + (u.seed.count > 0) +
         (u.finishPlain.count > 0) + 2 * (u.finishTension.count > 0);
    for (size_t it = 0; it < u.iter.size(); it++) k += 2 * (u.iter[it].count > 0) + (u.bodyIter[it].count > 0);
  }
  return k;
}

// Launches one frame of the schedule on the batch's stream.
int run_frame(p4a_batch* b, const Schedule& sch, int nSlots) {
  cudaStream_t st = b->stream;
  DevScene& d = b->d;
  for (size_t s = 0; s < sch.subs.size(); s++) {
    const Schedule::Sub& u = sch.subs[s];
    BatchWork w;
    w.params = b->dParams + s * (size_t)nSlots;
    auto at = [&](const Seg& g) {
      BatchWork x = w;
      x.items = b->dItems + g.off;
      return x;
    };
    launch_key_count_b(at(u.key), u.key.count, d, st);
    BTRY(b, cudaMemsetAsync(d.scanState, 0, (size_t)u.scan.count * 8, st));
    {
      // the scan addresses its tile states from 0: pass the segment's items
      BatchWork x = at(u.scan);
      launch_scan_b(x, u.scan.count, d, 1u, st);
    }
    launch_fill_b(at(u.part), u.part.count, d, st);
    launch_reorder_b(at(u.part), u.part.count, d, st);
    launch_body_seed_b(at(u.seed), u.seed.count, d, st);
    for (int it = 0; it < (int)u.iter.size(); it++) {
      launch_lambda_b(at(u.iter[it]), u.iter[it].count, d, it, st);
      launch_delta_b(at(u.iter[it]), u.iter[it].count, d, it, st);
      launch_body_match_b(at(u.bodyIter[it]), u.bodyIter[it].count, d, it, st);
    }
    launch_xsph_finalize_b(at(u.finishPlain), u.finishPlain.count, d, (int)s, st);
    launch_xsph_normals_b(at(u.finishTension), u.finishTension.count, d, st);
    launch_tension_finalize_b(at(u.finishTension), u.finishTension.count, d, (int)s, st);
  }
  BTRY(b, cudaGetLastError());
  return P4A_OK;
}

__global__ void k_zero_stats(uint32_t* __restrict__ stats, const uint2* __restrict__ items, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count * 8) stats[items[t / 8].x * 8 + (t % 8)] = 0u;
}

int ensure_items(p4a_batch* b, int64_t nItems) {
  if (nItems <= b->itemsCap) return P4A_OK;
  BTRY(b, cudaStreamSynchronize(b->stream));
  if (b->dItems) {
    cudaFree(b->dItems);
    b->dItems = nullptr;
  }
  const int64_t cap = std::max<int64_t>(nItems * 2, 4096);
  BTRY(b, cudaMalloc((void**)&b->dItems, (size_t)cap * sizeof(uint2)));
  b->itemsCap = cap;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graphKey.clear();
  }
  return P4A_OK;
}

int ensure_staging(p4a_batch* b, size_t bytes) {
  if (bytes <= b->stagingCap) return P4A_OK;
  for (int k = 0; k < 2; k++) {
    if (b->stagingDone[k]) cudaEventSynchronize(b->stagingDone[k]);
    if (b->staging[k]) cudaFreeHost(b->staging[k]);
    b->staging[k] = nullptr;
  }
  const size_t cap = std::max<size_t>(bytes * 2, 1 << 16);
  for (int k = 0; k < 2; k++) BTRY(b, cudaHostAlloc((void**)&b->staging[k], cap, cudaHostAllocDefault));
  b->stagingCap = cap;
  return P4A_OK;
}

// Uploads params tables + items and runs the frame (graph replay when the
// schedule's shape is unchanged). zeroItems lists the scenes whose stats restart.
int execute(p4a_batch* b, const Schedule& sch, const std::vector<SimParams>& params, int nSlots,
            const Seg& zeroSeg, const std::vector<int64_t>& key) {
  const size_t pBytes = params.size() * sizeof(SimParams);
  const size_t iBytes = sch.items.size() * sizeof(uint2);
  int rc;
  if ((rc = ensure_items(b, (int64_t)sch.items.size()))) return rc;
  if ((rc = ensure_staging(b, pBytes + iBytes))) return rc;
  const int k = b->stagingIdx;
  b->stagingIdx ^= 1;
  BTRY(b, cudaEventSynchronize(b->stagingDone[k]));  // the copy two frames ago has finished
  std::memcpy(b->staging[k], params.data(), pBytes);
  std::memcpy(b->staging[k] + pBytes, sch.items.data(), iBytes);
  BTRY(b, cudaMemcpyAsync(b->dParams, b->staging[k], pBytes, cudaMemcpyHostToDevice, b->stream));
  BTRY(b, cudaMemcpyAsync(b->dItems, b->staging[k] + pBytes, iBytes, cudaMemcpyHostToDevice, b->stream));
  BTRY(b, cudaEventRecord(b->stagingDone[k], b->stream));
  count_launches(frame_kernels(sch) + (zeroSeg.count > 0 ? 1 : 0));
  auto body = [&]() -> int {
    if (zeroSeg.count > 0)
      k_zero_stats<<<(zeroSeg.count * 8 + 255) / 256, 256, 0, b->stream>>>(b->d.statsOut, b->dItems + zeroSeg.off,
                                                                           zeroSeg.count);
    return run_frame(b, sch, nSlots);
  };
  if (!b->useGraphs) return body();
  if (!b->graph || b->graphKey != key) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    BTRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int brc = body();
    const cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
    if (brc) {
      if (g) cudaGraphDestroy(g);
      return brc;
    }
    if (ec != cudaSuccess) return bfail(b, P4A_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return bfail(b, P4A_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    b->graphKey = key;
  }
  BTRY(b, cudaGraphLaunch(b->graph, b->stream));
  return P4A_OK;
}

int scene_ok(p4a_batch* b, int32_t id) {
  if (!b) return P4A_ERR_ARG;
  if (id < 0 || id >= (int32_t)b->scenes.size() || !b->scenes[id].live)
    return bfail(b, P4A_ERR_ARG, "no live scene %d", id);
  return P4A_OK;
}

// Admits a host scene: arena ranges, uploads, prime (src/sim.js:66-253).
int admit(p4a_batch* b, const p4a_params& params, HostScene& sc, int pourBudget, int32_t* outId) {
  int slot = -1;
  for (int k = 0; k < (int)b->scenes.size(); k++)
    if (!b->scenes[k].live) {
      slot = k;
      break;
    }
  if (slot < 0) return bfail(b, P4A_ERR_CAPACITY, "all %d scene slots are in use", b->cfg.max_scenes);
  BScene s;
  s.params = params;
  s.specs.assign(params.bodies, params.bodies + (params.bodies ? params.n_bodies : 0));
  s.params.bodies = s.specs.empty() ? nullptr : s.specs.data();
  s.params.n_bodies = (int32_t)s.specs.size();
  s.h = sc.h;
  s.mass = sc.mass;
  s.denomRest = sc.denomRest;
  s.n = sc.n;
  s.nFluid = sc.nFluid;
  s.cap = sc.n + std::max(0, pourBudget);
  for (int k = 0; k < 3; k++) s.gridDim[k] = (int)std::max(1.0, std::floor(params.box[k] / s.h));
  s.nCells = s.gridDim[0] * s.gridDim[1] * s.gridDim[2];
  s.nBodies = (int)sc.bodyDensity.size();
  s.nBodyParts = sc.nBody;
  HostBoundary hb;
  build_boundary(params.box, params.rest_density, params.spacing, s.h, s.gridDim, hb);
  s.nBoundary = hb.count;
  // arena ranges (nothing is kept if any arena is full)
  const int64_t cellsPadded = (int64_t)((s.nCells + 2 + kScanTile - 1) / kScanTile) * kScanTile;
  s.part = {b->partA.alloc(std::max(1, s.cap), kBlock), std::max(1, s.cap)};
  s.cells = {b->cellA.alloc(cellsPadded, kScanTile), cellsPadded};
  s.bodies = {b->bodyA.alloc(s.nBodies + 1, 1), s.nBodies + 1};
  s.list = {b->listA.alloc(std::max(1, s.nBodyParts), 1), std::max(1, s.nBodyParts)};
  s.bound = {b->boundA.alloc(std::max(1, s.nBoundary), 1), std::max(1, s.nBoundary)};
  if (s.part.off < 0 || s.cells.off < 0 || s.bodies.off < 0 || s.list.off < 0 || s.bound.off < 0) {
    const bool p = s.part.off < 0, c = s.cells.off < 0;
    release_scene(b, s);
    return bfail(b, P4A_ERR_CAPACITY, "no room for a %d-particle scene (%s full)", sc.n,
                 p ? "particle arena" : c ? "cell arena" : "body/boundary arena");
  }
  // counts and fixed-point scales (src/sim.js:163-171)
  std::vector<int> counts(s.nBodies, 0);
  for (int i = 0; i < s.n; i++) {
    const uint32_t id = sc.phase[(size_t)i * 4];
    if (id >= 1 && (int)id <= s.nBodies) counts[id - 1]++;
  }
  double maxCount = 1, maxRest = 1e-3;
  for (int k = 0; k < s.nBodies; k++) maxCount = std::max(maxCount, (double)counts[k]);
  for (int i = 0; i < s.n; i++) {
    const double r = std::hypot((double)sc.rest[(size_t)i * 4], (double)sc.rest[(size_t)i * 4 + 1],
                                (double)sc.rest[(size_t)i * 4 + 2]);
    if (r > maxRest) maxRest = r;
  }
  const double extent = std::max(params.box[0], std::max(params.box[1], params.box[2]));
  s.bodyScale = 1e9 / (extent * maxCount);
  s.covScale = 1e9 / (extent * maxRest * maxCount);
  DevScene& d = b->d;
  cudaStream_t st = b->stream;
  // particles into parity 0 of the range; everything else of the range cleared
  const size_t po = (size_t)s.part.off, nb = (size_t)s.n * 16;
  for (int t = 0; t < 2; t++) {
    BTRY(b, cudaMemsetAsync(d.pos[t] + po, 0, (size_t)s.part.size * 16, st));
    BTRY(b, cudaMemsetAsync(d.vel[t] + po, 0, (size_t)s.part.size * 16, st));
    BTRY(b, cudaMemsetAsync(d.pred[t] + po, 0, (size_t)s.part.size * 16, st));
    BTRY(b, cudaMemsetAsync(d.body[t] + po, 0, (size_t)s.part.size * 16, st));
    BTRY(b, cudaMemsetAsync(d.rest[t] + po, 0, (size_t)s.part.size * 16, st));
  }
  if (s.n > 0) {
    BTRY(b, cudaMemcpyAsync(d.pos[0] + po, sc.pos.data(), nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.vel[0] + po, sc.vel.data(), nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.pred[0] + po, sc.pos.data(), nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.body[0] + po, sc.phase.data(), nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.rest[0] + po, sc.rest.data(), nb, cudaMemcpyHostToDevice, st));
  }
  // boundary samples and their cellStart in arena indices
  std::vector<uint32_t> bcs(hb.cellStart);
  for (auto& v : bcs) v += (uint32_t)s.bound.off;
  BTRY(b, cudaMemcpyAsync(d.bpos + s.bound.off, hb.pos.data(), hb.pos.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bpsi + s.bound.off, hb.psi.data(), hb.psi.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bcellStart + s.cells.off, bcs.data(), bcs.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemsetAsync(d.cellStart + s.cells.off, 0, (size_t)(s.nCells + 2) * 4, st));
  // bodies (src/sim.js:129-161)
  const int nb1 = s.nBodies + 1;
  std::vector<float> info((size_t)nb1 * 4, 0.0f), centre((size_t)nb1 * 4, 0.0f), rot((size_t)nb1 * 12, 0.0f);
  std::vector<uint32_t> bstart((size_t)nb1, 0u);
  uint32_t run = (uint32_t)s.list.off;
  for (int k = 0; k < s.nBodies; k++) {
    info[k * 4] = (float)(1 / std::max(1e-6, sc.bodyDensity[k]));
    for (int c = 0; c < 3; c++) centre[k * 4 + c] = (float)sc.bodyCentre[k * 3 + c];
    for (int r = 0; r < 3; r++) rot[k * 12 + r * 4 + r] = 1.0f;
    bstart[k] = run;
    run += (uint32_t)counts[k];
  }
  bstart[s.nBodies] = run;
  const size_t bo = (size_t)s.bodies.off;
  BTRY(b, cudaMemcpyAsync(d.bodyInfo + bo, info.data(), info.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyCentre + bo, centre.data(), centre.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyRef + bo, centre.data(), centre.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyRot + bo, rot.data(), rot.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyStart + bo, bstart.data(), bstart.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemsetAsync(d.bodyAccum + bo * 4, 0, (size_t)nb1 * 16, st));
  BTRY(b, cudaMemsetAsync(d.bodyCov + bo * 9, 0, (size_t)nb1 * 36, st));
  BTRY(b, cudaMemsetAsync(d.bodyFill + bo, 0, (size_t)nb1 * 4, st));
  BTRY(b, cudaMemsetAsync(d.statsOut + (size_t)slot * 8, 0, 32, st));
  // primeGrid (src/sim.js:223-253): a grid pass with dt = 0 from parity 0
  s.parity = 0;
  s.live = true;
  pack(s, 0.0, slot);
  b->scenes[slot] = std::move(s);
  BScene& S = b->scenes[slot];
  S.specs.assign(params.bodies, params.bodies + (params.bodies ? params.n_bodies : 0));
  S.params.bodies = S.specs.empty() ? nullptr : S.specs.data();
  Schedule sch;
  sch.subs.resize(1);
  const int64_t keyTiles = groups(std::max(S.n, S.nBodies));
  sch.subs[0].key = push_tiles(sch.items, (uint32_t)slot, keyTiles);
  sch.subs[0].scan = push_tiles(sch.items, (uint32_t)slot, scan_tiles(S.nCells));
  sch.subs[0].part = push_tiles(sch.items, (uint32_t)slot, groups(S.n));
  std::vector<SimParams> params1((size_t)slot + 1);
  params1[slot] = S.P;
  const bool graphs = b->useGraphs;
  b->useGraphs = false;
  const int rc = execute(b, sch, params1, slot + 1, Seg{}, {});
  b->useGraphs = graphs;
  if (rc) {
    release_scene(b, S);
    return rc;
  }
  BTRY(b, cudaStreamSynchronize(st));  // host vectors above go out of scope
  S.parity = 1;
  S.gen++;
  *outId = slot;
  return P4A_OK;
}

}  // namespace

extern "C" {

int p4a_batch_create(int device, const p4a_batch_config* cfg, p4a_batch** out) {
  if (!cfg || !out || cfg->max_particles <= 0 || cfg->max_cells <= 0 || cfg->max_scenes <= 0 ||
      cfg->max_particles > 0x7fffffffLL || cfg->max_cells > 0x7fffffffLL)
    return P4A_ERR_ARG;
  *out = nullptr;
  const int chk = p4a_device_check(device);
  if (chk != P4A_OK) return chk;
  if (cudaSetDevice(device) != cudaSuccess) return P4A_ERR_CUDA;
  p4a_batch* b = new p4a_batch();
  b->device = device;
  b->cfg = *cfg;
  if (b->cfg.max_bodies < 1) b->cfg.max_bodies = 1;
  if (b->cfg.max_body_parts < 1) b->cfg.max_body_parts = 1;
  if (b->cfg.max_boundary < 1) b->cfg.max_boundary = 1;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return P4A_ERR_CUDA;
  }
  b->ownStream = true;
  for (int k = 0; k < 2; k++) cudaEventCreateWithFlags(&b->stagingDone[k], cudaEventDisableTiming);
  const int64_t P = cfg->max_particles, Cc = cfg->max_cells + (int64_t)cfg->max_scenes * (kScanTile + 2);
  b->scanTilesCap = Cc / kScanTile + cfg->max_scenes + 1;
  DevScene& d = b->d;
  int rc = P4A_OK;
  for (int t = 0; t < 2 && !rc; t++) {
    if ((rc = balloc(b, &d.pos[t], P)) || (rc = balloc(b, &d.vel[t], P)) || (rc = balloc(b, &d.pred[t], P)) ||
        (rc = balloc(b, &d.body[t], P)) || (rc = balloc(b, &d.rest[t], P)))
      break;
  }
  const int64_t B1 = b->cfg.max_bodies;
  if (!rc &&
      ((rc = balloc(b, &d.lambda, P)) || (rc = balloc(b, &d.density, P)) || (rc = balloc(b, &d.corr, P)) ||
       (rc = balloc(b, &d.normal, P)) || (rc = balloc(b, &d.key, P)) || (rc = balloc(b, &d.rank, P)) ||
       (rc = balloc(b, &d.unordered, P)) || (rc = balloc(b, &d.nbMask, P * 9)) ||
       (rc = balloc(b, &d.nbLong, P)) || (rc = balloc(b, &d.cellCount, Cc)) ||
       (rc = balloc(b, &d.cellStart, Cc)) || (rc = balloc(b, &d.bcellStart, Cc)) ||
       (rc = balloc(b, &d.scanState, b->scanTilesCap)) || (rc = balloc(b, &d.scanTicket, 4)) ||
       (rc = balloc(b, &d.errorWord, 4)) || (rc = balloc(b, &d.bpos, b->cfg.max_boundary)) ||
       (rc = balloc(b, &d.bpsi, b->cfg.max_boundary)) || (rc = balloc(b, &d.bodyAccum, B1 * 4)) ||
       (rc = balloc(b, &d.bodyCov, B1 * 9)) || (rc = balloc(b, &d.bodyCentre, B1)) ||
       (rc = balloc(b, &d.bodyRef, B1)) || (rc = balloc(b, &d.bodyRot, B1 * 3)) ||
       (rc = balloc(b, &d.bodyInfo, B1)) || (rc = balloc(b, &d.bodyStart, B1)) ||
       (rc = balloc(b, &d.bodyFill, B1)) || (rc = balloc(b, &d.bodyList, b->cfg.max_body_parts)) ||
       (rc = balloc(b, &d.statsOut, (int64_t)cfg->max_scenes * 8)) ||
       (rc = balloc(b, &b->dParams, (int64_t)kMaxSubsteps * cfg->max_scenes))))
    ;
  if (rc) {
    p4a_batch_destroy(b);
    return rc;
  }
  d.cap = (uint32_t)P;
  b->partA.init(P);
  b->cellA.init(Cc);
  b->boundA.init(b->cfg.max_boundary);
  b->bodyA.init(b->cfg.max_bodies);
  b->listA.init(b->cfg.max_body_parts);
  b->scenes.resize(cfg->max_scenes);
  *out = b;
  return P4A_OK;
}

int p4a_batch_destroy(p4a_batch* b) {
  if (!b) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (void* p : b->allocs) cudaFree(p);
  if (b->dItems) cudaFree(b->dItems);
  for (int k = 0; k < 2; k++) {
    if (b->staging[k]) cudaFreeHost(b->staging[k]);
    if (b->stagingDone[k]) cudaEventDestroy(b->stagingDone[k]);
  }
  if (b->ownStream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return P4A_OK;
}

const char* p4a_batch_last_error(const p4a_batch* b) { return b ? b->err.c_str() : "null handle"; }

int p4a_batch_set_stream(p4a_batch* b, void* stream) {
  if (!b) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  BTRY(b, cudaStreamSynchronize(b->stream));
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graphKey.clear();
  }
  if (stream) {
    if (b->ownStream) cudaStreamDestroy(b->stream);
    b->stream = (cudaStream_t)stream;
    b->ownStream = false;
  } else if (!b->ownStream) {
    BTRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->ownStream = true;
  }
  return P4A_OK;
}

int p4a_batch_use_graphs(p4a_batch* b, int32_t on) {
  if (!b) return P4A_ERR_ARG;
  b->useGraphs = on != 0;
  return P4A_OK;
}

int p4a_batch_add_scene(p4a_batch* b, const p4a_params* params, const p4a_scene_desc* sd, int32_t* id) {
  if (!b || !params || !sd || !id || sd->n < 0 || (sd->n > 0 && !sd->pos) || !(params->spacing > 0) ||
      sd->n_bodies < 0 || (sd->n_bodies > 0 && (!sd->body_density || !sd->body_centre)))
    return bfail(b, P4A_ERR_ARG, "p4a_batch_add_scene: invalid scene");
  cudaSetDevice(b->device);
  HostScene sc;
  const size_t n = (size_t)sd->n;
  sc.n = sd->n;
  sc.d = params->spacing;
  sc.h = 2 * params->spacing;
  sc.pos.assign(sd->pos, sd->pos + n * 4);
  sc.vel = sd->vel ? std::vector<float>(sd->vel, sd->vel + n * 4) : std::vector<float>(n * 4, 0.0f);
  sc.rest = sd->rest ? std::vector<float>(sd->rest, sd->rest + n * 4) : std::vector<float>(n * 4, 0.0f);
  sc.phase = sd->phase ? std::vector<uint32_t>(sd->phase, sd->phase + n * 4) : std::vector<uint32_t>(n * 4, 0u);
  int nFluid = 0;
  for (size_t i = 0; i < n; i++) {
    const uint32_t bid = sc.phase[i * 4];
    if (bid == 0) nFluid++;
    else if ((int)bid > sd->n_bodies) return bfail(b, P4A_ERR_ARG, "particle %zu: body id %u > n_bodies", i, bid);
  }
  sc.nFluid = nFluid;
  sc.nBody = sd->n - nFluid;
  sc.bodyDensity.assign(sd->body_density, sd->body_density + sd->n_bodies);
  sc.bodyCentre.assign(sd->body_centre, sd->body_centre + 3 * (size_t)sd->n_bodies);
  sc.mass = sd->mass;
  sc.denomRest = sd->denom_rest;
  const bool doMass = !(sd->mass > 0), doDenom = !(sd->denom_rest > 0);
  if (doMass || doDenom) calibrate_scene(*params, sc, doMass, doDenom);
  return admit(b, *params, sc, sd->pour_budget, id);
}

int p4a_batch_add_preset(p4a_batch* b, const p4a_params* params, int32_t* id) {
  if (!b || !params || !id || !(params->spacing > 0)) return bfail(b, P4A_ERR_ARG, "invalid params");
  cudaSetDevice(b->device);
  HostScene sc;
  build_scene(*params, sc);
  return admit(b, *params, sc, params->pour ? sc.nFluid : 0, id);
}

int p4a_batch_remove_scene(p4a_batch* b, int32_t id) {
  int rc = scene_ok(b, id);
  if (rc) return rc;
  cudaSetDevice(b->device);
  BTRY(b, cudaStreamSynchronize(b->stream));
  release_scene(b, b->scenes[id]);
  return P4A_OK;
}

int p4a_batch_step(p4a_batch* b, const int32_t* ids, int32_t count, double frameDt) {
  if (!b || count < 0 || (count > 0 && !ids)) return bfail(b, P4A_ERR_ARG, "p4a_batch_step: bad list");
  cudaSetDevice(b->device);
  int nSlots = 0;
  std::vector<int> subs(count, 0);
  int maxSub = 0;
  for (int k = 0; k < count; k++) {
    int rc = scene_ok(b, ids[k]);
    if (rc) return rc;
    BScene& s = b->scenes[ids[k]];
    // time bank (src/sim.js:418-429)
    const int base = std::max(1, s.params.substeps);
    const double dtTarget = (1.0 / 60) / base;
    s.timeBank = s.timeBank + frameDt;
    double subD = std::floor(s.timeBank / dtTarget + 1e-4);
    const double workCap = base * 8;
    if (subD > workCap) {
      subD = workCap;
      s.timeBank = 0;
    } else {
      s.timeBank -= subD * dtTarget;
    }
    subs[k] = std::min((int)subD, kMaxSubsteps);
    s.lastSubsteps = subs[k];
    s.lastAdvanced = subs[k] < 1 ? 0 : subD * dtTarget;
    maxSub = std::max(maxSub, subs[k]);
    nSlots = std::max(nSlots, ids[k] + 1);
  }
  if (maxSub == 0) return P4A_OK;
  // schedule and per-substep params
  Schedule sch;
  sch.subs.resize(maxSub);
  std::vector<SimParams> params((size_t)maxSub * nSlots);
  std::vector<int64_t> key;
  key.push_back(nSlots);
  Seg zero;
  zero.off = 0;
  for (int k = 0; k < count; k++)
    if (subs[k] > 0) append_to(zero, sch.items, (uint32_t)ids[k], 1);
  // items of zero are (slot, 0): the zero kernel reads .x only
  for (int s = 0; s < maxSub; s++) {
    Schedule::Sub& u = sch.subs[s];
    int maxIt = 0;
    for (int k = 0; k < count; k++)
      if (subs[k] > s) maxIt = std::max(maxIt, std::max(1, b->scenes[ids[k]].params.iterations));
    u.iter.resize(maxIt);
    u.bodyIter.resize(maxIt);
    auto each = [&](auto&& fn) {
      for (int k = 0; k < count; k++)
        if (subs[k] > s) fn(b->scenes[ids[k]], (uint32_t)ids[k]);
    };
    each([&](BScene& S, uint32_t slot) { append_to(u.key, sch.items, slot, groups(std::max(S.n, S.nBodies))); });
    each([&](BScene& S, uint32_t slot) { append_to(u.scan, sch.items, slot, scan_tiles(S.nCells)); });
    each([&](BScene& S, uint32_t slot) { append_to(u.part, sch.items, slot, groups(S.n)); });
    each([&](BScene& S, uint32_t slot) {
      if (S.nBodyParts > 0 && S.nBodies > 0) append_to(u.seed, sch.items, slot, S.nBodies);
    });
    for (int it = 0; it < maxIt; it++) {
      each([&](BScene& S, uint32_t slot) {
        if (std::max(1, S.params.iterations) > it) append_to(u.iter[it], sch.items, slot, groups(S.n));
      });
      each([&](BScene& S, uint32_t slot) {
        if (std::max(1, S.params.iterations) > it && S.nBodyParts > 0 && S.nBodies > 0)
          append_to(u.bodyIter[it], sch.items, slot, S.nBodies);
      });
    }
    each([&](BScene& S, uint32_t slot) {
      if (!(S.params.surface_tension_k > 0)) append_to(u.finishPlain, sch.items, slot, groups(S.n));
    });
    each([&](BScene& S, uint32_t slot) {
      if (S.params.surface_tension_k > 0) append_to(u.finishTension, sch.items, slot, groups(S.n));
    });
    for (int k = 0; k < count; k++) {
      if (subs[k] <= s) continue;
      BScene& S = b->scenes[ids[k]];
      const double dt = (1.0 / 60) / std::max(1, S.params.substeps);
      pack(S, dt, ids[k]);
      S.P.parity = (uint32_t)(S.parity ^ (s & 1));
      S.P.subs = (uint32_t)subs[k];
      params[(size_t)s * nSlots + ids[k]] = S.P;
    }
    key.insert(key.end(), {u.key.count, u.scan.count, u.part.count, u.seed.count, (int64_t)u.iter.size(),
                           u.finishPlain.count, u.finishTension.count});
    for (int it = 0; it < maxIt; it++) key.insert(key.end(), {u.iter[it].count, u.bodyIter[it].count});
  }
  // the graph bakes the item segment offsets; the items themselves are uploaded per frame
  for (auto& u : sch.subs) key.insert(key.end(), {u.key.off, u.scan.off, u.part.off});
  key.push_back(zero.count);
  int rc = execute(b, sch, params, nSlots, zero, key);
  if (rc) return rc;
  for (int k = 0; k < count; k++) {
    BScene& S = b->scenes[ids[k]];
    if (subs[k] < 1) continue;
    S.parity ^= (subs[k] & 1);
    S.simTime += subs[k] * ((1.0 / 60) / std::max(1, S.params.substeps));
    S.statsValid = true;
  }
  return P4A_OK;
}

int p4a_batch_synchronize(p4a_batch* b) {
  if (!b) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  BTRY(b, cudaStreamSynchronize(b->stream));
  uint32_t w = 0;
  BTRY(b, cudaMemcpy(&w, b->d.errorWord, 4, cudaMemcpyDeviceToHost));
  if (w & ERR_SCAN_TIMEOUT) return bfail(b, P4A_ERR_TIMEOUT, "cell scan: a bounded wait gave up");
  return P4A_OK;
}

int p4a_batch_usage_get(const p4a_batch* b, p4a_batch_usage* o) {
  if (!b || !o) return P4A_ERR_ARG;
  *o = p4a_batch_usage{};
  o->free_particles = b->partA.free_total();
  o->free_cells = b->cellA.free_total();
  o->free_boundary = b->boundA.free_total();
  o->free_body_parts = b->listA.free_total();
  o->free_bodies = (int32_t)b->bodyA.free_total();
  int live = 0;
  for (auto& s : b->scenes) live += s.live ? 1 : 0;
  o->live_scenes = live;
  o->free_scenes = (int32_t)b->scenes.size() - live;
  o->device_bytes = (int64_t)b->deviceBytes;
  return P4A_OK;
}

int p4a_batch_scene_info(p4a_batch* b, int32_t id, p4a_info* o) {
  int rc = scene_ok(b, id);
  if (rc) return rc;
  if (!o) return P4A_ERR_ARG;
  const BScene& s = b->scenes[id];
  *o = p4a_info{};
  o->n = s.n; o->n_fluid = s.nFluid; o->n_body_parts = s.nBodyParts; o->n_bodies = s.nBodies;
  o->n_boundary = s.nBoundary; o->cap = s.cap; o->pour_budget = s.cap - s.n;
  for (int k = 0; k < 3; k++) o->grid_dim[k] = s.gridDim[k];
  o->n_cells = s.nCells; o->parity = s.parity; o->pred_parity = s.parity; o->gen = s.gen;
  o->last_substeps = s.lastSubsteps; o->h = s.h; o->mass = s.mass; o->denom_rest = s.denomRest;
  o->sim_time = s.simTime; o->last_advanced = s.lastAdvanced; o->time_bank = s.timeBank;
  o->body_scale = s.bodyScale; o->cov_scale = s.covScale; o->held_body = -1;
  return P4A_OK;
}

// Device pointer, element size and element count of a scene's view of a buffer.
static int scene_buffer(p4a_batch* b, const BScene& s, int32_t id, int32_t which, void** p, size_t* bytes) {
  const int w = which < 0 ? s.parity : (which & 1);
  DevScene& d = b->d;
  const size_t po = (size_t)s.part.off, n = (size_t)s.cap, bo = (size_t)s.bodies.off;
  const size_t nb1 = (size_t)std::max(1, s.nBodies);
  switch (id) {
    case P4A_BUF_POS: *p = d.pos[w] + po; *bytes = n * 16; break;
    case P4A_BUF_VEL: *p = d.vel[w] + po; *bytes = n * 16; break;
    case P4A_BUF_PRED: *p = d.pred[w] + po; *bytes = n * 16; break;
    case P4A_BUF_BODY: *p = d.body[w] + po; *bytes = n * 16; break;
    case P4A_BUF_REST: *p = d.rest[w] + po; *bytes = n * 16; break;
    case P4A_BUF_DENSITY: *p = d.density + po; *bytes = n * 4; break;
    case P4A_BUF_LAMBDA: *p = d.lambda + po; *bytes = n * 4; break;
    case P4A_BUF_CORR: *p = d.corr + po; *bytes = n * 16; break;
    case P4A_BUF_NORMAL: *p = d.normal + po; *bytes = n * 16; break;
    case P4A_BUF_CELL_START: *p = d.cellStart + s.cells.off; *bytes = ((size_t)s.nCells + 2) * 4; break;
    case P4A_BUF_BODY_CENTRE: *p = d.bodyCentre + bo; *bytes = nb1 * 16; break;
    case P4A_BUF_BODY_REF: *p = d.bodyRef + bo; *bytes = nb1 * 16; break;
    case P4A_BUF_BODY_ROT: *p = d.bodyRot + bo * 3; *bytes = nb1 * 48; break;
    case P4A_BUF_BODY_INFO: *p = d.bodyInfo + bo; *bytes = nb1 * 16; break;
    default: return bfail(b, P4A_ERR_ARG, "buffer id %d is not available per batched scene", id);
  }
  return P4A_OK;
}

int p4a_batch_read(p4a_batch* b, int32_t id, int32_t bid, int32_t which, void* host, size_t offset, size_t bytes) {
  int rc = scene_ok(b, id);
  if (rc) return rc;
  if (!host && bytes) return P4A_ERR_ARG;
  const BScene& s = b->scenes[id];
  void* p = nullptr;
  size_t total = 0;
  if ((rc = scene_buffer(b, s, bid, which, &p, &total))) return rc;
  if (offset > total || bytes > total - offset) return bfail(b, P4A_ERR_ARG, "read beyond the scene's buffer");
  if (!bytes) return P4A_OK;
  cudaSetDevice(b->device);
  BTRY(b, cudaMemcpyAsync(host, (const char*)p + offset, bytes, cudaMemcpyDeviceToHost, b->stream));
  BTRY(b, cudaStreamSynchronize(b->stream));
  if (bid == P4A_BUF_CELL_START) {  // arena indices -> the scene's own indices
    uint32_t* v = (uint32_t*)host;
    const size_t first = offset / 4, count = bytes / 4;
    for (size_t k = 0; k < count; k++)
      if (first + k <= (size_t)s.nCells) v[k] -= (uint32_t)s.part.off;
  }
  return P4A_OK;
}

int p4a_batch_write(p4a_batch* b, int32_t id, int32_t bid, int32_t which, const void* host, size_t offset,
                    size_t bytes) {
  int rc = scene_ok(b, id);
  if (rc) return rc;
  if (!host && bytes) return P4A_ERR_ARG;
  if (bid == P4A_BUF_CELL_START) return bfail(b, P4A_ERR_ARG, "cellStart is written by the sort only");
  const BScene& s = b->scenes[id];
  void* p = nullptr;
  size_t total = 0;
  if ((rc = scene_buffer(b, s, bid, which, &p, &total))) return rc;
  if (offset > total || bytes > total - offset) return bfail(b, P4A_ERR_ARG, "write beyond the scene's buffer");
  if (!bytes) return P4A_OK;
  cudaSetDevice(b->device);
  BTRY(b, cudaMemcpyAsync((char*)p + offset, host, bytes, cudaMemcpyHostToDevice, b->stream));
  BTRY(b, cudaStreamSynchronize(b->stream));
  return P4A_OK;
}

int p4a_batch_stats(p4a_batch* b, int32_t id, p4a_stats* o) {
  int rc = scene_ok(b, id);
  if (rc) return rc;
  if (!o) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  uint32_t v[8];
  BTRY(b, cudaMemcpyAsync(v, b->d.statsOut + (size_t)id * 8, 32, cudaMemcpyDeviceToHost, b->stream));
  BTRY(b, cudaStreamSynchronize(b->stream));
  const BScene& s = b->scenes[id];
  *o = p4a_stats{};
  const double SCALE = 1024;
  o->avg_rho = s.statsValid ? v[0] / SCALE / std::max(1, s.n) : 1;
  o->max_rho = s.statsValid ? v[1] / SCALE : 1;
  o->max_speed = v[2] / SCALE;
  o->ke = v[3] / SCALE;
  for (int k = 0; k < 4; k++) o->raw[k] = v[k];
  o->valid = s.statsValid ? 1 : 0;
  return P4A_OK;
}

}  // extern "C"
