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
#include "batch_internal.h"
#include "p4a_internal.h"
#include "scene.h"

using namespace p4a;

namespace p4a {

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

}  // namespace p4a

namespace {

const double kPi = 3.14159265358979323846;

template <class T>
int balloc(p4a_batch* b, T** out, int64_t count) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(16, (size_t)count * sizeof(T));
  if (b->sizeOnly) {  // p4a_batch_footprint: count the bytes, allocate nothing
    b->deviceBytes += bytes;
    *out = nullptr;
    return P4A_OK;
  }
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
  F.skinH2 = (float)((h + kSkin * h) * (h + kSkin * h));
  F.skinHalf = (float)((kSkin * h - 1e-4 * h) * 0.5);
  F.volSpiky = F.volume * F.spikyGrad;
}

// Kinds of the launches of a frame, in the order a substep issues them.
enum LaunchKind : int {
  LK_ZERO, LK_KEY, LK_SCAN_SUMS, LK_SCAN_OFFSETS, LK_SCAN, LK_FILL, LK_REORDER, LK_SEED, LK_LAMBDA, LK_DELTA, LK_MATCH,
  LK_FINISH, LK_NORMALS, LK_TENSION
};

struct LaunchRec {
  int kind, sub, it;
  WorkSeg seg;
};

// One frame: the work items of every launch (item .x = the scene's row in the
// frame's params table), the launches in issue order, and the params rows
// [sub][row] of the frame's scenes. `shape` (substeps, then the iteration count of
// each substep) fixes the launch sequence: frames of one shape replay one graph.
struct Frame {
  std::vector<uint2> items;
  std::vector<LaunchRec> launches;
  std::vector<SimParams> params;
  int nSubs = 0, nRows = 0;
  int variant[TK_COUNT] = {0, 0, 0, 0};  // launch shapes of the tuned kernels
  std::vector<int> shape;
};

WorkSeg push_items(Frame& F, uint32_t row, int64_t count, WorkSeg seg) {
  if (seg.count == 0) seg.off = (uint32_t)F.items.size();
  for (int64_t t = 0; t < count; t++) F.items.push_back(make_uint2(row, (uint32_t)t));
  seg.count += (uint32_t)count;
  return seg;
}

void add_launch(Frame& F, int kind, int sub, int it, WorkSeg seg) { F.launches.push_back({kind, sub, it, seg}); }

constexpr const char* kLaunchNames[] = {"zero_stats", "key_count", "scan_sums", "scan_offsets", "scan", "fill",
                                         "reorder", "body_seed",
                                         "lambda", "delta", "body_match", "xsph_finalize", "xsph_normals",
                                         "tension_finalize"};
constexpr int kLaunchKinds = (int)(sizeof(kLaunchNames) / sizeof(kLaunchNames[0]));

// Launches one frame on the batch's stream. Graph form: every launch of the shape
// is issued with the resident grid and fixed-size clears (counts are read on the
// device); direct form: empty launches are skipped and grids fit the counts.
// With `ev` (launches + 1 events), ev[L] is recorded before launch L and the last
// one after the last launch (as event-record nodes when the stream is captured).
int run_frame(p4a_batch* b, const Frame& F, bool graphForm, uint64_t* launched,
              const std::vector<cudaEvent_t>* ev = nullptr) {
  p4a_batch::Lane& Ln = *b->lane;
  cudaStream_t st = Ln.stream;
  DevScene& d = b->d;
  const int stride = b->cfg.max_scenes;
  uint64_t n = 0;
  auto record = [&](size_t k) {
    return graphForm ? cudaEventRecordWithFlags((*ev)[k], st, cudaEventRecordExternal)
                     : cudaEventRecord((*ev)[k], st);
  };
  BTRY(b, cudaMemsetAsync(Ln.dCursors, 0, F.launches.size() * sizeof(uint32_t), st));
  for (size_t L = 0; L < F.launches.size(); L++) {
    const LaunchRec& r = F.launches[L];
    if (ev) BTRY(b, record(L));
    if (!graphForm && r.seg.count == 0) continue;
    BatchWork w;
    w.params = Ln.dParams + (size_t)r.sub * stride;
    w.items = Ln.dItems;
    w.seg = Ln.dSegs + L;
    w.cursor = Ln.dCursors + L;
    const int maxItems = graphForm ? 0x7fffffff : (int)r.seg.count;
    switch (r.kind) {
      case LK_ZERO: launch_zero_stats_b(w, d.statsOut, st); break;
      case LK_KEY: launch_key_count_b(w, maxItems, d, st); break;
      case LK_SCAN_SUMS: launch_scan_sums_b(w, maxItems, d, st); break;
      case LK_SCAN_OFFSETS: launch_scan_offsets_b(w, maxItems, d, st); break;
      case LK_SCAN: launch_scan_apply_b(w, maxItems, d, st); break;
      case LK_FILL: launch_fill_b(w, maxItems, d, st); break;
      case LK_REORDER: launch_reorder_b(w, maxItems, d, st); break;
      case LK_SEED: launch_body_seed_b(w, maxItems, d, st); break;
      case LK_LAMBDA: launch_lambda_b(w, maxItems, d, r.it, st, F.variant[TK_LAMBDA]); break;
      case LK_DELTA: launch_delta_b(w, maxItems, d, r.it, st, F.variant[TK_DELTA]); break;
      case LK_MATCH: launch_body_match_b(w, maxItems, d, r.it, st); break;
      case LK_FINISH: launch_xsph_finalize_b(w, maxItems, d, r.sub, st); break;
      case LK_NORMALS: launch_xsph_normals_b(w, maxItems, d, st, F.variant[TK_NORMALS]); break;
      case LK_TENSION: launch_tension_finalize_b(w, maxItems, d, r.sub, st); break;
    }
    n++;
  }
  if (ev) BTRY(b, record(F.launches.size()));
  BTRY(b, cudaGetLastError());
  if (launched) *launched = n;
  return P4A_OK;
}

// Adds the intervals of every profiled frame queued so far to the per-kernel totals.
int resolve_profile(p4a_batch* b) {
  for (auto& pf : b->profPending) {
    BTRY(b, cudaEventSynchronize(pf.ev.back()));
    for (size_t k = 0; k + 1 < pf.ev.size(); k++) {
      if (pf.kinds[k] < 0) continue;
      float ms = 0.0f;
      BTRY(b, cudaEventElapsedTime(&ms, pf.ev[k], pf.ev[k + 1]));
      b->profMs[pf.kinds[k]] += ms;
      b->profLaunches[pf.kinds[k]]++;
    }
    b->profFree.push_back(std::move(pf.ev));
  }
  b->profPending.clear();
  return P4A_OK;
}

// A set of `count` timing events from the pool (created on demand).
int take_events(p4a_batch* b, size_t count, std::vector<cudaEvent_t>* out) {
  for (size_t k = 0; k < b->profFree.size(); k++) {
    if (b->profFree[k].size() == count) {
      *out = std::move(b->profFree[k]);
      b->profFree.erase(b->profFree.begin() + (long)k);
      return P4A_OK;
    }
  }
  out->assign(count, nullptr);
  for (auto& e : *out) BTRY(b, cudaEventCreate(&e));
  return P4A_OK;
}

void drop_profile_events(p4a_batch* b) {
  for (auto& pf : b->profPending) b->profFree.push_back(std::move(pf.ev));
  b->profPending.clear();
  for (auto& set : b->profFree)
    for (auto e : set) cudaEventDestroy(e);
  b->profFree.clear();
}

void drop_graphs(p4a_batch* b) {
  for (auto& Ln : b->lanes) {
    for (auto& kv : Ln.graphs) cudaGraphExecDestroy(kv.second);
    Ln.graphs.clear();
  }
  for (auto& kv : b->profNodes)
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  b->profNodes.clear();
}

int ensure_device_lists(p4a_batch* b, int64_t nItems, int64_t nLaunches) {
  p4a_batch::Lane& Ln = *b->lane;
  if (nItems <= Ln.itemsCap && nLaunches <= Ln.launchCap) return P4A_OK;
  for (auto& l : b->lanes)
    if (l.stream) BTRY(b, cudaStreamSynchronize(l.stream));
  drop_graphs(b);  // graphs hold the old addresses
  if (nItems > Ln.itemsCap) {
    if (Ln.dItems) cudaFree(Ln.dItems);
    Ln.dItems = nullptr;
    const int64_t cap = std::max<int64_t>(nItems * 2, 4096);
    BTRY(b, cudaMalloc((void**)&Ln.dItems, (size_t)cap * sizeof(uint2)));
    Ln.itemsCap = cap;
  }
  if (nLaunches > Ln.launchCap) {
    if (Ln.dSegs) cudaFree(Ln.dSegs);
    if (Ln.dCursors) cudaFree(Ln.dCursors);
    Ln.dSegs = nullptr;
    Ln.dCursors = nullptr;
    const int64_t cap = std::max<int64_t>(nLaunches * 2, 256);
    BTRY(b, cudaMalloc((void**)&Ln.dSegs, (size_t)cap * sizeof(WorkSeg)));
    BTRY(b, cudaMalloc((void**)&Ln.dCursors, (size_t)cap * sizeof(uint32_t)));
    Ln.launchCap = cap;
  }
  return P4A_OK;
}

int ensure_staging(p4a_batch* b, size_t bytes) {
  p4a_batch::Lane& Ln = *b->lane;
  if (bytes <= Ln.stagingCap) return P4A_OK;
  for (int k = 0; k < 2; k++) {
    if (Ln.stagingDone[k]) cudaEventSynchronize(Ln.stagingDone[k]);
    if (Ln.staging[k]) cudaFreeHost(Ln.staging[k]);
    Ln.staging[k] = nullptr;
  }
  const size_t cap = std::max<size_t>(bytes * 2, 1 << 16);
  for (int k = 0; k < 2; k++) BTRY(b, cudaHostAlloc((void**)&Ln.staging[k], cap, cudaHostAllocDefault));
  Ln.stagingCap = cap;
  return P4A_OK;
}

// Uploads the frame's params rows, items and segments, then runs it: a replay of
// the graph of its shape when graphs are on (captured on first use).
int execute(p4a_batch* b, const Frame& F, bool allowGraph) {
  const size_t rowBytes = (size_t)F.nRows * sizeof(SimParams);
  const size_t pBytes = rowBytes * F.nSubs;
  const size_t iBytes = F.items.size() * sizeof(uint2);
  const size_t sBytes = F.launches.size() * sizeof(WorkSeg);
  int rc;
  if ((rc = ensure_device_lists(b, (int64_t)F.items.size(), (int64_t)F.launches.size()))) return rc;
  if ((rc = ensure_staging(b, pBytes + iBytes + sBytes))) return rc;
  p4a_batch::Lane& Ln = *b->lane;
  const int k = Ln.stagingIdx;
  Ln.stagingIdx ^= 1;
  BTRY(b, cudaEventSynchronize(Ln.stagingDone[k]));  // the lane's upload two frames ago has finished
  unsigned char* h = Ln.staging[k];
  std::memcpy(h, F.params.data(), pBytes);
  std::memcpy(h + pBytes, F.items.data(), iBytes);
  WorkSeg* segs = reinterpret_cast<WorkSeg*>(h + pBytes + iBytes);
  for (size_t L = 0; L < F.launches.size(); L++) segs[L] = F.launches[L].seg;
  for (int s = 0; s < F.nSubs; s++)
    BTRY(b, cudaMemcpyAsync(Ln.dParams + (size_t)s * b->cfg.max_scenes, h + rowBytes * s, rowBytes,
                            cudaMemcpyHostToDevice, Ln.stream));
  if (iBytes) BTRY(b, cudaMemcpyAsync(Ln.dItems, h + pBytes, iBytes, cudaMemcpyHostToDevice, Ln.stream));
  BTRY(b, cudaMemcpyAsync(Ln.dSegs, segs, sBytes, cudaMemcpyHostToDevice, Ln.stream));
  BTRY(b, cudaEventRecord(Ln.stagingDone[k], Ln.stream));
  const size_t nEv = F.launches.size() + 1;
  p4a_batch::ProfPending pf;
  if (b->prof) {
    if (b->profPending.size() >= 64 && (rc = resolve_profile(b))) return rc;
    if ((rc = take_events(b, nEv, &pf.ev))) return rc;
    pf.kinds.assign(nEv, -1);
  }
  if (!(allowGraph && b->useGraphs)) {
    uint64_t n = 0;
    rc = run_frame(b, F, false, &n, b->prof ? &pf.ev : nullptr);
    count_launches(n);
    if (b->prof) {
      for (size_t L = 0; L < F.launches.size(); L++)
        if (F.launches[L].seg.count) pf.kinds[L] = F.launches[L].kind;
      b->profPending.push_back(std::move(pf));
    }
    return rc;
  }
  std::vector<int> key = F.shape;
  if (b->prof) key.push_back(-1);  // the profiled graph of the shape has event nodes
  auto it = Ln.graphs.find(key);
  if (it == Ln.graphs.end()) {
    if (Ln.graphs.size() >= 16) {
      for (auto& l : b->lanes)
        if (l.stream) BTRY(b, cudaStreamSynchronize(l.stream));
      drop_graphs(b);
    }
    cudaGraph_t g = nullptr;
    BTRY(b, cudaStreamBeginCapture(Ln.stream, cudaStreamCaptureModeThreadLocal));
    const int brc = run_frame(b, F, true, nullptr, b->prof ? &pf.ev : nullptr);
    const cudaError_t ec = cudaStreamEndCapture(Ln.stream, &g);
    if (brc) {
      if (g) cudaGraphDestroy(g);
      return brc;
    }
    if (ec != cudaSuccess) return bfail(b, P4A_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
    cudaGraphExec_t ge = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    if (ei != cudaSuccess) {
      cudaGraphDestroy(g);
      return bfail(b, P4A_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    }
    if (b->prof) {
      // the event-record node of each event of the capture, by the event's index
      p4a_batch::ProfNodes pn;
      pn.graph = g;
      pn.nodes.assign(nEv, nullptr);
      size_t count = 0;
      BTRY(b, cudaGraphGetNodes(g, nullptr, &count));
      std::vector<cudaGraphNode_t> all(count);
      BTRY(b, cudaGraphGetNodes(g, all.data(), &count));
      for (auto node : all) {
        cudaGraphNodeType t;
        BTRY(b, cudaGraphNodeGetType(node, &t));
        if (t != cudaGraphNodeTypeEventRecord) continue;
        cudaEvent_t e = nullptr;
        BTRY(b, cudaGraphEventRecordNodeGetEvent(node, &e));
        for (size_t k = 0; k < nEv; k++)
          if (pf.ev[k] == e) pn.nodes[k] = node;
      }
      for (auto node : pn.nodes)
        if (!node) {
          cudaGraphExecDestroy(ge);
          cudaGraphDestroy(g);
          return bfail(b, P4A_ERR_CUDA, "profiled graph: an event-record node is missing");
        }
      b->profNodes[key] = std::move(pn);
    } else {
      cudaGraphDestroy(g);
    }
    it = Ln.graphs.emplace(key, ge).first;
  }
  if (b->prof) {
    // later replays may still be reading this set's events: point the nodes at it
    const auto& pn = b->profNodes[key];
    for (size_t k = 0; k < nEv; k++)
      BTRY(b, cudaGraphExecEventRecordNodeSetEvent(it->second, pn.nodes[k], pf.ev[k]));
    for (size_t L = 0; L < F.launches.size(); L++) pf.kinds[L] = F.launches[L].kind;
  }
  BTRY(b, cudaGraphLaunch(it->second, Ln.stream));
  count_launches(F.launches.size());
  if (b->prof) b->profPending.push_back(std::move(pf));
  return P4A_OK;
}

int scene_ok(p4a_batch* b, int32_t id) {
  if (!b) return P4A_ERR_ARG;
  if (id < 0 || id >= (int32_t)b->scenes.size() || !b->scenes[id].live)
    return bfail(b, P4A_ERR_ARG, "no live scene %d", id);
  return P4A_OK;
}

}  // namespace

namespace p4a {

void release_scene(p4a_batch* b, BScene& s) {
  if (s.part.off >= 0) b->partA.release(s.part.off, s.part.size);
  if (s.cells.off >= 0) b->cellA.release(s.cells.off, s.cells.size);
  if (s.bodies.off >= 0) b->bodyA.release(s.bodies.off, s.bodies.size);
  if (s.list.off >= 0) b->listA.release(s.list.off, s.list.size);
  if (s.bound.off >= 0) b->boundA.release(s.bound.off, s.bound.size);
  s = BScene();
}

static size_t a16(size_t v) { return (v + 15) & ~(size_t)15; }

int prepare_scene(const p4a_params& params, HostScene& sc, int pourBudget, PreparedScene& ps,
                  std::string& err) {
  BScene& s = ps.s;
  s = BScene();
  s.params = params;
  s.specs.assign(params.bodies, params.bodies + (params.bodies ? params.n_bodies : 0));
  s.params.bodies = nullptr;  // re-pointed at s.specs when the scene is placed
  s.params.n_bodies = (int32_t)s.specs.size();
  s.h = sc.h;
  s.mass = sc.mass;
  s.denomRest = sc.denomRest;
  s.n = sc.n;
  s.nFluid = sc.nFluid;
  s.cap = sc.n + std::max(0, pourBudget);
  for (int k = 0; k < 3; k++) s.gridDim[k] = (int)std::max(1.0, std::floor(params.box[k] / s.h));
  const double cells = (double)s.gridDim[0] * s.gridDim[1] * s.gridDim[2];
  if (cells > 0x7fff0000) {
    err = "scene grid has too many cells";
    return P4A_ERR_CAPACITY;
  }
  s.nCells = s.gridDim[0] * s.gridDim[1] * s.gridDim[2];
  s.nBodies = (int)sc.bodyDensity.size();
  s.nBodyParts = sc.nBody;
  build_boundary(params.box, params.rest_density, params.spacing, s.h, s.gridDim, ps.hb);
  s.nBoundary = ps.hb.count;
  // counts and fixed-point scales (src/sim.js:163-171)
  ps.bodyCounts.assign(s.nBodies, 0);
  for (int i = 0; i < s.n; i++) {
    const uint32_t id = sc.phase[(size_t)i * 4];
    if (id >= 1 && (int)id <= s.nBodies) ps.bodyCounts[id - 1]++;
  }
  double maxCount = 1, maxRest = 1e-3;
  for (int k = 0; k < s.nBodies; k++) maxCount = std::max(maxCount, (double)ps.bodyCounts[k]);
  for (int i = 0; i < s.n; i++) {
    const double r = std::hypot((double)sc.rest[(size_t)i * 4], (double)sc.rest[(size_t)i * 4 + 1],
                                (double)sc.rest[(size_t)i * 4 + 2]);
    if (r > maxRest) maxRest = r;
  }
  const double extent = std::max(params.box[0], std::max(params.box[1], params.box[2]));
  s.bodyScale = 1e9 / (extent * maxCount);
  s.covScale = 1e9 / (extent * maxRest * maxCount);
  // blob layout
  ps.nb1 = s.nBodies + 1;
  const size_t n16 = (size_t)s.n * 16;
  size_t o = 0;
  ps.oPos = o; o = a16(o + n16);
  ps.oVel = o; o = a16(o + n16);
  ps.oPhase = o; o = a16(o + n16);
  ps.oRest = o; o = a16(o + n16);
  ps.oBpos = o; o = a16(o + ps.hb.pos.size() * 4);
  ps.oBpsi = o; o = a16(o + ps.hb.psi.size() * 4);
  ps.oBcs = o; o = a16(o + ps.hb.cellStart.size() * 4);
  ps.oInfo = o; o = a16(o + (size_t)ps.nb1 * 16);
  ps.oCentre = o; o = a16(o + (size_t)ps.nb1 * 16);
  ps.oRot = o; o = a16(o + (size_t)ps.nb1 * 48);
  ps.oBstart = o; o = a16(o + (size_t)ps.nb1 * 4);
  ps.bytes = o;
  ps.sc = std::move(sc);  // the particle arrays, until write_blob
  return P4A_OK;
}

void write_blob(const PreparedScene& ps, unsigned char* blob) {
  const BScene& s = ps.s;
  const HostScene& sc = ps.sc;
  const size_t n16 = (size_t)s.n * 16;
  if (n16) {
    std::memcpy(blob + ps.oPos, sc.pos.data(), n16);
    std::memcpy(blob + ps.oVel, sc.vel.data(), n16);
    std::memcpy(blob + ps.oPhase, sc.phase.data(), n16);
    std::memcpy(blob + ps.oRest, sc.rest.data(), n16);
  }
  std::memcpy(blob + ps.oBpos, ps.hb.pos.data(), ps.hb.pos.size() * 4);
  std::memcpy(blob + ps.oBpsi, ps.hb.psi.data(), ps.hb.psi.size() * 4);
  std::memcpy(blob + ps.oBcs, ps.hb.cellStart.data(), ps.hb.cellStart.size() * 4);
  // bodies (src/sim.js:129-161); bodyStart relative to the scene's list range
  float* info = reinterpret_cast<float*>(blob + ps.oInfo);
  float* centre = reinterpret_cast<float*>(blob + ps.oCentre);
  float* rot = reinterpret_cast<float*>(blob + ps.oRot);
  uint32_t* bstart = reinterpret_cast<uint32_t*>(blob + ps.oBstart);
  std::memset(info, 0, (size_t)ps.nb1 * 16);
  std::memset(centre, 0, (size_t)ps.nb1 * 16);
  std::memset(rot, 0, (size_t)ps.nb1 * 48);
  uint32_t run = 0;
  for (int k = 0; k < s.nBodies; k++) {
    info[k * 4] = (float)(1 / std::max(1e-6, sc.bodyDensity[k]));
    for (int c = 0; c < 3; c++) centre[k * 4 + c] = (float)sc.bodyCentre[k * 3 + c];
    for (int r = 0; r < 3; r++) rot[k * 12 + r * 4 + r] = 1.0f;
    bstart[k] = run;
    run += (uint32_t)ps.bodyCounts[k];
  }
  bstart[s.nBodies] = run;
}

int place_scene(p4a_batch* b, PreparedScene& ps, unsigned char* blob, cudaStream_t st, int32_t* outSlot) {
  int slot = -1;
  for (int k = 0; k < (int)b->scenes.size(); k++)
    if (!b->scenes[k].live) {
      slot = k;
      break;
    }
  if (slot < 0) return bfail(b, P4A_ERR_CAPACITY, "all %d scene slots are in use", b->cfg.max_scenes);
  BScene s = ps.s;
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
    return bfail(b, P4A_ERR_CAPACITY, "no room for a %d-particle scene (%s full)", s.n,
                 p ? "particle arena" : c ? "cell arena" : "body/boundary arena");
  }
  // arena offsets into the blob's index-valued pieces
  uint32_t* bcs = reinterpret_cast<uint32_t*>(blob + ps.oBcs);
  for (size_t k = 0; k < ps.hb.cellStart.size(); k++) bcs[k] += (uint32_t)s.bound.off;
  uint32_t* bstart = reinterpret_cast<uint32_t*>(blob + ps.oBstart);
  for (int k = 0; k < ps.nb1; k++) bstart[k] += (uint32_t)s.list.off;
  DevScene& d = b->d;
  // particles into parity 0 of the range; everything else of the range cleared
  const size_t po = (size_t)s.part.off, nb = (size_t)s.n * 16, pr = (size_t)s.part.size * 16;
  for (int t = 0; t < 2; t++) {
    BTRY(b, cudaMemsetAsync(d.pos[t] + po, 0, pr, st));
    BTRY(b, cudaMemsetAsync(d.vel[t] + po, 0, pr, st));
    BTRY(b, cudaMemsetAsync(d.pred[t] + po, 0, pr, st));
    BTRY(b, cudaMemsetAsync(d.body[t] + po, 0, pr, st));
    BTRY(b, cudaMemsetAsync(d.rest[t] + po, 0, pr, st));
  }
  if (nb) {
    BTRY(b, cudaMemcpyAsync(d.pos[0] + po, blob + ps.oPos, nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.vel[0] + po, blob + ps.oVel, nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.pred[0] + po, blob + ps.oPos, nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.body[0] + po, blob + ps.oPhase, nb, cudaMemcpyHostToDevice, st));
    BTRY(b, cudaMemcpyAsync(d.rest[0] + po, blob + ps.oRest, nb, cudaMemcpyHostToDevice, st));
  }
  // boundary samples and their cellStart in arena indices
  BTRY(b, cudaMemcpyAsync(d.bpos + s.bound.off, blob + ps.oBpos, ps.hb.pos.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bpsi + s.bound.off, blob + ps.oBpsi, ps.hb.psi.size() * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bcellStart + s.cells.off, blob + ps.oBcs, ps.hb.cellStart.size() * 4,
                          cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemsetAsync(d.cellStart + s.cells.off, 0, (size_t)(s.nCells + 2) * 4, st));
  const size_t bo = (size_t)s.bodies.off, nb1 = (size_t)ps.nb1;
  BTRY(b, cudaMemcpyAsync(d.bodyInfo + bo, blob + ps.oInfo, nb1 * 16, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyCentre + bo, blob + ps.oCentre, nb1 * 16, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyRef + bo, blob + ps.oCentre, nb1 * 16, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyRot + bo * 3, blob + ps.oRot, nb1 * 48, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemcpyAsync(d.bodyStart + bo, blob + ps.oBstart, nb1 * 4, cudaMemcpyHostToDevice, st));
  BTRY(b, cudaMemsetAsync(d.bodyAccum + bo * 4, 0, nb1 * 16, st));
  BTRY(b, cudaMemsetAsync(d.bodyCov + bo * 9, 0, nb1 * 36, st));
  BTRY(b, cudaMemsetAsync(d.bodyFill + bo, 0, nb1 * 4, st));
  BTRY(b, cudaMemsetAsync(d.statsOut + (size_t)slot * 8, 0, 32, st));
  s.parity = 0;
  s.live = true;
  s.primed = false;
  b->scenes[slot] = std::move(s);
  BScene& S = b->scenes[slot];
  S.params.bodies = S.specs.empty() ? nullptr : S.specs.data();
  *outSlot = slot;
  return P4A_OK;
}

int prime_scenes(p4a_batch* b, const std::vector<int>& slots) {
  if (slots.empty()) return P4A_OK;
  Frame F;
  F.nSubs = 1;
  F.nRows = (int)slots.size();
  F.params.resize(slots.size());
  WorkSeg key{0, 0}, scan{0, 0}, part{0, 0};
  for (size_t k = 0; k < slots.size(); k++) {
    BScene& S = b->scenes[slots[k]];
    S.parity = 0;
    pack(S, 0.0, slots[k]);
    F.params[k] = S.P;
  }
  for (size_t k = 0; k < slots.size(); k++) {
    const BScene& S = b->scenes[slots[k]];
    key = push_items(F, (uint32_t)k, groups(std::max(S.n, S.nBodies)), key);
  }
  for (size_t k = 0; k < slots.size(); k++) scan = push_items(F, (uint32_t)k, scan_tiles(b->scenes[slots[k]].nCells), scan);
  for (size_t k = 0; k < slots.size(); k++) part = push_items(F, (uint32_t)k, groups(b->scenes[slots[k]].n), part);
  add_launch(F, LK_KEY, 0, 0, key);
  add_launch(F, LK_SCAN_SUMS, 0, 0, scan);
  add_launch(F, LK_SCAN_OFFSETS, 0, 0, scan);
  add_launch(F, LK_SCAN, 0, 0, scan);
  add_launch(F, LK_FILL, 0, 0, part);
  add_launch(F, LK_REORDER, 0, 0, part);
  const int rc = execute(b, F, false);
  if (rc) return rc;
  for (int slot : slots) {
    BScene& S = b->scenes[slot];
    S.parity = 1;
    S.primed = true;
    S.gen++;
  }
  return P4A_OK;
}

int step_frame(p4a_batch* b, const int32_t* ids, const double* frameDt, int32_t count) {
  std::vector<int> subs(count, 0);
  int maxSub = 0;
  for (int k = 0; k < count; k++) {
    BScene& s = b->scenes[ids[k]];
    // time bank (src/sim.js:418-429)
    const int base = std::max(1, s.params.substeps);
    const double dtTarget = (1.0 / 60) / base;
    s.timeBank = s.timeBank + frameDt[k];
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
  }
  if (maxSub == 0) return P4A_OK;
  Frame F;
  F.nSubs = maxSub;
  F.nRows = count;
  F.params.resize((size_t)maxSub * count);
  int64_t total = 0;
  for (int k = 0; k < count; k++) total += b->scenes[ids[k]].n;
  for (int k = 0; k < TK_COUNT; k++) {
    F.variant[k] = tuned_variant_batched(k, total);
    F.shape.push_back(F.variant[k]);
  }
  F.shape.push_back(maxSub);
  WorkSeg zero{0, 0};
  for (int k = 0; k < count; k++)
    if (subs[k] > 0) zero = push_items(F, (uint32_t)k, 1, zero);
  add_launch(F, LK_ZERO, 0, 0, zero);
  std::map<std::vector<int64_t>, WorkSeg> segCache;
  for (int s = 0; s < maxSub; s++) {
    int maxIt = 0;
    for (int k = 0; k < count; k++)
      if (subs[k] > s) maxIt = std::max(maxIt, std::max(1, b->scenes[ids[k]].params.iterations));
    F.shape.push_back(maxIt);
    // launches with the same (scene, item count) list share one segment of items
    auto seg = [&](auto&& countOf) {
      std::vector<int64_t> sig;
      for (int k = 0; k < count; k++) {
        if (subs[k] <= s) continue;
        const int64_t c = countOf(b->scenes[ids[k]]);
        if (c > 0) sig.insert(sig.end(), {(int64_t)k, c});
      }
      auto hit = segCache.find(sig);
      if (hit != segCache.end()) return hit->second;
      WorkSeg g{0, 0};
      for (size_t q = 0; q < sig.size(); q += 2) g = push_items(F, (uint32_t)sig[q], sig[q + 1], g);
      segCache.emplace(std::move(sig), g);
      return g;
    };
    const WorkSeg key = seg([](const BScene& S) { return (int64_t)groups(std::max(S.n, S.nBodies)); });
    const WorkSeg scan = seg([](const BScene& S) { return (int64_t)scan_tiles(S.nCells); });
    const WorkSeg part = seg([](const BScene& S) { return (int64_t)groups(S.n); });
    const WorkSeg seed = seg([](const BScene& S) { return (int64_t)(S.nBodyParts > 0 ? S.nBodies : 0); });
    add_launch(F, LK_KEY, s, 0, key);
    add_launch(F, LK_SCAN_SUMS, s, 0, scan);
    add_launch(F, LK_SCAN_OFFSETS, s, 0, scan);
    add_launch(F, LK_SCAN, s, 0, scan);
    add_launch(F, LK_FILL, s, 0, part);
    add_launch(F, LK_REORDER, s, 0, part);
    add_launch(F, LK_SEED, s, 0, seed);
    for (int it = 0; it < maxIt; it++) {
      const WorkSeg iter = seg([&](const BScene& S) {
        return (int64_t)(std::max(1, S.params.iterations) > it ? groups(S.n) : 0);
      });
      const WorkSeg match = seg([&](const BScene& S) {
        return (int64_t)(std::max(1, S.params.iterations) > it && S.nBodyParts > 0 ? S.nBodies : 0);
      });
      add_launch(F, LK_LAMBDA, s, it, iter);
      add_launch(F, LK_DELTA, s, it, iter);
      add_launch(F, LK_MATCH, s, it, match);
    }
    const WorkSeg plain = seg([](const BScene& S) {
      return (int64_t)(S.params.surface_tension_k > 0 ? 0 : groups(S.n));
    });
    const WorkSeg tension = seg([](const BScene& S) {
      return (int64_t)(S.params.surface_tension_k > 0 ? groups(S.n) : 0);
    });
    add_launch(F, LK_FINISH, s, 0, plain);
    add_launch(F, LK_NORMALS, s, 0, tension);
    add_launch(F, LK_TENSION, s, 0, tension);
    for (int k = 0; k < count; k++) {
      if (subs[k] <= s) continue;
      BScene& S = b->scenes[ids[k]];
      const double dt = (1.0 / 60) / std::max(1, S.params.substeps);
      pack(S, dt, ids[k]);
      S.P.parity = (uint32_t)(S.parity ^ (s & 1));
      S.P.subs = (uint32_t)subs[k];
      F.params[(size_t)s * count + k] = S.P;
    }
  }
  const int rc = execute(b, F, true);
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

// One frame of the listed scenes: on lane 0, or, with L > 1 lanes and a frame of at
// least laneMinParticles, as L parts of about equal particle counts that run at once,
// one per lane. Scenes are independent, so each scene gets the bits the whole frame
// gives it; the batch's stream waits for every part. Profiled frames stay whole, on
// one lane, so that their per-launch intervals do not overlap.
int step_scenes(p4a_batch* b, const int32_t* ids, const double* dts, int32_t count) {
  b->lane = &b->lanes[0];
  int64_t total = 0;
  for (int k = 0; k < count; k++) total += b->scenes[ids[k]].n;
  const int L = std::min(b->laneCount, (int)count);
  if (L < 2 || b->prof || total < b->laneMinParticles) return step_frame(b, ids, dts, count);
  // largest scenes first, each to the part with the fewest particles so far; each
  // part keeps the list order
  std::vector<int> order((size_t)count);
  for (int k = 0; k < count; k++) order[(size_t)k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b->scenes[ids[x]].n > b->scenes[ids[y]].n; });
  std::vector<int> part((size_t)count, 0);
  int64_t load[p4a_batch::kMaxLanes] = {};
  for (int k : order) {
    int q = 0;
    for (int t = 1; t < L; t++)
      if (load[t] < load[q]) q = t;
    part[(size_t)k] = q;
    load[q] += b->scenes[ids[k]].n;
  }
  std::vector<int32_t> id[p4a_batch::kMaxLanes];
  std::vector<double> dt[p4a_batch::kMaxLanes];
  for (int k = 0; k < count; k++) {
    id[part[(size_t)k]].push_back(ids[k]);
    dt[part[(size_t)k]].push_back(dts[k]);
  }
  BTRY(b, cudaEventRecord(b->laneFork, b->stream));
  int rc = P4A_OK;
  for (int q = 0; q < L; q++) {
    if (id[q].empty()) continue;
    if (q > 0) BTRY(b, cudaStreamWaitEvent(b->lanes[q].stream, b->laneFork, 0));
    if (!rc) {
      b->lane = &b->lanes[q];
      rc = step_frame(b, id[q].data(), dt[q].data(), (int32_t)id[q].size());
      b->lane = &b->lanes[0];
    }
    // whatever happened, later work on the batch's stream comes after this lane's
    if (q > 0) {
      BTRY(b, cudaEventRecord(b->laneJoin[q], b->lanes[q].stream));
      BTRY(b, cudaStreamWaitEvent(b->stream, b->laneJoin[q], 0));
    }
  }
  return rc;
}

}  // namespace p4a

namespace {

// Admits a host scene on the batch's stream and waits for it (src/sim.js:66-253).
int admit(p4a_batch* b, const p4a_params& params, HostScene& sc, int pourBudget, int32_t* outId) {
  PreparedScene ps;
  std::string err;
  int rc = prepare_scene(params, sc, pourBudget, ps, err);
  if (rc) return bfail(b, rc, "%s", err.c_str());
  std::vector<unsigned char> blob(ps.bytes);
  write_blob(ps, blob.data());
  int32_t slot = -1;
  if ((rc = place_scene(b, ps, blob.data(), b->stream, &slot))) return rc;
  rc = prime_scenes(b, {slot});
  if (rc) {
    cudaStreamSynchronize(b->stream);
    release_scene(b, b->scenes[slot]);
    return rc;
  }
  BTRY(b, cudaStreamSynchronize(b->stream));  // the blob goes out of scope
  *outId = slot;
  return P4A_OK;
}

bool config_ok(const p4a_batch_config* cfg) {
  return cfg && cfg->max_particles > 0 && cfg->max_cells > 0 && cfg->max_scenes > 0 &&
         cfg->max_particles <= 0x7fffffffLL && cfg->max_cells <= 0x7fffffffLL;
}

p4a_batch_config normalised(p4a_batch_config c) {
  if (c.max_bodies < 1) c.max_bodies = 1;
  if (c.max_body_parts < 1) c.max_body_parts = 1;
  if (c.max_boundary < 1) c.max_boundary = 1;
  return c;
}

// Every arena of a batch, sized from b->cfg (its minimums already applied). With
// b->sizeOnly set nothing is allocated and b->deviceBytes receives the total.
int alloc_arenas(p4a_batch* b) {
  const p4a_batch_config* cfg = &b->cfg;
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
       (rc = balloc(b, &d.unordered, P)) || (rc = balloc(b, &d.nbList, P * kListCap)) || (rc = balloc(b, &d.nbCount, P)) ||
       (rc = balloc(b, &d.nbCell, P)) || (rc = balloc(b, &d.disp, (int64_t)cfg->max_scenes * kDispSlots)) ||
       (rc = balloc(b, &d.cellDisp, (int64_t)kDispSlots * Cc)) || (rc = balloc(b, &d.nbRef, P)) || (rc = balloc(b, &d.predLam, P)) ||
       (rc = balloc(b, &d.velRho, P)) || (rc = balloc(b, &d.normRho, P)) ||
       (rc = balloc(b, &d.cellCount, Cc)) ||
       (rc = balloc(b, &d.cellStart, Cc)) || (rc = balloc(b, &d.bcellStart, Cc)) ||
       (rc = balloc(b, &d.scanState, b->scanTilesCap)) || (rc = balloc(b, &d.scanTicket, 4)) ||
       (rc = balloc(b, &d.errorWord, 4)) || (rc = balloc(b, &d.bpos, b->cfg.max_boundary)) ||
       (rc = balloc(b, &d.bpsi, b->cfg.max_boundary)) || (rc = balloc(b, &d.bodyAccum, B1 * 4)) ||
       (rc = balloc(b, &d.bodyCov, B1 * 9)) || (rc = balloc(b, &d.bodyCentre, B1)) ||
       (rc = balloc(b, &d.bodyRef, B1)) || (rc = balloc(b, &d.bodyRot, B1 * 3)) ||
       (rc = balloc(b, &d.bodyInfo, B1)) || (rc = balloc(b, &d.bodyStart, B1)) ||
       (rc = balloc(b, &d.bodyFill, B1)) || (rc = balloc(b, &d.bodyList, b->cfg.max_body_parts)) ||
       (rc = balloc(b, &d.statsOut, (int64_t)cfg->max_scenes * 8)) ||
       (rc = balloc(b, &b->lanes[0].dParams, (int64_t)kMaxSubsteps * cfg->max_scenes)) ||
       (rc = balloc(b, &b->lanes[1].dParams, (int64_t)kMaxSubsteps * cfg->max_scenes)) ||
       (rc = balloc(b, &b->lanes[2].dParams, (int64_t)kMaxSubsteps * cfg->max_scenes)) ||
       (rc = balloc(b, &b->lanes[3].dParams, (int64_t)kMaxSubsteps * cfg->max_scenes))))
    ;
  return rc;
}

}  // namespace


extern "C" {

int p4a_batch_footprint(const p4a_batch_config* cfg, int64_t* bytes) {
  if (!bytes || !config_ok(cfg)) return P4A_ERR_ARG;
  p4a_batch b;
  b.sizeOnly = true;
  b.cfg = normalised(*cfg);
  const int rc = alloc_arenas(&b);
  *bytes = (int64_t)b.deviceBytes;
  return rc;
}

int p4a_batch_create(int device, const p4a_batch_config* cfg, p4a_batch** out) {
  if (!config_ok(cfg) || !out) return P4A_ERR_ARG;
  *out = nullptr;
  const int chk = p4a_device_check(device);
  if (chk != P4A_OK) return chk;
  if (cudaSetDevice(device) != cudaSuccess) return P4A_ERR_CUDA;
  p4a_batch* b = new p4a_batch();
  b->device = device;
  b->cfg = normalised(*cfg);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return P4A_ERR_CUDA;
  }
  b->ownStream = true;
  b->lanes[0].stream = b->stream;
  for (int q = 1; q < p4a_batch::kMaxLanes; q++)
    if (cudaStreamCreateWithFlags(&b->lanes[q].stream, cudaStreamNonBlocking) != cudaSuccess) {
      p4a_batch_destroy(b);
      return P4A_ERR_CUDA;
    }
  for (auto& Ln : b->lanes)
    for (int k = 0; k < 2; k++) cudaEventCreateWithFlags(&Ln.stagingDone[k], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&b->laneFork, cudaEventDisableTiming);
  for (auto& e : b->laneJoin) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  const int64_t P = cfg->max_particles, Cc = cfg->max_cells + (int64_t)cfg->max_scenes * (kScanTile + 2);
  int rc = alloc_arenas(b);
  if (rc) {
    p4a_batch_destroy(b);
    return rc;
  }
  b->d.cap = (uint32_t)P;
  b->d.cellStride = (uint32_t)Cc;
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
  for (int q = 1; q < p4a_batch::kMaxLanes; q++)
    if (b->lanes[q].stream) cudaStreamSynchronize(b->lanes[q].stream);
  drop_graphs(b);
  drop_profile_events(b);
  for (void* p : b->allocs) cudaFree(p);
  for (auto& Ln : b->lanes) {
    if (Ln.dItems) cudaFree(Ln.dItems);
    if (Ln.dSegs) cudaFree(Ln.dSegs);
    if (Ln.dCursors) cudaFree(Ln.dCursors);
    for (int k = 0; k < 2; k++) {
      if (Ln.staging[k]) cudaFreeHost(Ln.staging[k]);
      if (Ln.stagingDone[k]) cudaEventDestroy(Ln.stagingDone[k]);
    }
  }
  for (int q = 1; q < p4a_batch::kMaxLanes; q++)
    if (b->lanes[q].stream) cudaStreamDestroy(b->lanes[q].stream);
  if (b->laneFork) cudaEventDestroy(b->laneFork);
  for (auto e : b->laneJoin)
    if (e) cudaEventDestroy(e);
  if (b->upStream) cudaStreamDestroy(b->upStream);
  if (b->h2dStream) cudaStreamDestroy(b->h2dStream);
  if (b->d2hStream) cudaStreamDestroy(b->d2hStream);
  for (cudaEvent_t e : b->ioEvents) cudaEventDestroy(e);
  if (b->ownStream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return P4A_OK;
}

const char* p4a_batch_last_error(const p4a_batch* b) { return b ? b->err.c_str() : "null handle"; }

int p4a_batch_set_stream(p4a_batch* b, void* stream) {
  if (!b) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  BTRY(b, cudaStreamSynchronize(b->stream));
  for (int q = 1; q < p4a_batch::kMaxLanes; q++) BTRY(b, cudaStreamSynchronize(b->lanes[q].stream));
  drop_graphs(b);
  if (stream) {
    if (b->ownStream) cudaStreamDestroy(b->stream);
    b->stream = (cudaStream_t)stream;
    b->ownStream = false;
  } else if (!b->ownStream) {
    BTRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->ownStream = true;
  }
  b->lanes[0].stream = b->stream;
  return P4A_OK;
}

int p4a_batch_use_graphs(p4a_batch* b, int32_t on) {
  if (!b) return P4A_ERR_ARG;
  b->useGraphs = on != 0;
  return P4A_OK;
}

int p4a_batch_profile_enable(p4a_batch* b, int32_t on) {
  if (!b) return P4A_ERR_ARG;
  b->prof = on != 0;
  return P4A_OK;
}

int p4a_batch_profile_reset(p4a_batch* b) {
  if (!b) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  const int rc = resolve_profile(b);
  for (int k = 0; k < kLaunchKinds; k++) {
    b->profMs[k] = 0;
    b->profLaunches[k] = 0;
  }
  return rc;
}

int p4a_batch_profile_read(p4a_batch* b, p4a_phase_time* out, int32_t maxEntries, int32_t* count) {
  if (!b || (maxEntries > 0 && !out)) return P4A_ERR_ARG;
  cudaSetDevice(b->device);
  const int rc = resolve_profile(b);
  int c = 0;
  for (int k = 0; k < kLaunchKinds; k++) {
    if (b->profLaunches[k] == 0) continue;
    if (c < maxEntries) {
      std::snprintf(out[c].name, sizeof(out[c].name), "%s", kLaunchNames[k]);
      out[c].ms = b->profMs[k];
      out[c].launches = b->profLaunches[k];
    }
    c++;
  }
  if (count) *count = c;
  return rc;
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
  std::vector<char> seen(b->scenes.size(), 0);
  for (int k = 0; k < count; k++) {
    const int rc = scene_ok(b, ids[k]);
    if (rc) return rc;
    if (seen[ids[k]]++) return bfail(b, P4A_ERR_ARG, "p4a_batch_step: scene %d listed twice", ids[k]);
  }
  const std::vector<double> dts((size_t)count, frameDt);
  return step_scenes(b, ids, dts.data(), count);
}

int p4a_batch_set_lanes(p4a_batch* b, int32_t lanes, int64_t min_particles) {
  if (!b || lanes < 1 || lanes > p4a_batch::kMaxLanes || min_particles < 0)
    return bfail(b, P4A_ERR_ARG, "p4a_batch_set_lanes: bad value");
  b->laneCount = lanes;
  b->laneMinParticles = min_particles;
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

}  // extern "C"

// Device pointer, element size and element count of a scene's view of a buffer.
int p4a::scene_buffer(p4a_batch* b, const BScene& s, int32_t id, int32_t which, void** p, size_t* bytes) {
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

extern "C" {

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

// Asynchronous forms: the copy is queued on the batch's stream behind the frames
// already queued (and before the next ones); host memory stays in use until
// p4a_batch_synchronize. cellStart holds arena indices, so it is not offered here.
int p4a_batch_read_async(p4a_batch* b, int32_t id, int32_t bid, int32_t which, void* host, size_t offset,
                         size_t bytes) {
  int rc = scene_ok(b, id);
  if (rc) return rc;
  if (!host && bytes) return P4A_ERR_ARG;
  if (bid == P4A_BUF_CELL_START) return bfail(b, P4A_ERR_ARG, "cellStart is read with p4a_batch_read only");
  const BScene& s = b->scenes[id];
  void* p = nullptr;
  size_t total = 0;
  if ((rc = scene_buffer(b, s, bid, which, &p, &total))) return rc;
  if (offset > total || bytes > total - offset) return bfail(b, P4A_ERR_ARG, "read beyond the scene's buffer");
  if (!bytes) return P4A_OK;
  cudaSetDevice(b->device);
  BTRY(b, cudaMemcpyAsync(host, (const char*)p + offset, bytes, cudaMemcpyDeviceToHost, b->stream));
  return P4A_OK;
}

int p4a_batch_write_async(p4a_batch* b, int32_t id, int32_t bid, int32_t which, const void* host, size_t offset,
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
  return P4A_OK;
}

int p4a_batch_step_io(p4a_batch* b, const p4a_batch_io* io, int32_t count, double frameDt, int32_t groups) {
  if (!b || count < 0 || (count > 0 && !io) || groups < 0)
    return bfail(b, P4A_ERR_ARG, "p4a_batch_step_io: bad list");
  cudaSetDevice(b->device);
  std::vector<char> seen(b->scenes.size(), 0);
  int64_t total = 0;
  for (int k = 0; k < count; k++) {
    const int rc = scene_ok(b, io[k].scene_id);
    if (rc) return rc;
    if (seen[io[k].scene_id]++) return bfail(b, P4A_ERR_ARG, "p4a_batch_step_io: scene %d listed twice", io[k].scene_id);
    total += b->scenes[io[k].scene_id].n;
  }
  if (count == 0) return P4A_OK;
  // groups of about equal particle counts, in list order; group g runs on lane
  // g mod lanes. By default, with two or more frame lanes, one group per 750 k
  // particles (at most 8): consecutive groups run at once on different lanes, so a
  // group's launch tails overlap the other lanes' work and only the first group's
  // writes and the last groups' reads stay exposed (on the 6 M-particle mix with two
  // lanes: 391, 407, 417, 421 M particle-substeps/s end to end with 2, 4, 6, 8
  // groups). With one lane each split adds the launch tails of a whole frame (a frame
  // split in two took 6 % longer, in four 18 %): two groups from 3 M up, else one.
  const int nLanes = b->prof ? 1 : b->laneCount;
  int G = groups > 0 ? groups
                     : nLanes > 1 ? (int)std::min<int64_t>(8, std::max<int64_t>(1, total / 750000))
                                  : (total >= 3000000 ? 2 : 1);
  G = std::min(G, std::min(count, 64));
  std::vector<int> first((size_t)G + 1, count);
  first[0] = 0;
  {
    // group g starts after the first scene k at which the groups before it hold
    // g / G of the particles, or where each later group is left one scene
    int64_t acc = 0;
    int g = 1;
    for (int k = 0; k < count && g < G; k++) {
      acc += b->scenes[io[k].scene_id].n;
      const int left = count - (k + 1);
      if (acc * G >= total * g || left == G - g) first[(size_t)g++] = k + 1;
    }
  }
  if (!b->h2dStream) BTRY(b, cudaStreamCreateWithFlags(&b->h2dStream, cudaStreamNonBlocking));
  if (!b->d2hStream) BTRY(b, cudaStreamCreateWithFlags(&b->d2hStream, cudaStreamNonBlocking));
  while (b->ioEvents.size() < (size_t)(2 * G + 2)) {
    cudaEvent_t e = nullptr;
    BTRY(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ioEvents.push_back(e);
  }
  cudaEvent_t* ev = b->ioEvents.data();
  auto live = [&](const BScene& S, int32_t bid, void** p) -> int {
    size_t bytes = 0;
    const int rc = scene_buffer(b, S, bid, P4A_LIVE, p, &bytes);
    return rc ? rc : ((size_t)S.n * 16 > bytes ? bfail(b, P4A_ERR_ARG, "scene buffer too small") : P4A_OK);
  };
  // the copies start after everything queued on the batch's stream so far
  BTRY(b, cudaEventRecord(ev[0], b->stream));
  BTRY(b, cudaStreamWaitEvent(b->h2dStream, ev[0], 0));
  BTRY(b, cudaStreamWaitEvent(b->d2hStream, ev[0], 0));
  auto copies = [&](int g, bool in) -> int {
    for (int k = first[(size_t)g]; k < first[(size_t)g + 1]; k++) {
      const BScene& S = b->scenes[io[k].scene_id];
      const size_t bytes = (size_t)S.n * 16;
      const void* hp[2] = {in ? io[k].pos_in : io[k].pos_out, in ? io[k].vel_in : io[k].vel_out};
      for (int q = 0; q < 2; q++) {
        if (!hp[q] || !bytes) continue;
        void* p = nullptr;
        const int rc = live(S, q ? P4A_BUF_VEL : P4A_BUF_POS, &p);
        if (rc) return rc;
        if (in)
          BTRY(b, cudaMemcpyAsync(p, hp[q], bytes, cudaMemcpyHostToDevice, b->h2dStream));
        else
          BTRY(b, cudaMemcpyAsync(const_cast<void*>(hp[q]), p, bytes, cudaMemcpyDeviceToHost, b->d2hStream));
      }
    }
    return P4A_OK;
  };
  auto writes = [&](int g) -> int {
    const int rc = copies(g, true);
    if (rc) return rc;
    BTRY(b, cudaEventRecord(ev[1 + 2 * g], b->h2dStream));
    return P4A_OK;
  };
  std::vector<int32_t> ids;
  // group g on lane g mod lanes, so that consecutive groups' frames run at once;
  // profiled frames stay on lane 0
  auto frame = [&](int g) -> int {
    b->lane = &b->lanes[g % nLanes];
    cudaStream_t fs = b->lane->stream;
    // group g's frame waits for its own writes only
    BTRY(b, cudaStreamWaitEvent(fs, ev[1 + 2 * g], 0));
    ids.clear();
    for (int k = first[(size_t)g]; k < first[(size_t)g + 1]; k++) ids.push_back(io[k].scene_id);
    const std::vector<double> dts(ids.size(), frameDt);
    const int rc = step_frame(b, ids.data(), dts.data(), (int32_t)ids.size());
    b->lane = &b->lanes[0];
    if (rc) return rc;
    BTRY(b, cudaEventRecord(ev[2 + 2 * g], fs));
    return P4A_OK;
  };
  auto reads = [&](int g) -> int {
    // group g's reads wait for its own frame only
    BTRY(b, cudaStreamWaitEvent(b->d2hStream, ev[2 + 2 * g], 0));
    return copies(g, false);
  };
  // Issued as W0 F0, then W(g) F(g) R(g-1), then the last reads: a copy queued
  // behind one that waits for a frame never holds up an earlier frame, whether the
  // copy engines serve the two copy streams apart or in issue order.
  int rc = writes(0);
  if (!rc) rc = frame(0);
  for (int g = 1; g < G && !rc; g++) {
    rc = writes(g);
    if (!rc) rc = frame(g);
    if (!rc) rc = reads(g - 1);
  }
  if (!rc) rc = reads(G - 1);
  // later work on the batch's stream (and p4a_batch_synchronize) waits for every copy
  // and, through the reads' waits, for every group's frame
  b->lane = &b->lanes[0];
  BTRY(b, cudaEventRecord(ev[2 * G + 1], b->d2hStream));
  BTRY(b, cudaStreamWaitEvent(b->stream, ev[2 * G + 1], 0));
  BTRY(b, cudaEventRecord(ev[0], b->h2dStream));
  BTRY(b, cudaStreamWaitEvent(b->stream, ev[0], 0));
  return rc;
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
