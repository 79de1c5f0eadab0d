// api.cu — the C ABI of include/p4a.h: host orchestration of the simulation step.
//
// This replaces the reference's `class Sim` (src/sim.js:9-814). The schedule of a
// substep follows src/sim.js:458-596 with these B200-side fusions:
//   predict            recomputed inside the key and reorder passes (never stored)
//   grid pass          key_count -> scan -> fill -> reorder (kernels_grid.cu)
//   bodies pass        one CTA per body (kernels_body.cu)
//   k iterations       lambda, delta (+ velFromPos on the last), body_match
//   odd-k pred copy    fused into the finalize kernel
//   finish             xsph+finalize, or xsph+normals then tension+finalize
//   stats              fused into the last substep's finalize
// The time bank, substep count, uniform packing and parity bookkeeping are the
// reference's, in double precision like the JS.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/p4a.h"
#include "fmath.h"
#include "p4a_internal.h"
#include "scene.h"

using namespace p4a;

namespace {
const double kPi = 3.14159265358979323846;

// Kernel names for the per-kernel timing of p4a_profile_* (the counterpart of the
// reference's GpuTimer marks 'predict', 'grid', 'bodies', 'solve', 'finish', 'stats').
enum Phase {
  PH_DRAG, PH_KEY_COUNT, PH_SCAN, PH_FILL, PH_REORDER, PH_BODY_SEED, PH_LAMBDA, PH_DELTA,
  PH_BODY_MATCH, PH_XSPH_FINALIZE, PH_XSPH_NORMALS, PH_TENSION_FINALIZE, PH_ANISO, PH_IMPULSE,
  PH_RESIZE, PH_STATS_CLEAR, PH_MESH_FIELD, PH_MESH_BLUR, PH_MESH_MARCH, PH_SSFR, PH_RAY, PH_HOSE, PH_COUNT,
  PH_END = PH_COUNT
};
const char* const kPhaseNames[PH_COUNT] = {
    "body_drag", "key_count", "scan", "fill", "reorder", "body_seed", "lambda", "delta",
    "body_match", "xsph_finalize", "xsph_normals", "tension_finalize", "aniso", "impulse",
    "resize", "stats_clear", "mesh_field", "mesh_blur", "mesh_march", "ssfr", "ray", "hose"};

std::atomic<uint64_t> g_launches{0};
}  // namespace

struct p4a_sim {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  // asynchronous readbacks (p4a_read_async): a copy stream ordered after the sim's
  // stream by copyReady; copyDone marks the last queued copy
  cudaStream_t copyStream = nullptr;
  cudaEvent_t copyReady = nullptr, copyDone = nullptr;
  uint64_t copyInFlight = 0;  // buffer ids read by copies the sim's stream is not yet ordered after
  bool copyHost = false;      // copies whose host data p4a_read_wait has not waited for
  std::string err;
  p4a_params params{};
  std::vector<p4a_body_spec> specs;
  HostScene sc;
  int n = 0, cap = 0, pourBudget = 0, nBoundary = 0, nBodies = 0, nBodyParts = 0;
  double h = 0;
  int gridDim[3] = {1, 1, 1};
  int nCells = 1;
  DevScene d{};
  std::vector<void*> sceneAllocs;  // freed on reset / destroy
  std::vector<void*> cellAllocs;   // freed on reset / resize
  std::vector<void*> boundaryAllocs;
  std::vector<uint32_t> bodyStartHost;
  double bodyScale = 0, covScale = 0;
  int parity = 0, predParity = 0, gen = 0;
  double simTime = 0, timeBank = 0, lastAdvanced = 0;
  int lastSubsteps = 0;
  int heldBody = -1;
  double heldTarget[3] = {0, 0, 0}, heldRate = 10, heldLimit = 4;
  SimParams P{};
  uint32_t scanEpoch = 0;
  // readback (stats, error word, pose), latest-completed semantics
  uint32_t* pinned = nullptr;  // [8 stats][1 err][pad] then pose floats
  size_t pinnedBytes = 0;
  cudaEvent_t readEvent = nullptr;
  bool readPending = false;
  bool readStale = false;  // a step finished after the last readback was issued
  bool poseValid = false;
  p4a_stats stats{};
  std::vector<float> pose;  // per body: centre xyz, then 3 rows xyz(w)
  // aniso outputs
  float4* smoothPos = nullptr;
  float4* anisoG = nullptr;
  size_t anisoCap = 0;
  int anisoGen = 0;
  // surface mesh (p4a_mesh)
  float* meshField[3] = {nullptr, nullptr, nullptr};  // field, normal field, blur scratch
  uint32_t* meshCounts = nullptr;                     // per voxel, zero between calls
  uint32_t* meshOffsets = nullptr;                    // [nvox + 1]
  unsigned long long* meshScan = nullptr;
  uint32_t* meshTicket = nullptr;
  uint2* meshVerts = nullptr;
  size_t meshVertCap = 0, meshVoxCap = 0, meshTriCap = 0;
  int fieldSlot = 0, nfieldSlot = 1;  // which of meshField[] hold the fields
  int meshGen = 0;
  int32_t meshDim[3] = {0, 0, 0};
  double meshOrigin = 0, meshVoxel = 0;
  int64_t meshTris = 0;
  size_t meshNvox = 0;  // voxels of the last p4a_mesh: meshOffsets[meshNvox] is its triangle count
  uint32_t meshEpoch = 0;
  // screen-space fluid rendering (p4a_ssfr)
  std::vector<void*> ssfrAllocs;
  SsfrFrame ssfr{};
  int ssfrW = 0, ssfrH = 0, ssfrMapW = 0, ssfrMapH = 0, ssfrThW = 0, ssfrThH = 0, ssfrGen = 0;
  float4* ssfrBodies = nullptr;
  int ssfrBodyCap = 0;
  ushort4* envCube = nullptr;  // p4a_set_environment: 6 faces of envSize^2 rgba16float texels
  int envSize = 0;
  uchar4* rayImage = nullptr;  // p4a_ray
  char* raySurf = nullptr;     // p4a_ray's mesh surface maps, rayCap pixels
  size_t rayCap = 0;
  int rayW = 0, rayH = 0;
  bool ready = false;
  // every particle lies within the last substep's recorded iteration
  // displacements of the position the sort binned it by: true after a step, until
  // positions are written, appended, resized or reset
  bool sortedMoves = false;
  // per-kernel timing (p4a_profile_*)
  bool prof = false;
  std::vector<cudaEvent_t> evPool;
  std::vector<int> evPhase;
  int evUsed = 0;
  double phaseMs[PH_COUNT] = {};
  long long phaseLaunches[PH_COUNT] = {};
};

namespace {

int fail(p4a_sim* s, int code, const char* fmt, ...) {
  if (s) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    s->err = buf;
  }
  return code;
}

#define CUDA_TRY(s, call)                                                              \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      return fail((s), e_ == cudaErrorMemoryAllocation ? P4A_ERR_OOM : P4A_ERR_CUDA,   \
                  "%s: %s", #call, cudaGetErrorString(e_));                            \
    }                                                                                  \
  } while (0)

// Orders the sim's stream after the asynchronous readbacks of any buffer in
// `writes` (a mask of buffer-id bits), so that work queued next cannot change
// what those copies read. No host wait.
void after_reads(p4a_sim* s, uint64_t writes) {
  if (s->copyInFlight & writes) {
    cudaStreamWaitEvent(s->stream, s->copyDone, 0);
    s->copyInFlight = 0;  // copyDone covers every copy queued so far
  }
}
constexpr uint64_t kAllBuffers = ~0ull;
constexpr uint64_t buf_bit(int id) { return 1ull << id; }

// Host wait for every asynchronous readback: before device memory is freed or
// reallocated, and by p4a_read_wait / p4a_synchronize.
int drain_reads(p4a_sim* s) {
  if (s->copyHost) {
    s->copyHost = false;
    s->copyInFlight = 0;
    CUDA_TRY(s, cudaEventSynchronize(s->copyDone));
  }
  return P4A_OK;
}

// Accumulates the recorded kernel intervals into the per-kernel totals.
int resolve_marks(p4a_sim* s) {
  if (s->evUsed == 0) return P4A_OK;
  CUDA_TRY(s, cudaEventSynchronize(s->evPool[s->evUsed - 1]));
  for (int k = 0; k + 1 < s->evUsed; k++) {
    const int ph = s->evPhase[k];
    if (ph >= PH_COUNT) continue;
    float ms = 0.0f;
    CUDA_TRY(s, cudaEventElapsedTime(&ms, s->evPool[k], s->evPool[k + 1]));
    s->phaseMs[ph] += ms;
    s->phaseLaunches[ph]++;
  }
  s->evUsed = 0;
  return P4A_OK;
}

// Called before each kernel the handle launches (and with PH_END after the last):
// counts launches and, with profiling on, records the event that opens the interval.
void mark(p4a_sim* s, int phase) {
  // the SSFR phase counts its own launches (several kernels per phase)
  if (phase < PH_COUNT && phase != PH_STATS_CLEAR && phase != PH_SSFR && phase != PH_RAY) g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!s->prof) return;
  if (s->evUsed == (int)s->evPool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    s->evPool.push_back(e);
    s->evPhase.push_back(PH_END);
  }
  cudaEventRecord(s->evPool[s->evUsed], s->stream);
  s->evPhase[s->evUsed] = phase;
  s->evUsed++;
  if (phase == PH_END && s->evUsed >= 4096) resolve_marks(s);  // keeps the event pool bounded
}

template <class T>
int dalloc(p4a_sim* s, std::vector<void*>& list, T** out, size_t count) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(16, count * sizeof(T));
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess)
    return fail(s, P4A_ERR_OOM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  e = cudaMemsetAsync(p, 0, bytes, s->stream);
  if (e != cudaSuccess) {
    cudaFree(p);
    return fail(s, P4A_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
  }
  list.push_back(p);
  *out = (T*)p;
  return P4A_OK;
}

void free_list(std::vector<void*>& list) {
  for (void* p : list) cudaFree(p);
  list.clear();
}

// uploadParams(dt) (src/sim.js:371-413).
void pack_params(p4a_sim* s, double dt) {
  const p4a_params& p = s->params;
  SimParams& F = s->P;
  const double h = s->h, d = p.spacing;
  F.boxMin[0] = F.boxMin[1] = F.boxMin[2] = 0.0f;
  F.dt = (float)dt;
  for (int k = 0; k < 3; k++) F.boxMax[k] = (float)p.box[k];
  F.h = (float)h;
  for (int k = 0; k < 3; k++) F.gridDim[k] = s->gridDim[k];
  F.h2 = (float)(h * h);
  const double halfD = 0.5 * d;
  for (int k = 0; k < 3; k++) F.clampMin[k] = (float)halfD;
  const double poly6 = 315 / (64 * kPi * std::pow(h, 9));
  F.poly6 = (float)poly6;
  for (int k = 0; k < 3; k++) F.clampMax[k] = (float)(p.box[k] - halfD);
  F.spikyGrad = (float)(-45 / (kPi * std::pow(h, 6)));
  F.gravity = (float)p.gravity;
  F.mass = (float)s->sc.mass;
  F.rho0 = (float)p.rest_density;
  F.invRho0 = (float)(1 / p.rest_density);
  F.cfmEps = (float)(p.cfm_epsilon_abs > 0 ? p.cfm_epsilon_abs
                                           : std::max(1e-9, p.cfm_epsilon_rel * s->sc.denomRest));
  F.sCorrK = (float)(p.s_corr_k / (s->sc.denomRest * std::max(1, p.iterations)));
  const double rq = p.s_corr_dq * h, tq = h * h - rq * rq;
  const double wq = poly6 * tq * tq * tq;
  F.sCorrWq = (float)(wq > 0 ? 1 / wq : 0);
  F.xsphC = (float)p.xsph_c;
  F.n = (uint32_t)s->n;
  F.nCells = (uint32_t)s->nCells;
  F.nBoundary = p.no_boundary ? 0u : (uint32_t)s->nBoundary;
  F.nBodyParts = (uint32_t)s->nBodyParts;
  F.nBodies = (uint32_t)s->nBodies;
  F.bodyScale = (float)s->bodyScale;
  F.covScale = (float)s->covScale;
  F.omega = (float)p.omega;
  F.sorAverage = p.sor_average ? 1u : 0u;
  F.invDt = (float)(dt > 0 ? 1 / dt : 0);
  F.volume = (float)(s->sc.mass / p.rest_density);
  F.tension = (float)p.surface_tension_k;
  F.cohes = (float)(32 / (kPi * std::pow(h, 9)));
  F.cohesTerm = (float)(std::pow(h, 6) / 64);
  F.pOff = 0;
  F.pEnd = (uint32_t)s->n;
  F.cOff = 0;
  F.bOff = 0;
  F.parity = (uint32_t)s->parity;
  F.iters = (uint32_t)std::max(1, p.iterations);
  F.subs = 1;
  F.slot = 0;
  F.skinH2 = (float)((h + kSkin * h) * (h + kSkin * h));
  F.skinHalf = (float)((kSkin * h - 1e-4 * h) * 0.5);
  F.volSpiky = F.volume * F.spikyGrad;
}

uint32_t next_epoch(p4a_sim* s) {
  s->scanEpoch = (s->scanEpoch + 1) & 0x3fffffffu;
  if (s->scanEpoch == 0) s->scanEpoch = 1;
  return s->scanEpoch;
}

// Cell arrays: histogram, cellStart, scan tile state (src/sim.js:107-110).
int alloc_cells(p4a_sim* s) {
  free_list(s->cellAllocs);
  int rc;
  if ((rc = dalloc(s, s->cellAllocs, &s->d.cellCount, (size_t)s->nCells + 1))) return rc;
  if ((rc = dalloc(s, s->cellAllocs, &s->d.cellStart, (size_t)s->nCells + 2))) return rc;
  if ((rc = dalloc(s, s->cellAllocs, &s->d.scanState, (size_t)scan_tiles(s->nCells)))) return rc;
  if ((rc = dalloc(s, s->cellAllocs, &s->d.scanTicket, 4))) return rc;
  s->d.cellStride = (uint32_t)s->nCells + 1;
  if ((rc = dalloc(s, s->cellAllocs, &s->d.cellDisp, (size_t)kDispSlots * s->d.cellStride))) return rc;
  return P4A_OK;
}

// boundaryParticles + sortBoundary, uploaded (src/sim.js:112-127, 721-736).
int upload_boundary(p4a_sim* s) {
  HostBoundary hb;
  build_boundary(s->params.box, s->params.rest_density, s->params.spacing, s->h, s->gridDim, hb);
  free_list(s->boundaryAllocs);
  int rc;
  const int nb = hb.count;
  if ((rc = dalloc(s, s->boundaryAllocs, &s->d.bpos, (size_t)std::max(1, nb)))) return rc;
  if ((rc = dalloc(s, s->boundaryAllocs, &s->d.bpsi, (size_t)std::max(1, nb)))) return rc;
  if ((rc = dalloc(s, s->boundaryAllocs, &s->d.bcellStart, (size_t)s->nCells + 2))) return rc;
  CUDA_TRY(s, cudaMemcpyAsync(s->d.bpos, hb.pos.data(), hb.pos.size() * 4, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaMemcpyAsync(s->d.bpsi, hb.psi.data(), hb.psi.size() * 4, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaMemcpyAsync(s->d.bcellStart, hb.cellStart.data(), hb.cellStart.size() * 4,
                              cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));  // host vectors go out of scope
  s->nBoundary = nb;
  return P4A_OK;
}

// The grid pass at parity `par` into parity par^1 (src/sim.js:473-492).
void grid_pass(p4a_sim* s, int par) {
  DevScene& d = s->d;
  cudaStream_t st = s->stream;
  s->P.parity = (uint32_t)par;
  mark(s, PH_KEY_COUNT);
  launch_key_count(s->P, d, st);
  mark(s, PH_SCAN);
  launch_scan(d.cellCount, d.cellStart, s->nCells, d.scanState, d.scanTicket, next_epoch(s),
              d.errorWord, st);
  mark(s, PH_FILL);
  launch_fill(s->P, d, st);
  mark(s, PH_REORDER);
  launch_reorder(s->P, d, st);
}

int reset_common(p4a_sim* s) {
  const int drc = drain_reads(s);  // the buffers are reallocated
  if (drc) return drc;
  s->sortedMoves = false;
  HostScene& sc = s->sc;
  const p4a_params& p = s->params;
  s->ready = false;
  s->simTime = 0;
  s->gen++;
  const int n = sc.n;
  s->h = sc.h;
  for (int k = 0; k < 3; k++) s->gridDim[k] = (int)std::max(1.0, std::floor(p.box[k] / s->h));
  s->nCells = s->gridDim[0] * s->gridDim[1] * s->gridDim[2];
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  free_list(s->sceneAllocs);
  s->d = DevScene{};
  const size_t cap = (size_t)n + s->pourBudget;
  s->cap = (int)cap;
  int rc;
  auto& L = s->sceneAllocs;
  for (int t = 0; t < 2; t++) {
    if ((rc = dalloc(s, L, &s->d.pos[t], cap)) || (rc = dalloc(s, L, &s->d.vel[t], cap)) ||
        (rc = dalloc(s, L, &s->d.pred[t], cap)) || (rc = dalloc(s, L, &s->d.body[t], cap)) ||
        (rc = dalloc(s, L, &s->d.rest[t], cap)))
      return rc;
  }
  if ((rc = dalloc(s, L, &s->d.lambda, cap)) || (rc = dalloc(s, L, &s->d.density, cap)) ||
      (rc = dalloc(s, L, &s->d.corr, cap)) || (rc = dalloc(s, L, &s->d.normal, cap)) ||
      (rc = dalloc(s, L, &s->d.key, cap)) || (rc = dalloc(s, L, &s->d.rank, cap)) ||
      (rc = dalloc(s, L, &s->d.unordered, cap)) || (rc = dalloc(s, L, &s->d.statsOut, 8)) ||
      (rc = dalloc(s, L, &s->d.errorWord, 4)) || (rc = dalloc(s, L, &s->d.nbList, cap * kListCap)) ||
      (rc = dalloc(s, L, &s->d.nbCount, cap)) || (rc = dalloc(s, L, &s->d.nbCell, cap)) ||
      (rc = dalloc(s, L, &s->d.disp, kDispSlots)) || (rc = dalloc(s, L, &s->d.nbRef, cap)) ||
      (rc = dalloc(s, L, &s->d.predLam, cap)) || (rc = dalloc(s, L, &s->d.velRho, cap)) ||
      (rc = dalloc(s, L, &s->d.normRho, cap)))
    return rc;
  s->d.cap = (uint32_t)cap;
  if ((rc = alloc_cells(s))) return rc;
  if ((rc = upload_boundary(s))) return rc;
  // bodies (src/sim.js:129-161)
  const int nBodies = (int)sc.bodyDensity.size();
  s->nBodies = nBodies;
  s->nBodyParts = sc.nBody;
  const int nb1 = std::max(1, nBodies);
  if ((rc = dalloc(s, L, &s->d.bodyAccum, (size_t)nb1 * 4)) || (rc = dalloc(s, L, &s->d.bodyCov, (size_t)nb1 * 9)) ||
      (rc = dalloc(s, L, &s->d.bodyCentre, nb1)) || (rc = dalloc(s, L, &s->d.bodyRef, nb1)) ||
      (rc = dalloc(s, L, &s->d.bodyRot, (size_t)nb1 * 3)) || (rc = dalloc(s, L, &s->d.bodyInfo, nb1)) ||
      (rc = dalloc(s, L, &s->d.bodyStart, (size_t)nb1 + 1)) || (rc = dalloc(s, L, &s->d.bodyFill, nb1)) ||
      (rc = dalloc(s, L, &s->d.bodyList, (size_t)std::max(1, sc.nBody))))
    return rc;
  std::vector<int> counts(nBodies, 0);
  for (int i = 0; i < n; i++) {
    const uint32_t b = sc.phase[(size_t)i * 4];
    if (b >= 1 && (int)b <= nBodies) counts[b - 1]++;
  }
  s->bodyStartHost.assign(nb1 + 1, 0u);
  for (int b = 0; b < nBodies; b++) s->bodyStartHost[b + 1] = s->bodyStartHost[b] + counts[b];
  if (nBodies) {
    std::vector<float> info((size_t)nBodies * 4, 0.0f), centre((size_t)nBodies * 4, 0.0f),
        rot((size_t)nBodies * 12, 0.0f);
    for (int i = 0; i < nBodies; i++) {
      info[i * 4] = (float)(1 / std::max(1e-6, sc.bodyDensity[i]));
      for (int k = 0; k < 3; k++) centre[i * 4 + k] = (float)sc.bodyCentre[i * 3 + k];
      for (int r = 0; r < 3; r++) rot[i * 12 + r * 4 + r] = 1.0f;
    }
    CUDA_TRY(s, cudaMemcpyAsync(s->d.bodyInfo, info.data(), info.size() * 4, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.bodyCentre, centre.data(), centre.size() * 4, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.bodyRef, centre.data(), centre.size() * 4, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.bodyRot, rot.data(), rot.size() * 4, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.bodyStart, s->bodyStartHost.data(), s->bodyStartHost.size() * 4,
                                cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  }
  // fixed-point scales (src/sim.js:163-171)
  double maxCount = 1, maxRest = 1e-3;
  for (int b = 0; b < nBodies; b++) maxCount = std::max(maxCount, (double)counts[b]);
  for (int i = 0; i < n; i++) {
    const double r = std::hypot((double)sc.rest[(size_t)i * 4], (double)sc.rest[(size_t)i * 4 + 1],
                                (double)sc.rest[(size_t)i * 4 + 2]);
    if (r > maxRest) maxRest = r;
  }
  const double extent = std::max(p.box[0], std::max(p.box[1], p.box[2]));
  s->bodyScale = 1e9 / (extent * maxCount);
  s->covScale = 1e9 / (extent * maxRest * maxCount);
  // pinned readback: 8 stats words, error word, pose (16 floats per body)
  const size_t want = 64 + (size_t)nb1 * 16 * sizeof(float);
  if (s->pinnedBytes < want) {
    if (s->readEvent) cudaEventSynchronize(s->readEvent);
    if (s->pinned) cudaFreeHost(s->pinned);
    s->pinned = nullptr;
    CUDA_TRY(s, cudaHostAlloc((void**)&s->pinned, want, cudaHostAllocDefault));
    s->pinnedBytes = want;
  }
  s->readPending = false;
  s->readStale = false;
  s->poseValid = false;
  s->stats = p4a_stats{};
  s->stats.avg_rho = 1;
  s->stats.max_rho = 1;
  s->pose.assign((size_t)nBodies * 12, 0.0f);
  for (int b = 0; b < nBodies; b++) {
    for (int k = 0; k < 3; k++) s->pose[b * 12 + k] = (float)sc.bodyCentre[b * 3 + k];
    for (int r = 0; r < 3; r++) s->pose[b * 12 + 3 + r * 3 + r] = 1.0f;
  }
  // initial particle state into parity A (src/sim.js:191-195)
  const size_t nb = (size_t)n * 16;
  if (n > 0) {
    CUDA_TRY(s, cudaMemcpyAsync(s->d.pos[0], sc.pos.data(), nb, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.vel[0], sc.vel.data(), nb, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.pred[0], sc.pos.data(), nb, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.body[0], sc.phase.data(), nb, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(s->d.rest[0], sc.rest.data(), nb, cudaMemcpyHostToDevice, s->stream));
  }
  s->n = n;
  s->parity = 0;
  s->predParity = 0;
  s->heldBody = -1;
  s->heldTarget[0] = s->heldTarget[1] = s->heldTarget[2] = 0;
  s->heldRate = 10;
  s->heldLimit = 4;
  // primeGrid (src/sim.js:223-253)
  pack_params(s, 0);
  grid_pass(s, s->parity);
  mark(s, PH_END);
  s->parity ^= 1;
  s->predParity = s->parity;
  pack_params(s, 1.0 / 240);
  CUDA_TRY(s, cudaGetLastError());
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  s->ready = true;
  return P4A_OK;
}

void copy_params(p4a_sim* s, const p4a_params* p) {
  s->params = *p;
  s->specs.assign(p->bodies, p->bodies + (p->bodies ? p->n_bodies : 0));
  s->params.bodies = s->specs.empty() ? nullptr : s->specs.data();
  s->params.n_bodies = (int32_t)s->specs.size();
}

int check_error_word(p4a_sim* s) {
  const uint32_t w = s->pinned ? s->pinned[8] : 0u;
  if (w & ERR_SCAN_TIMEOUT)
    return fail(s, P4A_ERR_TIMEOUT, "cell scan: a bounded wait on a predecessor tile gave up");
  return P4A_OK;
}

// Queues the copy of statsOut, the error word and the body pose into pinned memory
// behind the work already on the stream (src/sim.js:604-614).
int issue_readback(p4a_sim* s) {
  cudaStream_t st = s->stream;
  DevScene& d = s->d;
  CUDA_TRY(s, cudaMemcpyAsync(s->pinned, d.statsOut, 32, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(s, cudaMemcpyAsync(s->pinned + 8, d.errorWord, 4, cudaMemcpyDeviceToHost, st));
  if (s->nBodies) {
    float* f = (float*)(s->pinned + 16);
    CUDA_TRY(s, cudaMemcpyAsync(f, d.bodyCentre, (size_t)s->nBodies * 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(s, cudaMemcpyAsync(f + (size_t)s->nBodies * 4, d.bodyRot, (size_t)s->nBodies * 48,
                                cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(s, cudaEventRecord(s->readEvent, st));
  s->readPending = true;
  s->readStale = false;
  return P4A_OK;
}

// Completes an outstanding readback if it finished (or waits for it).
int poll_readback(p4a_sim* s, bool wait) {
  if (!s->readPending) return P4A_OK;
  if (wait) {
    CUDA_TRY(s, cudaEventSynchronize(s->readEvent));
  } else {
    const cudaError_t q = cudaEventQuery(s->readEvent);
    if (q == cudaErrorNotReady) return P4A_OK;
    if (q != cudaSuccess) return fail(s, P4A_ERR_CUDA, "readback: %s", cudaGetErrorString(q));
  }
  s->readPending = false;
  const uint32_t* v = s->pinned;
  const double SCALE = 1024;
  s->stats.avg_rho = v[0] / SCALE / std::max(1, s->n);
  s->stats.max_rho = v[1] / SCALE;
  s->stats.max_speed = v[2] / SCALE;
  s->stats.ke = v[3] / SCALE;
  for (int k = 0; k < 4; k++) s->stats.raw[k] = v[k];
  s->stats.valid = 1;
  if (s->nBodies) {
    const float* f = (const float*)(s->pinned + 16);
    for (int b = 0; b < s->nBodies; b++) {
      for (int k = 0; k < 3; k++) s->pose[b * 12 + k] = f[b * 4 + k];
      const float* rows = f + (size_t)s->nBodies * 4 + (size_t)b * 12;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) s->pose[b * 12 + 3 + r * 3 + c] = rows[r * 4 + c];
    }
    s->poseValid = true;
  }
  return check_error_word(s);
}

int buffer_ptr(p4a_sim* s, int32_t id, int32_t which, void** p, size_t* bytes) {
  const int w = which < 0 ? s->parity : (which & 1);
  const size_t cap = (size_t)s->cap;
  const size_t nb1 = (size_t)std::max(1, s->nBodies);
  const size_t nbd = (size_t)std::max(1, s->nBoundary);
  const size_t cells = (size_t)s->nCells + 2;
  switch (id) {
    case P4A_BUF_POS: *p = s->d.pos[w]; *bytes = cap * 16; break;
    case P4A_BUF_VEL: *p = s->d.vel[w]; *bytes = cap * 16; break;
    case P4A_BUF_PRED: *p = s->d.pred[w]; *bytes = cap * 16; break;
    case P4A_BUF_BODY: *p = s->d.body[w]; *bytes = cap * 16; break;
    case P4A_BUF_REST: *p = s->d.rest[w]; *bytes = cap * 16; break;
    case P4A_BUF_DENSITY: *p = s->d.density; *bytes = cap * 4; break;
    case P4A_BUF_LAMBDA: *p = s->d.lambda; *bytes = cap * 4; break;
    case P4A_BUF_CORR: *p = s->d.corr; *bytes = cap * 16; break;
    case P4A_BUF_NORMAL: *p = s->d.normal; *bytes = cap * 16; break;
    case P4A_BUF_CELL_START: *p = s->d.cellStart; *bytes = cells * 4; break;
    case P4A_BUF_BPOS: *p = s->d.bpos; *bytes = nbd * 16; break;
    case P4A_BUF_BPSI: *p = s->d.bpsi; *bytes = nbd * 4; break;
    case P4A_BUF_BCELL_START: *p = s->d.bcellStart; *bytes = cells * 4; break;
    case P4A_BUF_BODY_CENTRE: *p = s->d.bodyCentre; *bytes = nb1 * 16; break;
    case P4A_BUF_BODY_REF: *p = s->d.bodyRef; *bytes = nb1 * 16; break;
    case P4A_BUF_BODY_ROT: *p = s->d.bodyRot; *bytes = nb1 * 48; break;
    case P4A_BUF_BODY_INFO: *p = s->d.bodyInfo; *bytes = nb1 * 16; break;
    case P4A_BUF_STATS_OUT: *p = s->d.statsOut; *bytes = 32; break;
    case P4A_BUF_SMOOTH_POS: *p = s->smoothPos; *bytes = s->smoothPos ? (size_t)s->n * 16 : 0; break;
    case P4A_BUF_ANISO_G: *p = s->anisoG; *bytes = s->anisoG ? (size_t)s->n * 32 : 0; break;
    case P4A_BUF_MESH_FIELD:
    case P4A_BUF_MESH_NFIELD: {
      const size_t nv = (size_t)s->meshDim[0] * s->meshDim[1] * s->meshDim[2];
      *p = s->meshField[id == P4A_BUF_MESH_FIELD ? s->fieldSlot : s->nfieldSlot];
      *bytes = *p ? nv * 4 : 0;
      break;
    }
    case P4A_BUF_MESH_VERTS:
      *p = s->meshVerts;
      *bytes = s->meshVerts ? (size_t)std::min<int64_t>(s->meshTris, (int64_t)s->meshTriCap) * 24 : 0;
      break;
    default: return fail(s, P4A_ERR_ARG, "unknown buffer id %d", id);
  }
  return P4A_OK;
}

}  // namespace

extern "C" {

int p4a_abi_version(void) { return P4A_ABI_VERSION; }

const char* p4a_status_string(int status) {
  switch (status) {
    case P4A_OK: return "ok";
    case P4A_ERR_ARG: return "invalid argument";
    case P4A_ERR_OOM: return "out of memory";
    case P4A_ERR_CUDA: return "CUDA error";
    case P4A_ERR_TIMEOUT: return "device wait timed out";
    case P4A_ERR_CAPACITY: return "capacity exceeded";
    case P4A_ERR_STATE: return "invalid state";
    case P4A_ERR_NODEV: return "no usable CUDA device";
    default: return "unknown status";
  }
}

int p4a_default_params(const char* preset, p4a_params* out) {
  static const p4a_body_spec kDefaultBodies[3] = {
      {P4A_SHAPE_SPHERE, 0.5, 0.75}, {P4A_SHAPE_TORUS, 0.8, 0.75}, {P4A_SHAPE_BOX, 1.4, 0.75}};
  if (!out) return P4A_ERR_ARG;
  p4a_params p{};
  p.spacing = 0.02;
  p.rest_density = 1000;
  p.gravity = 9.81;
  p.substeps = 4;
  p.iterations = 4;
  p.cfm_epsilon_rel = 0.01;
  p.s_corr_k = 0.1;
  p.s_corr_dq = 0.3;
  p.xsph_c = 0.05;
  p.omega = 1.0;
  p.sor_average = 0;
  p.surface_tension_k = 0;
  p.target_particle_count = 60000;
  p.box[0] = 1.5; p.box[1] = 1.5; p.box[2] = 1.0;
  p.n_bodies = 3;
  p.bodies = kDefaultBodies;
  p.body_size = 0;
  p.no_boundary = 0;
  p.pour = 1;
  p.cfm_epsilon_abs = 0;
  if (preset && std::strcmp(preset, "extreme") == 0) {  // src/scene.js:7-8
    p.target_particle_count = 1000000;
    p.box[0] = p.box[1] = p.box[2] = 3.0;
  }
  *out = p;
  return P4A_OK;
}

int p4a_device_check(int device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return P4A_ERR_NODEV;
  if (device < 0 || device >= count) return P4A_ERR_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return P4A_ERR_NODEV;
  return prop.major == 10 && prop.minor == 0 ? P4A_OK : P4A_ERR_NODEV;
}

int p4a_create(int device, p4a_sim** out) {
  if (!out) return P4A_ERR_ARG;
  *out = nullptr;
  const int chk = p4a_device_check(device);
  if (chk != P4A_OK) return chk;
  p4a_sim* s = new p4a_sim();
  s->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->readEvent, cudaEventDisableTiming) != cudaSuccess) {
    delete s;
    return P4A_ERR_CUDA;
  }
  s->ownStream = true;
  *out = s;
  return P4A_OK;
}

int p4a_destroy(p4a_sim* s) {
  if (!s) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  drain_reads(s);
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_list(s->sceneAllocs);
  free_list(s->cellAllocs);
  free_list(s->boundaryAllocs);
  if (s->smoothPos) cudaFree(s->smoothPos);
  if (s->anisoG) cudaFree(s->anisoG);
  for (float* f : s->meshField)
    if (f) cudaFree(f);
  if (s->meshCounts) cudaFree(s->meshCounts);
  if (s->meshOffsets) cudaFree(s->meshOffsets);
  if (s->meshScan) cudaFree(s->meshScan);
  if (s->meshTicket) cudaFree(s->meshTicket);
  if (s->meshVerts) cudaFree(s->meshVerts);
  free_list(s->ssfrAllocs);
  if (s->ssfrBodies) cudaFree(s->ssfrBodies);
  if (s->rayImage) cudaFree(s->rayImage);
  if (s->raySurf) cudaFree(s->raySurf);
  if (s->envCube) cudaFree(s->envCube);
  if (s->pinned) cudaFreeHost(s->pinned);
  if (s->readEvent) cudaEventDestroy(s->readEvent);
  for (cudaEvent_t e : s->evPool) cudaEventDestroy(e);
  if (s->copyReady) cudaEventDestroy(s->copyReady);
  if (s->copyDone) cudaEventDestroy(s->copyDone);
  if (s->copyStream) cudaStreamDestroy(s->copyStream);
  if (s->ownStream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return P4A_OK;
}

const char* p4a_last_error(const p4a_sim* s) { return s ? s->err.c_str() : "null handle"; }

int p4a_set_stream(p4a_sim* s, void* stream) {
  if (!s) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  int rc = drain_reads(s);
  if (rc) return rc;
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  if (stream) {
    if (s->ownStream) cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->ownStream = false;
  } else if (!s->ownStream) {
    CUDA_TRY(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->ownStream = true;
  }
  return P4A_OK;
}

int p4a_synchronize(p4a_sim* s) {
  if (!s) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  const int rc = drain_reads(s);
  if (rc) return rc;
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return poll_readback(s, true);
}

int p4a_reset(p4a_sim* s, const p4a_params* params) {
  if (!s || !params || !(params->spacing > 0) || params->n_bodies < 0 ||
      (params->n_bodies > 0 && !params->bodies))
    return fail(s, P4A_ERR_ARG, "p4a_reset: invalid params");
  cudaSetDevice(s->device);
  copy_params(s, params);
  build_scene(s->params, s->sc);
  s->pourBudget = params->pour ? s->sc.nFluid : 0;
  return reset_common(s);
}

int p4a_reset_scene(p4a_sim* s, const p4a_params* params, const p4a_scene_desc* sd) {
  if (!s || !params || !sd || sd->n < 0 || (sd->n > 0 && !sd->pos) || !(params->spacing > 0) ||
      sd->n_bodies < 0 || (sd->n_bodies > 0 && (!sd->body_density || !sd->body_centre)))
    return fail(s, P4A_ERR_ARG, "p4a_reset_scene: invalid scene");
  cudaSetDevice(s->device);
  copy_params(s, params);
  HostScene& sc = s->sc;
  sc = HostScene();
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
    const uint32_t b = sc.phase[i * 4];
    if (b == 0) nFluid++;
    else if ((int)b > sd->n_bodies) return fail(s, P4A_ERR_ARG, "particle %zu: body id %u > n_bodies", i, b);
  }
  sc.nFluid = nFluid;
  sc.nBody = sd->n - nFluid;
  sc.bodyDensity.assign(sd->body_density, sd->body_density + sd->n_bodies);
  sc.bodyCentre.assign(sd->body_centre, sd->body_centre + 3 * (size_t)sd->n_bodies);
  sc.mass = sd->mass;
  sc.denomRest = sd->denom_rest;
  const bool doMass = !(sd->mass > 0), doDenom = !(sd->denom_rest > 0);
  if (doMass || doDenom) calibrate_scene(s->params, sc, doMass, doDenom);
  s->pourBudget = std::max(0, sd->pour_budget);
  return reset_common(s);
}

int p4a_step(p4a_sim* s, double frameDt, int32_t* substeps_out) {
  if (!s) return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "p4a_step before p4a_reset");
  cudaSetDevice(s->device);
  after_reads(s, kAllBuffers);
  const p4a_params& p = s->params;
  // time bank (src/sim.js:418-429)
  const int base = std::max(1, p.substeps);
  const double dtTarget = (1.0 / 60) / base;
  s->timeBank = s->timeBank + frameDt;
  double subD = std::floor(s->timeBank / dtTarget + 1e-4);
  const double workCap = base * 8;
  if (subD > workCap) {
    subD = workCap;
    s->timeBank = 0;
  } else {
    s->timeBank -= subD * dtTarget;
  }
  const int sub = (int)subD;
  s->lastSubsteps = sub;
  s->lastAdvanced = subD * dtTarget;
  if (substeps_out) *substeps_out = sub;
  if (sub < 1) {
    s->lastAdvanced = 0;
    return P4A_OK;
  }
  const double dt = dtTarget;
  {
    const int rc = poll_readback(s, false);  // a finished readback frees the slot
    if (rc) return rc;
  }
  pack_params(s, dt);
  const SimParams& P = s->P;
  DevScene& d = s->d;
  cudaStream_t st = s->stream;
  const bool bodies = s->nBodyParts > 0 && s->nBodies > 0;
  const bool dragging = s->heldBody >= 1 && s->nBodyParts > 0;
  const float blend = (float)(1 - std::exp(-std::max(dt, 0.0) / 0.02));
  const float goal[3] = {(float)s->heldTarget[0], (float)s->heldTarget[1], (float)s->heldTarget[2]};
  const int iters = std::max(1, p.iterations);
  const bool tension = p.surface_tension_k > 0;
  for (int step = 0; step < sub; step++) {
    const int par = s->parity, q = par ^ 1;
    if (dragging) {
      const uint32_t hb = (uint32_t)s->heldBody;
      mark(s, PH_DRAG);
      launch_body_drag(d, d.vel[par], d.body[par], hb, s->bodyStartHost[hb] - s->bodyStartHost[hb - 1],
                       s->bodyStartHost[hb - 1], goal, (float)s->heldRate, blend, (float)s->heldLimit, st);
    }
    s->P.subs = (uint32_t)sub;
    grid_pass(s, par);  // sets P.parity = par: the passes below read parity par ^ 1
    s->parity = q;
    s->predParity = q;
    if (bodies) {
      mark(s, PH_BODY_SEED);
      launch_body_seed(P, d, st);
    }
    for (int it = 0; it < iters; it++) {
      mark(s, PH_LAMBDA);
      launch_lambda(P, d, it, st);
      mark(s, PH_DELTA);
      launch_delta(P, d, it, st);
      if (bodies) {
        mark(s, PH_BODY_MATCH);
        launch_body_match(P, d, it, st);
      }
    }
    if (step == sub - 1) {
      mark(s, PH_STATS_CLEAR);
      CUDA_TRY(s, cudaMemsetAsync(d.statsOut, 0, 32, st));
    }
    if (tension) {
      mark(s, PH_XSPH_NORMALS);
      launch_xsph_normals(P, d, st);
      mark(s, PH_TENSION_FINALIZE);
      launch_tension_finalize(P, d, step, st);
    } else {
      mark(s, PH_XSPH_FINALIZE);
      launch_xsph_finalize(P, d, step, st);
    }
    s->simTime += dt;
  }
  if (sub > 0) s->sortedMoves = true;
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  // stats and pose readback (src/sim.js:598-655), at most one in flight
  if (!s->readPending) return issue_readback(s);
  s->readStale = true;
  return P4A_OK;
}

int p4a_append_fluid(p4a_sim* s, const float* pos3, const float* vel3, int32_t count, int32_t* added) {
  if (!s || count < 0 || (count > 0 && (!pos3 || !vel3))) return fail(s, P4A_ERR_ARG, "appendFluid: bad arguments");
  if (!s->ready) return fail(s, P4A_ERR_STATE, "appendFluid before reset");
  cudaSetDevice(s->device);
  after_reads(s, kAllBuffers);
  s->sortedMoves = false;
  const int room = std::max(0, s->cap - s->n);
  const int c = std::min(count, room);
  if (added) *added = std::max(0, c);
  if (c <= 0) return P4A_OK;
  std::vector<float> p4((size_t)c * 4), v4((size_t)c * 4, 0.0f), rho((size_t)c, (float)s->params.rest_density);
  for (int i = 0; i < c; i++) {
    for (int k = 0; k < 3; k++) {
      p4[i * 4 + k] = pos3[i * 3 + k];
      v4[i * 4 + k] = vel3[i * 3 + k];
    }
    p4[i * 4 + 3] = 1.0f;
  }
  const size_t o4 = (size_t)s->n, bytes4 = (size_t)c * 16, bytes1 = (size_t)c * 4;
  cudaStream_t st = s->stream;
  DevScene& d = s->d;
  CUDA_TRY(s, cudaMemcpyAsync(d.pos[s->parity] + o4, p4.data(), bytes4, cudaMemcpyHostToDevice, st));
  CUDA_TRY(s, cudaMemcpyAsync(d.vel[s->parity] + o4, v4.data(), bytes4, cudaMemcpyHostToDevice, st));
  CUDA_TRY(s, cudaMemcpyAsync(d.pred[s->predParity] + o4, p4.data(), bytes4, cudaMemcpyHostToDevice, st));
  CUDA_TRY(s, cudaMemcpyAsync(d.density + o4, rho.data(), bytes1, cudaMemcpyHostToDevice, st));
  CUDA_TRY(s, cudaMemsetAsync(d.lambda + o4, 0, bytes1, st));
  CUDA_TRY(s, cudaMemsetAsync(d.corr + o4, 0, bytes4, st));
  CUDA_TRY(s, cudaMemsetAsync(d.normal + o4, 0, bytes4, st));
  for (int t = 0; t < 2; t++) {
    CUDA_TRY(s, cudaMemsetAsync(d.body[t] + o4, 0, bytes4, st));
    CUDA_TRY(s, cudaMemsetAsync(d.rest[t] + o4, 0, bytes4, st));
  }
  CUDA_TRY(s, cudaStreamSynchronize(st));  // host staging vectors go out of scope
  s->n += c;
  return P4A_OK;
}

int p4a_hose_emit(p4a_sim* s, const p4a_hose* hose, int64_t emission, int32_t* added) {
  if (!s || !hose || emission < 0 || hose->per_step < 0 || !(hose->spacing > 0) || !(hose->jitter >= 0))
    return fail(s, P4A_ERR_ARG, "hose_emit: bad arguments");
  if (!s->ready) return fail(s, P4A_ERR_STATE, "hose_emit before reset");
  const int room = std::max(0, s->cap - s->n);
  const int want = hose->count < 0 ? hose->per_step : std::min(hose->count, hose->per_step);
  const int c = std::min(want, room);
  if (added) *added = std::max(0, c);
  if (c <= 0) return P4A_OK;
  cudaSetDevice(s->device);
  after_reads(s, kAllBuffers);
  s->sortedMoves = false;
  HoseEmit H{};
  uint32_t k = 1;
  while ((int64_t)k * k < hose->per_step) k++;
  for (int a = 0; a < 3; a++) H.nozzle[a] = hose->nozzle[a];
  H.spacing = hose->spacing;
  H.centre = (float)(k - 1) * 0.5f;
  H.jitter = hose->jitter;
  H.speed = hose->speed;
  H.rho0 = (float)s->params.rest_density;
  H.k = k;
  H.count = (uint32_t)c;
  H.first = (uint32_t)s->n;
  H.seed = hose->seed;
  H.emission = (uint64_t)emission;
  mark(s, PH_HOSE);
  launch_hose_emit(H, s->d, s->parity, s->predParity, s->stream);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  s->n += c;
  return P4A_OK;
}

int p4a_apply_ray_impulse(p4a_sim* s, const double origin[3], const double dir[3], const double impulse[3],
                          double radius, double speedLimit) {
  if (!s || !origin || !dir || !impulse) return fail(s, P4A_ERR_ARG, "applyRayImpulse: null argument");
  if (!s->ready) return fail(s, P4A_ERR_STATE, "applyRayImpulse before reset");
  if (!s->n || radius <= 0) return P4A_OK;
  const double len = std::hypot(impulse[0], impulse[1], impulse[2]);
  if (len <= 0) return P4A_OK;
  double dl = std::hypot(dir[0], dir[1], dir[2]);
  if (!(dl != 0)) dl = 1;
  cudaSetDevice(s->device);
  after_reads(s, kAllBuffers);
  const float o[3] = {(float)origin[0], (float)origin[1], (float)origin[2]};
  const float dr[3] = {(float)(dir[0] / dl), (float)(dir[1] / dl), (float)(dir[2] / dl)};
  const float im[3] = {(float)impulse[0], (float)impulse[1], (float)impulse[2]};
  mark(s, PH_IMPULSE);
  launch_impulse((uint32_t)s->n, s->d.pos[s->parity], s->d.vel[s->parity], o, dr, im, (float)radius,
                 (float)speedLimit, s->stream);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  return P4A_OK;
}

int p4a_hold_body(p4a_sim* s, int32_t body1, const double target[3], double rate, double limit) {
  if (!s || !target) return fail(s, P4A_ERR_ARG, "holdBody: null argument");
  s->heldBody = (body1 >= 1 && body1 <= s->nBodies) ? body1 : -1;
  for (int k = 0; k < 3; k++) s->heldTarget[k] = target[k];
  s->heldRate = rate;
  s->heldLimit = limit;
  return P4A_OK;
}

int p4a_release_body(p4a_sim* s) {
  if (!s) return P4A_ERR_ARG;
  s->heldBody = -1;
  return P4A_OK;
}

int p4a_resize_box(p4a_sim* s, const double newBox[3]) {
  if (!s || !newBox) return fail(s, P4A_ERR_ARG, "resizeBox: null argument");
  if (!s->ready) return fail(s, P4A_ERR_STATE, "resizeBox before reset");
  cudaSetDevice(s->device);
  {
    const int drc = drain_reads(s);  // the grid buffers may be reallocated
    if (drc) return drc;
  }
  s->sortedMoves = false;
  p4a_params& p = s->params;
  const double oldBox[3] = {p.box[0], p.box[1], p.box[2]};
  bool moved = false;
  for (int a = 0; a < 3; a++)
    if (std::fabs(newBox[a] - oldBox[a]) > 1e-9) moved = true;
  if (!moved) return P4A_OK;
  for (int a = 0; a < 3; a++) p.box[a] = newBox[a];
  for (int k = 0; k < 3; k++) s->gridDim[k] = (int)std::max(1.0, std::floor(newBox[k] / s->h));
  const int cells = s->gridDim[0] * s->gridDim[1] * s->gridDim[2];
  const bool changed = cells != s->nCells;
  s->nCells = cells;
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  int rc;
  if (changed && (rc = alloc_cells(s))) return rc;
  if ((rc = upload_boundary(s))) return rc;
  s->gen++;
  const float halfD = (float)(0.5 * p.spacing);
  const float oldS[3] = {(float)oldBox[0], (float)oldBox[1], (float)oldBox[2]};
  const float newS[3] = {(float)newBox[0], (float)newBox[1], (float)newBox[2]};
  const float cMin[3] = {halfD, halfD, halfD};
  const float cMax[3] = {(float)(newBox[0] - 0.5 * p.spacing), (float)(newBox[1] - 0.5 * p.spacing),
                         (float)(newBox[2] - 0.5 * p.spacing)};
  mark(s, PH_RESIZE);
  launch_resize((uint32_t)s->n, s->d.pos[s->parity], oldS, newS, cMin, cMax, s->stream);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  return P4A_OK;
}

int p4a_get_info(const p4a_sim* s, p4a_info* o) {
  if (!s || !o) return P4A_ERR_ARG;
  *o = p4a_info{};
  o->n = s->n; o->n_fluid = s->sc.nFluid; o->n_body_parts = s->nBodyParts; o->n_bodies = s->nBodies;
  o->n_boundary = s->nBoundary; o->cap = s->cap; o->pour_budget = s->pourBudget;
  for (int k = 0; k < 3; k++) o->grid_dim[k] = s->gridDim[k];
  o->n_cells = s->nCells; o->parity = s->parity; o->pred_parity = s->predParity; o->gen = s->gen;
  o->last_substeps = s->lastSubsteps; o->h = s->h; o->mass = s->sc.mass; o->denom_rest = s->sc.denomRest;
  o->sim_time = s->simTime; o->last_advanced = s->lastAdvanced; o->time_bank = s->timeBank;
  o->body_scale = s->bodyScale; o->cov_scale = s->covScale; o->held_body = s->heldBody;
  o->aniso_gen = s->anisoGen;
  return P4A_OK;
}

int p4a_buffer(p4a_sim* s, int32_t id, int32_t which, void** dptr, size_t* bytes) {
  if (!s || !dptr) return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "buffer query before reset");
  size_t b = 0;
  const int rc = buffer_ptr(s, id, which, dptr, &b);
  if (bytes) *bytes = b;
  return rc;
}

int p4a_read(p4a_sim* s, int32_t id, int32_t which, void* host, size_t offset, size_t bytes) {
  if (!s || (!host && bytes)) return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "read before reset");
  void* p = nullptr;
  size_t total = 0;
  int rc = buffer_ptr(s, id, which, &p, &total);
  if (rc) return rc;
  if (offset > total || bytes > total - offset)
    return fail(s, P4A_ERR_ARG, "read of %zu bytes at %zu beyond buffer size %zu", bytes, offset, total);
  if (!bytes) return P4A_OK;
  cudaSetDevice(s->device);
  CUDA_TRY(s, cudaMemcpyAsync(host, (const char*)p + offset, bytes, cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return P4A_OK;
}

int p4a_read_async(p4a_sim* s, int32_t id, int32_t which, void* host, size_t offset, size_t bytes) {
  if (!s || (!host && bytes)) return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "read before reset");
  void* p = nullptr;
  size_t total = 0;
  int rc = buffer_ptr(s, id, which, &p, &total);
  if (rc) return rc;
  if (offset > total || bytes > total - offset)
    return fail(s, P4A_ERR_ARG, "read of %zu bytes at %zu beyond buffer size %zu", bytes, offset, total);
  if (!bytes) return P4A_OK;
  cudaSetDevice(s->device);
  if (!s->copyStream) {
    CUDA_TRY(s, cudaStreamCreateWithFlags(&s->copyStream, cudaStreamNonBlocking));
    CUDA_TRY(s, cudaEventCreateWithFlags(&s->copyReady, cudaEventDisableTiming));
    CUDA_TRY(s, cudaEventCreateWithFlags(&s->copyDone, cudaEventDisableTiming));
  }
  CUDA_TRY(s, cudaEventRecord(s->copyReady, s->stream));
  CUDA_TRY(s, cudaStreamWaitEvent(s->copyStream, s->copyReady, 0));
  CUDA_TRY(s, cudaMemcpyAsync(host, (const char*)p + offset, bytes, cudaMemcpyDeviceToHost, s->copyStream));
  CUDA_TRY(s, cudaEventRecord(s->copyDone, s->copyStream));
  s->copyInFlight |= buf_bit(id);
  s->copyHost = true;
  return P4A_OK;
}

int p4a_read_wait(p4a_sim* s) {
  if (!s) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  return drain_reads(s);
}

int p4a_write(p4a_sim* s, int32_t id, int32_t which, const void* host, size_t offset, size_t bytes) {
  if (!s || (!host && bytes)) return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "write before reset");
  void* p = nullptr;
  size_t total = 0;
  int rc = buffer_ptr(s, id, which, &p, &total);
  if (rc) return rc;
  if (offset > total || bytes > total - offset)
    return fail(s, P4A_ERR_ARG, "write of %zu bytes at %zu beyond buffer size %zu", bytes, offset, total);
  if (!bytes) return P4A_OK;
  cudaSetDevice(s->device);
  after_reads(s, buf_bit(id));
  s->sortedMoves = false;
  CUDA_TRY(s, cudaMemcpyAsync((char*)p + offset, host, bytes, cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return P4A_OK;
}

// wait = 1: the values of the last step, read back now if its own readback was
// skipped because an earlier one was still in flight.
static int refresh_readback(p4a_sim* s, bool wait) {
  int rc = poll_readback(s, wait);
  if (rc || !wait || !s->readStale || !s->ready) return rc;
  if ((rc = issue_readback(s))) return rc;
  return poll_readback(s, true);
}

int p4a_get_stats(p4a_sim* s, int32_t wait, p4a_stats* out) {
  if (!s || !out) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  const int rc = refresh_readback(s, wait != 0);
  *out = s->stats;
  return rc;
}

int p4a_body_pose(p4a_sim* s, int32_t wait, float* centre3, float* rot9, int32_t maxBodies) {
  if (!s) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  const int rc = refresh_readback(s, wait != 0);
  const int nb = std::min(maxBodies, s->nBodies);
  for (int b = 0; b < nb; b++) {
    if (centre3)
      for (int k = 0; k < 3; k++) centre3[b * 3 + k] = s->pose[b * 12 + k];
    if (rot9)  // column-major, as Sim.bodyPose (src/sim.js:648-650)
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) rot9[b * 9 + c * 3 + r] = s->pose[b * 12 + 3 + r * 3 + c];
  }
  return rc;
}

int p4a_default_aniso_params(p4a_aniso_params* a) {
  if (!a) return P4A_ERR_ARG;
  a->ratio = 4.0;
  a->ks = 1.0;
  a->stretch = 2.0;
  a->lonely = 1.0;
  a->min_neighbours = 25;
  a->lambda = 0.9;
  a->radius_scale = 2.0;
  a->min_extent = 0.0;
  return P4A_OK;
}

int p4a_aniso(p4a_sim* s, const p4a_aniso_params* ap) {
  if (!s || !ap) return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "aniso before reset");
  const int n = s->n;
  if (n <= 0) return P4A_OK;
  cudaSetDevice(s->device);
  after_reads(s, buf_bit(P4A_BUF_SMOOTH_POS) | buf_bit(P4A_BUF_ANISO_G));
  if ((size_t)n > s->anisoCap) {  // src/mesh.js:210-220
    const int drc = drain_reads(s);
    if (drc) return drc;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->smoothPos) cudaFree(s->smoothPos);
    if (s->anisoG) cudaFree(s->anisoG);
    s->smoothPos = nullptr;
    s->anisoG = nullptr;
    s->anisoCap = 0;
    CUDA_TRY(s, cudaMalloc((void**)&s->smoothPos, (size_t)n * 16));
    CUDA_TRY(s, cudaMalloc((void**)&s->anisoG, (size_t)n * 32));
    s->anisoCap = (size_t)n;
    s->anisoGen++;
  }
  const double support = s->h;
  const double radius = ap->radius_scale * support;
  const double sigmaBulk = 0.15 * radius * radius;
  AnisoParams A{};
  A.count = (uint32_t)n;
  A.lambda = (float)ap->lambda;
  A.invSupport = (float)(1 / support);
  A.support = (float)support;
  A.boxMin[0] = A.boxMin[1] = A.boxMin[2] = 0.0f;
  A.radius = (float)radius;
  for (int k = 0; k < 3; k++) A.gridDim[k] = s->gridDim[k];
  A.cells = (int32_t)std::ceil(ap->radius_scale);
  A.kr = (float)ap->ratio;
  A.kn = (float)ap->lonely;
  A.ks = (float)(ap->ks / sigmaBulk);
  A.stretch = (float)ap->stretch;
  A.minExtent = (float)ap->min_extent;
  A.neps = ap->min_neighbours;
  // the row trimming needs every particle within the recorded displacements of
  // the position the sort binned it by: true right after a step
  A.disp = s->d.disp;
  const int iters = std::max(1, s->params.iterations);  // as p4a_step runs them
  A.dispCount = s->sortedMoves && iters <= kDispSlots ? iters : 0;
  mark(s, PH_ANISO);
  launch_aniso(A, s->d.pos[s->parity], s->d.cellStart, s->smoothPos, s->anisoG, s->stream);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  return P4A_OK;
}

int p4a_default_mesh_params(p4a_mesh_params* m) {
  if (!m) return P4A_ERR_ARG;
  *m = p4a_mesh_params{};
  m->resolution = 128;  // src/main.js:320
  m->iso = 0.4;         // src/main.js:321
  m->field_passes = 0;  // src/main.js:323
  m->normal_passes = 2; // src/main.js:324
  m->max_triangles = 3000000;  // src/mesh.js:17
  m->blur_axes = 0;
  return P4A_OK;
}

// SurfaceMesh.configure + generate (src/mesh.js:99-146, 326-352) on the live buffers.
int p4a_mesh(p4a_sim* s, const p4a_mesh_params* mp, int64_t* triangles) {
  if (!s || !mp || mp->resolution < 1 || mp->max_triangles < 0 || mp->field_passes < 0 ||
      mp->normal_passes < 0 || mp->max_triangles > 0x7fffffffLL)
    return P4A_ERR_ARG;
  if (!s->ready) return fail(s, P4A_ERR_STATE, "mesh before reset");
  cudaSetDevice(s->device);
  const double* box = s->params.box;
  const double longest = std::max(box[0], std::max(box[1], box[2]));
  const double voxel = longest / mp->resolution;
  int32_t dim[3];
  for (int k = 0; k < 3; k++) dim[k] = (int32_t)std::ceil(box[k] / voxel) + 2 + 1;
  const double nv = (double)dim[0] * dim[1] * dim[2];
  if (nv > 0x7fffffff || std::max(dim[0], std::max(dim[1], dim[2])) > 8192)
    return fail(s, P4A_ERR_CAPACITY, "mesh grid too large");
  const size_t nVerts = (size_t)nv;
  const size_t nvox = (size_t)(dim[0] - 1) * (dim[1] - 1) * (dim[2] - 1);
  const size_t tris = (size_t)mp->max_triangles;
  after_reads(s, buf_bit(P4A_BUF_MESH_FIELD) | buf_bit(P4A_BUF_MESH_NFIELD) | buf_bit(P4A_BUF_MESH_VERTS));
  if (nVerts > s->meshVertCap || nvox > s->meshVoxCap || tris != s->meshTriCap) {  // src/mesh.js:105-125
    const int drc = drain_reads(s);
    if (drc) return drc;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (nVerts > s->meshVertCap) {
      for (float*& f : s->meshField) {
        if (f) cudaFree(f);
        f = nullptr;
      }
      s->meshVertCap = 0;
      for (float*& f : s->meshField) CUDA_TRY(s, cudaMalloc((void**)&f, nVerts * 4));
      s->meshVertCap = nVerts;
    }
    if (nvox > s->meshVoxCap) {
      if (s->meshCounts) cudaFree(s->meshCounts);
      if (s->meshOffsets) cudaFree(s->meshOffsets);
      if (s->meshScan) cudaFree(s->meshScan);
      s->meshCounts = s->meshOffsets = nullptr;
      s->meshScan = nullptr;
      s->meshVoxCap = 0;
      CUDA_TRY(s, cudaMalloc((void**)&s->meshCounts, nvox * 4));
      CUDA_TRY(s, cudaMemset(s->meshCounts, 0, nvox * 4));
      CUDA_TRY(s, cudaMalloc((void**)&s->meshOffsets, (nvox + 1) * 4));
      CUDA_TRY(s, cudaMalloc((void**)&s->meshScan, (size_t)scan_tiles((int)nvox) * 8));
      CUDA_TRY(s, cudaMemset(s->meshScan, 0, (size_t)scan_tiles((int)nvox) * 8));
      if (!s->meshTicket) {
        CUDA_TRY(s, cudaMalloc((void**)&s->meshTicket, 16));
        CUDA_TRY(s, cudaMemset(s->meshTicket, 0, 16));
      }
      s->meshVoxCap = nvox;
    }
    if (tris != s->meshTriCap) {
      if (s->meshVerts) cudaFree(s->meshVerts);
      s->meshVerts = nullptr;
      s->meshTriCap = 0;
      CUDA_TRY(s, cudaMalloc((void**)&s->meshVerts, std::max<size_t>(1, tris) * 24));
      s->meshTriCap = tris;
    }
    s->meshGen++;
  }
  // uniform (src/mesh.js:137-153)
  const double h = s->h;
  MeshParams M{};
  for (int k = 0; k < 3; k++) {
    M.vertDim[k] = dim[k];
    M.gridOrigin[k] = (float)(0.0 - voxel);
    M.boxMin[k] = 0.0f;
    M.simGridDim[k] = s->gridDim[k];
  }
  M.voxel = (float)voxel;
  M.iso = (float)mp->iso;
  M.invSupport = (float)(1 / h);
  M.support2 = (float)(h * h);
  M.poly6 = (float)(315 / (64 * kPi * std::pow(h, 9)));
  M.mass = (float)s->sc.mass;
  M.rho0 = (float)s->params.rest_density;
  M.maxTris = (uint32_t)tris;
  M.skipBodies = s->nBodyParts > 0 ? 1u : 0u;
  cudaStream_t st = s->stream;
  const int par = s->parity;
  float* buf[3] = {s->meshField[0], s->meshField[1], s->meshField[2]};
  mark(s, PH_MESH_FIELD);
  launch_mesh_field(M, s->d.pos[par], s->d.density, s->d.cellStart, s->d.body[par], (uint32_t)s->n, buf[0], st);
  // blur passes: consecutive passes along one axis run in one launch
  auto blur = [&](int from, int to, int steps) -> int {
    int cur = from;
    for (int k = 0; k < steps;) {
      const int axis = mp->blur_axes ? k % 3 : 0;
      int run = 1;
      while (k + run < steps && (mp->blur_axes ? (k + run) % 3 : 0) == axis) run++;
      const int dst = (k + run == steps) ? to : (cur == 2 ? to : 2);
      const cudaError_t e = launch_mesh_blur(M, buf[cur], buf[dst], axis, run, st);
      if (e != cudaSuccess) return fail(s, P4A_ERR_CUDA, "mesh blur: %s", cudaGetErrorString(e));
      cur = dst;
      k += run;
    }
    return P4A_OK;
  };
  mark(s, PH_MESH_BLUR);
  int rc;
  if ((rc = blur(0, 0, 3 * mp->field_passes))) return rc;
  s->fieldSlot = 0;
  if (mp->normal_passes > 0) {
    if ((rc = blur(0, 1, 3 * mp->normal_passes))) return rc;
    s->nfieldSlot = 1;
  } else {
    s->nfieldSlot = 0;
  }
  mark(s, PH_MESH_MARCH);
  launch_mesh_count(M, buf[0], s->meshCounts, (uint32_t)nvox, st);
  launch_scan(s->meshCounts, s->meshOffsets, (int)nvox, s->meshScan, s->meshTicket, ++s->meshEpoch & 0x3fffffffu,
              s->d.errorWord, st);
  launch_mesh_emit(M, buf[0], buf[s->nfieldSlot], s->meshOffsets, (uint32_t)nvox, s->meshVerts, st);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  for (int k = 0; k < 3; k++) s->meshDim[k] = dim[k];
  s->meshOrigin = -voxel;
  s->meshVoxel = voxel;
  s->meshNvox = nvox;
  if (triangles) {
    uint32_t t = 0;
    CUDA_TRY(s, cudaMemcpyAsync(&t, s->meshOffsets + nvox, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(s, cudaStreamSynchronize(st));
    s->meshTris = t;
    *triangles = t;
  } else {
    s->meshTris = (int64_t)tris;  // unknown until waited for: the stored capacity bounds it
  }
  return P4A_OK;
}

int p4a_default_ssfr_params(p4a_ssfr_params* o) {
  if (!o) return P4A_ERR_ARG;
  *o = p4a_ssfr_params{};
  // an identity camera: callers set the four matrices and the eye
  for (int k = 0; k < 4; k++) o->view[k * 5] = o->proj[k * 5] = o->inv_view_proj[k * 5] = o->inv_view[k * 5] = 1.0f;
  o->width = 640;
  o->height = 480;
  o->render_scale = 1.0;  // FluidSSFR constructor defaults (src/ssfr.js:9-47)
  o->splat_radius = 1.0;
  o->thickness_radius = 0.62;
  o->thickness_scale = 3.0;
  o->thickness_filter_size = 8;
  o->thickness_half_res = 1;
  o->filter = 2;
  o->filter_iterations = 2;
  o->cleanup_pass = 1;
  o->cleanup_radius = 4;
  o->filter_max_radius = 32;
  o->depth_cull_neighbours = 0;
  o->filter_sigma = 0.7;
  o->narrow_delta = 10.0;
  o->narrow_mu = 1.0;
  o->bilateral_range = 2.0;
  o->ior = 1.333;
  o->absorption = 1.0;
  o->transmit[0] = 0.35;
  o->transmit[1] = 0.62;
  o->transmit[2] = 0.78;
  o->roughness = 0.055;
  o->sun_intensity = 3.0;
  o->sun_elevation = 38.0;
  o->sun_azimuth = 40.0;
  o->exposure = 1.0;
  o->ground_reflection = 0.0;
  o->floor_plane = 1;
  o->debug = 0;
  o->env_intensity = 1.0;  // Environment constructor (src/env.js:151-153)
  o->env_yaw = 0.0;
  return P4A_OK;
}

// The environment uniforms of a render pass (src/ssfr.js:205-207, src/ray.js:66-68):
// hasEnvMap, the intensity and the yaw as float32, the yaw's cosine and sine taken
// once here instead of per pixel.
static EnvMap env_uniform(const p4a_sim* s, double intensity, double yaw) {
  EnvMap E{};
  E.texels = s->envCube;
  E.size = s->envCube ? s->envSize : 0;
  E.intensity = (float)intensity;
  const float y = (float)yaw;
  E.yawCos = (float)std::cos((double)y);
  E.yawSin = (float)std::sin((double)y);
  return E;
}

int p4a_set_environment(p4a_sim* s, const float* rgb, int32_t width, int32_t height) {
  if (!s) return P4A_ERR_ARG;
  if (rgb && (width < 2 || height < 1 || width > 65536 || height > 32768))
    return fail(s, P4A_ERR_ARG, "p4a_set_environment: bad panorama size %d x %d", width, height);
  if (rgb && (width < 2 * height - 2 || width > 2 * height + 2))  // src/env.js:183-184
    return fail(s, P4A_ERR_ARG, "p4a_set_environment: the panorama is %dx%d - an equirectangular panorama is 2:1",
                width, height);
  cudaSetDevice(s->device);
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));  // renders in flight may still read the old map
  if (s->envCube) cudaFree(s->envCube);
  s->envCube = nullptr;
  s->envSize = 0;
  if (!rgb) return P4A_OK;  // Environment.clear
  const int size = env_face_size(width);
  std::vector<uint16_t> host((size_t)6 * size * size * 4);
  build_env_cube(rgb, width, height, size, host.data());
  CUDA_TRY(s, cudaMalloc((void**)&s->envCube, host.size() * 2));
  CUDA_TRY(s, cudaMemcpy(s->envCube, host.data(), host.size() * 2, cudaMemcpyHostToDevice));
  s->envSize = size;
  return P4A_OK;
}

int p4a_environment_read(p4a_sim* s, int32_t* faceSize, void* host, size_t bytes) {
  if (!s) return P4A_ERR_ARG;
  if (faceSize) *faceSize = s->envCube ? s->envSize : 0;
  if (!host || !s->envCube) return P4A_OK;
  const size_t have = (size_t)6 * s->envSize * s->envSize * 8;
  if (bytes > have)
    return fail(s, P4A_ERR_ARG, "p4a_environment_read: %zu bytes asked, the map holds %zu", bytes, have);
  cudaSetDevice(s->device);
  CUDA_TRY(s, cudaMemcpy(host, s->envCube, bytes, cudaMemcpyDeviceToHost));
  return P4A_OK;
}

static int upload_bodies(p4a_sim* s, const float* bodies, int32_t bodyCount);

int p4a_ssfr(p4a_sim* s, const p4a_ssfr_params* sp, const float* bodies, int32_t bodyCount) {
  if (!s || !sp || sp->width < 1 || sp->height < 1 || sp->width > 16384 || sp->height > 16384 ||
      bodyCount < 0 || (bodyCount > 0 && !bodies) || sp->filter < 0 || sp->filter > 2 ||
      sp->filter_iterations < 0 || sp->filter_iterations > 16 || sp->cleanup_radius < 0 ||
      sp->cleanup_radius > 64 || sp->filter_max_radius < 0 || sp->filter_max_radius > 256 ||
      sp->thickness_filter_size < 0 || sp->thickness_filter_size > 2 * kSsfrMaxBlur)
    return fail(s, P4A_ERR_ARG, "p4a_ssfr: invalid parameters");
  if (!s->ready) return fail(s, P4A_ERR_STATE, "ssfr before reset");
  if ((size_t)s->n > s->anisoCap || (s->n > 0 && !s->smoothPos))
    return fail(s, P4A_ERR_STATE, "ssfr needs the anisotropic pass (p4a_aniso) of the current particles");
  cudaSetDevice(s->device);
  const p4a_ssfr_params& q = *sp;
  // render targets (src/ssfr.js:95-130, 173-178)
  const double rs = std::min(1.0, std::max(0.25, q.render_scale));
  const int mapW = std::max(1, (int)std::floor(q.width * rs + 0.5));
  const int mapH = std::max(1, (int)std::floor(q.height * rs + 0.5));
  const bool half = q.thickness_half_res && q.thickness_filter_size >= 4;
  const int tw = half ? (mapW + 1) >> 1 : mapW, th = half ? (mapH + 1) >> 1 : mapH;
  SsfrFrame& F = s->ssfr;
  if (mapW != s->ssfrMapW || mapH != s->ssfrMapH || tw != s->ssfrThW || th != s->ssfrThH ||
      q.width != s->ssfrW || q.height != s->ssfrH) {
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    free_list(s->ssfrAllocs);
    s->ssfrMapW = s->ssfrMapH = s->ssfrThW = s->ssfrThH = s->ssfrW = s->ssfrH = 0;
    const size_t mapN = (size_t)mapW * mapH, thN = (size_t)tw * th;
    int rc;
    if ((rc = dalloc(s, s->ssfrAllocs, &F.depthKey, mapN)) || (rc = dalloc(s, s->ssfrAllocs, &F.thickAcc, thN)) ||
        (rc = dalloc(s, s->ssfrAllocs, &F.eyeZ[0], mapN)) || (rc = dalloc(s, s->ssfrAllocs, &F.eyeZ[1], mapN)) ||
        (rc = dalloc(s, s->ssfrAllocs, &F.raw, mapN)) || (rc = dalloc(s, s->ssfrAllocs, &F.thickMap, thN)) ||
        (rc = dalloc(s, s->ssfrAllocs, &F.thickTmp, thN)) || (rc = dalloc(s, s->ssfrAllocs, &F.bodyT, mapN)) ||
        (rc = dalloc(s, s->ssfrAllocs, &F.image, (size_t)q.width * q.height)))
      return rc;
    s->ssfrMapW = mapW;
    s->ssfrMapH = mapH;
    s->ssfrThW = tw;
    s->ssfrThH = th;
    s->ssfrW = q.width;
    s->ssfrH = q.height;
    s->ssfrGen++;
  }
  {
    const int rc = upload_bodies(s, bodies, bodyCount);
    if (rc) return rc;
  }
  F.mapW = mapW;
  F.mapH = mapH;
  F.thickW = tw;
  F.thickH = th;
  F.smoothPos = s->smoothPos;
  F.g = s->anisoG;
  F.phase = s->d.body[s->parity];
  F.bodies = s->ssfrBodies;
  // host constants (src/ssfr.js:173-226), in double, stored as float
  const double kPiD = 3.14159265358979323846;
  const double el = q.sun_elevation * kPiD / 180, az = q.sun_azimuth * kPiD / 180;
  const double sun[3] = {std::cos(el) * std::sin(az), std::sin(el), std::cos(el) * std::cos(az)};
  const double sl = std::sqrt(sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2]);
  double absorb[3];
  for (int k = 0; k < 3; k++) absorb[k] = q.absorption * -std::log(std::min(1.0, std::max(1e-3, q.transmit[k])));
  const double spacing = s->params.spacing, support = s->h;
  const double scale = q.splat_radius * spacing / support;
  const double r = 0.5 * spacing;
  const double thickRadius = q.thickness_radius * spacing;
  const bool skipBodies = s->nBodyParts > 0;
  float pv[16];
  for (int c = 0; c < 4; c++)
    for (int rr = 0; rr < 4; rr++)
      pv[c * 4 + rr] = std::fma(q.proj[12 + rr], q.view[c * 4 + 3],
                                std::fma(q.proj[8 + rr], q.view[c * 4 + 2],
                                         std::fma(q.proj[4 + rr], q.view[c * 4 + 1], q.proj[rr] * q.view[c * 4])));
  auto splat = [&](SsfrSplat& S, int vw, int vh, double quadRadius, double maxNb) {
    memcpy(S.view, q.view, 64);
    memcpy(S.proj, q.proj, 64);
    memcpy(S.ivp, q.inv_view_proj, 64);
    memcpy(S.pv, pv, 64);
    S.vw = (float)vw;
    S.vh = (float)vh;
    S.kernelScale = (float)scale;
    S.quadRadius = (float)quadRadius;
    S.thickRadius = (float)thickRadius;
    S.maxNeighbours = (float)maxNb;
    S.skipBodies = skipBodies ? 1u : 0u;
    S.count = (uint32_t)std::max(0, s->n);
  };
  splat(F.depth, mapW, mapH, 0.0, (double)q.depth_cull_neighbours);
  splat(F.thick, tw, th, thickRadius, 0.0);
  // thickness blur (src/ssfr.js:227-233)
  const int blurSize = q.thickness_filter_size == 0 ? 0
                       : (tw < mapW ? std::max(1, q.thickness_filter_size >> 1) : q.thickness_filter_size);
  if (blurSize > kSsfrMaxBlur) return fail(s, P4A_ERR_ARG, "p4a_ssfr: thickness blur wider than %d", kSsfrMaxBlur);
  for (int p = 0; p < 2; p++) {
    SsfrBlur& B = F.blur[p];
    B = SsfrBlur{};
    B.dirX = p == 0 ? 1 : 0;
    B.dirY = p == 0 ? 0 : 1;
    B.size = blurSize;
    const float sigma = std::max((float)blurSize / 3.0f, 1.0e-3f);
    const float twoSigma2 = 2.0f * sigma * sigma;
    for (int i = -blurSize; i <= blurSize; i++) B.w[i + blurSize] = fm_exp(-(float)(i * i) / twoSigma2);
  }
  // depth filter uniforms (src/ssfr.js:151-164, 235-237)
  auto filt = [&](SsfrFilter& Fl, int dx, int dy, int clean) {
    Fl = SsfrFilter{};
    Fl.dirX = dx;
    Fl.dirY = dy;
    Fl.maxRadius = q.filter_max_radius;
    Fl.mode = q.filter;
    Fl.sigmaWorld = (float)(q.filter_sigma * r);
    Fl.proj11 = q.proj[5];
    Fl.viewH = (float)mapH;
    Fl.delta = (float)(q.narrow_delta * r);
    Fl.mu = (float)(q.narrow_mu * r);
    Fl.rangeSigma = (float)std::max(q.bilateral_range * r, 1e-4);
    Fl.clean = clean;
    Fl.cleanRadius = q.cleanup_radius;
  };
  filt(F.filter[0], 1, 0, 0);
  filt(F.filter[1], 0, 1, 0);
  filt(F.filter[2], 0, 0, 1);
  F.filterPasses = 0;
  for (int it = 0; it < q.filter_iterations * 2; it++) F.filterSlot[F.filterPasses++] = it % 2;
  if (q.cleanup_pass && q.filter_iterations > 0) F.filterSlot[F.filterPasses++] = 2;
  // composite uniform (src/ssfr.js:183-213)
  SsfrComp& C = F.comp;
  C = SsfrComp{};
  memcpy(C.ivp, q.inv_view_proj, 64);
  memcpy(C.iv, q.inv_view, 64);
  for (int k = 0; k < 3; k++) {
    C.eye[k] = q.eye[k];
    C.boxMin[k] = 0.0f;
    C.boxMax[k] = (float)s->params.box[k];
    C.absorb[k] = (float)absorb[k];
    C.sunDir[k] = (float)(sun[k] / sl);
  }
  C.proj00 = q.proj[0];
  C.proj11 = q.proj[5];
  C.ior = (float)q.ior;
  C.sunIntensity = (float)q.sun_intensity;
  C.roughness = (float)q.roughness;
  C.exposure = (float)q.exposure;
  C.groundReflection = (float)q.ground_reflection;
  C.thicknessScale = (float)q.thickness_scale;
  C.bodyCount = bodyCount;
  C.floorPlane = q.floor_plane ? 1 : 0;
  C.debug = q.debug;
  C.mapScaleX = (float)((double)mapW / std::max(1, q.width));
  C.mapScaleY = (float)((double)mapH / std::max(1, q.height));
  C.width = q.width;
  C.height = q.height;
  C.mapW = mapW;
  C.mapH = mapH;
  C.thickW = tw;
  C.thickH = th;
  C.env = env_uniform(s, q.env_intensity, q.env_yaw);
  mark(s, PH_SSFR);
  launch_ssfr(F, s->stream);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  return P4A_OK;
}

int p4a_ssfr_get_info(p4a_sim* s, p4a_ssfr_info* o) {
  if (!s || !o) return P4A_ERR_ARG;
  *o = p4a_ssfr_info{};
  o->width = s->ssfrW;
  o->height = s->ssfrH;
  o->map_w = s->ssfrMapW;
  o->map_h = s->ssfrMapH;
  o->thick_w = s->ssfrThW;
  o->thick_h = s->ssfrThH;
  o->ssfr_gen = s->ssfrGen;
  return P4A_OK;
}

int p4a_ssfr_buffer(p4a_sim* s, int32_t which, void** dptr, size_t* bytes) {
  if (!s || !dptr || !bytes) return P4A_ERR_ARG;
  if (s->ssfrW == 0) return fail(s, P4A_ERR_STATE, "p4a_ssfr_buffer before p4a_ssfr");
  const SsfrFrame& F = s->ssfr;
  const size_t mapN = (size_t)s->ssfrMapW * s->ssfrMapH, thN = (size_t)s->ssfrThW * s->ssfrThH;
  switch (which) {
    case P4A_SSFR_EYEZ: {
      // the filter's last output: eyeZ[passes % 2]
      *dptr = F.eyeZ[F.filterPasses % 2];
      *bytes = mapN * 4;
      return P4A_OK;
    }
    case P4A_SSFR_RAWZ: *dptr = F.raw; *bytes = mapN * 4; return P4A_OK;
    case P4A_SSFR_THICK: *dptr = F.thickMap; *bytes = thN * 4; return P4A_OK;
    case P4A_SSFR_IMAGE: *dptr = F.image; *bytes = (size_t)s->ssfrW * s->ssfrH * 4; return P4A_OK;
    case P4A_SSFR_BODYT: *dptr = F.bodyT; *bytes = mapN * 4; return P4A_OK;
    default: return fail(s, P4A_ERR_ARG, "p4a_ssfr_buffer: unknown buffer %d", which);
  }
}

int p4a_ssfr_read(p4a_sim* s, int32_t which, void* host, size_t bytes) {
  if (!s || (!host && bytes)) return P4A_ERR_ARG;
  void* p = nullptr;
  size_t have = 0;
  const int rc = p4a_ssfr_buffer(s, which, &p, &have);
  if (rc) return rc;
  if (bytes > have) return fail(s, P4A_ERR_ARG, "p4a_ssfr_read: %zu bytes asked, buffer holds %zu", bytes, have);
  cudaSetDevice(s->device);
  CUDA_TRY(s, cudaMemcpyAsync(host, p, bytes, cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return P4A_OK;
}

// Uploads the caller's packed bodies into the sim's body buffer (shared by the
// render passes); waits, since the host array may go away.
static int upload_bodies(p4a_sim* s, const float* bodies, int32_t bodyCount) {
  if (bodyCount > s->ssfrBodyCap) {
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->ssfrBodies) cudaFree(s->ssfrBodies);
    s->ssfrBodies = nullptr;
    s->ssfrBodyCap = 0;
    CUDA_TRY(s, cudaMalloc((void**)&s->ssfrBodies, (size_t)bodyCount * 6 * 16));
    s->ssfrBodyCap = bodyCount;
  }
  if (bodyCount > 0) {
    CUDA_TRY(s, cudaMemcpyAsync(s->ssfrBodies, bodies, (size_t)bodyCount * 6 * 16, cudaMemcpyHostToDevice,
                                s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  }
  return P4A_OK;
}

int p4a_default_ray_params(p4a_ray_params* o) {
  if (!o) return P4A_ERR_ARG;
  *o = p4a_ray_params{};
  for (int k = 0; k < 4; k++) o->proj[k * 5] = o->inv_view_proj[k * 5] = o->inv_view[k * 5] = 1.0f;
  o->width = 640;
  o->height = 480;
  o->iso = 0.4;  // RayMarch constructor defaults (src/ray.js:16-29), meshIso (src/main.js:320)
  o->ior = 1.333;
  o->absorption = 1.0;
  o->transmit[0] = 0.35;
  o->transmit[1] = 0.62;
  o->transmit[2] = 0.78;
  o->thickness_steps = 48;
  o->floor_plane = 1;
  o->ground_reflection = 0.0;
  o->skin_width = 0.05;
  o->roughness = 0.055;
  o->sun_intensity = 3.0;
  o->sun_elevation = 38.0;
  o->sun_azimuth = 40.0;
  o->exposure = 1.0;
  o->debug = 0;
  o->use_surface = 1;  // raySurface (src/main.js)
  o->env_intensity = 1.0;
  o->env_yaw = 0.0;
  for (int k = 0; k < 4; k++) o->view[k * 5] = 1.0f;
  return P4A_OK;
}

int p4a_ray(p4a_sim* s, const p4a_ray_params* rp, const float* bodies, int32_t bodyCount) {
  if (!s || !rp || rp->width < 1 || rp->height < 1 || rp->width > 16384 || rp->height > 16384 || bodyCount < 0 ||
      (bodyCount > 0 && !bodies) || rp->thickness_steps < 0 || rp->thickness_steps > 4096)
    return fail(s, P4A_ERR_ARG, "p4a_ray: invalid parameters");
  if (!s->ready) return fail(s, P4A_ERR_STATE, "ray before reset");
  if (s->meshDim[0] < 2 || !s->meshField[s->fieldSlot])
    return fail(s, P4A_ERR_STATE, "ray needs the density field of p4a_mesh");
  if (rp->use_surface && s->meshTriCap >= (1u << 30))  // the depth test keys hold triangle * 4 + fan index
    return fail(s, P4A_ERR_CAPACITY, "p4a_ray: the mesh surface pass takes at most 2^30 triangles");
  cudaSetDevice(s->device);
  const size_t px = (size_t)rp->width * rp->height;
  if (px > s->rayCap) {
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->rayImage) cudaFree(s->rayImage);
    s->rayImage = nullptr;
    s->rayCap = 0;
    if (s->raySurf) cudaFree(s->raySurf);
    s->raySurf = nullptr;
    CUDA_TRY(s, cudaMalloc((void**)&s->rayImage, px * 4));
    CUDA_TRY(s, cudaMalloc((void**)&s->raySurf, px * (8 + 4 + 16)));
    s->rayCap = px;
  }
  int rc = upload_bodies(s, bodies, bodyCount);
  if (rc) return rc;
  const p4a_ray_params& q = *rp;
  RayParams R{};
  memcpy(R.ivp, q.inv_view_proj, 64);
  memcpy(R.iv, q.inv_view, 64);
  memcpy(R.view, q.view, 64);
  for (int c = 0; c < 4; c++)
    for (int rr = 0; rr < 4; rr++)
      R.vp[c * 4 + rr] = std::fma(q.proj[12 + rr], q.view[c * 4 + 3],
                                  std::fma(q.proj[8 + rr], q.view[c * 4 + 2],
                                           std::fma(q.proj[4 + rr], q.view[c * 4 + 1], q.proj[rr] * q.view[c * 4])));
  R.useSurface = q.use_surface ? 1 : 0;
  R.env = env_uniform(s, q.env_intensity, q.env_yaw);
  const double kPiD = 3.14159265358979323846;
  const double el = q.sun_elevation * kPiD / 180, az = q.sun_azimuth * kPiD / 180;
  const double sun[3] = {std::cos(el) * std::sin(az), std::sin(el), std::cos(el) * std::cos(az)};
  const double sl = std::sqrt(sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2]);
  for (int k = 0; k < 3; k++) {
    R.eye[k] = q.eye[k];
    R.gridOrigin[k] = (float)s->meshOrigin;
    R.boxMin[k] = 0.0f;
    R.boxMax[k] = (float)s->params.box[k];
    R.absorb[k] = (float)(q.absorption * -std::log(std::min(1.0, std::max(1e-3, q.transmit[k]))));
    R.sunDir[k] = (float)(sun[k] / sl);
    R.vertDim[k] = s->meshDim[k];
  }
  R.voxel = (float)s->meshVoxel;
  R.iso = (float)q.iso;
  R.ior = (float)q.ior;
  R.skin = (float)q.skin_width;
  R.sunIntensity = (float)q.sun_intensity;
  R.roughness = (float)q.roughness;
  R.exposure = (float)q.exposure;
  R.groundReflection = (float)q.ground_reflection;
  R.proj00 = q.proj[0];
  R.proj11 = q.proj[5];
  R.thickSteps = q.thickness_steps;
  R.bodyCount = bodyCount;
  R.floorPlane = q.floor_plane ? 1 : 0;
  R.debug = q.debug;
  R.width = q.width;
  R.height = q.height;
  const double deg[4] = {5.0, 10.0, 20.0, 40.0};
  for (int k = 0; k < 4; k++) R.cosDeg[k] = (float)std::cos(deg[k] * kPiD / 180);
  mark(s, PH_RAY);
  // surface maps: normals, then 8-byte depth-test keys, then eye z
  float4* surfN = (float4*)s->raySurf;
  unsigned long long* key = (unsigned long long*)(s->raySurf + px * 16);
  float* surfZ = (float*)(s->raySurf + px * 24);
  if (R.useSurface)
    launch_surface(R, s->meshVerts, s->meshOffsets + s->meshNvox, (uint32_t)s->meshTriCap, R.gridOrigin, R.vertDim,
                   R.voxel, key, surfZ, surfN, s->stream);
  launch_ray(R, s->meshField[s->fieldSlot], s->ssfrBodies, surfZ, surfN, s->rayImage, s->stream);
  mark(s, PH_END);
  CUDA_TRY(s, cudaGetLastError());
  s->rayW = q.width;
  s->rayH = q.height;
  return P4A_OK;
}

int p4a_ray_buffer(p4a_sim* s, void** dptr, size_t* bytes, int32_t* width, int32_t* height) {
  if (!s || !dptr || !bytes) return P4A_ERR_ARG;
  if (s->rayW == 0) return fail(s, P4A_ERR_STATE, "p4a_ray_buffer before p4a_ray");
  *dptr = s->rayImage;
  *bytes = (size_t)s->rayW * s->rayH * 4;
  if (width) *width = s->rayW;
  if (height) *height = s->rayH;
  return P4A_OK;
}

int p4a_ray_read(p4a_sim* s, void* host, size_t bytes) {
  if (!s || (!host && bytes)) return P4A_ERR_ARG;
  void* p = nullptr;
  size_t have = 0;
  const int rc = p4a_ray_buffer(s, &p, &have, nullptr, nullptr);
  if (rc) return rc;
  if (bytes > have) return fail(s, P4A_ERR_ARG, "p4a_ray_read: %zu bytes asked, image holds %zu", bytes, have);
  cudaSetDevice(s->device);
  CUDA_TRY(s, cudaMemcpyAsync(host, p, bytes, cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return P4A_OK;
}

int p4a_mesh_get_info(p4a_sim* s, p4a_mesh_info* o) {
  if (!s || !o) return P4A_ERR_ARG;
  *o = p4a_mesh_info{};
  for (int k = 0; k < 3; k++) {
    o->vert_dim[k] = s->meshDim[k];
    o->origin[k] = s->meshOrigin;
  }
  o->voxel = s->meshVoxel;
  o->triangles = s->meshTris;
  o->mesh_gen = s->meshGen;
  return P4A_OK;
}

int p4a_profile_enable(p4a_sim* s, int32_t on) {
  if (!s) return P4A_ERR_ARG;
  if (!on && s->prof) {
    mark(s, PH_END);
    const int rc = resolve_marks(s);
    s->prof = false;
    return rc;
  }
  s->prof = on != 0;
  return P4A_OK;
}

int p4a_profile_reset(p4a_sim* s) {
  if (!s) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  const int rc = resolve_marks(s);
  for (int k = 0; k < PH_COUNT; k++) {
    s->phaseMs[k] = 0;
    s->phaseLaunches[k] = 0;
  }
  return rc;
}

int p4a_profile_read(p4a_sim* s, p4a_phase_time* out, int32_t maxEntries, int32_t* count) {
  if (!s || (!out && maxEntries > 0)) return P4A_ERR_ARG;
  cudaSetDevice(s->device);
  const int rc = resolve_marks(s);
  int c = 0;
  for (int k = 0; k < PH_COUNT; k++) {
    if (!s->phaseLaunches[k]) continue;
    if (c < maxEntries) {
      std::snprintf(out[c].name, sizeof(out[c].name), "%s", kPhaseNames[k]);
      out[c].ms = s->phaseMs[k];
      out[c].launches = s->phaseLaunches[k];
    }
    c++;
  }
  if (count) *count = c;
  return rc;
}

uint64_t p4a_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

}  // extern "C"

namespace p4a {
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

std::atomic<uint32_t> g_op_spin_limit{kScanSpinLimit};
std::atomic<int32_t> g_op_skip_first_tile{0};

int grid_sort_check(const p4a_grid* g, int32_t n, long long maxCells, long long* cells) {
  if (!g || n < 0 || !(g->h > 0)) return P4A_ERR_ARG;
  long long c = 1;
  for (int k = 0; k < 3; k++) {
    if (g->dim[k] < 1) return P4A_ERR_ARG;
    // checked one factor at a time, so the product never overflows
    if ((long long)g->dim[k] > maxCells / c) return P4A_ERR_CAPACITY;
    c *= g->dim[k];
  }
  *cells = c;
  return P4A_OK;
}

int grid_sort_launch(const p4a_grid& g, int32_t n, float dt, float gravity, const float* pos, const float* vel,
                     const uint32_t* body, const float* rest, float* posOut, float* velOut, float* predOut,
                     uint32_t* bodyOut, float* restOut, uint32_t* cellStart, uint32_t* slotOut, uint32_t* key,
                     uint32_t* rank, uint32_t* unordered, uint32_t* cellCount, unsigned long long* state,
                     uint32_t* ticket, uint32_t* err, uint32_t* status, cudaStream_t st) {
  // test hook (p4a_test_scan_wait): start the tickets at 1, so tile 0 is never
  // scanned and tile 1's lookback waits on a flag that nothing sets
  if (g_op_skip_first_tile.load(std::memory_order_relaxed) &&
      cudaMemsetAsync(ticket, 1, 1, st) != cudaSuccess)
    return P4A_ERR_CUDA;
  g_launches.fetch_add(4, std::memory_order_relaxed);
  if (run_grid_sort(g, n, dt, gravity, pos, vel, body, rest, posOut, velOut, predOut, bodyOut, restOut, cellStart,
                    slotOut, key, rank, unordered, cellCount, state, ticket, err, st,
                    g_op_spin_limit.load(std::memory_order_relaxed)) != cudaSuccess)
    return P4A_ERR_CUDA;
  if (status) {  // the caller reads the error word when it reads the outputs
    return cudaMemcpyAsync(status, err, 4, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? P4A_OK : P4A_ERR_CUDA;
  }
  uint32_t word = 0;
  if (cudaMemcpyAsync(&word, err, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return P4A_ERR_CUDA;
  return (word & ERR_SCAN_TIMEOUT) ? P4A_ERR_TIMEOUT : P4A_OK;
}

int resident_grid(const void* kernel, int block) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, kernel);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int perSM = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, block, 0) != cudaSuccess || perSM < 1)
    perSM = 1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
  const int g = perSM * sms;
  cache[key] = g;
  return g;
}
}  // namespace p4a

extern "C" {

// ---- operator entry: predict + grid pass on caller buffers ---------------
static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t p4a_grid_sort_workspace_size(int32_t n, int32_t nCells) {
  if (n < 0 || nCells <= 0) return 0;
  const size_t un = (size_t)std::max(1, n);
  return 3 * align256(un * 4) + align256(((size_t)nCells + 1) * 4) +
         align256((size_t)scan_tiles(nCells) * 8) + align256(4) + align256(4);
}

int p4a_test_scan_wait(uint32_t spin_limit, int32_t skip_first_tile) {
  if (skip_first_tile != 0 && skip_first_tile != 1) return P4A_ERR_ARG;
  p4a::g_op_spin_limit.store(spin_limit ? spin_limit : p4a::kScanSpinLimit, std::memory_order_relaxed);
  p4a::g_op_skip_first_tile.store(skip_first_tile, std::memory_order_relaxed);
  return P4A_OK;
}

int p4a_grid_sort(const p4a_grid* grid, int32_t n, float dt, float gravity, const float* pos,
                  const float* vel, const uint32_t* body, const float* rest, float* pos_out,
                  float* vel_out, float* pred_out, uint32_t* body_out, float* rest_out,
                  uint32_t* cell_start, uint32_t* slot_out, void* workspace, size_t workspace_bytes,
                  uint32_t* status, void* stream) {
  using namespace p4a;
  long long cellsLL = 0;
  int rc = grid_sort_check(grid, n, 0x7fffffffLL, &cellsLL);
  if (rc != P4A_OK) return rc;
  const int nCells = (int)cellsLL;
  if (n > 0 && (!pos || !vel || !pos_out || !vel_out || !pred_out)) return P4A_ERR_ARG;
  if ((body && !body_out) || (rest && !rest_out) || !cell_start) return P4A_ERR_ARG;
  if (!workspace || workspace_bytes < p4a_grid_sort_workspace_size(n, nCells)) return P4A_ERR_CAPACITY;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)workspace;
  const size_t un = (size_t)std::max(1, n);
  uint32_t* key = (uint32_t*)w; w += align256(un * 4);
  uint32_t* rank = (uint32_t*)w; w += align256(un * 4);
  uint32_t* unordered = (uint32_t*)w; w += align256(un * 4);
  uint32_t* cellCount = (uint32_t*)w; w += align256(((size_t)nCells + 1) * 4);
  unsigned long long* state = (unsigned long long*)w; w += align256((size_t)scan_tiles(nCells) * 8);
  uint32_t* ticket = (uint32_t*)w; w += align256(4);
  uint32_t* errw = (uint32_t*)w;
  const size_t zeroBytes = (size_t)((char*)errw + 4 - (char*)cellCount);
  if (cudaMemsetAsync(cellCount, 0, zeroBytes, st) != cudaSuccess) return P4A_ERR_CUDA;
  return grid_sort_launch(*grid, n, dt, gravity, pos, vel, body, rest, pos_out, vel_out, pred_out, body_out,
                          rest_out, cell_start, slot_out, key, rank, unordered, cellCount, state, ticket, errw,
                          status, st);
}

}  // extern "C"
