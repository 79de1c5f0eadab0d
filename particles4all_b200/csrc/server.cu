// server.cu — the serving loop (p4a_server_*): continuous batching of create /
// step / destroy requests for many scenes kept resident on one GPU.
//
// Threads
//   clients   submit requests into the inbox from any thread and poll completions;
//   builders  build created scenes on the host (the reference's buildScene, or an
//             explicit scene with its mass calibration), then the boundary samples
//             and scales, into a pinned upload blob;
//   engine    owns the batch and its streams. Each turn it takes new requests,
//             retires finished frames (readbacks copied out, completions posted,
//             latencies recorded), admits built scenes while scene slots and arena
//             ranges are free (uploads on a second stream, then one prime frame
//             for all of them), releases destroyed scenes' ranges once the last
//             frame that touched them has finished, and launches the next frame
//             with every live scene that has a pending step while up to
//             max_frames_in_flight earlier frames are still on the GPU.
// A scene's arena ranges are handed out again only after every frame that used
// them has finished, so uploads on the second stream never race a running frame.
// With plain = 1 the same loop serves each scene with its own plain Sim, stepped
// one after another on the engine's stream (the comparison for the batched form);
// its admission applies the same particle budget and scene-count limits.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/p4a.h"
#include "batch_internal.h"
#include "p4a_internal.h"
#include "scene.h"

using namespace p4a;

namespace {

using Clock = std::chrono::steady_clock;
constexpr double kAdmitSecondsPerTurn = 0.004;

// First-fit ranges of one pinned host slab, shared by threads.
class PinnedPool {
 public:
  ~PinnedPool() {
    if (base_) cudaFreeHost(base_);
  }
  int init(size_t bytes) {
    if (cudaHostAlloc((void**)&base_, bytes, cudaHostAllocPortable) != cudaSuccess) {
      base_ = nullptr;
      return P4A_ERR_OOM;
    }
    cap_ = bytes;
    ranges_.init((int64_t)bytes);
    return P4A_OK;
  }
  size_t capacity() const { return cap_; }
  unsigned char* try_get(size_t bytes) {
    std::lock_guard<std::mutex> l(mu_);
    const int64_t off = ranges_.alloc((int64_t)bytes, 256);
    return off < 0 ? nullptr : base_ + off;
  }
  // Waits until `bytes` fit; nullptr when they never can or `stop` is set.
  unsigned char* get(size_t bytes, const std::atomic<bool>& stop) {
    if (bytes > cap_) return nullptr;
    std::unique_lock<std::mutex> l(mu_);
    for (;;) {
      const int64_t off = ranges_.alloc((int64_t)bytes, 256);
      if (off >= 0) return base_ + off;
      if (stop.load()) return nullptr;
      cv_.wait_for(l, std::chrono::milliseconds(20));
    }
  }
  void put(unsigned char* p, size_t bytes) {
    if (!p) return;
    {
      std::lock_guard<std::mutex> l(mu_);
      ranges_.release(p - base_, (int64_t)bytes);
    }
    cv_.notify_all();
  }

 private:
  unsigned char* base_ = nullptr;
  size_t cap_ = 0;
  RangeAlloc ranges_;
  std::mutex mu_;
  std::condition_variable cv_;
};

struct StepReq {
  int64_t id = 0;
  double dt = 0, tSubmit = 0;
  float* pos = nullptr;
  float* vel = nullptr;
  size_t outBytes = 0;
};

struct CreateReq {
  p4a_params params{};
  std::vector<p4a_body_spec> specs;
  std::unique_ptr<HostScene> scene;  // explicit scene, or null for buildScene
  int pourBudget = 0;
};

struct Req {
  int kind = 0;
  int64_t id = 0;
  int32_t scene = -1;
  double t = 0;
  std::unique_ptr<CreateReq> create;
  StepReq step;
};

enum SceneState { S_BUILDING, S_READY, S_LIVE };

struct SScene {
  int state = S_BUILDING;
  int64_t createReq = 0;
  double tSubmit = 0;
  int64_t n = 0;
  p4a_params params{};
  std::vector<p4a_body_spec> specs;
  int slot = -1;            // batch slot
  p4a_sim* sim = nullptr;   // plain form
  std::deque<StepReq> steps;
  bool destroyWanted = false;
  int64_t destroyReq = -1;
  double tDestroy = 0;
  uint64_t lastSeq = 0;     // last frame that used the scene's device memory
  std::unique_ptr<PreparedScene> prep;
  std::unique_ptr<HostScene> host;  // plain form: the built scene
  unsigned char* blob = nullptr;
  size_t blobBytes = 0;
};

struct BuildJob {
  int32_t handle = -1;
  std::unique_ptr<CreateReq> req;
};

struct BuildResult {
  int32_t handle = -1;
  int status = P4A_OK;
  std::string err;
  int64_t n = 0;
  std::unique_ptr<PreparedScene> prep;
  std::unique_ptr<HostScene> host;
  unsigned char* blob = nullptr;
  size_t bytes = 0;
};

struct Readback {
  unsigned char* pinned = nullptr;
  size_t bytes = 0;
  void* dst = nullptr;
};

struct FrameRec {
  uint64_t seq = 0;
  cudaEvent_t start = nullptr, done = nullptr;
  double tLaunch = 0;
  std::vector<std::pair<int32_t, StepReq>> steps;
  std::vector<int> substeps;
  std::vector<int64_t> particles;
  std::vector<Readback> rbs;
  std::vector<int32_t> primed;  // scenes whose create completes with this frame
  std::vector<std::pair<unsigned char*, size_t>> blobs;
  uint64_t kernels = 0;
};

double quantile(std::vector<double> v, double q) {
  if (v.empty()) return 0;
  const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + (long)k, v.end());
  return v[k];
}

}  // namespace

struct p4a_server {
  int device = 0;
  p4a_server_config cfg{};
  Clock::time_point t0;
  p4a_batch* batch = nullptr;
  cudaStream_t stream = nullptr;  // the engine's stream (the batch's, or its own when plain)
  bool ownStream = false;
  cudaStream_t up = nullptr;
  cudaEvent_t upEvent = nullptr;
  uint32_t* errPinned = nullptr;  // device error word, copied after every frame
  PinnedPool uploads, readbacks;
  // client side
  std::mutex mu;
  std::condition_variable cvPoll;
  std::vector<Req> inbox;
  std::deque<p4a_completion> done;
  std::string err;
  int64_t nextReq = 1;
  int32_t nextScene = 0;
  std::atomic<bool> stop{false};
  std::atomic<bool> failed{false};
  // builders
  std::mutex bmu;
  std::condition_variable bcv;
  std::deque<BuildJob> buildQ;
  std::vector<BuildResult> built;
  std::vector<std::thread> builders;
  std::thread engine;
  // engine state
  std::unordered_map<int32_t, SScene> scenes;
  std::deque<int32_t> admitQ;
  std::deque<FrameRec> inflight;
  std::vector<cudaEvent_t> evPool;
  uint64_t seq = 0, doneSeq = 0;
  int building = 0;
  int64_t plainParticles = 0;
  int plainScenes = 0;
  // statistics (under mu)
  p4a_server_stats st{};
  std::vector<double> stepMs, admitMs;
  double frameScenes = 0;
  int64_t stepFrames = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void set_err(p4a_server* S, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  std::lock_guard<std::mutex> l(S->mu);
  S->err = buf;
}

void post(p4a_server* S, const p4a_completion& c) {
  {
    std::lock_guard<std::mutex> l(S->mu);
    S->done.push_back(c);
  }
  S->cvPoll.notify_all();
}

p4a_completion completion(int kind, int64_t id, int32_t scene, int status, double tSubmit, double tStart,
                          double tEnd, int64_t particles, int substeps = 0) {
  p4a_completion c{};
  c.request = id;
  c.kind = kind;
  c.scene = scene;
  c.status = status;
  c.substeps = substeps;
  c.particles = particles;
  c.submitted = tSubmit;
  c.started = tStart;
  c.finished = tEnd;
  return c;
}

cudaEvent_t take_event(p4a_server* S) {
  if (!S->evPool.empty()) {
    cudaEvent_t e = S->evPool.back();
    S->evPool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// ---- builders ---------------------------------------------------------------

void builder_main(p4a_server* S) {
  omp_set_num_threads(2);
  for (;;) {
    BuildJob job;
    {
      std::unique_lock<std::mutex> l(S->bmu);
      S->bcv.wait(l, [&] { return S->stop.load() || !S->buildQ.empty(); });
      if (S->stop.load()) return;
      job = std::move(S->buildQ.front());
      S->buildQ.pop_front();
    }
    BuildResult r;
    r.handle = job.handle;
    CreateReq& c = *job.req;
    c.params.bodies = c.specs.empty() ? nullptr : c.specs.data();
    c.params.n_bodies = (int32_t)c.specs.size();
    std::unique_ptr<HostScene> sc;
    if (c.scene) {
      sc = std::move(c.scene);
      const bool doMass = !(sc->mass > 0), doDenom = !(sc->denomRest > 0);
      if (doMass || doDenom) calibrate_scene(c.params, *sc, doMass, doDenom);
    } else {
      sc.reset(new HostScene());
      build_scene(c.params, *sc);
      if (c.params.pour) c.pourBudget = sc->nFluid;
    }
    r.n = sc->n;
    if (S->cfg.plain) {
      r.host = std::move(sc);
    } else {
      r.prep.reset(new PreparedScene());
      r.status = prepare_scene(c.params, *sc, c.pourBudget, *r.prep, r.err);
      if (r.status == P4A_OK) {
        r.bytes = r.prep->bytes;
        r.blob = S->uploads.get(r.bytes, S->stop);
        if (!r.blob) {
          r.status = P4A_ERR_CAPACITY;
          r.err = "scene larger than the upload staging";
        } else {
          write_blob(*r.prep, r.blob);
          r.prep->sc = HostScene();  // the blob holds the particles now
        }
      }
    }
    {
      std::lock_guard<std::mutex> l(S->bmu);
      S->built.push_back(std::move(r));
    }
  }
}

// ---- engine -------------------------------------------------------------------

void take_request(p4a_server* S, Req& r) {
  if (r.kind == P4A_REQ_CREATE) {
    const int pending = S->building + (int)S->admitQ.size();
    if (S->cfg.max_pending_creates > 0 && pending >= S->cfg.max_pending_creates) {
      post(S, completion(P4A_REQ_CREATE, r.id, r.scene, P4A_ERR_CAPACITY, r.t, r.t, S->now(), 0));
      std::lock_guard<std::mutex> l(S->mu);
      S->st.rejected++;
      return;
    }
    SScene& sc = S->scenes[r.scene];
    sc.state = S_BUILDING;
    sc.createReq = r.id;
    sc.tSubmit = r.t;
    sc.params = r.create->params;
    sc.specs = r.create->specs;
    sc.params.bodies = nullptr;
    S->building++;
    {
      std::lock_guard<std::mutex> l(S->bmu);
      BuildJob j;
      j.handle = r.scene;
      j.req = std::move(r.create);
      S->buildQ.push_back(std::move(j));
    }
    S->bcv.notify_one();
    return;
  }
  auto it = S->scenes.find(r.scene);
  const bool gone = it == S->scenes.end() || it->second.destroyWanted;
  if (r.kind == P4A_REQ_STEP) {
    if (gone) {
      post(S, completion(P4A_REQ_STEP, r.id, r.scene, P4A_ERR_STATE, r.t, r.t, S->now(), 0));
      return;
    }
    it->second.steps.push_back(r.step);
    return;
  }
  // destroy
  if (gone) {
    post(S, completion(P4A_REQ_DESTROY, r.id, r.scene, P4A_ERR_STATE, r.t, r.t, S->now(), 0));
    return;
  }
  it->second.destroyWanted = true;
  it->second.destroyReq = r.id;
  it->second.tDestroy = r.t;
}

void drop_scene(p4a_server* S, int32_t h, int createStatus) {
  SScene& sc = S->scenes[h];
  const double t = S->now();
  if (sc.blob) S->uploads.put(sc.blob, sc.blobBytes);
  for (const StepReq& q : sc.steps) post(S, completion(P4A_REQ_STEP, q.id, h, P4A_ERR_STATE, q.tSubmit, t, t, sc.n));
  post(S, completion(P4A_REQ_CREATE, sc.createReq, h, createStatus, sc.tSubmit, t, t, sc.n));
  if (sc.destroyWanted) post(S, completion(P4A_REQ_DESTROY, sc.destroyReq, h, P4A_OK, sc.tDestroy, t, t, sc.n));
  S->scenes.erase(h);
}

bool collect_built(p4a_server* S) {
  std::vector<BuildResult> got;
  {
    std::lock_guard<std::mutex> l(S->bmu);
    got.swap(S->built);
  }
  for (BuildResult& r : got) {
    S->building--;
    SScene& sc = S->scenes[r.handle];
    sc.n = r.n;
    sc.blob = r.blob;
    sc.blobBytes = r.bytes;
    if (r.status != P4A_OK) {
      set_err(S, "scene %d: %s", r.handle, r.err.c_str());
      {
        std::lock_guard<std::mutex> l(S->mu);
        S->st.rejected++;
      }
      drop_scene(S, r.handle, r.status);
      continue;
    }
    if (sc.destroyWanted) {
      drop_scene(S, r.handle, P4A_ERR_STATE);
      continue;
    }
    sc.prep = std::move(r.prep);
    sc.host = std::move(r.host);
    sc.state = S_READY;
    S->admitQ.push_back(r.handle);
  }
  return !got.empty();
}

void record_admit(p4a_server* S, SScene& sc, double t) {
  std::lock_guard<std::mutex> l(S->mu);
  S->st.admitted++;
  S->admitMs.push_back((t - sc.tSubmit) * 1e3);
}

bool expired(const p4a_server* S, const SScene& sc, double t) {
  return S->cfg.admit_timeout > 0 && t - sc.tSubmit > S->cfg.admit_timeout;
}

void reject(p4a_server* S, int32_t h) {
  {
    std::lock_guard<std::mutex> l(S->mu);
    S->st.rejected++;
  }
  drop_scene(S, h, P4A_ERR_CAPACITY);
}

int admit_plain(p4a_server* S, SScene& sc) {
  if (S->plainScenes >= S->cfg.arenas.max_scenes || S->plainParticles + sc.n > S->cfg.arenas.max_particles)
    return P4A_ERR_CAPACITY;
  p4a_sim* sim = nullptr;
  int rc = p4a_create(S->device, &sim);
  if (rc) return rc;
  if ((rc = p4a_set_stream(sim, S->stream))) {
    p4a_destroy(sim);
    return rc;
  }
  const HostScene& h = *sc.host;
  p4a_scene_desc d{};
  d.n = h.n;
  d.pos = h.pos.data();
  d.vel = h.vel.data();
  d.phase = h.phase.data();
  d.rest = h.rest.data();
  d.n_bodies = (int32_t)h.bodyDensity.size();
  d.body_density = h.bodyDensity.data();
  d.body_centre = h.bodyCentre.data();
  d.mass = h.mass;
  d.denom_rest = h.denomRest;
  p4a_params p = sc.params;
  p.bodies = sc.specs.empty() ? nullptr : sc.specs.data();
  p.n_bodies = (int32_t)sc.specs.size();
  rc = p4a_reset_scene(sim, &p, &d);
  if (rc) {
    p4a_destroy(sim);
    return rc == P4A_ERR_OOM ? P4A_ERR_CAPACITY : rc;
  }
  sc.sim = sim;
  sc.host.reset();
  S->plainScenes++;
  S->plainParticles += sc.n;
  return P4A_OK;
}

bool admit(p4a_server* S) {
  if (S->admitQ.empty()) return false;
  bool progress = false;
  std::vector<int> slots;
  std::vector<int32_t> handles;
  std::vector<std::pair<unsigned char*, size_t>> blobs;
  const double t = S->now();
  for (auto it = S->admitQ.begin(); it != S->admitQ.end();) {
    // bounded admission work per engine turn, so frames keep flowing
    if (S->now() - t > kAdmitSecondsPerTurn) break;
    const int32_t h = *it;
    SScene& sc = S->scenes[h];
    if (sc.destroyWanted) {
      drop_scene(S, h, P4A_ERR_STATE);
      it = S->admitQ.erase(it);
      progress = true;
      continue;
    }
    int rc;
    if (S->cfg.plain) {
      rc = admit_plain(S, sc);
    } else {
      int32_t slot = -1;
      rc = place_scene(S->batch, *sc.prep, sc.blob, S->up, &slot);
      if (rc == P4A_OK) {
        sc.slot = slot;
        slots.push_back(slot);
        handles.push_back(h);
        blobs.emplace_back(sc.blob, sc.blobBytes);
        sc.blob = nullptr;
        sc.prep.reset();
      }
    }
    if (rc == P4A_OK) {
      sc.state = S_LIVE;
      record_admit(S, sc, t);
      if (S->cfg.plain) post(S, completion(P4A_REQ_CREATE, sc.createReq, h, P4A_OK, sc.tSubmit, t, S->now(), sc.n));
      it = S->admitQ.erase(it);
      progress = true;
    } else if (rc == P4A_ERR_CAPACITY) {
      if (expired(S, sc, t)) {
        reject(S, h);
        it = S->admitQ.erase(it);
        progress = true;
      } else {
        ++it;
      }
    } else {
      set_err(S, "admission of scene %d failed (%d): %s", h, rc,
              S->batch ? p4a_batch_last_error(S->batch) : "plain sim");
      S->failed = true;
      return true;
    }
  }
  if (slots.empty()) return progress;
  // one prime frame for the admitted scenes, after their uploads
  FrameRec F;
  F.seq = ++S->seq;
  F.start = take_event(S);
  F.done = take_event(S);
  F.tLaunch = S->now();
  const uint64_t k0 = p4a_kernel_launches();
  cudaEventRecord(S->upEvent, S->up);
  cudaStreamWaitEvent(S->stream, S->upEvent, 0);
  cudaEventRecord(F.start, S->stream);
  const int rc = prime_scenes(S->batch, slots);
  if (rc) {
    set_err(S, "prime frame: %s", p4a_batch_last_error(S->batch));
    S->failed = true;
  }
  cudaEventRecord(F.done, S->stream);
  F.kernels = p4a_kernel_launches() - k0;
  F.primed = handles;
  F.blobs = blobs;
  for (int32_t h : handles) S->scenes[h].lastSeq = F.seq;
  S->inflight.push_back(std::move(F));
  return true;
}

int step_frames_in_flight(const p4a_server* S) {
  int n = 0;
  for (const FrameRec& f : S->inflight) n += f.steps.empty() ? 0 : 1;
  return n;
}

bool launch(p4a_server* S) {
  if (step_frames_in_flight(S) >= std::max(1, S->cfg.max_frames_in_flight)) return false;
  std::vector<int32_t> hs;
  for (auto& kv : S->scenes)
    if (kv.second.state == S_LIVE && !kv.second.steps.empty()) hs.push_back(kv.first);
  if (hs.empty()) return false;
  std::sort(hs.begin(), hs.end());
  // readback staging for the whole frame, or wait for frames to retire
  FrameRec F;
  std::vector<std::pair<int32_t, int>> rbWho;  // (scene, 0 = pos / 1 = vel)
  for (int32_t h : hs) {
    SScene& sc = S->scenes[h];
    const StepReq& q = sc.steps.front();
    const size_t want = std::min((size_t)sc.n * 16, q.outBytes);
    for (int w = 0; w < 2; w++) {
      if (!(w == 0 ? (void*)q.pos : (void*)q.vel) || want == 0) continue;
      if (want > S->readbacks.capacity()) continue;  // completes with P4A_ERR_CAPACITY
      unsigned char* p = S->readbacks.try_get(want);
      if (!p) {
        for (Readback& r : F.rbs) S->readbacks.put(r.pinned, r.bytes);
        if (!S->inflight.empty()) return false;
        set_err(S, "readback staging exhausted with no frame in flight");
        S->failed = true;
        return true;
      }
      F.rbs.push_back({p, want, w == 0 ? (void*)q.pos : (void*)q.vel});
      rbWho.emplace_back(h, w);
    }
  }
  F.seq = ++S->seq;
  F.start = take_event(S);
  F.done = take_event(S);
  F.tLaunch = S->now();
  const uint64_t k0 = p4a_kernel_launches();
  cudaEventRecord(F.start, S->stream);
  int rc = P4A_OK;
  if (S->cfg.plain) {
    for (int32_t h : hs) {
      SScene& sc = S->scenes[h];
      int32_t subs = 0;
      rc = p4a_step(sc.sim, sc.steps.front().dt, &subs);
      if (rc) {
        set_err(S, "plain step of scene %d: %s", h, p4a_last_error(sc.sim));
        break;
      }
      F.substeps.push_back(subs);
    }
  } else {
    std::vector<int32_t> ids;
    std::vector<double> dts;
    for (int32_t h : hs) {
      ids.push_back(S->scenes[h].slot);
      dts.push_back(S->scenes[h].steps.front().dt);
    }
    rc = step_scenes(S->batch, ids.data(), dts.data(), (int32_t)ids.size());
    if (rc) set_err(S, "frame: %s", p4a_batch_last_error(S->batch));
    for (int32_t h : hs) F.substeps.push_back(S->batch->scenes[S->scenes[h].slot].lastSubsteps);
  }
  if (rc) {
    S->failed = true;
    return true;
  }
  for (size_t k = 0; k < F.rbs.size(); k++) {
    SScene& sc = S->scenes[rbWho[k].first];
    const int32_t buf = rbWho[k].second == 0 ? P4A_BUF_POS : P4A_BUF_VEL;
    void* src = nullptr;
    size_t bytes = 0;
    if (S->cfg.plain) {
      rc = p4a_buffer(sc.sim, buf, P4A_LIVE, &src, &bytes);
    } else {
      rc = scene_buffer(S->batch, S->batch->scenes[sc.slot], buf, P4A_LIVE, &src, &bytes);
    }
    if (rc == P4A_OK) cudaMemcpyAsync(F.rbs[k].pinned, src, F.rbs[k].bytes, cudaMemcpyDeviceToHost, S->stream);
  }
  if (!S->cfg.plain) cudaMemcpyAsync(S->errPinned, S->batch->d.errorWord, 4, cudaMemcpyDeviceToHost, S->stream);
  cudaEventRecord(F.done, S->stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err(S, "frame launch: %s", cudaGetErrorString(e));
    S->failed = true;
  }
  F.kernels = p4a_kernel_launches() - k0;
  for (int32_t h : hs) {
    SScene& sc = S->scenes[h];
    F.steps.emplace_back(h, sc.steps.front());
    F.particles.push_back(sc.n);
    sc.steps.pop_front();
    sc.lastSeq = F.seq;
  }
  S->inflight.push_back(std::move(F));
  return true;
}

bool retire(p4a_server* S) {
  bool progress = false;
  while (!S->inflight.empty()) {
    FrameRec& F = S->inflight.front();
    const cudaError_t q = cudaEventQuery(F.done);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) {
      set_err(S, "frame %llu: %s", (unsigned long long)F.seq, cudaGetErrorString(q));
      S->failed = true;
      return true;
    }
    const double t = S->now();
    float ms = 0;
    cudaEventElapsedTime(&ms, F.start, F.done);
    const bool deviceErr = !S->cfg.plain && !F.steps.empty() && *S->errPinned != 0u;
    for (Readback& r : F.rbs) {
      std::memcpy(r.dst, r.pinned, r.bytes);
      S->readbacks.put(r.pinned, r.bytes);
    }
    double ps = 0;
    for (size_t k = 0; k < F.steps.size(); k++) {
      const StepReq& q2 = F.steps[k].second;
      const size_t want = std::min((size_t)F.particles[k] * 16, q2.outBytes);
      const bool rbTooBig = (q2.pos || q2.vel) && want > S->readbacks.capacity();
      const int status = deviceErr ? P4A_ERR_TIMEOUT : rbTooBig ? P4A_ERR_CAPACITY : P4A_OK;
      post(S, completion(P4A_REQ_STEP, q2.id, F.steps[k].first, status, q2.tSubmit, F.tLaunch, t,
                         F.particles[k], F.substeps[k]));
      ps += (double)F.particles[k] * F.substeps[k];
    }
    for (int32_t h : F.primed) {
      SScene& sc = S->scenes[h];
      post(S, completion(P4A_REQ_CREATE, sc.createReq, h, P4A_OK, sc.tSubmit, F.tLaunch, t, sc.n));
    }
    for (auto& b : F.blobs) S->uploads.put(b.first, b.second);
    {
      std::lock_guard<std::mutex> l(S->mu);
      S->st.gpu_seconds += ms * 1e-3;
      S->st.kernel_launches += (int64_t)F.kernels;
      if (!F.steps.empty()) {
        S->st.frames++;
        S->stepFrames++;
        S->frameScenes += (double)F.steps.size();
        S->st.steps += (int64_t)F.steps.size();
        S->st.particle_substeps += ps;
        S->st.last_finish = t;
        for (auto& s : F.steps) S->stepMs.push_back((t - s.second.tSubmit) * 1e3);
      }
    }
    if (deviceErr) {
      set_err(S, "a bounded device wait gave up (cell scan)");
      S->failed = true;
    }
    S->doneSeq = F.seq;
    S->evPool.push_back(F.start);
    S->evPool.push_back(F.done);
    S->inflight.pop_front();
    progress = true;
  }
  return progress;
}

// Destroys take effect once a scene's earlier steps are done and its last frame
// has finished.
bool bury(p4a_server* S) {
  std::vector<int32_t> gone;
  for (auto& kv : S->scenes) {
    SScene& sc = kv.second;
    if (!sc.destroyWanted || sc.state != S_LIVE || !sc.steps.empty() || sc.lastSeq > S->doneSeq) continue;
    if (S->cfg.plain) {
      p4a_destroy(sc.sim);
      sc.sim = nullptr;
      S->plainScenes--;
      S->plainParticles -= sc.n;
    } else {
      release_scene(S->batch, S->batch->scenes[sc.slot]);
    }
    const double t = S->now();
    post(S, completion(P4A_REQ_DESTROY, sc.destroyReq, kv.first, P4A_OK, sc.tDestroy, t, t, sc.n));
    gone.push_back(kv.first);
  }
  for (int32_t h : gone) S->scenes.erase(h);
  if (!gone.empty()) {
    std::lock_guard<std::mutex> l(S->mu);
    S->st.destroyed += (int64_t)gone.size();
  }
  return !gone.empty();
}

void publish_counts(p4a_server* S) {
  int live = 0, ready = 0;
  for (auto& kv : S->scenes) {
    live += kv.second.state == S_LIVE ? 1 : 0;
    ready += kv.second.state == S_READY ? 1 : 0;
  }
  std::lock_guard<std::mutex> l(S->mu);
  S->st.live_scenes = live;
  S->st.queued_creates = ready;
  S->st.building = S->building;
  S->st.max_queued_creates = std::max(S->st.max_queued_creates, ready + S->building);
}

void engine_main(p4a_server* S) {
  cudaSetDevice(S->device);
  for (;;) {
    bool progress = false;
    std::vector<Req> in;
    {
      std::lock_guard<std::mutex> l(S->mu);
      in.swap(S->inbox);
    }
    for (Req& r : in) take_request(S, r);
    progress |= !in.empty();
    progress |= collect_built(S);
    progress |= retire(S);
    if (S->failed.load()) break;
    const bool stopping = S->stop.load();
    if (!stopping) {
      progress |= admit(S);
      progress |= launch(S);
    }
    progress |= bury(S);
    publish_counts(S);
    if (S->failed.load()) break;
    if (stopping && S->inflight.empty()) break;
    if (!progress) {
      if (!S->inflight.empty()) {
        // wait for the oldest frame, waking up now and then for new requests
        for (int k = 0; k < 20 && cudaEventQuery(S->inflight.front().done) == cudaErrorNotReady; k++)
          std::this_thread::sleep_for(std::chrono::microseconds(50));
      } else {
        std::this_thread::sleep_for(std::chrono::microseconds(200));
      }
    }
  }
  cudaStreamSynchronize(S->stream);
  if (S->up) cudaStreamSynchronize(S->up);
  while (!S->inflight.empty()) {
    FrameRec& F = S->inflight.front();
    for (Readback& r : F.rbs) S->readbacks.put(r.pinned, r.bytes);
    for (auto& b : F.blobs) S->uploads.put(b.first, b.second);
    S->evPool.push_back(F.start);
    S->evPool.push_back(F.done);
    S->inflight.pop_front();
  }
}

int submit(p4a_server* S, Req&& r, int64_t* request) {
  {
    std::lock_guard<std::mutex> l(S->mu);
    if (S->failed.load() || S->stop.load()) return P4A_ERR_STATE;
    r.id = S->nextReq++;
    r.t = S->now();
    if (r.kind == P4A_REQ_CREATE) {
      r.scene = S->nextScene++;
      S->st.creates++;
      if (S->st.first_submit == 0) S->st.first_submit = r.t;
    }
    if (request) *request = r.id;
    S->inbox.push_back(std::move(r));
  }
  return P4A_OK;
}

}  // namespace

extern "C" {

int p4a_server_default_config(p4a_server_config* c) {
  if (!c) return P4A_ERR_ARG;
  *c = p4a_server_config{};
  c->arenas.max_particles = 1 << 24;
  c->arenas.max_cells = 1 << 24;
  c->arenas.max_boundary = 1 << 23;
  c->arenas.max_scenes = 1024;
  c->arenas.max_bodies = 4096;
  c->arenas.max_body_parts = 1 << 22;
  c->builder_threads = 4;
  c->max_frames_in_flight = 2;
  c->admit_timeout = 0;
  c->max_pending_creates = 0;
  c->use_graphs = 1;
  c->plain = 0;
  c->upload_bytes = 1LL << 30;
  c->readback_bytes = 1LL << 30;
  c->frame_lanes = 2;
  c->lane_min_particles = 1000000;
  return P4A_OK;
}

int p4a_server_create(int device, const p4a_server_config* cfg, p4a_server** out) {
  if (!cfg || !out || cfg->builder_threads < 1 || cfg->arenas.max_scenes < 1 || cfg->upload_bytes < 4096 ||
      cfg->readback_bytes < 4096)
    return P4A_ERR_ARG;
  *out = nullptr;
  const int chk = p4a_device_check(device);
  if (chk != P4A_OK) return chk;
  if (cudaSetDevice(device) != cudaSuccess) return P4A_ERR_CUDA;
  std::unique_ptr<p4a_server> S(new p4a_server());
  S->device = device;
  S->cfg = *cfg;
  S->t0 = Clock::now();
  int rc;
  if (!cfg->plain) {
    if ((rc = p4a_batch_create(device, &cfg->arenas, &S->batch))) return rc;
    p4a_batch_use_graphs(S->batch, cfg->use_graphs);
    if ((rc = p4a_batch_set_lanes(S->batch, std::max(1, cfg->frame_lanes), cfg->lane_min_particles))) return rc;
    S->stream = S->batch->stream;
    if (cudaStreamCreateWithFlags(&S->up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->upEvent, cudaEventDisableTiming) != cudaSuccess) {
      p4a_batch_destroy(S->batch);
      return P4A_ERR_CUDA;
    }
  } else {
    if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess) return P4A_ERR_CUDA;
    S->ownStream = true;
  }
  if (cudaHostAlloc((void**)&S->errPinned, 16, cudaHostAllocDefault) != cudaSuccess ||
      (rc = S->uploads.init((size_t)cfg->upload_bytes)) || (rc = S->readbacks.init((size_t)cfg->readback_bytes))) {
    if (S->batch) p4a_batch_destroy(S->batch);
    if (S->up) cudaStreamDestroy(S->up);
    if (S->upEvent) cudaEventDestroy(S->upEvent);
    if (S->ownStream) cudaStreamDestroy(S->stream);
    if (S->errPinned) cudaFreeHost(S->errPinned);
    return P4A_ERR_OOM;
  }
  *S->errPinned = 0u;
  p4a_server* raw = S.release();
  for (int k = 0; k < cfg->builder_threads; k++) raw->builders.emplace_back(builder_main, raw);
  raw->engine = std::thread(engine_main, raw);
  *out = raw;
  return P4A_OK;
}

int p4a_server_destroy(p4a_server* S) {
  if (!S) return P4A_ERR_ARG;
  S->stop = true;
  S->bcv.notify_all();
  if (S->engine.joinable()) S->engine.join();
  for (auto& t : S->builders)
    if (t.joinable()) t.join();
  cudaSetDevice(S->device);
  for (auto& kv : S->scenes) {
    if (kv.second.sim) p4a_destroy(kv.second.sim);
    if (kv.second.blob) S->uploads.put(kv.second.blob, kv.second.blobBytes);
  }
  for (BuildResult& r : S->built)
    if (r.blob) S->uploads.put(r.blob, r.bytes);
  for (cudaEvent_t e : S->evPool) cudaEventDestroy(e);
  if (S->batch) p4a_batch_destroy(S->batch);
  if (S->up) cudaStreamDestroy(S->up);
  if (S->upEvent) cudaEventDestroy(S->upEvent);
  if (S->ownStream && S->stream) cudaStreamDestroy(S->stream);
  if (S->errPinned) cudaFreeHost(S->errPinned);
  delete S;
  return P4A_OK;
}

const char* p4a_server_last_error(const p4a_server* S) {
  if (!S) return "null handle";
  return S->err.c_str();
}

double p4a_server_clock(const p4a_server* S) { return S ? S->now() : 0.0; }

int p4a_server_create_scene(p4a_server* S, const p4a_params* params, const p4a_scene_desc* sd, int32_t* sceneId,
                            int64_t* request) {
  if (!S || !params || !sceneId || !(params->spacing > 0) || params->n_bodies < 0 ||
      (params->n_bodies > 0 && !params->bodies))
    return P4A_ERR_ARG;
  Req r;
  r.kind = P4A_REQ_CREATE;
  r.create.reset(new CreateReq());
  CreateReq& c = *r.create;
  c.params = *params;
  c.specs.assign(params->bodies, params->bodies + (params->bodies ? params->n_bodies : 0));
  c.params.bodies = nullptr;
  if (sd) {
    if (sd->n < 0 || (sd->n > 0 && !sd->pos) || sd->n_bodies < 0 ||
        (sd->n_bodies > 0 && (!sd->body_density || !sd->body_centre)))
      return P4A_ERR_ARG;
    const size_t n = (size_t)sd->n;
    c.scene.reset(new HostScene());
    HostScene& h = *c.scene;
    h.n = sd->n;
    h.d = params->spacing;
    h.h = 2 * params->spacing;
    h.pos.assign(sd->pos, sd->pos + n * 4);
    h.vel = sd->vel ? std::vector<float>(sd->vel, sd->vel + n * 4) : std::vector<float>(n * 4, 0.0f);
    h.rest = sd->rest ? std::vector<float>(sd->rest, sd->rest + n * 4) : std::vector<float>(n * 4, 0.0f);
    h.phase = sd->phase ? std::vector<uint32_t>(sd->phase, sd->phase + n * 4) : std::vector<uint32_t>(n * 4, 0u);
    int nFluid = 0;
    for (size_t i = 0; i < n; i++) {
      const uint32_t b = h.phase[i * 4];
      if (b == 0) nFluid++;
      else if ((int)b > sd->n_bodies) return P4A_ERR_ARG;
    }
    h.nFluid = nFluid;
    h.nBody = sd->n - nFluid;
    h.bodyDensity.assign(sd->body_density, sd->body_density + sd->n_bodies);
    h.bodyCentre.assign(sd->body_centre, sd->body_centre + 3 * (size_t)sd->n_bodies);
    h.mass = sd->mass;
    h.denomRest = sd->denom_rest;
    c.pourBudget = std::max(0, sd->pour_budget);
  }
  const int rc = submit(S, std::move(r), request);
  if (rc == P4A_OK) {
    std::lock_guard<std::mutex> l(S->mu);
    *sceneId = S->nextScene - 1;
  }
  return rc;
}

int p4a_server_step(p4a_server* S, int32_t sceneId, double frameDt, float* pos, float* vel, size_t outBytes,
                    int64_t* request) {
  if (!S || !(frameDt >= 0) || ((pos || vel) && outBytes == 0)) return P4A_ERR_ARG;
  Req r;
  r.kind = P4A_REQ_STEP;
  r.scene = sceneId;
  r.step.dt = frameDt;
  r.step.pos = pos;
  r.step.vel = vel;
  r.step.outBytes = (pos || vel) ? outBytes : 0;
  int rc;
  {
    std::lock_guard<std::mutex> l(S->mu);
    if (S->failed.load() || S->stop.load()) return P4A_ERR_STATE;
    r.id = S->nextReq++;
    r.t = S->now();
    r.step.id = r.id;
    r.step.tSubmit = r.t;
    if (request) *request = r.id;
    S->inbox.push_back(std::move(r));
    rc = P4A_OK;
  }
  return rc;
}

int p4a_server_destroy_scene(p4a_server* S, int32_t sceneId, int64_t* request) {
  if (!S) return P4A_ERR_ARG;
  Req r;
  r.kind = P4A_REQ_DESTROY;
  r.scene = sceneId;
  return submit(S, std::move(r), request);
}

int p4a_server_poll(p4a_server* S, p4a_completion* out, int32_t max, int32_t* count, double wait) {
  if (!S || !count || max < 0 || (max > 0 && !out)) return P4A_ERR_ARG;
  std::unique_lock<std::mutex> l(S->mu);
  if (S->done.empty() && wait > 0 && !S->failed.load())
    S->cvPoll.wait_for(l, std::chrono::duration<double>(wait), [&] { return !S->done.empty() || S->failed.load(); });
  int32_t c = 0;
  while (c < max && !S->done.empty()) {
    out[c++] = S->done.front();
    S->done.pop_front();
  }
  *count = c;
  return S->failed.load() && c == 0 ? P4A_ERR_CUDA : P4A_OK;
}

int p4a_server_get_stats(p4a_server* S, p4a_server_stats* out) {
  if (!S || !out) return P4A_ERR_ARG;
  std::lock_guard<std::mutex> l(S->mu);
  *out = S->st;
  out->step_p50_ms = quantile(S->stepMs, 0.50);
  out->step_p99_ms = quantile(S->stepMs, 0.99);
  double sum = 0, mx = 0;
  for (double v : S->stepMs) {
    sum += v;
    mx = std::max(mx, v);
  }
  out->step_mean_ms = S->stepMs.empty() ? 0 : sum / (double)S->stepMs.size();
  out->step_max_ms = mx;
  out->admit_p50_ms = quantile(S->admitMs, 0.50);
  out->admit_p99_ms = quantile(S->admitMs, 0.99);
  out->mean_frame_scenes = S->stepFrames ? S->frameScenes / (double)S->stepFrames : 0;
  return P4A_OK;
}

}  // extern "C"
