// cg_server.cu — the served form: render requests over resident scenes.
//
// A worker thread owns two pipelines ("lanes", each a Renderer with its own
// stream and ray queues).  Requests wait until their film plus their share of
// path state fits the HBM budget, then join the active set; both admission
// and dispatch go shortest first (fewest samples left), except that a request
// waiting longer than kAgingSeconds goes before every younger one, oldest
// first, so large requests are not starved.  Each idle lane gets one
// wavefront chunk for one scene: the scene of the first request in that
// order, filled with slices of that scene's active requests in the same
// order, so requests that arrive while others are on the GPU start with the
// next chunk and share the device with them (continuous batching); with two
// chunks in flight the host builds and retires chunks while the GPU stays
// busy.  A request finishes
// when its last pixel is resolved: the worker enqueues the film's copy into a
// pinned staging buffer (a copy-engine transfer, so it does not wait for SMs
// that the other lane's kernels hold) and goes on dispatching; a copy-out
// thread waits for that copy, packs it into the caller's buffer (whose page
// tables a prefault thread populated after the submit) and completes the
// request.
// Sample streams are keyed by (request seed, pixel, sample), so a result does
// not depend on the requests it was batched with.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cg_cuda.h"
#include "cg_api_internal.h"

namespace cg {
namespace {

double nowSeconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct ServerReq {
  uint64_t id = 0;
  cg_request req{};
  float* out = nullptr;
  double submit_s = 0, start_s = 0, finish_s = 0;
  int status = CG_OK;
  bool done = false, cancelled = false;
  uint32_t npx = 0, next_pixel = 0, resolved = 0;
  size_t bytes = 0;
  float4* film = nullptr;
};

}  // namespace
}  // namespace cg

// One pipeline of the server: its own stream and ray queues, the view table
// of the chunk it runs, and the event that marks the chunk's end.  Two lanes
// keep the device busy while the host retires one chunk and builds the next,
// and let two chunks (of the same or different scenes) share the GPU.
struct ServerLane {
  cg::Renderer rend;
  cg::ViewDev* table = nullptr;
  size_t table_cap = 0;
  std::vector<cg::ViewDev> slices;
  std::vector<cg::ServerReq*> slice_req;
  uint32_t used = 0;
  bool busy = false;
  uint32_t* status_host = nullptr;  // pinned: the chunk's status word
  cudaEvent_t done = nullptr;
  ~ServerLane() {
    if (done) cudaEventDestroy(done);
    if (status_host) cudaFreeHost(status_host);
    if (table) cudaFree(table);
  }
};

struct StagingBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool busy = false;
};

// A finished film on its way to the caller: its pinned staging buffer, the
// event after its device-to-host copy.
struct CopyJob {
  cg::ServerReq* r = nullptr;
  StagingBuf* buf = nullptr;
  cudaEvent_t ev = nullptr;
};

struct cg_server_s {
  static constexpr int kLanes = 2;
  std::vector<cg::SceneDev*> scenes;
  uint64_t budget = 0;
  ServerLane lanes[kLanes];
  cudaStream_t alloc_stream = nullptr;  // film allocations (synchronised before use)
  cg_conf conf{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<cg::ServerReq*> pending;
  std::vector<cg::ServerReq*> active;
  std::unordered_map<uint64_t, std::unique_ptr<cg::ServerReq>> reqs;
  bool stop = false;
  int fatal = CG_OK;
  std::string fatal_msg;
  uint64_t next_id = 1;
  cg_server_stats st{};
  // copy-out thread and its queue; staging buffers and events are reused
  std::thread copier;
  std::mutex copy_mu;
  std::condition_variable copy_cv;
  std::deque<CopyJob> copy_q;
  bool copy_stop = false;
  std::vector<cudaEvent_t> free_events;  // guarded by copy_mu
  // prefault thread: populates each submitted film buffer while the GPU works
  std::thread prefaulter;
  std::mutex pf_mu;
  std::condition_variable pf_cv;
  std::deque<std::pair<void*, size_t>> pf_q;
  bool pf_stop = false;
  ~cg_server_s() {
    for (cudaEvent_t e : free_events) cudaEventDestroy(e);
    if (alloc_stream) cudaStreamDestroy(alloc_stream);
  }
};

namespace cg {
namespace {

// Film bytes plus the path state the request can occupy in one chunk.
size_t requestBytes(const cg_server_s& sv, const SceneDev& scene, const cg_request& r) {
  const size_t npx = size_t(r.view.width) * r.view.height;
  const LevelPlan plan = planLevels(capsOf(sv.conf), std::max(1u, scene.max_lobes));
  const size_t per_sample = 12 + plan.max_product * (36 + 20 + 36);
  const size_t samples =
      std::min<size_t>(npx * r.view.spp, sv.lanes[0].rend.chunkSamples(scene, capsOf(sv.conf)));
  return npx * 16 + samples * per_sample;
}

void finishRequest(cg_server_s& sv, ServerReq* r, int status) {
  r->status = status;
  r->finish_s = nowSeconds();
  r->done = true;
  sv.st.bytes_in_use -= r->bytes;
  if (status == CG_OK)
    ++sv.st.completed;
  else if (status == CG_E_CANCELLED)
    ++sv.st.cancelled;
}

// Scheduling order (admission and dispatch): a request that has waited
// longer than this since its submit goes before every younger one, the oldest
// first; the others go shortest first (fewest samples left to schedule), the
// older first among equals.  Shortest first finishes the many small requests
// of a mixed stream early (lower median latency than first come, first
// served, at the same throughput); the aging bound keeps the tail finite when
// small requests keep arriving.
constexpr double kAgingSeconds = 1.0;

uint64_t samplesLeft(const ServerReq* r) {
  return uint64_t(r->npx - r->next_pixel) * r->req.view.spp;
}

// True when a goes before b.
bool schedulesBefore(const ServerReq* a, const ServerReq* b, double now) {
  const bool aged_a = now - a->submit_s > kAgingSeconds, aged_b = now - b->submit_s > kAgingSeconds;
  if (aged_a != aged_b) return aged_a;
  if (aged_a) return a->id < b->id;
  const uint64_t la = samplesLeft(a), lb = samplesLeft(b);
  if (la != lb) return la < lb;
  return a->id < b->id;
}

// Builds one chunk in `lane` for the scene of the first request in
// scheduling order, filled with that scene's requests in the same order.
// Returns false when no request has pixels left to schedule.
bool buildChunk(cg_server_s* sv, ServerLane& lane, const Caps& caps, SceneDev*& scene_out,
                ChunkDesc& ch) {
  std::vector<ServerReq*> order;
  for (ServerReq* r : sv->active)
    if (!r->cancelled && r->next_pixel < r->npx) order.push_back(r);
  if (order.empty()) return false;
  const double now = nowSeconds();
  std::sort(order.begin(), order.end(),
            [now](const ServerReq* a, const ServerReq* b) { return schedulesBefore(a, b, now); });
  const uint32_t scene_idx = order.front()->req.scene;
  SceneDev& scene = *sv->scenes[scene_idx];
  const uint32_t cap = lane.rend.chunkSamples(scene, caps);
  lane.slices.clear();
  lane.slice_req.clear();
  uint32_t used = 0;
  auto take = [&](ServerReq* r, uint32_t budget_samples) {
    const uint32_t spp = r->req.view.spp;
    uint32_t px = std::min<uint32_t>(budget_samples / spp, r->npx - r->next_pixel);
    px = std::min<uint32_t>(px, (cap - used) / spp);
    if (px == 0) return;
    ViewDev v;
    std::memset(&v, 0, sizeof(v));
    cameraBasis(r->req.view.camera, v);
    v.width = r->req.view.width;
    v.height = r->req.view.height;
    v.spp = spp;
    v.seed = r->req.view.seed;
    v.frame = 0;
    v.sample_weight = 1.0f;
    v.pixel_base = r->next_pixel;
    v.pixel_count = px;
    v.film = r->film;
    v.rgba = nullptr;
    lane.slices.push_back(v);
    lane.slice_req.push_back(r);
    r->next_pixel += px;
    used += px * spp;
  };
  for (ServerReq* r : order)
    if (r->req.scene == scene_idx) take(r, cap);
  layoutViews(lane.slices);
  ch = ChunkDesc{0, 0, used, 0};
  for (const ViewDev& v : lane.slices) ch.pixel_count += v.pixel_count;
  lane.used = used;
  scene_out = &scene;
  return true;
}

// Enqueues the lane's chunk: view table upload, the kernel sequence, the
// status word read into pinned memory, the completion event.
int enqueueLane(ServerLane& lane, SceneDev& scene, const ChunkDesc& ch, const Caps& caps) {
  if (lane.slices.size() > lane.table_cap) {
    if (lane.table) cudaFree(lane.table);
    lane.table = nullptr;
    lane.table_cap = 0;
    if (cudaMalloc(&lane.table, lane.slices.size() * 2 * sizeof(ViewDev)) != cudaSuccess) {
      cudaGetLastError();
      return CG_E_OOM;
    }
    lane.table_cap = lane.slices.size() * 2;
  }
  cudaStream_t s = lane.rend.stream;
  if (cudaMemcpyAsync(lane.table, lane.slices.data(), lane.slices.size() * sizeof(ViewDev),
                      cudaMemcpyHostToDevice, s) != cudaSuccess)
    return CG_E_CUDA;
  RenderRecord rec;
  lane.rend.enqueueChunk(scene, static_cast<uint32_t>(lane.slices.size()), lane.table, ch, caps, s,
                         rec);
  if (cudaGetLastError() != cudaSuccess) return CG_E_CUDA;
  if (cudaMemcpyAsync(lane.status_host, lane.rend.wave.status, 4, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaEventRecord(lane.done, s) != cudaSuccess)
    return CG_E_CUDA;
  return CG_OK;
}

// Pinned staging buffers shared by every server of the process.  Pinning
// fresh memory zeroes and locks new pages, which on a busy host can take
// seconds for a burst of films; a server created later reuses the buffers
// instead.  Portable, so a server on any device can copy into them.
// cg_term frees the buffers no server holds.
struct StagingPool {
  std::mutex mu;
  std::vector<std::unique_ptr<StagingBuf>> bufs;
};
StagingPool& stagingPool() {
  static StagingPool pool;
  return pool;
}

// A free pinned staging buffer of at least `bytes` (the smallest that fits,
// allocated in whole MiB if none does), or null.
StagingBuf* takeStagingBuf(size_t bytes) {
  StagingPool& pool = stagingPool();
  std::lock_guard<std::mutex> lk(pool.mu);
  StagingBuf* best = nullptr;
  for (auto& b : pool.bufs)
    if (!b->busy && b->bytes >= bytes && (!best || b->bytes < best->bytes)) best = b.get();
  if (!best) {
    auto b = std::make_unique<StagingBuf>();
    const size_t size = (bytes + (size_t(1) << 20) - 1) & ~((size_t(1) << 20) - 1);
    if (cudaHostAlloc(&b->p, size, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    b->bytes = size;
    best = b.get();
    pool.bufs.push_back(std::move(b));
  }
  best->busy = true;
  return best;
}

void giveStagingBuf(StagingBuf* b) {
  std::lock_guard<std::mutex> lk(stagingPool().mu);
  b->busy = false;
}

// A staging buffer of at least `bytes` and an event; false if pinned memory
// or the event cannot be had.
bool takeStaging(cg_server_s* sv, size_t bytes, StagingBuf*& buf, cudaEvent_t& ev) {
  std::lock_guard<std::mutex> lk(sv->copy_mu);
  if (sv->free_events.empty()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    sv->free_events.push_back(e);
  }
  buf = takeStagingBuf(bytes);
  if (!buf) return false;
  ev = sv->free_events.back();
  sv->free_events.pop_back();
  return true;
}

constexpr int kCopyThreads = 4;

void copyLoop(cg_server_s* sv, int device) {
  cudaSetDevice(device);
  while (true) {
    CopyJob job;
    const void* src = nullptr;
    {
      std::unique_lock<std::mutex> lk(sv->copy_mu);
      sv->copy_cv.wait(lk, [&] { return sv->copy_stop || !sv->copy_q.empty(); });
      if (sv->copy_q.empty()) break;
      job = sv->copy_q.front();
      sv->copy_q.pop_front();
      src = job.buf->p;
    }
    const double t0 = nowSeconds();
    int st = CG_OK;
    if (cudaEventSynchronize(job.ev) != cudaSuccess) {
      cudaGetLastError();
      st = CG_E_CUDA;
    } else {
      // float4 -> three floats per pixel; large films are packed by
      // kCopyThreads threads (this one and helpers), so one slow core on a
      // busy host does not hold the request back
      const size_t npx = job.r->npx;
      float* dst = job.r->out;
      const float* from = static_cast<const float*>(src);
      auto pack = [dst, from](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
          dst[3 * i] = from[4 * i];
          dst[3 * i + 1] = from[4 * i + 1];
          dst[3 * i + 2] = from[4 * i + 2];
        }
      };
      const int parts = npx >= (size_t(1) << 18) ? kCopyThreads : 1;
      const size_t step = (npx + parts - 1) / parts;
      std::thread helpers[kCopyThreads];
      for (int k = 1; k < parts; ++k) {
        const size_t b = std::min(npx, step * k), e = std::min(npx, step * (k + 1));
        if (e > b) helpers[k] = std::thread(pack, b, e);
      }
      pack(0, std::min(npx, step));
      for (int k = 1; k < parts; ++k)
        if (helpers[k].joinable()) helpers[k].join();
    }
    giveStagingBuf(job.buf);
    {
      std::lock_guard<std::mutex> lk(sv->copy_mu);
      sv->free_events.push_back(job.ev);
    }
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->st.copy_out_s += nowSeconds() - t0;
      finishRequest(*sv, job.r, st);
    }
    sv->done_cv.notify_all();
    sv->cv.notify_all();  // its memory may let the worker admit a waiting request
  }
}

void prefaultLoop(cg_server_s* sv) {
  while (true) {
    std::pair<void*, size_t> job;
    {
      std::unique_lock<std::mutex> lk(sv->pf_mu);
      sv->pf_cv.wait(lk, [&] { return sv->pf_stop || !sv->pf_q.empty(); });
      if (sv->pf_stop) break;
      job = sv->pf_q.front();
      sv->pf_q.pop_front();
    }
    prefaultHostBuffer(job.first, job.second);
  }
}

}  // namespace

void releaseIdleStaging() {
  StagingPool& pool = stagingPool();
  std::lock_guard<std::mutex> lk(pool.mu);
  for (auto it = pool.bufs.begin(); it != pool.bufs.end();) {
    if (!(*it)->busy) {
      cudaFreeHost((*it)->p);
      it = pool.bufs.erase(it);
    } else {
      ++it;
    }
  }
}

namespace {

void failAll(cg_server_s* sv, int rc, const char* msg) {
  sv->fatal = rc;
  sv->fatal_msg = msg;
  for (ServerReq* r : sv->active) finishRequest(*sv, r, rc);
  sv->active.clear();
  for (ServerReq* r : sv->pending) finishRequest(*sv, r, rc);
  sv->pending.clear();
  sv->done_cv.notify_all();
}

void serverLoop(cg_server_s* sv) {
  cudaSetDevice(sv->lanes[0].rend.device);
  const Caps caps = capsOf(sv->conf);
  double busy_since = 0.0;  // start of the current stretch with a chunk in flight
  double all_since = 0.0;   // start of the current stretch with every lane busy
  std::unique_lock<std::mutex> lk(sv->mu);
  while (true) {
    // ---- admission under the HBM budget, in scheduling order ----
    while (!sv->pending.empty()) {
      auto pick = sv->pending.begin();
      const double now = nowSeconds();
      for (auto it = sv->pending.begin(); it != sv->pending.end(); ++it)
        if ((*it)->cancelled || schedulesBefore(*it, *pick, now)) {
          pick = it;
          if ((*it)->cancelled) break;
        }
      ServerReq* r = *pick;
      if (r->cancelled) {
        sv->pending.erase(pick);
        r->bytes = 0;
        finishRequest(*sv, r, CG_E_CANCELLED);
        sv->done_cv.notify_all();
        continue;
      }
      if (sv->st.bytes_in_use + r->bytes > sv->budget) {
        // wait for memory held by active requests or films being copied out
        // (the first request in order keeps its place, so it is not passed
        // over for ever by smaller ones)
        if (r->bytes <= sv->budget && sv->st.bytes_in_use > 0) break;
        sv->pending.erase(pick);  // can never fit
        r->bytes = 0;
        ++sv->st.rejected;
        finishRequest(*sv, r, CG_E_OOM);
        sv->done_cv.notify_all();
        continue;
      }
      sv->pending.erase(pick);
      const size_t fb = size_t(r->npx) * 16;
      void* film = nullptr;
      if (cudaMallocAsync(&film, fb, sv->alloc_stream) != cudaSuccess ||
          cudaStreamSynchronize(sv->alloc_stream) != cudaSuccess) {
        cudaGetLastError();
        r->bytes = 0;
        ++sv->st.rejected;
        finishRequest(*sv, r, CG_E_OOM);
        sv->done_cv.notify_all();
        continue;
      }
      r->film = static_cast<float4*>(film);
      r->start_s = nowSeconds();
      sv->st.bytes_in_use += r->bytes;
      sv->st.peak_bytes = std::max(sv->st.peak_bytes, sv->st.bytes_in_use);
      sv->active.push_back(r);
    }
    sv->st.active = static_cast<uint32_t>(sv->active.size());
    sv->st.pending = static_cast<uint32_t>(sv->pending.size());
    // ---- dispatch a chunk to every idle lane while there is work ----
    const bool was_busy = std::any_of(std::begin(sv->lanes), std::end(sv->lanes),
                                      [](const ServerLane& l) { return l.busy; });
    for (ServerLane& lane : sv->lanes) {
      if (lane.busy) continue;
      SceneDev* scene = nullptr;
      ChunkDesc ch{};
      if (!buildChunk(sv, lane, caps, scene, ch)) break;
      const int rc = enqueueLane(lane, *scene, ch, caps);
      if (rc != CG_OK) {
        failAll(sv, rc, "CUDA failure in the server loop");
        return;
      }
      lane.busy = true;
      ++sv->st.chunks;
      if (!was_busy && busy_since == 0.0) busy_since = nowSeconds();
    }
    if (all_since == 0.0 && std::all_of(std::begin(sv->lanes), std::end(sv->lanes),
                                        [](const ServerLane& l) { return l.busy; }))
      all_since = nowSeconds();
    const bool any_busy = std::any_of(std::begin(sv->lanes), std::end(sv->lanes),
                                      [](const ServerLane& l) { return l.busy; });
    if (!any_busy) {
      // nothing in flight: retire requests that were cancelled before they ran
      bool any = false;
      for (auto it = sv->active.begin(); it != sv->active.end();) {
        ServerReq* r = *it;
        if (r->cancelled && r->resolved == r->next_pixel) {
          cudaFreeAsync(r->film, sv->alloc_stream);
          r->film = nullptr;
          finishRequest(*sv, r, CG_E_CANCELLED);
          it = sv->active.erase(it);
          any = true;
        } else {
          ++it;
        }
      }
      if (any) {
        cudaStreamSynchronize(sv->alloc_stream);
        sv->done_cv.notify_all();
        continue;
      }
      if (sv->stop && sv->active.empty()) break;
      // idle (or only requests waiting for memory): sleep until a submit,
      // cancel or shutdown; the timeout re-checks in case a wake-up raced
      sv->cv.wait_for(lk, std::chrono::milliseconds(50));
      continue;
    }
    // ---- retire the first chunk to finish (a lane whose chunk is done must
    // not wait for a longer chunk on the other lane) ----
    lk.unlock();
    ServerLane* fin = nullptr;  // a lane whose chunk is done
    bool ok = true;
    while (!fin) {
      for (ServerLane& lane : sv->lanes) {  // `busy` is only written by this thread
        if (!lane.busy) continue;
        const cudaError_t e = cudaEventQuery(lane.done);
        if (e == cudaErrorNotReady) continue;
        ok = e == cudaSuccess;
        fin = &lane;
        break;
      }
      if (!fin) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    lk.lock();
    fin->busy = false;
    if (all_since != 0.0) {
      sv->st.all_busy_s += nowSeconds() - all_since;
      all_since = 0.0;
    }
    if (std::none_of(std::begin(sv->lanes), std::end(sv->lanes),
                     [](const ServerLane& l) { return l.busy; })) {
      sv->st.busy_s += nowSeconds() - busy_since;
      busy_since = 0.0;
    }
    if (!ok || *fin->status_host) {
      cudaGetLastError();
      failAll(sv, ok ? CG_E_DEVICE : CG_E_CUDA,
              ok ? "kernel status word set (stack or queue overflow)" : "CUDA failure in the server loop");
      return;
    }
    sv->st.samples += fin->used;
    for (size_t k = 0; k < fin->slice_req.size(); ++k)
      fin->slice_req[k]->resolved += fin->slices[k].pixel_count;
    bool any = false;
    cudaStream_t s = fin->rend.stream;
    for (auto it = sv->active.begin(); it != sv->active.end();) {
      ServerReq* r = *it;
      const bool complete = r->resolved == r->npx;
      if (complete || (r->cancelled && r->resolved == r->next_pixel)) {
        int st = CG_E_CANCELLED;
        if (complete && !r->cancelled) {
          // one contiguous copy of the float4 film into pinned staging; the
          // copy-out thread packs it and completes the request
          StagingBuf* buf = nullptr;
          cudaEvent_t ev = nullptr;
          const size_t bytes = size_t(r->npx) * 16;
          st = CG_E_OOM;
          if (takeStaging(sv, bytes, buf, ev)) {
            const bool queued =
                cudaMemcpyAsync(buf->p, r->film, bytes, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                cudaEventRecord(ev, s) == cudaSuccess;
            if (!queued) {
              cudaGetLastError();
              giveStagingBuf(buf);
            }
            std::lock_guard<std::mutex> clk(sv->copy_mu);
            if (queued) {
              sv->copy_q.push_back(CopyJob{r, buf, ev});
              sv->copy_cv.notify_one();
              st = CG_OK;
            } else {
              sv->free_events.push_back(ev);
              st = CG_E_CUDA;
            }
          }
        }
        cudaFreeAsync(r->film, s);  // after the copy in stream order
        r->film = nullptr;
        if (st != CG_OK) finishRequest(*sv, r, st);  // else the copy-out thread does
        it = sv->active.erase(it);
        any = true;
      } else {
        ++it;
      }
    }
    if (any) sv->done_cv.notify_all();
  }
}

}  // namespace
}  // namespace cg

using namespace cg;

extern "C" {

CG_API int cg_server_create(const cg_scene_t* scenes, uint32_t scene_count, uint64_t hbm_budget_bytes,
                            cg_server_t* out) {
  return guarded([&]() -> int {
    if (!scenes || scene_count == 0 || !out) return fail(CG_E_INVALID, "null argument");
    *out = nullptr;
    cg_conf conf;
    cg_tuning tuning;
    int device = 0;
    bool hero = false;
    uint32_t roulette = 0;
    {
      std::lock_guard<std::mutex> lk(g_env_mu);
      if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
      conf = g_env->conf;
      tuning = g_env->tuning;
      device = g_env->device;
      hero = g_env->spectral == CG_SPECTRAL_HERO;
      roulette = g_env->roulette;
    }
    for (uint32_t i = 0; i < scene_count; ++i)
      if (!scenes[i]) return fail(CG_E_INVALID, "null scene");
    auto sv = std::make_unique<cg_server_s>();
    for (uint32_t i = 0; i < scene_count; ++i) sv->scenes.push_back(reinterpret_cast<SceneDev*>(scenes[i]));
    sv->budget = hbm_budget_bytes;
    sv->conf = conf;
    for (ServerLane& lane : sv->lanes) {
      lane.rend.tuning = tuning;
      lane.rend.hero = hero;
      lane.rend.roulette = roulette;
      int rc = lane.rend.init(device);
      if (rc != CG_OK) return rc;
      rc = lane.rend.ensureWave(tuning.queue_capacity);
      if (rc != CG_OK) return rc;
      if (cudaMallocHost(&lane.status_host, sizeof(uint32_t)) != cudaSuccess ||
          cudaEventCreateWithFlags(&lane.done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return fail(CG_E_CUDA, "server lane setup failed");
      }
      *lane.status_host = 0u;
    }
    if (cudaStreamCreateWithFlags(&sv->alloc_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return fail(CG_E_CUDA, "server stream setup failed");
    }
    sv->worker = std::thread(serverLoop, sv.get());
    sv->copier = std::thread(copyLoop, sv.get(), device);
    sv->prefaulter = std::thread(prefaultLoop, sv.get());
    *out = sv.release();
    return CG_OK;
  });
}

CG_API int cg_server_destroy(cg_server_t server) {
  return guarded([&]() -> int {
    if (!server) return CG_OK;
    {
      std::lock_guard<std::mutex> lk(server->mu);
      for (ServerReq* r : server->pending) r->cancelled = true;
      for (ServerReq* r : server->active) r->cancelled = true;
      server->stop = true;
    }
    server->cv.notify_all();
    if (server->worker.joinable()) server->worker.join();
    {
      std::lock_guard<std::mutex> lk(server->copy_mu);
      server->copy_stop = true;  // the copier drains its queue first
    }
    server->copy_cv.notify_all();
    if (server->copier.joinable()) server->copier.join();
    {
      std::lock_guard<std::mutex> lk(server->pf_mu);
      server->pf_stop = true;  // buffers not yet populated are simply written later
    }
    server->pf_cv.notify_all();
    if (server->prefaulter.joinable()) server->prefaulter.join();
    delete server;
    return CG_OK;
  });
}

CG_API int cg_server_submit(cg_server_t server, const cg_request* request, float* film_xyz,
                            uint64_t* request_id) {
  return guarded([&]() -> int {
    if (!server || !request || !film_xyz) return fail(CG_E_INVALID, "null argument");
    const cg_view_desc& v = request->view;
    if (request->scene >= server->scenes.size()) return fail(CG_E_INVALID, "scene index out of range");
    if (v.width == 0 || v.height == 0 || v.spp == 0) return fail(CG_E_INVALID, "zero size or spp");
    SceneDev& scene = *server->scenes[request->scene];
    if (v.spp > server->lanes[0].rend.chunkSamples(scene, capsOf(server->conf)))
      return fail(CG_E_INVALID, "spp exceeds the wavefront chunk");
    if (uint64_t(v.width) * v.height > 0xffffffffull)
      return fail(CG_E_INVALID, "view has more than 2^32 - 1 pixels");
    auto r = std::make_unique<ServerReq>();
    r->req = *request;
    r->out = film_xyz;
    r->npx = v.width * v.height;
    r->submit_s = nowSeconds();
    r->bytes = requestBytes(*server, scene, *request);
    std::lock_guard<std::mutex> lk(server->mu);
    if (server->fatal != CG_OK) return fail(server->fatal, server->fatal_msg);
    if (server->stop) return fail(CG_E_INVALID, "server is shutting down");
    r->id = server->next_id++;
    if (request_id) *request_id = r->id;
    server->pending.push_back(r.get());
    {
      std::lock_guard<std::mutex> plk(server->pf_mu);
      server->pf_q.emplace_back(film_xyz, size_t(r->npx) * 12);
    }
    server->pf_cv.notify_one();
    server->reqs[r->id] = std::move(r);
    ++server->st.submitted;
    server->cv.notify_all();
    return CG_OK;
  });
}

CG_API int cg_server_wait(cg_server_t server, uint64_t request_id, int timeout_ms,
                          cg_request_result* result) {
  return guarded([&]() -> int {
    if (!server) return fail(CG_E_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(server->mu);
    auto it = server->reqs.find(request_id);
    if (it == server->reqs.end()) return fail(CG_E_INVALID, "unknown request id");
    ServerReq* r = it->second.get();
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0)
      server->done_cv.wait(lk, pred);
    else if (!server->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
      return fail(CG_E_TIMEOUT, "request not finished within the timeout");
    if (result) {
      result->status = r->status;
      result->submit_s = r->submit_s;
      result->start_s = r->start_s;
      result->finish_s = r->finish_s;
    }
    const int st = r->status;
    server->reqs.erase(it);
    if (st != CG_OK) return fail(st, st == CG_E_CANCELLED ? "request cancelled" : "request failed");
    return CG_OK;
  });
}

CG_API int cg_server_cancel(cg_server_t server, uint64_t request_id) {
  return guarded([&]() -> int {
    if (!server) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(server->mu);
    auto it = server->reqs.find(request_id);
    if (it == server->reqs.end()) return fail(CG_E_INVALID, "unknown request id");
    it->second->cancelled = true;
    server->cv.notify_all();
    return CG_OK;
  });
}

CG_API int cg_server_get_stats(cg_server_t server, cg_server_stats* out) {
  return guarded([&]() -> int {
    if (!server || !out) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(server->mu);
    *out = server->st;
    return CG_OK;
  });
}

}  // extern "C"
