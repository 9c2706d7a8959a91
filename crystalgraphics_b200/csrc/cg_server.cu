// cg_server.cu — the served form: render requests over resident scenes.
//
// A worker thread owns one Renderer (stream, ray queues).  Requests wait in
// a FIFO until their film plus their share of path state fits the HBM budget,
// then join the active set.  Every loop iteration builds one wavefront chunk
// for one scene out of slices of all its active requests (each gets an equal
// share of the chunk, the rest is filled first-come first-served), so
// requests that arrive while others are on the GPU start with the next chunk
// and share the device with them (continuous batching).  A request finishes
// when its last pixel is resolved; its film is copied out and its memory
// released.  Sample streams are keyed by (request seed, pixel, sample), so a
// result does not depend on the requests it was batched with.
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

struct cg_server_s {
  std::vector<cg::SceneDev*> scenes;
  uint64_t budget = 0;
  cg::Renderer rend;
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
  uint32_t rr = 0;
  cg::ViewDev* table = nullptr;
  size_t table_cap = 0;
  std::vector<cg::ViewDev> slices;
  std::vector<cg::ServerReq*> slice_req;
};

namespace cg {
namespace {

// Film bytes plus the path state the request can occupy in one chunk.
size_t requestBytes(const cg_server_s& sv, const SceneDev& scene, const cg_request& r) {
  const size_t npx = size_t(r.view.width) * r.view.height;
  const LevelPlan plan = planLevels(capsOf(sv.conf), std::max(1u, scene.max_lobes));
  const size_t per_sample = 12 + plan.max_product * (36 + 20 + 36);
  const size_t samples = std::min<size_t>(npx * r.view.spp, sv.rend.chunkSamples(scene, capsOf(sv.conf)));
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

void serverLoop(cg_server_s* sv) {
  cudaSetDevice(sv->rend.device);
  const Caps caps = capsOf(sv->conf);
  std::unique_lock<std::mutex> lk(sv->mu);
  while (true) {
    // ---- admission (FIFO under the HBM budget) ----
    while (!sv->pending.empty()) {
      ServerReq* r = sv->pending.front();
      if (r->cancelled) {
        sv->pending.pop_front();
        r->bytes = 0;
        finishRequest(*sv, r, CG_E_CANCELLED);
        sv->done_cv.notify_all();
        continue;
      }
      if (sv->st.bytes_in_use + r->bytes > sv->budget) {
        if (!sv->active.empty()) break;  // wait for memory to free up
        sv->pending.pop_front();         // can never fit
        r->bytes = 0;
        ++sv->st.rejected;
        finishRequest(*sv, r, CG_E_OOM);
        sv->done_cv.notify_all();
        continue;
      }
      sv->pending.pop_front();
      const size_t fb = size_t(r->npx) * 16;
      void* film = nullptr;
      if (cudaMallocAsync(&film, fb, sv->rend.stream) != cudaSuccess) {
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
    if (sv->active.empty()) {
      if (sv->stop) break;
      sv->cv.wait(lk);
      continue;
    }
    // ---- one chunk for one scene, round robin over scenes with work ----
    uint32_t scene_idx = UINT32_MAX;
    for (uint32_t k = 0; k < sv->scenes.size() && scene_idx == UINT32_MAX; ++k) {
      const uint32_t s = (sv->rr + k) % static_cast<uint32_t>(sv->scenes.size());
      for (ServerReq* r : sv->active)
        if (r->req.scene == s && !r->cancelled && r->next_pixel < r->npx) {
          scene_idx = s;
          break;
        }
    }
    if (scene_idx == UINT32_MAX) {  // only cancelled requests left
      for (ServerReq* r : sv->active) {
        cudaFreeAsync(r->film, sv->rend.stream);
        finishRequest(*sv, r, CG_E_CANCELLED);
      }
      sv->active.clear();
      cudaStreamSynchronize(sv->rend.stream);
      sv->done_cv.notify_all();
      continue;
    }
    sv->rr = scene_idx + 1;
    SceneDev& scene = *sv->scenes[scene_idx];
    const uint32_t cap = sv->rend.chunkSamples(scene, caps);
    std::vector<ServerReq*> mine;
    for (ServerReq* r : sv->active)
      if (r->req.scene == scene_idx && !r->cancelled && r->next_pixel < r->npx) mine.push_back(r);
    const uint32_t share = std::max<uint32_t>(1u, cap / static_cast<uint32_t>(mine.size()));
    sv->slices.clear();
    sv->slice_req.clear();
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
      sv->slices.push_back(v);
      sv->slice_req.push_back(r);
      r->next_pixel += px;
      used += px * spp;
    };
    for (ServerReq* r : mine) take(r, share);
    for (ServerReq* r : mine) take(r, cap);
    layoutViews(sv->slices);
    ChunkDesc ch{0, 0, used, 0};
    for (const ViewDev& v : sv->slices) ch.pixel_count += v.pixel_count;
    lk.unlock();
    // ---- run it ----
    int rc = CG_OK;
    if (sv->slices.size() > sv->table_cap) {
      if (sv->table) cudaFree(sv->table);
      sv->table = nullptr;
      sv->table_cap = 0;
      if (cudaMalloc(&sv->table, sv->slices.size() * 2 * sizeof(ViewDev)) == cudaSuccess)
        sv->table_cap = sv->slices.size() * 2;
      else
        rc = CG_E_OOM;
    }
    RenderRecord rec;
    if (rc == CG_OK &&
        cudaMemcpyAsync(sv->table, sv->slices.data(), sv->slices.size() * sizeof(ViewDev),
                        cudaMemcpyHostToDevice, sv->rend.stream) != cudaSuccess)
      rc = CG_E_CUDA;
    if (rc == CG_OK) {
      sv->rend.enqueueChunk(scene, static_cast<uint32_t>(sv->slices.size()), sv->table, ch, caps,
                            sv->rend.stream, rec);
      if (cudaGetLastError() != cudaSuccess) rc = CG_E_CUDA;
    }
    uint32_t status = 0;
    if (rc == CG_OK &&
        (cudaMemcpyAsync(&status, sv->rend.wave.status, 4, cudaMemcpyDeviceToHost, sv->rend.stream) !=
             cudaSuccess ||
         cudaStreamSynchronize(sv->rend.stream) != cudaSuccess))
      rc = CG_E_CUDA;
    if (rc == CG_OK && status) rc = CG_E_DEVICE;
    lk.lock();
    if (rc != CG_OK) {
      sv->fatal = rc;
      sv->fatal_msg = rc == CG_E_DEVICE ? "kernel status word set (stack or queue overflow)"
                                        : "CUDA failure in the server loop";
      for (ServerReq* r : sv->active) finishRequest(*sv, r, rc);
      sv->active.clear();
      for (ServerReq* r : sv->pending) finishRequest(*sv, r, rc);
      sv->pending.clear();
      sv->done_cv.notify_all();
      break;
    }
    sv->st.samples += used;
    // ---- completions ----
    for (size_t k = 0; k < sv->slice_req.size(); ++k) sv->slice_req[k]->resolved += sv->slices[k].pixel_count;
    bool any = false;
    for (auto it = sv->active.begin(); it != sv->active.end();) {
      ServerReq* r = *it;
      const bool complete = r->resolved == r->npx;
      if (complete || (r->cancelled && r->resolved == r->next_pixel)) {
        int st = CG_E_CANCELLED;
        if (complete && !r->cancelled) {
          st = cudaMemcpy2DAsync(r->out, 12, r->film, 16, 12, r->npx, cudaMemcpyDeviceToHost,
                                 sv->rend.stream) == cudaSuccess
                   ? CG_OK
                   : CG_E_CUDA;
        }
        cudaFreeAsync(r->film, sv->rend.stream);
        r->film = nullptr;
        cudaStreamSynchronize(sv->rend.stream);
        finishRequest(*sv, r, st);
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
  if (!scenes || scene_count == 0 || !out) return fail(CG_E_INVALID, "null argument");
  *out = nullptr;
  cg_conf conf;
  cg_tuning tuning;
  int device = 0;
  {
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    conf = g_env->conf;
    tuning = g_env->tuning;
    device = g_env->device;
  }
  for (uint32_t i = 0; i < scene_count; ++i)
    if (!scenes[i]) return fail(CG_E_INVALID, "null scene");
  auto sv = std::make_unique<cg_server_s>();
  for (uint32_t i = 0; i < scene_count; ++i) sv->scenes.push_back(reinterpret_cast<SceneDev*>(scenes[i]));
  sv->budget = hbm_budget_bytes;
  sv->conf = conf;
  sv->rend.tuning = tuning;
  int rc = sv->rend.init(device);
  if (rc != CG_OK) return rc;
  rc = sv->rend.ensureWave(tuning.queue_capacity);
  if (rc != CG_OK) return rc;
  sv->worker = std::thread(serverLoop, sv.get());
  *out = sv.release();
  return CG_OK;
}

CG_API int cg_server_destroy(cg_server_t server) {
  if (!server) return CG_OK;
  {
    std::lock_guard<std::mutex> lk(server->mu);
    for (ServerReq* r : server->pending) r->cancelled = true;
    for (ServerReq* r : server->active) r->cancelled = true;
    server->stop = true;
  }
  server->cv.notify_all();
  if (server->worker.joinable()) server->worker.join();
  if (server->table) cudaFree(server->table);
  delete server;
  return CG_OK;
}

CG_API int cg_server_submit(cg_server_t server, const cg_request* request, float* film_xyz,
                            uint64_t* request_id) {
  if (!server || !request || !film_xyz) return fail(CG_E_INVALID, "null argument");
  const cg_view_desc& v = request->view;
  if (request->scene >= server->scenes.size()) return fail(CG_E_INVALID, "scene index out of range");
  if (v.width == 0 || v.height == 0 || v.spp == 0) return fail(CG_E_INVALID, "zero size or spp");
  SceneDev& scene = *server->scenes[request->scene];
  if (v.spp > server->rend.chunkSamples(scene, capsOf(server->conf)))
    return fail(CG_E_INVALID, "spp exceeds the wavefront chunk");
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
  server->reqs[r->id] = std::move(r);
  ++server->st.submitted;
  server->cv.notify_all();
  return CG_OK;
}

CG_API int cg_server_wait(cg_server_t server, uint64_t request_id, int timeout_ms,
                          cg_request_result* result) {
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
}

CG_API int cg_server_cancel(cg_server_t server, uint64_t request_id) {
  if (!server) return fail(CG_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(server->mu);
  auto it = server->reqs.find(request_id);
  if (it == server->reqs.end()) return fail(CG_E_INVALID, "unknown request id");
  it->second->cancelled = true;
  server->cv.notify_all();
  return CG_OK;
}

CG_API int cg_server_get_stats(cg_server_t server, cg_server_stats* out) {
  if (!server || !out) return fail(CG_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(server->mu);
  *out = server->st;
  return CG_OK;
}

}  // extern "C"
