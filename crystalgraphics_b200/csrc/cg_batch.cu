// cg_batch.cu — the batched form: many views of one scene in one wavefront.
//
// The reference renders one view per View() call (one dispatch of
// compute.wesl:32 over the window).  Here a batch of views of uneven
// resolution and spp shares the same chunked ray queues, so small views fill
// the GPU together; the whole launch sequence of a batch is captured once as
// a CUDA graph and replayed.  The autotuner picks the queue capacity and the
// block sizes of the traversal and shading kernels per scene.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/cg_cuda.h"
#include "cg_api_internal.h"

namespace cg {

namespace {
bool sameViews(const std::vector<cg_view_desc>& a, const cg_view_desc* b, uint32_t n) {
  return a.size() == n && (n == 0 || std::memcmp(a.data(), b, n * sizeof(cg_view_desc)) == 0);
}
}  // namespace

void Env::dropGraphsFor(uint64_t tag) {
  graphs.erase(std::remove_if(graphs.begin(), graphs.end(),
                              [&](const std::unique_ptr<BatchGraph>& g) { return g->scene_tag == tag; }),
               graphs.end());
  if (view_graph.exec && view_graph.scene_tag == tag) dropViewGraph();
}
void Env::dropAllGraphs() {
  graphs.clear();
  dropViewGraph();
}
void Env::dropViewGraph() {
  if (view_graph.exec) cudaGraphExecDestroy(view_graph.exec);
  view_graph = ViewGraph{};
}

// Builds the view table of a batch into `g` (films allocated per view).
static int buildBatch(Env& env, const SceneDev& scene, const cg_view_desc* views, uint32_t n,
                      BatchGraph& g, std::vector<ViewDev>& vd) {
  size_t film_bytes = 0;
  g.film_off.resize(n);
  g.rgba_off.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    const cg_view_desc& v = views[i];
    if (v.width == 0 || v.height == 0 || v.spp == 0)
      return fail(CG_E_INVALID, "view " + std::to_string(i) + " has a zero size or spp");
    g.film_off[i] = film_bytes;
    film_bytes += align256(size_t(v.width) * v.height * 16);
  }
  for (uint32_t i = 0; i < n; ++i) {
    g.rgba_off[i] = film_bytes;
    film_bytes += align256(size_t(views[i].width) * views[i].height * 4);
  }
  const size_t table_off = film_bytes;
  film_bytes += align256(n * sizeof(ViewDev));
  int rc = g.films.alloc(film_bytes);
  if (rc != CG_OK) return rc;
  char* base = static_cast<char*>(g.films.base);
  vd.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    ViewDev& d = vd[i];
    std::memset(&d, 0, sizeof(d));
    cameraBasis(views[i].camera, d);
    d.width = views[i].width;
    d.height = views[i].height;
    d.spp = views[i].spp;
    d.seed = views[i].seed;
    d.frame = 0;
    d.sample_weight = 1.0f;
    d.pixel_base = 0;
    d.pixel_count = d.width * d.height;
    d.film = reinterpret_cast<float4*>(base + g.film_off[i]);
    d.rgba = reinterpret_cast<uchar4*>(base + g.rgba_off[i]);
  }
  layoutViews(vd);
  CG_CUDA(cudaMemcpyAsync(base + table_off, vd.data(), n * sizeof(ViewDev), cudaMemcpyHostToDevice,
                          env.stream));
  g.scene_tag = scene.tag;
  g.views.assign(views, views + n);
  g.table_off = table_off;
  return CG_OK;
}

// Renders a batch on env.stream; leaves the films on the device in `gp`.
static int runBatch(Env& env, const SceneDev& scene, const cg_view_desc* views, uint32_t n,
                    BatchGraph*& gp, RenderRecord& rec, float& ms) {
  const Caps caps = capsOf(env.conf);
  int rc = env.ensureWave(env.tuning.queue_capacity);
  if (rc != CG_OK) return rc;
  if (env.tuning.pipelines > 1u) {  // before any capture
    rc = env.ensurePipelines(static_cast<int>(env.tuning.pipelines));
    if (rc != CG_OK) return rc;
  }
  gp = nullptr;
  const bool use_graph = env.tuning.use_graph && !env.profiling;
  if (use_graph) {
    for (auto& g : env.graphs)
      if (g->scene_tag == scene.tag && sameViews(g->views, views, n)) gp = g.get();
  }
  std::unique_ptr<BatchGraph> fresh;
  if (!gp) {
    fresh = std::make_unique<BatchGraph>();
    std::vector<ViewDev> vd;
    rc = buildBatch(env, scene, views, n, *fresh, vd);
    if (rc != CG_OK) return rc;
    const ViewDev* table = reinterpret_cast<const ViewDev*>(static_cast<char*>(fresh->films.base) +
                                                           fresh->table_off);
    if (use_graph) {
      CG_CUDA(cudaStreamSynchronize(env.stream));
      cudaGraph_t graph = nullptr;
      CG_CUDA(cudaStreamBeginCapture(env.stream, cudaStreamCaptureModeThreadLocal));
      RenderRecord r;
      rc = env.enqueueViews(scene, vd, table, caps, env.stream, r);
      cudaError_t ce = cudaStreamEndCapture(env.stream, &graph);
      if (rc != CG_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ce != cudaSuccess) return cudaFail(ce, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&fresh->exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return cudaFail(ce, "cudaGraphInstantiate");
      fresh->rec = r;
    } else {
      fresh->rec = RenderRecord{};
      CG_CUDA(cudaEventRecord(env.ev0, env.stream));
      rc = env.enqueueViews(scene, vd, table, caps, env.stream, fresh->rec);
      if (rc != CG_OK) return rc;
      CG_CUDA(cudaEventRecord(env.ev1, env.stream));
      CG_CUDA(cudaEventSynchronize(env.ev1));
      cudaEventElapsedTime(&ms, env.ev0, env.ev1);
      rec = fresh->rec;
      gp = fresh.get();
      env.graphs.push_back(std::move(fresh));
      if (env.graphs.size() > 8) env.graphs.erase(env.graphs.begin());
      return CG_OK;
    }
    gp = fresh.get();
    env.graphs.push_back(std::move(fresh));
    if (env.graphs.size() > 8) env.graphs.erase(env.graphs.begin());
  }
  CG_CUDA(cudaEventRecord(env.ev0, env.stream));
  CG_CUDA(cudaGraphLaunch(gp->exec, env.stream));
  CG_CUDA(cudaEventRecord(env.ev1, env.stream));
  CG_CUDA(cudaEventSynchronize(env.ev1));
  cudaEventElapsedTime(&ms, env.ev0, env.ev1);
  rec = gp->rec;
  return CG_OK;
}

}  // namespace cg

using namespace cg;

extern "C" {

CG_API int cg_batch_render(cg_scene_t scene, const cg_view_desc* views, uint32_t view_count,
                           float* films_xyz, uint8_t* films_rgba8) {
  return guarded([&]() -> int {
    if (!scene || (view_count && !views)) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    if (view_count == 0) return CG_OK;
    Env& env = *g_env;
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    CG_CUDA(cudaSetDevice(env.device));
    int rc = env.ensureWave(env.tuning.queue_capacity);
    if (rc != CG_OK) return rc;
    rc = env.beginStats(env.stream);
    if (rc != CG_OK) return rc;
    BatchGraph* g = nullptr;
    RenderRecord rec;
    float ms = 0.0f;
    rc = runBatch(env, *s, views, view_count, g, rec, ms);
    if (rc != CG_OK) return rc;
    rc = env.endStats(env.stream, rec, ms);
    if (rc != CG_OK) return rc;
    // readback
    const char* base = static_cast<const char*>(g->films.base);
    if (films_xyz) {
      size_t total = 0;
      for (uint32_t i = 0; i < view_count; ++i) total += size_t(views[i].width) * views[i].height;
      std::vector<float> tmp;
      size_t out = 0;
      for (uint32_t i = 0; i < view_count; ++i) {
        const size_t npx = size_t(views[i].width) * views[i].height;
        tmp.resize(npx * 4);
        CG_CUDA(cudaMemcpyAsync(tmp.data(), base + g->film_off[i], npx * 16, cudaMemcpyDeviceToHost,
                                env.stream));
        CG_CUDA(cudaStreamSynchronize(env.stream));
        for (size_t p = 0; p < npx; ++p) {
          films_xyz[3 * (out + p)] = tmp[4 * p];
          films_xyz[3 * (out + p) + 1] = tmp[4 * p + 1];
          films_xyz[3 * (out + p) + 2] = tmp[4 * p + 2];
        }
        out += npx;
      }
      (void)total;
    }
    if (films_rgba8) {
      size_t out = 0;
      for (uint32_t i = 0; i < view_count; ++i) {
        const size_t npx = size_t(views[i].width) * views[i].height;
        CG_CUDA(cudaMemcpyAsync(films_rgba8 + out, base + g->rgba_off[i], npx * 4,
                                cudaMemcpyDeviceToHost, env.stream));
        out += npx * 4;
      }
      CG_CUDA(cudaStreamSynchronize(env.stream));
    }
    return CG_OK;
  });
}

CG_API int cg_autotune_views(cg_scene_t scene, const cg_view_desc* views, uint32_t count,
                             cg_tuning* best) {
  return guarded([&]() -> int {
    if (!scene || !views || count == 0) return fail(CG_E_INVALID, "null argument or no views");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    CG_CUDA(cudaSetDevice(env.device));
    const cg_tuning saved = env.tuning;
    // Time of the probe views under tuning t: one untimed run, then two timed
    // (un-captured, so every launch shape change takes effect); +inf if a run fails.
    auto measure = [&](const cg_tuning& t) {
      env.tuning = t;
      env.tuning.use_graph = 0;
      env.dropAllGraphs();
      float total = 0.0f;
      for (int rep = 0; rep < 3; ++rep) {
        BatchGraph* g = nullptr;
        RenderRecord rec;
        float ms = 0.0f;
        if (runBatch(env, *s, views, count, g, rec, ms) != CG_OK) return 1e30f;
        if (rep > 0) total += ms;
      }
      return total;
    };
    // Coordinate descent from the current tuning: kernel variant, then queue
    // capacity, then the traversal and shading block sizes.
    cg_tuning winner = saved;
    float best_ms = measure(winner);
    auto consider = [&](cg_tuning t) {
      const float ms = measure(t);
      if (ms < best_ms) {
        best_ms = ms;
        winner = t;
      }
    };
    // kernel variants: (node width, persistent lane refill 1 on / 2 off, shading
    // order 1 level-wide sort / 3 per-block sort / 2 none, bits per child box bound)
    const uint32_t variants[][4] = {
        {4u, 1u, 1u, 32u}, {4u, 2u, 1u, 32u}, {4u, 1u, 1u, 8u}, {4u, 1u, 3u, 32u},
        {4u, 1u, 2u, 32u}, {2u, 1u, 1u, 32u}, {2u, 2u, 1u, 32u}};
    {
      const cg_tuning base = winner;
      for (const auto& var : variants) {
        cg_tuning t = base;
        t.bvh_width = var[0];
        t.persistent = var[1];
        t.shade_sort = var[2];
        t.box_bits = var[3];
        consider(t);
      }
    }
    {  // pipelines together with the traversal grids' residency: fewer traversal
       // threads per SM let one pipeline's shading run beside another's traversal
      const cg_tuning base = winner;
      for (uint32_t pl : {1u, 2u, 3u, 4u})
        for (uint32_t tt : {1024u, 768u}) {
          cg_tuning t = base;
          t.pipelines = pl;
          t.traversal_threads = tt % t.extend_block ? 1024u : tt;
          consider(t);
        }
    }
    {
      const cg_tuning base = winner;
      for (uint32_t q : {16u << 20, 64u << 20, 128u << 20}) {
        cg_tuning t = base;
        t.queue_capacity = q;
        consider(t);
      }
    }
    {
      const cg_tuning base = winner;
      for (uint32_t b : {64u, 128u, 256u}) {
        cg_tuning t = base;
        t.extend_block = b;
        if (t.traversal_threads % b) t.traversal_threads = 1024u;
        consider(t);
      }
    }
    {
      const cg_tuning base = winner;
      for (uint32_t b : {64u, 128u, 256u}) {
        cg_tuning t = base;
        t.shade_block = b;
        consider(t);
      }
    }
    env.dropAllGraphs();
    winner.use_graph = saved.use_graph;
    env.tuning = winner;
    // release an oversized queue if a smaller capacity won
    if (env.wave.capacity > winner.queue_capacity) {
      env.wave_arena.release();
      env.wave = WaveBuffers{};
    }
    if (best) *best = winner;
    if (best_ms >= 1e30f) return fail(CG_E_CUDA, "autotune: no configuration ran");
    return CG_OK;
  });
}

CG_API int cg_autotune(cg_scene_t scene, const cg_view_desc* view, cg_tuning* best) {
  return guarded([&]() -> int {
    return cg_autotune_views(scene, view, view ? 1u : 0u, best);
  });
}

}  // extern "C"
