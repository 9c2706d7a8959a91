// cg_api_internal.h — host-side state shared by the C ABI implementation
// files (cg_api.cu, cg_batch.cu, cg_server.cu).
#ifndef CG_API_INTERNAL_H_
#define CG_API_INTERNAL_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cg_cuda.h"
#include "cg_kernels.h"
#include "cg_scene.h"

namespace cg {

extern thread_local std::string tl_error;
int fail(int code, const std::string& msg);

// Runs the body of a C-ABI entry point: a C++ exception (a host allocation
// that failed, a thread that could not start) becomes an error status instead
// of crossing the ABI.
template <class Body>
int guarded(Body&& body) {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return fail(CG_E_OOM, "out of host memory");
  } catch (const std::exception& e) {
    return fail(CG_E_INVALID, e.what());
  }
}
int cudaFail(cudaError_t e, const char* what);

// The identity of the calling thread's current CUDA context: a 64-bit id the
// driver never reuses within a process (cuCtxGetId, reached through the
// runtime's driver entry points so that the library does not link libcuda).
// A device reset or a context switch changes it.  Returns CG_OK or an error.
int currentContextId(unsigned long long* id);

#define CG_CUDA(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cudaFail(e_, #call); \
  } while (0)

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Populates the page tables of a caller's host buffer (the whole pages inside
// it) as if written, without changing its contents, so a later copy into a
// freshly allocated buffer does not take one page fault per 4 KB page.  Best
// effort: errors (an older kernel, a pinned or unmapped range) are ignored.
void prefaultHostBuffer(void* p, size_t bytes);

// Frees the pinned film staging buffers that no server holds (cg_term).
void releaseIdleStaging();

struct DeviceArena {
  void* base = nullptr;
  size_t size = 0;
  int alloc(size_t bytes);
  void release();
  DeviceArena() = default;
  DeviceArena(const DeviceArena&) = delete;
  DeviceArena& operator=(const DeviceArena&) = delete;
  ~DeviceArena() { release(); }
};

// An uploaded scene (cg_scene_t).  Immutable after cg_scene_create.
struct SceneDev {
  HostScene host;     // packing result; big arrays are dropped after upload
  DeviceArena arena;
  SceneView view;
  size_t eprim_off = 0, alias_off = 0;
  uint32_t max_lobes = 1;
  uint64_t tag = 0;
  cg_scene_info info{};
  // where the device buffers live: the device current at upload and its
  // context (entry points that run on the caller's current device check both)
  int device = -1;
  unsigned long long ctx_id = 0;
};

int uploadScene(const HostScene& h, SceneDev& s);

// The traversal's node format for a tuning (binary, or four-wide with 32-bit
// or 8-bit child boxes).
inline int nodeFormatOf(const cg_tuning& t) {
  if (t.bvh_width == 2u) return kNodesBinary;
  return t.box_bits == 8u ? kNodesWide4Q : kNodesWide4;
}

struct LevelPlan {
  uint32_t levels = 0;      // depths that can hold rays
  bool shadow[64] = {};     // depths that can draw a light sample
  uint64_t max_product = 1; // most rays one sample can have at one depth
};
LevelPlan planLevels(const Caps& caps, uint32_t max_lobes);
Caps capsOf(const cg_conf& c);
void cameraBasis(const cg_camera& cam, ViewDev& v);
// Fills the views' global pixel / sample offsets from pixel_count and spp.
void layoutViews(std::vector<ViewDev>& views);

struct RenderRecord {
  uint64_t samples = 0;
  uint32_t chunks = 0;
  uint32_t launches = 0;
};

// Device resources of one launch stream: wavelength tables, ray queues and
// the launch shape.  The View() environment and each server own one.
struct Renderer {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float* wl_tree = nullptr;
  float* wl_const = nullptr;
  // pinned: each pipeline's statistics (64 B) and status word, read back
  // with asynchronous copies and one synchronisation
  static constexpr size_t kStatsHostStride = 128;
  unsigned char* stats_host = nullptr;
  bool counting = false;
  // 64M rays per level queue (~11.1 GB of path state): large chunks keep every
  // level's launch full
  cg_tuning tuning{64u << 20, 128u, 128u, 1u, 4u, 1u, 1u, 32u, 2u, 1024u};
  DeviceArena wave_arena;
  WaveBuffers wave{};
  // the extra chunk pipelines of enqueueViews (pipeline 0 is `stream` with
  // `wave`): their ray queues, streams and join events, and the fork event;
  // allocated on first use
  static constexpr int kMaxPipelines = 4;
  DeviceArena xwave_arena[kMaxPipelines - 1];
  WaveBuffers xwave[kMaxPipelines - 1]{};
  // hero-wavelength mode: the extra per-ray and per-sample buffers of every
  // allocated queue set (WaveBuffers::ray_w, sh_w, s_L4), attached while
  // `hero` is set
  bool hero = false;
  DeviceArena hero_arena, xhero_arena[kMaxPipelines - 1];
  // Russian roulette from this hit depth on (0 = off, as the reference)
  uint32_t roulette = 0;
  // (Re)attaches or releases the hero buffers of the allocated queue sets to
  // match `hero` (never inside a stream capture)
  int syncHero();
  cudaStream_t xstream[kMaxPipelines - 1] = {};
  cudaEvent_t fork_ev = nullptr, xjoin_ev[kMaxPipelines - 1] = {};
  // allocates pipelines 1 .. count - 1 (never inside a stream capture:
  // cudaMalloc is not allowed there)
  int ensurePipelines(int count);

  int init(int dev);
  // Takes over prev's wavelength tables and ray queues (after its stream has
  // drained); call before init().
  void adoptBuffers(Renderer& prev);
  int ensureWave(uint32_t capacity);
  // Samples one chunk may hold for this scene and caps (whole trees fit the
  // queues).
  uint32_t chunkSamples(const SceneDev& scene, const Caps& caps) const;
  // Enqueues the chunked wavefront over `views` (laid out by layoutViews; the
  // same table already on the device at `table`).  No host<->device copies
  // and no synchronisation: the sequence can be captured into a CUDA graph.
  int enqueueViews(const SceneDev& scene, const std::vector<ViewDev>& views, const ViewDev* table,
                   const Caps& caps, cudaStream_t s, RenderRecord& rec);
  // Enqueues one chunk covering all of `views` (their samples must fit), on
  // the ray queues `wbp` (default: `wave`).
  void enqueueChunk(const SceneDev& scene, uint32_t view_count, const ViewDev* table,
                    const ChunkDesc& ch, const Caps& caps, cudaStream_t s, RenderRecord& rec,
                    const WaveBuffers* wbp = nullptr);
  int beginStats(cudaStream_t s);
  int readStats(cudaStream_t s, const RenderRecord& rec, float ms, cg_stats& out);

  // Per-kernel CUDA-event timing (off by default; never inside a capture).
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;  // pairs
  std::vector<int> prof_kind;
  size_t prof_used = 0;
  cg_profile prof{};
  void profBegin(int kind, cudaStream_t s);
  void profEnd(cudaStream_t s);
  void profCollect();  // after the stream is synchronised
  ~Renderer();
};

// A captured batch: the graph replays the whole chunk sequence of one
// (scene, views) pair into the films it was captured with.
struct BatchGraph {
  uint64_t scene_tag = 0;
  std::vector<cg_view_desc> views;
  cudaGraphExec_t exec = nullptr;
  DeviceArena films;        // float4 films, rgba8 films, then the view table
  std::vector<size_t> film_off, rgba_off;
  size_t table_off = 0;
  RenderRecord rec;
  ~BatchGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

// The process-global environment (the reference's global::env,
// src/global.h:14): the View() film and its frame history.
struct Env : Renderer {
  cg_conf conf{};
  int spectral = CG_SPECTRAL_REFERENCE;  // cg_set_spectral
  void* film = nullptr;   // float4 per pixel
  void* rgba = nullptr;   // uchar4 per pixel
  float* film_pack = nullptr;  // three floats per pixel: the XYZ / RGB readback
  // FrameHistory (src/wgpu/frame_history.h)
  bool has_prev = false;
  uint64_t prev_tag = 0;
  cg_camera prev_cam{};
  uint32_t frame_count = 0;
  uint32_t seed = 0;
  void* views_dev = nullptr;
  size_t view_cap = 0;
  cg_stats last{};
  std::vector<std::unique_ptr<BatchGraph>> graphs;
  // View()'s launch sequence, captured once per scene and replayed (the view
  // table it reads is uploaded before every replay); valid while the scene,
  // the counting mode and the table's address are the ones it was captured
  // with (tuning changes drop it)
  struct ViewGraph {
    uint64_t scene_tag = 0;
    bool counting = false;
    const void* table = nullptr;
    cudaGraphExec_t exec = nullptr;
    RenderRecord rec;
  } view_graph;
  void dropViewGraph();

  int uploadViews(const std::vector<ViewDev>& views, cudaStream_t s);
  int endStats(cudaStream_t s, const RenderRecord& rec, float ms) {
    return readStats(s, rec, ms, last);
  }
  void dropGraphsFor(uint64_t tag);
  void dropAllGraphs();
  ~Env();
};

extern Env* g_env;
extern std::mutex g_env_mu;

}  // namespace cg

#endif
