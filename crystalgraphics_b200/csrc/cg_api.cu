// cg_api.cu — the C ABI of libcg_cuda.so (include/cg_cuda.h).
//
// Host side of the View() hot path: the environment (EnvInit/EnvTerm), scene
// upload (LoadScene), the chunked wavefront frame loop, film readback and the
// parity ray query.  The batched form is in cg_batch.cu, the served form in
// cg_server.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cg_cuda.h"
#include "cg_api_internal.h"
#include "cg_bvh.h"
#include "cg_kernels.h"
#include "cg_scene.h"

#include <sys/mman.h>
#include <unistd.h>

namespace cg {

void prefaultHostBuffer(void* p, size_t bytes) {
#ifdef MADV_POPULATE_WRITE
  static const uintptr_t page = static_cast<uintptr_t>(sysconf(_SC_PAGESIZE));
  const uintptr_t lo = (reinterpret_cast<uintptr_t>(p) + page - 1) & ~(page - 1);
  const uintptr_t hi = (reinterpret_cast<uintptr_t>(p) + bytes) & ~(page - 1);
  if (hi > lo) (void)madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_POPULATE_WRITE);
#else
  (void)p;
  (void)bytes;
#endif
}

thread_local std::string tl_error;

int fail(int code, const std::string& msg) {
  tl_error = msg;
  return code;
}

int cudaFail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a non-sticky error so the next call starts clean
  return fail(e == cudaErrorMemoryAllocation ? CG_E_OOM : CG_E_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

int currentContextId(unsigned long long* id) {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(fn);
    fn = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(fn);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return fail(CG_E_CUDA, "the driver has no cuCtxGetId");
  void* ctx = nullptr;
  if (get_current(&ctx) != 0) return fail(CG_E_CUDA, "cuCtxGetCurrent failed");
  if (!ctx) {
    // nothing current yet: the runtime's primary context of the current
    // device (cudaSetDevice initialises it; it allocates nothing)
    int dev = 0;
    CG_CUDA(cudaGetDevice(&dev));
    CG_CUDA(cudaSetDevice(dev));
    if (get_current(&ctx) != 0 || !ctx) return fail(CG_E_CUDA, "no current CUDA context");
  }
  if (get_id(ctx, id) != 0) return fail(CG_E_CUDA, "cuCtxGetId failed");
  return CG_OK;
}

int DeviceArena::alloc(size_t bytes) {
  release();
  if (bytes == 0) bytes = 256;
  cudaError_t e = cudaMalloc(&base, bytes);
  if (e != cudaSuccess) {
    base = nullptr;
    cudaGetLastError();
    return cudaFail(e, "cudaMalloc");
  }
  size = bytes;
  return CG_OK;
}
void DeviceArena::release() {
  if (base) cudaFree(base);
  base = nullptr;
  size = 0;
}

// ---- scenes -------------------------------------------------------------------
namespace {
std::atomic<uint64_t> g_tag_counter{0x5eed0000u};
template <class T>
size_t bytesOf(const std::vector<T>& v) {
  return v.size() * sizeof(T);
}
}  // namespace

int uploadScene(const HostScene& h, SceneDev& s) {
  struct Part {
    const void* src;
    size_t bytes;
    size_t off;
  };
  std::vector<Part> parts = {
      {h.tlas.data(), bytesOf(h.tlas), 0},       {h.blas.data(), bytesOf(h.blas), 0},
      {h.tris.data(), bytesOf(h.tris), 0},       {h.tri_vidx.data(), bytesOf(h.tri_vidx), 0},
      {h.vnormal.data(), bytesOf(h.vnormal), 0}, {h.inst.data(), bytesOf(h.inst), 0},
      {h.mat.data(), bytesOf(h.mat), 0},         {h.eprim.data(), bytesOf(h.eprim), 0},
      {h.alias.data(), bytesOf(h.alias), 0},     {h.light_bvh.data(), bytesOf(h.light_bvh), 0},
      {h.ltri.data(), bytesOf(h.ltri), 0},       {h.env.data(), bytesOf(h.env), 0},
      {h.tlas4.data(), bytesOf(h.tlas4), 0},     {h.blas4.data(), bytesOf(h.blas4), 0},
      {h.tlas4q.data(), bytesOf(h.tlas4q), 0},   {h.blas4q.data(), bytesOf(h.blas4q), 0},
      {h.mattex.data(), bytesOf(h.mattex), 0},   {h.tex.data(), bytesOf(h.tex), 0},
      {h.vuv.data(), bytesOf(h.vuv), 0}};
  size_t total = 0;
  for (auto& p : parts) {
    p.off = total;
    total += align256(std::max<size_t>(p.bytes, 16));
  }
  CG_CUDA(cudaGetDevice(&s.device));
  int rc = currentContextId(&s.ctx_id);
  if (rc != CG_OK) return rc;
  rc = s.arena.alloc(total);
  if (rc != CG_OK) return rc;
  char* base = static_cast<char*>(s.arena.base);
  for (auto& p : parts)
    if (p.bytes) CG_CUDA(cudaMemcpy(base + p.off, p.src, p.bytes, cudaMemcpyHostToDevice));
  SceneView& v = s.view;
  v.tlas = reinterpret_cast<const BvhNode*>(base + parts[0].off);
  v.blas = reinterpret_cast<const BvhNode*>(base + parts[1].off);
  v.tris = reinterpret_cast<const float4*>(base + parts[2].off);
  v.tri_vidx = reinterpret_cast<const uint4*>(base + parts[3].off);
  v.vnormal = reinterpret_cast<const float4*>(base + parts[4].off);
  v.inst = reinterpret_cast<const DevInstance*>(base + parts[5].off);
  v.mat = reinterpret_cast<const DevMaterial*>(base + parts[6].off);
  v.eprim = reinterpret_cast<const DevEmissivePrim*>(base + parts[7].off);
  v.alias = reinterpret_cast<const DevAlias*>(base + parts[8].off);
  v.light_bvh = reinterpret_cast<const BvhNode*>(base + parts[9].off);
  v.light_tri = reinterpret_cast<const DevLightTri*>(base + parts[10].off);
  v.env = reinterpret_cast<const float4*>(base + parts[11].off);
  v.tlas4 = reinterpret_cast<const Bvh4Node*>(base + parts[12].off);
  v.blas4 = reinterpret_cast<const Bvh4Node*>(base + parts[13].off);
  v.tlas4q = reinterpret_cast<const Bvh4QNode*>(base + parts[14].off);
  v.blas4q = reinterpret_cast<const Bvh4QNode*>(base + parts[15].off);
  v.mattex = reinterpret_cast<const DevMatTex*>(base + parts[16].off);
  v.tex = reinterpret_cast<const uchar4*>(base + parts[17].off);
  v.vuv = reinterpret_cast<const float4*>(base + parts[18].off);
  v.tex_w = h.tex_w;
  v.tex_h = h.tex_h;
  v.tex_layers = h.tex_layers;
  v.env_w = h.env_w;
  v.env_h = h.env_h;
  v.emissive_count = static_cast<uint32_t>(h.eprim.size());
  v.instance_count = static_cast<uint32_t>(h.inst.size());
  v.has_tlas = h.inst.empty() ? 0u : 1u;
  v.has_lights = h.eprim.empty() ? 0u : 1u;
  s.eprim_off = parts[7].off;
  s.alias_off = parts[8].off;
  return CG_OK;
}

// ---- frame planning ---------------------------------------------------------------
Caps capsOf(const cg_conf& c) {
  Caps k;
  k.trace_depth = std::clamp(c.trace_depth, 1u, 64u);
  k.transport_cap = c.max_transport_sample_count;
  k.emission_cap = c.max_emission_sample_count;
  k.diffuse_cap = c.max_diffuse_sample_count;
  k.rough_cap = c.max_rough_sample_count;
  return k;
}

// The transport and light sample budgets per depth (sample.wesl:215-233 with
// lod.wesl:16-18), in the kernels' float arithmetic: which depths can hold
// rays, which can draw light samples, and the most rays a sample can have at
// one depth (each lobe gets at most one sample, so a hit has at most
// min(budget, lobes) children).
LevelPlan planLevels(const Caps& caps, uint32_t max_lobes) {
  LevelPlan p;
  const int32_t D = static_cast<int32_t>(caps.trace_depth);
  const uint32_t cut = std::max(1u, std::min(caps.trace_depth, 64u)) - 1u;
  uint64_t prod = 1, maxprod = 1;
  for (int32_t d = 0; d < D; ++d) {
    p.levels = static_cast<uint32_t>(d) + 1u;
    const float heur = static_cast<float>(D - d) / static_cast<float>(D);
    const float tf = heur * static_cast<float>(std::min(caps.transport_cap, 4u));
    const float ef = heur * static_cast<float>(std::min(caps.emission_cap, 1u));
    const uint32_t ta = tf > 0.0f ? static_cast<uint32_t>(tf) : 0u;
    const uint32_t ea = ef > 0.0f ? static_cast<uint32_t>(ef) : 0u;
    const bool shades = static_cast<uint32_t>(d) < cut;
    p.shadow[d] = shades && ea > 0u;
    const uint32_t fan = shades ? std::min(ta, max_lobes) : 0u;
    if (fan == 0) break;
    prod *= fan;
    maxprod = std::max(maxprod, prod);
  }
  p.max_product = maxprod;
  return p;
}

void layoutViews(std::vector<ViewDev>& views) {
  uint64_t px_off = 0, smp_off = 0;
  for (auto& v : views) {
    v.pixel_offset = px_off;
    v.sample_offset = smp_off;
    px_off += v.pixel_count;
    smp_off += uint64_t(v.pixel_count) * v.spp;
  }
}

void cameraBasis(const cg_camera& cam, ViewDev& v) {
  // cameraRay's basis (compute.wesl:68-74) in plain float, as the host
  // restatement computes it: dx = normalize(cross(dir, +z)) * viewport.x,
  // dy = normalize(cross(dir, dx)) * viewport.y.
  const float* d = cam.direction;
  const float cx[3] = {d[1] * 1.0f - 0.0f * d[2], d[2] * 0.0f - 1.0f * d[0],
                       d[0] * 0.0f - 0.0f * d[1]};
  const float l = std::sqrt(cx[0] * cx[0] + cx[1] * cx[1] + cx[2] * cx[2]);
  const float dx[3] = {cx[0] / l * cam.viewport[0], cx[1] / l * cam.viewport[0],
                       cx[2] / l * cam.viewport[0]};
  const float cy[3] = {d[1] * dx[2] - dx[1] * d[2], d[2] * dx[0] - dx[2] * d[0],
                       d[0] * dx[1] - dx[0] * d[1]};
  const float m = std::sqrt(cy[0] * cy[0] + cy[1] * cy[1] + cy[2] * cy[2]);
  for (int a = 0; a < 3; ++a) {
    v.pos[a] = cam.position[a];
    v.dir[a] = d[a];
    v.dx[a] = dx[a];
    v.dy[a] = cy[a] / m * cam.viewport[1];
  }
}

// ---- Renderer ------------------------------------------------------------------------
int Renderer::init(int dev) {
  device = dev;
  CG_CUDA(cudaSetDevice(dev));
  CG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CG_CUDA(cudaEventCreate(&ev0));
  CG_CUDA(cudaEventCreate(&ev1));
  CG_CUDA(cudaMallocHost(&stats_host, kMaxPipelines * kStatsHostStride));
  configureKernels();
  if (wl_tree) return CG_OK;  // adopted from a previous renderer
  CG_CUDA(cudaMalloc(&wl_tree, 65535 * sizeof(float)));
  CG_CUDA(cudaMalloc(&wl_const, 4 * sizeof(float)));
  launchWavelengthTree(wl_tree, wl_const, stream);
  CG_CUDA(cudaGetLastError());
  CG_CUDA(cudaStreamSynchronize(stream));
  return CG_OK;
}

void Renderer::adoptBuffers(Renderer& prev) {
  if (prev.stream) cudaStreamSynchronize(prev.stream);
  for (cudaStream_t x : prev.xstream)
    if (x) cudaStreamSynchronize(x);
  std::swap(wl_tree, prev.wl_tree);
  std::swap(wl_const, prev.wl_const);
  std::swap(wave_arena.base, prev.wave_arena.base);
  std::swap(wave_arena.size, prev.wave_arena.size);
  std::swap(hero_arena.base, prev.hero_arena.base);
  std::swap(hero_arena.size, prev.hero_arena.size);
  std::swap(wave, prev.wave);
  std::swap(hero, prev.hero);
  for (int k = 0; k < kMaxPipelines - 1; ++k) {
    std::swap(xwave_arena[k].base, prev.xwave_arena[k].base);
    std::swap(xwave_arena[k].size, prev.xwave_arena[k].size);
    std::swap(xhero_arena[k].base, prev.xhero_arena[k].base);
    std::swap(xhero_arena[k].size, prev.xhero_arena[k].size);
    std::swap(xwave[k], prev.xwave[k]);
  }
}

Renderer::~Renderer() {
  if (stream) cudaStreamSynchronize(stream);
  for (cudaStream_t x : xstream)
    if (x) cudaStreamSynchronize(x);
  for (cudaEvent_t e : prof_events) cudaEventDestroy(e);
  wave_arena.release();
  hero_arena.release();
  for (int k = 0; k < kMaxPipelines - 1; ++k) {
    xwave_arena[k].release();
    xhero_arena[k].release();
    if (xjoin_ev[k]) cudaEventDestroy(xjoin_ev[k]);
    if (xstream[k]) cudaStreamDestroy(xstream[k]);
  }
  if (fork_ev) cudaEventDestroy(fork_ev);
  if (wl_tree) cudaFree(wl_tree);
  if (wl_const) cudaFree(wl_const);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (stats_host) cudaFreeHost(stats_host);
  if (stream) cudaStreamDestroy(stream);
}

namespace {
// Carves one set of ray queues, sample slots and counters of `capacity` rays
// out of a fresh allocation.
int allocWave(DeviceArena& arena, WaveBuffers& w, uint32_t capacity) {
  const size_t Q = capacity;
  const size_t parts[] = {Q * 16, Q * 16, Q * 16, Q * 16, Q * 4, Q * 4,  // ray queues
                          Q * 16, Q * 4,                                 // hits
                          Q * 16, Q * 16, Q * 4,                         // shadow queue
                          Q * 4,  Q * 4,  Q * 4,                         // sample slots
                          Q,      Q * 4,                                 // shading key, order
                          256,    256,    256,                           // counts, stats, status
                          Q * 16, Q * 4};                                // light-pdf deferral
  size_t total = 0;
  for (size_t b : parts) total += align256(b);
  w = WaveBuffers{};
  int rc = arena.alloc(total);
  if (rc != CG_OK) return rc;
  char* p = static_cast<char*>(arena.base);
  size_t off = 0;
  auto take = [&](size_t b) {
    char* r = p + off;
    off += align256(b);
    return r;
  };
  w.ray_o[0] = reinterpret_cast<float4*>(take(Q * 16));
  w.ray_o[1] = reinterpret_cast<float4*>(take(Q * 16));
  w.ray_d[0] = reinterpret_cast<float4*>(take(Q * 16));
  w.ray_d[1] = reinterpret_cast<float4*>(take(Q * 16));
  w.ray_slot[0] = reinterpret_cast<uint32_t*>(take(Q * 4));
  w.ray_slot[1] = reinterpret_cast<uint32_t*>(take(Q * 4));
  w.hit = reinterpret_cast<float4*>(take(Q * 16));
  w.hit_inst = reinterpret_cast<int32_t*>(take(Q * 4));
  w.sh_o = reinterpret_cast<float4*>(take(Q * 16));
  w.sh_d = reinterpret_cast<float4*>(take(Q * 16));
  w.sh_slot = reinterpret_cast<uint32_t*>(take(Q * 4));
  w.s_L = reinterpret_cast<float*>(take(Q * 4));
  w.s_lambda = reinterpret_cast<float*>(take(Q * 4));
  w.s_prob = reinterpret_cast<float*>(take(Q * 4));
  w.shade_key = reinterpret_cast<uint8_t*>(take(Q));
  w.shade_perm = reinterpret_cast<uint32_t*>(take(Q * 4));
  w.counts = reinterpret_cast<uint32_t*>(take(256));
  w.stats = reinterpret_cast<unsigned long long*>(take(256));
  w.status = reinterpret_cast<uint32_t*>(take(256));
  w.defer = reinterpret_cast<float4*>(take(Q * 16));
  w.defer_dist = reinterpret_cast<float*>(take(Q * 4));
  w.capacity = capacity;
  w.sample_capacity = capacity;
  CG_CUDA(cudaMemset(w.counts, 0, 256));
  CG_CUDA(cudaMemset(w.stats, 0, 256));
  CG_CUDA(cudaMemset(w.status, 0, 256));
  return CG_OK;
}
}  // namespace

// The hero-wavelength buffers of one queue set: per queued ray (both queues)
// and per shadow ray a float4, per sample slot a float4.
int attachHero(DeviceArena& arena, WaveBuffers& w) {
  const size_t Q = w.capacity, S = w.sample_capacity;
  const size_t q16 = align256(Q * 16);
  int rc = arena.alloc(4 * q16 + align256(S * 16));
  if (rc != CG_OK) return rc;
  char* p = static_cast<char*>(arena.base);
  w.ray_w[0] = reinterpret_cast<float4*>(p);
  w.ray_w[1] = reinterpret_cast<float4*>(p + q16);
  w.sh_w = reinterpret_cast<float4*>(p + 2 * q16);
  w.defer_w = reinterpret_cast<float4*>(p + 3 * q16);
  w.s_L4 = reinterpret_cast<float4*>(p + 4 * q16);
  w.hero = 1u;
  return CG_OK;
}

void detachHero(DeviceArena& arena, WaveBuffers& w) {
  arena.release();
  w.ray_w[0] = w.ray_w[1] = w.sh_w = w.s_L4 = w.defer_w = nullptr;
  w.hero = 0u;
}

int Renderer::syncHero() {
  auto one = [&](DeviceArena& queues, DeviceArena& extra, WaveBuffers& w) -> int {
    if (!queues.base) return CG_OK;
    if (hero && !w.hero) return attachHero(extra, w);
    if (!hero && w.hero) detachHero(extra, w);
    return CG_OK;
  };
  bool detach = !hero && wave.hero;
  for (int k = 0; k < kMaxPipelines - 1; ++k) detach = detach || (!hero && xwave[k].hero);
  if (detach) {  // buffers in use by queued work stay until it is done
    if (stream) CG_CUDA(cudaStreamSynchronize(stream));
    for (cudaStream_t x : xstream)
      if (x) CG_CUDA(cudaStreamSynchronize(x));
  }
  int rc = one(wave_arena, hero_arena, wave);
  for (int k = 0; k < kMaxPipelines - 1 && rc == CG_OK; ++k)
    rc = one(xwave_arena[k], xhero_arena[k], xwave[k]);
  return rc;
}

int Renderer::ensureWave(uint32_t capacity) {
  if (wave_arena.base && wave.capacity == capacity) return syncHero();
  if (stream) CG_CUDA(cudaStreamSynchronize(stream));
  for (int k = 0; k < kMaxPipelines - 1; ++k) {  // the extra sets follow the first one's capacity
    if (xstream[k]) CG_CUDA(cudaStreamSynchronize(xstream[k]));
    xwave_arena[k].release();
    xhero_arena[k].release();
    xwave[k] = WaveBuffers{};
  }
  hero_arena.release();
  const int rc = allocWave(wave_arena, wave, capacity);
  if (rc != CG_OK) return rc;
  return syncHero();
}

int Renderer::ensurePipelines(int count) {
  if (!fork_ev) CG_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  for (int k = 0; k + 1 < count && k < kMaxPipelines - 1; ++k) {
    if (!xstream[k]) {
      CG_CUDA(cudaStreamCreateWithFlags(&xstream[k], cudaStreamNonBlocking));
      CG_CUDA(cudaEventCreateWithFlags(&xjoin_ev[k], cudaEventDisableTiming));
    }
    if (!(xwave_arena[k].base && xwave[k].capacity == wave.capacity)) {
      xhero_arena[k].release();
      int rc = allocWave(xwave_arena[k], xwave[k], wave.capacity);
      if (rc != CG_OK) return rc;
      if (hero) {
        rc = attachHero(xhero_arena[k], xwave[k]);
        if (rc != CG_OK) return rc;
      }
    }
  }
  return CG_OK;
}

uint32_t Renderer::chunkSamples(const SceneDev& scene, const Caps& caps) const {
  const LevelPlan plan = planLevels(caps, std::max(1u, scene.max_lobes));
  return static_cast<uint32_t>(std::min<uint64_t>(
      wave.sample_capacity, wave.capacity / std::max<uint64_t>(1, plan.max_product)));
}

void Renderer::enqueueChunk(const SceneDev& scene, uint32_t view_count, const ViewDev* table,
                            const ChunkDesc& ch, const Caps& caps, cudaStream_t s,
                            RenderRecord& rec, const WaveBuffers* wbp) {
  const WaveBuffers& wb = wbp ? *wbp : wave;
  const LevelPlan plan = planLevels(caps, std::max(1u, scene.max_lobes));
  FrameConst fc;
  fc.views = table;
  fc.view_count = view_count;
  fc.caps = caps;
  fc.wl_tree = wl_tree;
  fc.wl_const = wl_const;
  fc.roulette = roulette;
  LaunchShape ls;
  ls.extend_block = tuning.extend_block;
  ls.shade_block = tuning.shade_block;
  ls.nodes = nodeFormatOf(tuning);
  ls.persistent = tuning.persistent != 2u;
  ls.spec = tuning.persistent == 3u;
  ls.traversal_threads = tuning.traversal_threads ? tuning.traversal_threads : 1024u;
  const uint32_t cut_depth = std::max(1u, std::min(caps.trace_depth, 64u)) - 1u;
  ls.shade_sort = tuning.shade_sort == 2u   ? kShadeSortNone
                  : tuning.shade_sort == 3u ? kShadeSortBlock
                                            : kShadeSortGlobal;
  if (wb.hero) ls.shade_sort = kShadeSortGlobal;  // the hero kernels take the level-wide order
  profBegin(CG_K_GEN, s);
  launchGen(fc, wb, ch, s);
  profEnd(s);
  ++rec.launches;
  for (uint32_t d = 0; d < plan.levels; ++d) {
    const int parity = static_cast<int>(d & 1u);
    profBegin(CG_K_EXTEND, s);
    launchExtend(scene.view, wb, parity, counting, ls, d >= cut_depth, s);
    profEnd(s);
    profBegin(CG_K_SHADE, s);
    const int shade_kernels =
        launchShade(scene.view, fc, wb, static_cast<int>(d), parity, ls, s, plan.shadow[d]);
    profEnd(s);
    rec.launches += 1 + static_cast<uint32_t>(shade_kernels);
    if (plan.shadow[d]) {
      profBegin(CG_K_SHADOW, s);
      launchShadow(scene.view, wb, counting, ls, s);
      profEnd(s);
      ++rec.launches;
    }
  }
  profBegin(CG_K_RESOLVE, s);
  launchResolve(fc, wb, ch, s);
  profEnd(s);
  ++rec.launches;
  ++rec.chunks;
  rec.samples += ch.sample_count;
}

int Renderer::enqueueViews(const SceneDev& scene, const std::vector<ViewDev>& views,
                           const ViewDev* table, const Caps& caps, cudaStream_t s,
                           RenderRecord& rec) {
  if (views.empty()) return CG_OK;
  int rc = ensureWave(tuning.queue_capacity);
  if (rc != CG_OK) return rc;
  const uint32_t sample_cap = chunkSamples(scene, caps);
  for (const auto& v : views)
    if (v.spp > sample_cap)
      return fail(CG_E_INVALID, "spp " + std::to_string(v.spp) + " exceeds the wavefront chunk of " +
                                    std::to_string(sample_cap) + " samples");
  // chunks of whole pixels, each filled up to sample_cap samples
  std::vector<ChunkDesc> chunks;
  size_t vi = 0;
  uint64_t pix_in_view = 0, gpix = 0, gsmp = 0;
  while (vi < views.size()) {
    ChunkDesc ch;
    ch.sample_begin = gsmp;
    ch.pixel_begin = gpix;
    ch.sample_count = 0;
    ch.pixel_count = 0;
    while (vi < views.size()) {
      const ViewDev& v = views[vi];
      if (pix_in_view >= v.pixel_count) {
        ++vi;
        pix_in_view = 0;
        continue;
      }
      const uint64_t room = (sample_cap - ch.sample_count) / v.spp;
      if (room == 0) break;
      const uint64_t take = std::min<uint64_t>(room, v.pixel_count - pix_in_view);
      ch.sample_count += static_cast<uint32_t>(take * v.spp);
      ch.pixel_count += static_cast<uint32_t>(take);
      pix_in_view += take;
    }
    if (ch.pixel_count == 0) break;
    gpix += ch.pixel_count;
    gsmp += ch.sample_count;
    chunks.push_back(ch);
  }
  // P pipelines: chunk k runs on pipeline k mod P; pipeline 0 is `s` with
  // `wave`, the others are extra streams with their own ray queues, forked
  // from and joined back into `s` by events (also inside a stream capture), so
  // one chunk's sparse deep levels overlap another's launches.  Per-kernel
  // timing keeps one pipeline.
  int P = profiling ? 1 : static_cast<int>(std::clamp(tuning.pipelines, 1u, uint32_t(kMaxPipelines)));
  P = std::min<int>(P, static_cast<int>(chunks.size()));
  if (P > 1) {
    rc = ensurePipelines(P);
    if (rc != CG_OK) return rc;
    CG_CUDA(cudaEventRecord(fork_ev, s));
    for (int k = 0; k + 1 < P; ++k) CG_CUDA(cudaStreamWaitEvent(xstream[k], fork_ev, 0));
  }
  for (size_t k = 0; k < chunks.size(); ++k) {
    const int p = static_cast<int>(k % static_cast<size_t>(P));
    enqueueChunk(scene, static_cast<uint32_t>(views.size()), table, chunks[k], caps,
                 p ? xstream[p - 1] : s, rec, p ? &xwave[p - 1] : &wave);
  }
  for (int k = 0; k + 1 < P; ++k) {
    CG_CUDA(cudaEventRecord(xjoin_ev[k], xstream[k]));
    CG_CUDA(cudaStreamWaitEvent(s, xjoin_ev[k], 0));
  }
  return CG_OK;
}

void Renderer::profBegin(int kind, cudaStream_t s) {
  if (!profiling) return;
  if (prof_used + 2 > prof_events.size()) {
    for (int k = 0; k < 64; ++k) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return;
      prof_events.push_back(e);
    }
  }
  prof_kind.resize(prof_events.size() / 2 + 1);
  prof_kind[prof_used / 2] = kind;
  cudaEventRecord(prof_events[prof_used], s);
}

void Renderer::profEnd(cudaStream_t s) {
  if (!profiling || prof_used + 2 > prof_events.size()) return;
  cudaEventRecord(prof_events[prof_used + 1], s);
  prof_used += 2;
}

void Renderer::profCollect() {
  for (size_t i = 0; i + 1 < prof_used; i += 2) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, prof_events[i], prof_events[i + 1]) == cudaSuccess) {
      const int k = prof_kind[i / 2];
      prof.ms[k] += ms;
      ++prof.launches[k];
    }
  }
  prof_used = 0;
}

int Renderer::beginStats(cudaStream_t s) {
  CG_CUDA(cudaMemsetAsync(wave.stats, 0, 256, s));
  CG_CUDA(cudaMemsetAsync(wave.status, 0, 256, s));
  for (int k = 0; k < kMaxPipelines - 1; ++k)
    if (xwave_arena[k].base) {  // ordered before the fork the extra pipelines wait on
      CG_CUDA(cudaMemsetAsync(xwave[k].stats, 0, 256, s));
      CG_CUDA(cudaMemsetAsync(xwave[k].status, 0, 256, s));
    }
  return CG_OK;
}

int Renderer::readStats(cudaStream_t s, const RenderRecord& rec, float ms, cg_stats& out) {
  unsigned long long st[kMaxPipelines][8] = {};
  uint32_t status[kMaxPipelines] = {};
  bool used[kMaxPipelines] = {true};
  for (int k = 0; k < kMaxPipelines - 1; ++k)
    used[k + 1] = xwave_arena[k].base != nullptr;  // zeroed by beginStats; read after the join
  for (int p = 0; p < kMaxPipelines; ++p) {
    if (!used[p]) continue;
    const WaveBuffers& w = p ? xwave[p - 1] : wave;
    unsigned char* h = stats_host + p * kStatsHostStride;
    CG_CUDA(cudaMemcpyAsync(h, w.stats, sizeof(st[0]), cudaMemcpyDeviceToHost, s));
    CG_CUDA(cudaMemcpyAsync(h + sizeof(st[0]), w.status, 4, cudaMemcpyDeviceToHost, s));
  }
  CG_CUDA(cudaStreamSynchronize(s));
  for (int p = 0; p < kMaxPipelines; ++p) {
    if (!used[p]) continue;
    const unsigned char* h = stats_host + p * kStatsHostStride;
    std::memcpy(st[p], h, sizeof(st[0]));
    std::memcpy(&status[p], h + sizeof(st[0]), 4);
  }
  for (int p = 1; p < kMaxPipelines; ++p) {
    for (int k = 0; k < 8; ++k) st[0][k] += st[p][k];
    status[0] |= status[p];
  }
  profCollect();
  out.samples = rec.samples;
  out.extend_rays = st[0][0];
  out.shadow_rays = st[0][1];
  out.node_visits = st[0][2];
  out.tri_tests = st[0][3];
  out.inst_visits = st[0][4];
  out.nonfinite_samples = st[0][5];
  out.chunks = rec.chunks;
  out.kernel_launches = rec.launches;
  out.device_ms = ms;
  if (status[0] & 1u) return fail(CG_E_DEVICE, "traversal stack overflow in a kernel");
  if (status[0] & 2u) return fail(CG_E_DEVICE, "ray queue overflow in a kernel");
  return CG_OK;
}

// ---- the environment ---------------------------------------------------------------
Env* g_env = nullptr;
std::mutex g_env_mu;

int Env::uploadViews(const std::vector<ViewDev>& views, cudaStream_t s) {
  if (views.size() > view_cap) {
    if (views_dev) cudaFree(views_dev);
    views_dev = nullptr;
    view_cap = 0;
    CG_CUDA(cudaMalloc(&views_dev, views.size() * sizeof(ViewDev)));
    view_cap = views.size();
  }
  CG_CUDA(cudaMemcpyAsync(views_dev, views.data(), views.size() * sizeof(ViewDev),
                          cudaMemcpyHostToDevice, s));
  return CG_OK;
}

Env::~Env() {
  if (stream) cudaStreamSynchronize(stream);
  graphs.clear();
  dropViewGraph();
  if (views_dev) cudaFree(views_dev);
  if (film) cudaFree(film);
  if (rgba) cudaFree(rgba);
  if (film_pack) cudaFree(film_pack);
}

// `prev` (may be null) is the environment being replaced: on the same device
// its wavelength tables and ray queues, which do not depend on the film size,
// move to the new environment instead of being freed and allocated again.
static int createEnv(const cg_conf& conf_in, int device, std::unique_ptr<Env>& out, Env* prev) {
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(CG_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (device < 0 || device >= ndev) return fail(CG_E_INVALID, "device index out of range");
  if (conf_in.render_width == 0 || conf_in.render_height == 0)
    return fail(CG_E_INVALID, "render size must be nonzero");
  if (conf_in.sample_count == 0) return fail(CG_E_INVALID, "sample_count must be nonzero");
  auto env = std::make_unique<Env>();
  env->conf = conf_in;
  env->conf.trace_depth = std::clamp(conf_in.trace_depth, 1u, 64u);
  if (prev && prev->device == device) {
    if (prev->stream) cudaStreamSynchronize(prev->stream);
    prev->graphs.clear();  // captured graphs point at the adopted queues
    env->adoptBuffers(*prev);
  }
  int rc = env->init(device);
  if (rc != CG_OK) return rc;
  env->hero = false;  // a new environment samples like the reference until told otherwise
  rc = env->syncHero();
  if (rc != CG_OK) return rc;
  const size_t npx = size_t(env->conf.render_width) * env->conf.render_height;
  CG_CUDA(cudaMalloc(&env->film, npx * sizeof(float4)));
  CG_CUDA(cudaMalloc(&env->rgba, npx * sizeof(uchar4)));
  CG_CUDA(cudaMalloc(&env->film_pack, npx * 3 * sizeof(float)));
  CG_CUDA(cudaMemset(env->film, 0, npx * sizeof(float4)));
  CG_CUDA(cudaMemset(env->rgba, 0, npx * sizeof(uchar4)));
  out = std::move(env);
  return CG_OK;
}

// Renders one prepared view of `s` into the environment's film: uploads the
// view table and enqueues (or, when `allow_graph`, replays the captured)
// launch sequence, then waits and reads the statistics.
static int renderEnvView(Env& env, SceneDev* s, std::vector<ViewDev>& views, bool allow_graph) {
  layoutViews(views);
  const Caps caps = capsOf(env.conf);
  int rc = env.ensureWave(env.tuning.queue_capacity);
  if (rc != CG_OK) return rc;
  const bool use_graph = allow_graph && env.tuning.use_graph && !env.profiling;
  if (use_graph && env.tuning.pipelines > 1u) {  // before any capture
    rc = env.ensurePipelines(static_cast<int>(env.tuning.pipelines));
    if (rc != CG_OK) return rc;
  }
  rc = env.beginStats(env.stream);
  if (rc != CG_OK) return rc;
  rc = env.uploadViews(views, env.stream);
  if (rc != CG_OK) return rc;
  const ViewDev* table = static_cast<const ViewDev*>(env.views_dev);
  RenderRecord rec;
  if (use_graph) {
    // the launch sequence depends only on the scene, the conf, the tuning and
    // the buffers, so it is captured once and replayed: a small frame's ~60
    // launches then cost one graph launch
    Env::ViewGraph& vg = env.view_graph;
    if (!(vg.exec && vg.scene_tag == s->tag && vg.counting == env.counting && vg.table == table)) {
      env.dropViewGraph();
      CG_CUDA(cudaStreamSynchronize(env.stream));
      cudaGraph_t graph = nullptr;
      CG_CUDA(cudaStreamBeginCapture(env.stream, cudaStreamCaptureModeThreadLocal));
      RenderRecord r;
      rc = env.enqueueViews(*s, views, table, caps, env.stream, r);
      cudaError_t ce = cudaStreamEndCapture(env.stream, &graph);
      if (rc != CG_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ce != cudaSuccess) return cudaFail(ce, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&vg.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) {
        vg.exec = nullptr;
        return cudaFail(ce, "cudaGraphInstantiate");
      }
      vg.scene_tag = s->tag;
      vg.counting = env.counting;
      vg.table = table;
      vg.rec = r;
    }
    CG_CUDA(cudaEventRecord(env.ev0, env.stream));
    CG_CUDA(cudaGraphLaunch(vg.exec, env.stream));
    rec = vg.rec;
  } else {
    CG_CUDA(cudaEventRecord(env.ev0, env.stream));
    rc = env.enqueueViews(*s, views, table, caps, env.stream, rec);
    if (rc != CG_OK) return rc;
  }
  CG_CUDA(cudaEventRecord(env.ev1, env.stream));
  CG_CUDA(cudaGetLastError());
  CG_CUDA(cudaEventSynchronize(env.ev1));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, env.ev0, env.ev1);
  return env.endStats(env.stream, rec, ms);
}

}  // namespace cg

using namespace cg;

extern "C" {

CG_API const char* cg_version(void) { return "crystalgraphics-b200 0.1 (sm_100a)"; }

CG_API const char* cg_last_error(void) { return tl_error.c_str(); }

CG_API int cg_init(const cg_conf* conf, int device) {
  return guarded([&]() -> int {
    if (!conf) return fail(CG_E_INVALID, "conf is null");
    std::lock_guard<std::mutex> lk(g_env_mu);
    std::unique_ptr<Env> prev(g_env);
    g_env = nullptr;
    std::unique_ptr<Env> env;
    int rc = createEnv(*conf, device, env, prev.get());
    prev.reset();
    if (rc != CG_OK) return rc;
    g_env = env.release();
    return CG_OK;
  });
}

CG_API int cg_term(void) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_env_mu);
    delete g_env;
    g_env = nullptr;
    releaseIdleStaging();
    return CG_OK;
  });
}

CG_API int cg_status(void) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_env_mu);
    return g_env ? 1 : 0;
  });
}

CG_API int cg_get_conf(cg_conf* out) {
  return guarded([&]() -> int {
    if (!out) return fail(CG_E_INVALID, "out is null");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *out = g_env->conf;
    return CG_OK;
  });
}

CG_API int cg_scene_create(const cg_scene_desc* desc, cg_scene_t* out) {
  return guarded([&]() -> int {
    if (!out) return fail(CG_E_INVALID, "out is null");
    *out = nullptr;
    auto sd = std::make_unique<SceneDev>();
    std::string err;
    int rc = CG_OK;
    {
      std::lock_guard<std::mutex> lk(g_env_mu);
      if (g_env) cudaSetDevice(g_env->device);  // device BVH builds run there too
    }
    resetBvhBuildStats();
    try {
      rc = packScene(desc, sd->host, err);
    } catch (const std::exception& e) {
      return fail(CG_E_CUDA, std::string("scene build: ") + e.what());
    }
    if (rc != CG_OK) return fail(rc, err);
    const BvhBuildStats bstats = bvhBuildStats();
    if (sd->host.blas_depth + sd->host.tlas_depth + 2 > 64)
      return fail(CG_E_INVALID, "BVH too deep for the 64-entry traversal stack");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return fail(CG_E_CUDA, "no CUDA device");
    }
    {
      std::lock_guard<std::mutex> lk(g_env_mu);
      if (g_env) cudaSetDevice(g_env->device);
    }
    rc = uploadScene(sd->host, *sd);
    if (rc != CG_OK) return rc;
    sd->max_lobes = sd->host.max_lobes;
    sd->tag = ++g_tag_counter;
    cg_scene_info& in = sd->info;
    in.instance_count = static_cast<uint32_t>(sd->host.inst.size());
    in.mesh_count = sd->host.mesh_count;
    in.triangle_count = sd->host.triangle_count;
    in.material_count = static_cast<uint32_t>(sd->host.mat.size());
    in.emissive_count = static_cast<uint32_t>(sd->host.eprim.size());
    in.blas_node_count = static_cast<uint32_t>(sd->host.blas.size());
    in.tlas_node_count = static_cast<uint32_t>(sd->host.tlas.size());
    in.light_node_count = static_cast<uint32_t>(sd->host.light_bvh.size());
    in.device_bytes = sd->arena.size;
    in.tag = sd->tag;
    in.bvh_build_seconds = bstats.seconds;
    in.bvh_host_builds = bstats.host_builds;
    in.bvh_device_builds = bstats.device_builds;
    // the device holds the geometry now
    HostScene& h = sd->host;
    std::vector<BvhNode>().swap(h.blas);
    std::vector<Bvh4Node>().swap(h.blas4);
    std::vector<Bvh4QNode>().swap(h.blas4q);
    std::vector<float>().swap(h.tris);
    std::vector<uint32_t>().swap(h.tri_vidx);
    std::vector<float>().swap(h.vnormal);
    std::vector<uint32_t>().swap(h.tex);
    std::vector<float>().swap(h.vuv);
    *out = reinterpret_cast<cg_scene_t>(sd.release());
    return CG_OK;
  });
}

CG_API int cg_bvh_build(const float* boxes, uint32_t count, int mode, void* nodes_out,
                        uint32_t node_capacity, uint32_t* node_count, uint32_t* order_out) {
  return guarded([&]() -> int {
    if (!boxes || !node_count || (count && !order_out))
      return fail(CG_E_INVALID, "null argument");
    if (mode != kBuildHost && mode != kBuildDevice) return fail(CG_E_INVALID, "mode must be host or device");
    std::vector<Box> bx(count);
    std::memcpy(bx.data(), boxes, sizeof(Box) * size_t(count));
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> order;
    const int saved = bvhBuildMode();
    setBvhBuildMode(mode);
    try {
      BvhBuildOptions opt;
      buildBvh(bx, opt, 0, nodes, order);
    } catch (const std::exception& e) {
      setBvhBuildMode(saved);
      return fail(CG_E_CUDA, std::string("bvh build: ") + e.what());
    }
    setBvhBuildMode(saved);
    *node_count = static_cast<uint32_t>(nodes.size());
    if (nodes_out && node_capacity >= nodes.size())
      std::memcpy(nodes_out, nodes.data(), sizeof(BvhNode) * nodes.size());
    if (count) std::memcpy(order_out, order.data(), 4 * size_t(count));
    return CG_OK;
  });
}

CG_API int cg_set_bvh_build(int mode) {
  return guarded([&]() -> int {
    if (mode < kBuildAuto || mode > kBuildDevice) return fail(CG_E_INVALID, "unknown BVH build mode");
    setBvhBuildMode(mode);
    return CG_OK;
  });
}

CG_API int cg_scene_destroy(cg_scene_t scene) {
  return guarded([&]() -> int {
    if (!scene) return CG_OK;
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    {
      std::lock_guard<std::mutex> lk(g_env_mu);
      if (g_env) {
        cudaStreamSynchronize(g_env->stream);
        g_env->dropGraphsFor(s->tag);
      }
    }
    delete s;
    return CG_OK;
  });
}

CG_API int cg_scene_get_info(cg_scene_t scene, cg_scene_info* out) {
  return guarded([&]() -> int {
    if (!scene || !out) return fail(CG_E_INVALID, "null argument");
    *out = reinterpret_cast<SceneDev*>(scene)->info;
    return CG_OK;
  });
}

CG_API int cg_scene_read_emissive(cg_scene_t scene, cg_emissive_prim* prims, cg_alias_entry* alias,
                                  uint32_t capacity, uint32_t* count) {
  return guarded([&]() -> int {
    if (!scene) return fail(CG_E_INVALID, "scene is null");
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    const uint32_t n = s->info.emissive_count;
    if (count) *count = n;
    if (n == 0 || (!prims && !alias)) return CG_OK;  // count query
    if (capacity < n) return fail(CG_E_INVALID, "capacity below the emissive count");
    const char* base = static_cast<const char*>(s->arena.base);
    if (prims)
      CG_CUDA(cudaMemcpy(prims, base + s->eprim_off, n * sizeof(cg_emissive_prim),
                         cudaMemcpyDeviceToHost));
    if (alias)
      CG_CUDA(cudaMemcpy(alias, base + s->alias_off, n * sizeof(cg_alias_entry),
                         cudaMemcpyDeviceToHost));
    return CG_OK;
  });
}

CG_API int cg_alias_build(const double* weights, uint32_t count, cg_alias_entry* out) {
  return guarded([&]() -> int {
    if (count && (!weights || !out)) return fail(CG_E_INVALID, "null argument");
    buildAliasTable(weights, count, out);
    return CG_OK;
  });
}

CG_API int cg_view(cg_scene_t scene, const cg_camera* camera) {
  return guarded([&]() -> int {
    if (!scene || !camera) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    CG_CUDA(cudaSetDevice(env.device));
    // FrameHistory::NextIteration (src/wgpu/frame_history.h:12-23)
    const bool same = env.has_prev && env.prev_tag == s->tag &&
                      camera->position[0] == env.prev_cam.position[0] &&
                      camera->position[1] == env.prev_cam.position[1] &&
                      camera->position[2] == env.prev_cam.position[2] &&
                      camera->direction[0] == env.prev_cam.direction[0] &&
                      camera->direction[1] == env.prev_cam.direction[1] &&
                      camera->direction[2] == env.prev_cam.direction[2] &&
                      camera->viewport[0] == env.prev_cam.viewport[0] &&
                      camera->viewport[1] == env.prev_cam.viewport[1];
    uint32_t iter;
    if (!same) {
      env.has_prev = true;
      env.prev_tag = s->tag;
      env.prev_cam = *camera;
      env.frame_count = 1;
      iter = 0;
    } else {
      iter = env.frame_count++;
    }
    std::vector<ViewDev> views(1);
    ViewDev& v = views[0];
    std::memset(&v, 0, sizeof(v));
    cameraBasis(*camera, v);
    v.width = env.conf.render_width;
    v.height = env.conf.render_height;
    v.spp = env.conf.sample_count;
    v.seed = env.seed;
    v.frame = iter;
    v.sample_weight = 1.0f / static_cast<float>(iter + 1u);
    v.pixel_base = 0;
    v.pixel_count = v.width * v.height;
    v.film = static_cast<float4*>(env.film);
    v.rgba = static_cast<uchar4*>(env.rgba);
    return renderEnvView(env, s, views, true);
  });
}

CG_API int cg_view_samples(cg_scene_t scene, const cg_camera* camera, uint32_t sample_begin,
                           uint32_t sample_count) {
  return guarded([&]() -> int {
    if (!scene || !camera) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    if (sample_begin > env.conf.sample_count ||
        sample_count > env.conf.sample_count - sample_begin)
      return fail(CG_E_INVALID, "sample range beyond the conf's sample_count");
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    CG_CUDA(cudaSetDevice(env.device));
    env.has_prev = false;  // a share of a frame: the next View() starts a fresh mean
    const size_t npx = size_t(env.conf.render_width) * env.conf.render_height;
    if (sample_count == 0) {  // this share holds no samples
      CG_CUDA(cudaMemsetAsync(env.film, 0, npx * sizeof(float4), env.stream));
      launchFilmRgba8(static_cast<const float4*>(env.film), static_cast<uchar4*>(env.rgba), npx,
                      env.stream);
      CG_CUDA(cudaGetLastError());
      CG_CUDA(cudaStreamSynchronize(env.stream));
      env.last = cg_stats{};
      return CG_OK;
    }
    std::vector<ViewDev> views(1);
    ViewDev& v = views[0];
    std::memset(&v, 0, sizeof(v));
    cameraBasis(*camera, v);
    v.width = env.conf.render_width;
    v.height = env.conf.render_height;
    v.spp = sample_count;
    v.sample_base = sample_begin;
    v.spp_total = env.conf.sample_count;
    v.seed = env.seed;
    v.frame = 0;
    v.sample_weight = 1.0f;
    v.pixel_base = 0;
    v.pixel_count = v.width * v.height;
    v.film = static_cast<float4*>(env.film);
    v.rgba = static_cast<uchar4*>(env.rgba);
    // the chunking depends on the range, so the captured View() sequence does not apply
    return renderEnvView(env, s, views, false);
  });
}

CG_API int cg_film_device(void** film_xyzw, size_t* bytes) {
  return guarded([&]() -> int {
    if (!film_xyzw || !bytes) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *film_xyzw = g_env->film;
    *bytes = size_t(g_env->conf.render_width) * g_env->conf.render_height * sizeof(float4);
    return CG_OK;
  });
}

CG_API int cg_film_update_rgba8(void) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    CG_CUDA(cudaSetDevice(env.device));
    launchFilmRgba8(static_cast<const float4*>(env.film), static_cast<uchar4*>(env.rgba),
                    size_t(env.conf.render_width) * env.conf.render_height, env.stream);
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaStreamSynchronize(env.stream));
    return CG_OK;
  });
}

CG_API int cg_film_read(void* host, size_t bytes, int format) {
  return guarded([&]() -> int {
    if (!host) return fail(CG_E_INVALID, "host is null");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    const size_t npx = size_t(env.conf.render_width) * env.conf.render_height;
    CG_CUDA(cudaSetDevice(env.device));
    prefaultHostBuffer(host, std::min(bytes, npx * (format == CG_FILM_RGBA8 ? 4 : 12)));
    if (format == CG_FILM_RGBA8) {
      if (bytes < npx * 4) return fail(CG_E_INVALID, "buffer too small for RGBA8");
      CG_CUDA(cudaMemcpyAsync(host, env.rgba, npx * 4, cudaMemcpyDeviceToHost, env.stream));
      CG_CUDA(cudaStreamSynchronize(env.stream));
      return CG_OK;
    }
    if (format != CG_FILM_XYZ32F && format != CG_FILM_RGB32F)
      return fail(CG_E_INVALID, "unknown film format");
    if (bytes < npx * 12) return fail(CG_E_INVALID, "buffer too small for 3 floats per pixel");
    // packed (and for RGB converted) on the device, then one contiguous copy
    // (a direct DMA when `host` is pinned)
    launchFilmPack(static_cast<const float4*>(env.film), env.film_pack, npx,
                   format == CG_FILM_RGB32F, env.stream);
    CG_CUDA(cudaGetLastError());
    CG_CUDA(cudaMemcpyAsync(host, env.film_pack, npx * 12, cudaMemcpyDeviceToHost, env.stream));
    CG_CUDA(cudaStreamSynchronize(env.stream));
    return CG_OK;
  });
}

CG_API int cg_film_frames(uint32_t* frames) {
  return guarded([&]() -> int {
    if (!frames) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *frames = g_env->has_prev ? g_env->frame_count : 0u;
    return CG_OK;
  });
}

CG_API int cg_last_stats(cg_stats* out) {
  return guarded([&]() -> int {
    if (!out) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *out = g_env->last;
    return CG_OK;
  });
}

CG_API int cg_set_counting(int enable) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    g_env->counting = enable != 0;
    g_env->dropAllGraphs();
    return CG_OK;
  });
}

CG_API int cg_set_profiling(int enable) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    g_env->profiling = enable != 0;
    g_env->prof = cg_profile{};
    return CG_OK;
  });
}

CG_API int cg_profile_read(cg_profile* out) {
  return guarded([&]() -> int {
    if (!out) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *out = g_env->prof;
    g_env->prof = cg_profile{};
    return CG_OK;
  });
}

CG_API int cg_set_seed(uint32_t seed) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    g_env->seed = seed;
    return CG_OK;
  });
}

CG_API int cg_set_spectral(int mode) {
  return guarded([&]() -> int {
    if (mode != CG_SPECTRAL_REFERENCE && mode != CG_SPECTRAL_HERO)
      return fail(CG_E_INVALID, "unknown spectral sampling mode");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    if (env.spectral == mode) return CG_OK;
    CG_CUDA(cudaSetDevice(env.device));
    CG_CUDA(cudaStreamSynchronize(env.stream));
    env.dropAllGraphs();  // captured launch sequences use the other mode's kernels
    env.dropViewGraph();
    env.spectral = mode;
    env.hero = mode == CG_SPECTRAL_HERO;
    env.has_prev = false;  // the film's running mean restarts
    return env.syncHero();
  });
}

CG_API int cg_set_roulette(uint32_t start_depth) {
  return guarded([&]() -> int {
    if (start_depth > 64u) return fail(CG_E_INVALID, "roulette start depth beyond the trace depth cap");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    Env& env = *g_env;
    if (env.roulette == start_depth) return CG_OK;
    CG_CUDA(cudaSetDevice(env.device));
    CG_CUDA(cudaStreamSynchronize(env.stream));
    env.dropAllGraphs();  // captured launches hold the old setting
    env.dropViewGraph();
    env.roulette = start_depth;
    env.has_prev = false;  // the film's running mean restarts
    return CG_OK;
  });
}

CG_API int cg_get_spectral(int* mode) {
  return guarded([&]() -> int {
    if (!mode) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *mode = g_env->spectral;
    return CG_OK;
  });
}

CG_API int cg_set_tuning(const cg_tuning* t) {
  return guarded([&]() -> int {
    if (!t) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    // every field is checked before any is applied
    auto okBlock = [](uint32_t b) { return b == 0 || (b >= 32 && b <= 1024 && b % 32 == 0); };
    if (!okBlock(t->extend_block) || !okBlock(t->shade_block))
      return fail(CG_E_INVALID, "block sizes must be multiples of 32 in [32, 1024]");
    if (t->extend_block > 256u)  // the traversal kernels' launch bounds
      return fail(CG_E_INVALID, "extend_block must be at most 256");
    if (t->queue_capacity && (t->queue_capacity < 4096 || t->queue_capacity > (1u << 28)))
      return fail(CG_E_INVALID, "queue capacity must be in [4096, 2^28]");
    if (t->bvh_width && t->bvh_width != 2 && t->bvh_width != 4)
      return fail(CG_E_INVALID, "bvh_width must be 2 or 4");
    if (t->box_bits && t->box_bits != 8 && t->box_bits != 32)
      return fail(CG_E_INVALID, "box_bits must be 8 or 32");
    if (t->pipelines > static_cast<uint32_t>(Renderer::kMaxPipelines))
      return fail(CG_E_INVALID, "pipelines must be 1 to 4");
    if (t->shade_sort > 3u) return fail(CG_E_INVALID, "shade_sort must be 0..3");
    {
      const uint32_t eb = t->extend_block ? t->extend_block : g_env->tuning.extend_block;
      if (t->traversal_threads &&
          (t->traversal_threads > 1024u || t->traversal_threads < eb || t->traversal_threads % eb))
        return fail(CG_E_INVALID,
                    "traversal_threads must be a multiple of extend_block in [extend_block, 1024]");
    }
    cg_tuning& g = g_env->tuning;
    if (t->queue_capacity) g.queue_capacity = t->queue_capacity;
    if (t->box_bits) g.box_bits = t->box_bits;
    if (t->pipelines) g.pipelines = t->pipelines;
    if (t->extend_block) g.extend_block = t->extend_block;
    if (t->shade_block) g.shade_block = t->shade_block;
    if (t->bvh_width) g.bvh_width = t->bvh_width;
    if (t->persistent) g.persistent = t->persistent == 2u || t->persistent == 3u ? t->persistent : 1u;
    if (t->shade_sort) g.shade_sort = t->shade_sort;
    if (t->traversal_threads) g.traversal_threads = t->traversal_threads;
    if (g.traversal_threads % g.extend_block) g.traversal_threads = 1024u;  // a new block size
    g_env->tuning.use_graph = t->use_graph;
    g_env->dropAllGraphs();
    return CG_OK;
  });
}

CG_API int cg_get_tuning(cg_tuning* out) {
  return guarded([&]() -> int {
    if (!out) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    *out = g_env->tuning;
    return CG_OK;
  });
}

CG_API int cg_trace_closest(cg_scene_t scene, const float* rays, uint32_t n, cg_hit* hits) {
  return guarded([&]() -> int {
    if (!scene || (n && (!rays || !hits))) return fail(CG_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(g_env_mu);
    if (!g_env) return fail(CG_E_NOT_INIT, "Environment not initialized.");
    if (n == 0) return CG_OK;
    Env& env = *g_env;
    SceneDev* s = reinterpret_cast<SceneDev*>(scene);
    CG_CUDA(cudaSetDevice(env.device));
    DeviceArena a;
    const size_t rb = size_t(n) * 32, ob = size_t(n) * 16;
    int rc = a.alloc(align256(rb) + 2 * align256(ob) + 256);
    if (rc != CG_OK) return rc;
    char* p = static_cast<char*>(a.base);
    float4* d_rays = reinterpret_cast<float4*>(p);
    float4* d_tuv = reinterpret_cast<float4*>(p + align256(rb));
    int4* d_ids = reinterpret_cast<int4*>(p + align256(rb) + align256(ob));
    uint32_t* d_status = reinterpret_cast<uint32_t*>(p + align256(rb) + 2 * align256(ob));
    CG_CUDA(cudaMemcpyAsync(d_rays, rays, rb, cudaMemcpyHostToDevice, env.stream));
    CG_CUDA(cudaMemsetAsync(d_status, 0, 4, env.stream));
    launchTraceClosest(s->view, d_rays, n, d_tuv, d_ids, d_status, nodeFormatOf(env.tuning),
                       env.stream);
    CG_CUDA(cudaGetLastError());
    std::vector<float4> tuv(n);
    std::vector<int4> ids(n);
    uint32_t status = 0;
    CG_CUDA(cudaMemcpyAsync(tuv.data(), d_tuv, ob, cudaMemcpyDeviceToHost, env.stream));
    CG_CUDA(cudaMemcpyAsync(ids.data(), d_ids, ob, cudaMemcpyDeviceToHost, env.stream));
    CG_CUDA(cudaMemcpyAsync(&status, d_status, 4, cudaMemcpyDeviceToHost, env.stream));
    CG_CUDA(cudaStreamSynchronize(env.stream));
    if (status) return fail(CG_E_DEVICE, "traversal stack overflow in k_trace_closest");
    for (uint32_t i = 0; i < n; ++i) {
      cg_hit h{};
      h.t = tuv[i].x;
      h.u = tuv[i].y;
      h.v = tuv[i].z;
      h.instance = ids[i].x;
      h.triangle = ids[i].y;
      hits[i] = h;
    }
    return CG_OK;
  });
}

}  // extern "C"
