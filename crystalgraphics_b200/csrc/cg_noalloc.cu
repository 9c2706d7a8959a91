// cg_noalloc.cu — cg_render_noalloc: one view rendered with no allocation in
// the call.
//
// Some callers cannot call cudaMalloc while they render: a host application
// that owns the device memory budget and hands a plugin only the buffers it
// may touch, code that runs under a custom or pooled allocator that forbids
// driver allocations during a frame, or a real-time loop where an allocation
// (which may synchronise the device) would stall the frame.  For them this
// entry point runs the same wavefront kernels as cg_view / cg_batch_render,
// but its ray queues, sample slots, counters and wavelength table live in the
// file-scope device array `g_noalloc_scratch` below, which every GPU that
// loads this library holds until the process exits.  The caller passes the
// scene (uploaded earlier) and a film of its own; the call allocates nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/cg_cuda.h"
#include "cg_api_internal.h"

namespace cg {
namespace {

// Rays one level of the wavefront may hold in the scratch queues.
constexpr uint32_t kNoAllocRays = 1u << 17;
constexpr size_t Q = kNoAllocRays;
// Byte layout of the scratch (every part 256-byte aligned).
constexpr size_t kOffRayO0 = 0;
constexpr size_t kOffRayO1 = kOffRayO0 + Q * 16;
constexpr size_t kOffRayD0 = kOffRayO1 + Q * 16;
constexpr size_t kOffRayD1 = kOffRayD0 + Q * 16;
constexpr size_t kOffSlot0 = kOffRayD1 + Q * 16;
constexpr size_t kOffSlot1 = kOffSlot0 + Q * 4;
constexpr size_t kOffHit = kOffSlot1 + Q * 4;
constexpr size_t kOffHitInst = kOffHit + Q * 16;
constexpr size_t kOffShO = kOffHitInst + Q * 4;
constexpr size_t kOffShD = kOffShO + Q * 16;
constexpr size_t kOffShSlot = kOffShD + Q * 16;
constexpr size_t kOffSL = kOffShSlot + Q * 4;
constexpr size_t kOffSLambda = kOffSL + Q * 4;
constexpr size_t kOffSProb = kOffSLambda + Q * 4;
constexpr size_t kOffKey = kOffSProb + Q * 4;      // shading keys (1 B per ray)
constexpr size_t kOffPerm = kOffKey + Q;           // shading order
constexpr size_t kOffDefer = kOffPerm + Q * 4;     // light-pdf deferral (16 B per ray)
constexpr size_t kOffDeferDist = kOffDefer + Q * 16;  // its lobe values (4 B per ray)
constexpr size_t kOffCounts = kOffDeferDist + Q * 4;  // 256 B: queue counts
constexpr size_t kOffStats = kOffCounts + 256;     // 256 B: ray statistics
constexpr size_t kOffStatus = kOffStats + 256;     // 256 B: kernel status word
constexpr size_t kOffView = kOffStatus + 256;      // 256 B: the ViewDev table
constexpr size_t kOffWlTree = kOffView + 256;      // 65535 floats (+ pad)
constexpr size_t kOffWlConst = kOffWlTree + 65536 * 4;
constexpr size_t kScratchBytes = kOffWlConst + 256;
static_assert(sizeof(ViewDev) <= 256, "the view table slot holds one ViewDev");
static_assert(kOffCounts % 256 == 0 && kOffWlTree % 256 == 0, "256-byte aligned parts");

// ~21.9 MB per device; file scope so that only this file's host code asks for
// its address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceSetup {
  unsigned long long ctx_id = 0;  // the context the set-up belongs to (0 = none yet)
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch there
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

// Once per device and context, with that device current: the device address
// of the scratch (the host-side symbol is only a stand-in, never a device
// pointer) and the wavelength table, computed into the scratch.  A new context
// on the device (after a device reset, or another context made current) gets
// the set-up again: its copy of the array starts as zeros at a possibly new
// address.
int setupDevice(int dev, unsigned long long ctx, cudaStream_t stream, unsigned char** base) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (dev < 0 || dev >= kMaxDevices) return fail(CG_E_INVALID, "device index out of range");
  DeviceSetup& s = g_setup[dev];
  if (s.ctx_id != ctx) {
    s.ctx_id = 0;
    s.base = nullptr;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return cudaFail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    unsigned char* b = static_cast<unsigned char*>(ptr);
    launchWavelengthTree(reinterpret_cast<float*>(b + kOffWlTree),
                         reinterpret_cast<float*>(b + kOffWlConst), stream);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cudaFail(e, "wavelength table launch");
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cudaFail(e, "wavelength table");
    s.base = b;
    s.ctx_id = ctx;
  }
  *base = s.base;
  return CG_OK;
}

// The size of the device allocation that holds `p` from `p` on
// (cuMemGetAddressRange through the runtime's driver entry points); 0 when the
// driver cannot tell, in which case the caller's size is taken on trust.
size_t deviceBytesFrom(const void* p) {
  using GetRange = int (*)(unsigned long long*, size_t*, unsigned long long);
  static GetRange get_range = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_range = reinterpret_cast<GetRange>(fn);
    cudaGetLastError();
  });
  if (!get_range) return 0;
  unsigned long long lo = 0;
  size_t size = 0;
  const unsigned long long a = reinterpret_cast<unsigned long long>(p);
  if (get_range(&lo, &size, a) != 0 || a < lo || a - lo > size) return 0;
  return static_cast<size_t>(lo + size - a);
}

// A film argument must be device (or managed) memory of device `dev` with
// room for `bytes`.
int checkFilm(const void* p, size_t bytes, int dev, const char* name) {
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CG_E_INVALID, std::string(name) + " is not a device pointer");
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return fail(CG_E_INVALID, std::string(name) + " is not device memory");
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    return fail(CG_E_INVALID, std::string(name) + " belongs to device " + std::to_string(a.device) +
                                  ", not the current device " + std::to_string(dev));
  const size_t have = deviceBytesFrom(p);
  if (have != 0 && have < bytes)
    return fail(CG_E_INVALID, std::string(name) + " holds " + std::to_string(have) +
                                  " bytes from its start; the view needs " + std::to_string(bytes));
  return CG_OK;
}

WaveBuffers scratchBuffers(unsigned char* b) {
  WaveBuffers w{};
  w.ray_o[0] = reinterpret_cast<float4*>(b + kOffRayO0);
  w.ray_o[1] = reinterpret_cast<float4*>(b + kOffRayO1);
  w.ray_d[0] = reinterpret_cast<float4*>(b + kOffRayD0);
  w.ray_d[1] = reinterpret_cast<float4*>(b + kOffRayD1);
  w.ray_slot[0] = reinterpret_cast<uint32_t*>(b + kOffSlot0);
  w.ray_slot[1] = reinterpret_cast<uint32_t*>(b + kOffSlot1);
  w.hit = reinterpret_cast<float4*>(b + kOffHit);
  w.hit_inst = reinterpret_cast<int32_t*>(b + kOffHitInst);
  w.sh_o = reinterpret_cast<float4*>(b + kOffShO);
  w.sh_d = reinterpret_cast<float4*>(b + kOffShD);
  w.sh_slot = reinterpret_cast<uint32_t*>(b + kOffShSlot);
  w.s_L = reinterpret_cast<float*>(b + kOffSL);
  w.s_lambda = reinterpret_cast<float*>(b + kOffSLambda);
  w.s_prob = reinterpret_cast<float*>(b + kOffSProb);
  w.shade_key = b + kOffKey;
  w.shade_perm = reinterpret_cast<uint32_t*>(b + kOffPerm);
  w.defer = reinterpret_cast<float4*>(b + kOffDefer);
  w.defer_dist = reinterpret_cast<float*>(b + kOffDeferDist);
  w.counts = reinterpret_cast<uint32_t*>(b + kOffCounts);
  w.stats = reinterpret_cast<unsigned long long*>(b + kOffStats);
  w.status = reinterpret_cast<uint32_t*>(b + kOffStatus);
  w.capacity = kNoAllocRays;
  w.sample_capacity = kNoAllocRays;
  return w;
}

}  // namespace
}  // namespace cg

using namespace cg;

extern "C" CG_API int cg_render_noalloc(cg_scene_t scene, const cg_conf* conf,
                                        const cg_view_desc* view, void* film_xyzw,
                                        void* film_rgba8, void* stream) {
  return guarded([&]() -> int {
    if (!scene || !conf || !view || !film_xyzw)
      return fail(CG_E_INVALID, "null argument");
    if (view->width == 0 || view->height == 0 || view->spp == 0)
      return fail(CG_E_INVALID, "view has a zero size or spp");
    const uint64_t npx = uint64_t(view->width) * view->height;
    if (npx > 0xffffffffull)
      return fail(CG_E_INVALID, "view has more than 2^32 - 1 pixels");
    SceneDev& sd = *reinterpret_cast<SceneDev*>(scene);
    const Caps caps = capsOf(*conf);
    const LevelPlan plan = planLevels(caps, std::max(1u, sd.max_lobes));
    const uint64_t chunk = kNoAllocRays / std::max<uint64_t>(1, plan.max_product);
    if (view->spp > chunk)
      return fail(CG_E_INVALID,
                  "spp " + std::to_string(view->spp) + " exceeds the no-alloc scratch: at trace depth " +
                      std::to_string(caps.trace_depth) + " one chunk holds at most " +
                      std::to_string(chunk) + " samples (" + std::to_string(kNoAllocRays) +
                      " queued rays)");
    // everything runs on the caller's current device, which must be the one
    // (and the context) the scene was uploaded in
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cudaFail(e, "cudaGetDevice");
    if (dev != sd.device)
      return fail(CG_E_INVALID, "the scene was uploaded on device " + std::to_string(sd.device) +
                                    " but the current device is " + std::to_string(dev) +
                                    ": make the scene's device current first");
    unsigned long long ctx = 0;
    int rc = currentContextId(&ctx);
    if (rc != CG_OK) return rc;
    if (ctx != sd.ctx_id)
      return fail(CG_E_INVALID,
                  "the scene was uploaded in another CUDA context of this device (the device was "
                  "reset, or another context is current): its buffers are not valid here");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (s) {
      int sdev = -1;
      e = cudaStreamGetDevice(s, &sdev);
      if (e != cudaSuccess) return cudaFail(e, "cudaStreamGetDevice");
      if (sdev != dev)
        return fail(CG_E_INVALID, "the stream belongs to device " + std::to_string(sdev) +
                                      ", not the current device " + std::to_string(dev));
    }
    rc = checkFilm(film_xyzw, npx * 16, dev, "film_xyzw");
    if (rc != CG_OK) return rc;
    if (film_rgba8) {
      rc = checkFilm(film_rgba8, npx * 4, dev, "film_rgba8");
      if (rc != CG_OK) return rc;
    }
    unsigned char* base = nullptr;
    rc = setupDevice(dev, ctx, s, &base);
    if (rc != CG_OK) return rc;
    // what must start at zero: counters, statistics, status word
    e = cudaMemsetAsync(base + kOffCounts, 0, 3 * 256, s);
    if (e != cudaSuccess) return cudaFail(e, "cudaMemsetAsync(scratch counters)");
    ViewDev v;
    std::memset(&v, 0, sizeof(v));
    cameraBasis(view->camera, v);
    v.width = view->width;
    v.height = view->height;
    v.spp = view->spp;
    v.seed = view->seed;
    v.frame = 0;
    v.sample_weight = 1.0f;
    v.pixel_base = 0;
    v.pixel_count = static_cast<uint32_t>(npx);
    v.pixel_offset = 0;
    v.sample_offset = 0;
    v.film = static_cast<float4*>(film_xyzw);
    v.rgba = static_cast<uchar4*>(film_rgba8);
    // the view table goes into its scratch slot (a copy of a host struct, no
    // allocation); stream order keeps it ahead of the kernels
    e = cudaMemcpyAsync(base + kOffView, &v, sizeof(ViewDev), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cudaFail(e, "cudaMemcpyAsync(view table)");
    const WaveBuffers wb = scratchBuffers(base);
    FrameConst fc;
    fc.views = reinterpret_cast<const ViewDev*>(base + kOffView);
    fc.view_count = 1;
    fc.caps = caps;
    fc.wl_tree = reinterpret_cast<const float*>(base + kOffWlTree);
    fc.wl_const = reinterpret_cast<const float*>(base + kOffWlConst);
    LaunchShape ls;  // default block sizes
    const uint32_t cut_depth = std::max(1u, std::min(caps.trace_depth, 64u)) - 1u;
    uint64_t pix = 0, smp = 0;
    while (pix < npx) {  // the chunk sequence of Renderer::enqueueChunk
      ChunkDesc ch;
      ch.pixel_begin = pix;
      ch.sample_begin = smp;
      const uint64_t take = std::min<uint64_t>(npx - pix, chunk / v.spp);
      ch.pixel_count = static_cast<uint32_t>(take);
      ch.sample_count = static_cast<uint32_t>(take * v.spp);
      launchGen(fc, wb, ch, s);
      for (uint32_t d = 0; d < plan.levels; ++d) {
        const int parity = static_cast<int>(d & 1u);
        launchExtend(sd.view, wb, parity, false, ls, d >= cut_depth, s);
        launchShade(sd.view, fc, wb, static_cast<int>(d), parity, ls, s);
        if (plan.shadow[d]) launchShadow(sd.view, wb, false, ls, s);
      }
      launchResolve(fc, wb, ch, s);
      pix += take;
      smp += take * v.spp;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cudaFail(e, "wavefront launch");
    uint32_t status = 0;
    e = cudaMemcpyAsync(&status, base + kOffStatus, 4, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cudaFail(e, "cudaMemcpyAsync(status)");
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cudaFail(e, "cudaStreamSynchronize");
    if (status & 1u) return fail(CG_E_DEVICE, "traversal stack overflow in a kernel");
    if (status & 2u) return fail(CG_E_DEVICE, "ray queue overflow in a kernel");
    return CG_OK;
  });
}
