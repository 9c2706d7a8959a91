// cg_kernels.cu — the wavefront path tracer (sm_100a).
//
// The reference evaluates every camera sample as a depth-first tree inside
// one thread with a 64-frame private stack (trace.wesl:22-89).  Its result is
// linear in the children's radiance (backwardPass, shading.wesl:48-53), so
// here each tree node is a queued ray carrying the product of the transport
// coefficients above it; emission, environment and light-sample terms are
// added straight into the sample's radiance slot.  Trees are processed level
// by level: every level is one extend (closest hit), one shade and one shadow
// launch over all rays of that depth in the chunk.
#include "cg_kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <type_traits>

#include "cg_device.cuh"
#include "cg_traverse.cuh"

namespace cg {
namespace {

using namespace dev;

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }

// transpose(inv_trans) * vec4(n, 0) (bvh.wesl:110-111)
__device__ __forceinline__ V3 normalToWorld(const float* m, V3 n) {
  return {(m[0] * n.x + m[4] * n.y) + m[8] * n.z, (m[1] * n.x + m[5] * n.y) + m[9] * n.z,
          (m[2] * n.x + m[6] * n.y) + m[10] * n.z};
}

// ---- view lookup ------------------------------------------------------------
__device__ __forceinline__ uint32_t findViewBySample(const FrameConst& fc, uint64_t g) {
  uint32_t lo = 0, hi = fc.view_count;  // last view with sample_offset <= g
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (fc.views[mid].sample_offset <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}
__device__ __forceinline__ uint32_t findViewByPixel(const FrameConst& fc, uint64_t g) {
  uint32_t lo = 0, hi = fc.view_count;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (fc.views[mid].pixel_offset <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// ---- wavelength tree (physics/wavelength.wesl:24-45) ---------------------------
__global__ void k_wavelength_tree(float* tree, float* consts) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const float total = xyzMatchSumIntegral(380.0f, 720.0f);
  if (k == 0) {
    consts[0] = total;
    consts[1] = xyzMatchSumIntegral(380.0f, 720.0f) / 3.0f;
  }
  if (k >= 65535u) return;
  // replay the bisection path from the root to node k
  uint32_t path[16];
  int depth = 0;
  for (uint32_t x = k; x > 0; x = (x - 1u) >> 1) path[depth++] = x;
  float low = 380.0f, high = 720.0f;
  for (int i = depth - 1; i >= 0; --i) {
    const uint32_t x = path[i];
    const uint32_t parent = (x - 1u) >> 1;
    const float mid = 0.5f * (low + high);
    if (x == 2u * parent + 1u)
      high = mid;  // cdf >= target
    else
      low = mid;
  }
  const float mid = 0.5f * (low + high);
  tree[k] = xyzMatchSumIntegral(380.0f, mid) / total;
}

// ---- generate: one primary ray per sample (compute.wesl:32-62, render.wesl) ----
__global__ void k_gen(FrameConst fc, WaveBuffers wb, ChunkDesc ch) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    wb.counts[0] = ch.sample_count;
    wb.counts[2] = 0u;
    wb.counts[3] = 0u;  // work counters of the persistent traversal
    wb.counts[4] = 0u;
  }
  if (i >= ch.sample_count) return;
  const uint64_t g = ch.sample_begin + i;
  const ViewDev& v = fc.views[findViewBySample(fc, g)];
  const uint64_t local = g - v.sample_offset;
  const uint32_t lp = static_cast<uint32_t>(local / v.spp);
  const uint32_t k = static_cast<uint32_t>(local - uint64_t(lp) * v.spp);
  const uint32_t pixel = v.pixel_base + lp;
  const uint32_t px = pixel % v.width, py = pixel / v.width;
  const uint32_t key = sampleKey(v.seed, v.frame, pixel, k + v.sample_base);
  Rng wr;
  seedRng(wr, wavelengthKey(key));
  if (wb.hero) {  // the hero's offset; the four wavelengths follow from it
    wb.s_lambda[i] = heroOffset(randFloat(wr));
    wb.s_L4[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    wb.ray_w[0][i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  } else {
    const float lambda = sampleWavelengthTree(fc.wl_tree, randFloat(wr));
    const V3 xyz = xyzMatch(lambda);
    const float prob = fmaxf((xyz.x + xyz.y + xyz.z) / fc.wl_const[0], 1e-6f);
    wb.s_L[i] = 0.0f;
    wb.s_lambda[i] = lambda;
    wb.s_prob[i] = prob;
  }
  // cameraRay, rounded per operation like the host restatement
  const float cx = XS(XM(__fdiv_rn(static_cast<float>(px), static_cast<float>(v.width)), 2.0f), 1.0f);
  const float cy = XS(XM(__fdiv_rn(static_cast<float>(py), static_cast<float>(v.height)), 2.0f), 1.0f);
  float d[3];
  for (int a = 0; a < 3; ++a) d[a] = XA(XA(v.dir[a], XM(cx, v.dx[a])), XM(cy, v.dy[a]));
  const float len = __fsqrt_rn(XA(XA(XM(d[0], d[0]), XM(d[1], d[1])), XM(d[2], d[2])));
  wb.ray_o[0][i] = make_float4(v.pos[0], v.pos[1], v.pos[2], 1.0f);
  wb.ray_d[0][i] = make_float4(__fdiv_rn(d[0], len), __fdiv_rn(d[1], len), __fdiv_rn(d[2], len),
                               __uint_as_float(key));
  wb.ray_slot[0][i] = i;
}

// ---- shading keys (the level-wide shading order) ---------------------------------
// Key of a hit: 0 miss, 1 hit beyond the depth cut (no work), 2 + material
// kind; kNumKeys - 1 marks an empty slot.  The closest-hit kernel writes each
// ray's key and counts rays per key (counts[kKeyCount + k]); the block that
// finishes last turns the counts into the scatter cursors (counts[kKeyCursor
// + k], exclusive prefix sums) and zeroes the counts and the ticket
// (counts[kTicket]) for the next level.  No block waits for another.
constexpr int kNumKeys = 19;
constexpr int kTicket = 6, kKeyCount = 8, kKeyCursor = 32;

__device__ __forceinline__ int shadeKeyOf(const SceneView& sc, int32_t inst, bool cut) {
  if (inst < 0) return 0;
  if (cut) return 1;
  const uint4 meta = __ldg(reinterpret_cast<const uint4*>(sc.inst + inst) + 3);
  return 2 + static_cast<int>((sc.mat[meta.y].volume >> kKindShift) & 15u);
}

// The block's key counts of a keyed closest-hit launch (one shared array per
// block), flushed to the level's counts once at the end of the block.
__device__ __forceinline__ uint32_t* blockKeyCounts() {
  __shared__ uint32_t s_keycnt[kNumKeys];
  return s_keycnt;
}

// At the start of a keyed closest-hit launch (every thread of the block).
__device__ __forceinline__ void beginShadeKeys() {
  if (threadIdx.x < kNumKeys) blockKeyCounts()[threadIdx.x] = 0u;
  __syncthreads();
}

// keys: 0 none, 1 keys for a level shaded before the depth cut, 2 after it.
// Called by the lanes that finished a ray (one shared-memory atomic per
// distinct key among them).
__device__ __forceinline__ void writeShadeKey(const SceneView& sc, const WaveBuffers& wb, uint32_t i,
                                              int32_t inst, int keys) {
  const int key = shadeKeyOf(sc, inst, keys == 2);
  wb.shade_key[i] = static_cast<uint8_t>(key);
  const unsigned peers = __match_any_sync(__activemask(), key);
  if ((threadIdx.x & 31u) == static_cast<uint32_t>(__ffs(peers) - 1))
    atomicAdd(&blockKeyCounts()[key], static_cast<uint32_t>(__popc(peers)));
}

// At the end of a keyed closest-hit launch (every thread of the block): adds
// the block's counts to the level's, and the last block to finish turns the
// level's counts into the scatter cursors (exclusive scan).
__device__ __forceinline__ void finishShadeKeys(const WaveBuffers& wb) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x < kNumKeys) {
    const uint32_t c = blockKeyCounts()[threadIdx.x];
    if (c) atomicAdd(&wb.counts[kKeyCount + threadIdx.x], c);
    __threadfence();  // ordered before this block's ticket
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&wb.counts[kTicket], 1u) == gridDim.x - 1u;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    uint32_t off = 0;
    for (int k = 0; k < kNumKeys; ++k) {
      const uint32_t c = atomicExch(&wb.counts[kKeyCount + k], 0u);
      wb.counts[kKeyCursor + k] = off;
      off += c;
    }
    wb.counts[kTicket] = 0u;
  }
}

// ---- extend: closest hit --------------------------------------------------------
// Any hit / closest hit over the trees of node format kNodes (NodeFormat).
template <bool kAny, bool kCount, int kNodes>
__device__ __forceinline__ HitRec trace(const SceneView& sc, float4 o, float4 d, float tmax,
                                        TravCounters& cnt, uint32_t* status) {
  if (kNodes == kNodesWide4Q)
    return traceRay4<kAny, kCount, true>(sc, o.x, o.y, o.z, d.x, d.y, d.z, tmax, cnt, status);
  if (kNodes == kNodesWide4)
    return traceRay4<kAny, kCount, false>(sc, o.x, o.y, o.z, d.x, d.y, d.z, tmax, cnt, status);
  return traceRay<kAny, kCount>(sc, o.x, o.y, o.z, d.x, d.y, d.z, tmax, cnt, status);
}

// At most 64 registers per thread (4 blocks of 256 or 8 of 128 per SM).
// keys (writeShadeKey): also the level's shading keys and their counts.
template <bool kCount, int kNodes>
__global__ void __launch_bounds__(256, 4) k_extend(SceneView sc, WaveBuffers wb, int parity,
                                                   int keys) {
  // counts can exceed the capacity after an overflow (the appends are then
  // dropped and the status word set); never read past the queue
  const uint32_t n = min(wb.counts[parity], wb.capacity);
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    wb.counts[parity ^ 1] = 0u;
    wb.counts[2] = 0u;
    wb.counts[4] = 0u;
    atomicAdd(&wb.stats[0], static_cast<unsigned long long>(n));
  }
  if (keys) beginShadeKeys();
  TravCounters cnt{0u, 0u, 0u};
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = tid; i < n; i += stride) {
    const float4 o = wb.ray_o[parity][i];
    const float4 d = wb.ray_d[parity][i];
    HitRec h = trace<false, kCount, kNodes>(sc, o, d, MAXD, cnt, wb.status);
    wb.hit[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.tri));
    wb.hit_inst[i] = h.inst;
    if (keys) writeShadeKey(sc, wb, i, h.inst, keys);
  }
  if (keys) finishShadeKeys(wb);
  if (kCount) {
    unsigned long long a = cnt.nodes, b = cnt.tris, c = cnt.insts;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(kFull, a, o);
      b += __shfl_down_sync(kFull, b, o);
      c += __shfl_down_sync(kFull, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&wb.stats[2], a);
      atomicAdd(&wb.stats[3], b);
      atomicAdd(&wb.stats[4], c);
    }
  }
}

// ---- persistent traversal with lane refill -------------------------------------
// Secondary rays of one warp need very different numbers of steps; with one
// ray per lane the warp waits for its longest ray.  Here each warp loops over
// the queue: lanes advance their ray a bounded number of steps, and once at
// least kRefill lanes are idle the warp takes that many new rays from a
// per-launch work counter (one atomicAdd per refill).  kAny: shadow rays.
// An unoccluded shadow ray adds its light-sample term to its sample's slot
// (all four wavelengths' terms in hero-wavelength mode).
__device__ __forceinline__ void addShadowTerm(const WaveBuffers& wb, uint32_t i) {
  const uint32_t slot = wb.sh_slot[i];
  if (wb.hero) {
    const float4 x = wb.sh_w[i];
    atomicAdd(wb.s_L4 + slot, make_float4(wb.sh_o[i].w, x.x, x.y, x.z));
  } else {
    atomicAdd(&wb.s_L[slot], wb.sh_o[i].w);
  }
}

// (CG_STEP_BUDGET / CG_REFILL override them for measurements)
#ifndef CG_STEP_BUDGET
#define CG_STEP_BUDGET 16
#endif
#ifndef CG_REFILL
#define CG_REFILL 8
#endif
constexpr int kStepBudget = CG_STEP_BUDGET;
constexpr int kRefill = CG_REFILL;
// Closest-hit traversal stack entries per thread kept in shared memory
// (dynamic shared memory of the persistent closest-hit launch: kShortStack * 4
// bytes per thread).  Measured on the 1280x720 icosphere frame and the
// instanced scene: closest-hit launches 1-2% faster than with the whole stack
// in local memory, shadow launches 6-8% slower (their walks are short and the
// shared carve-out costs them L1), so shadow rays keep a local stack.
constexpr int kShortStack = 16;

// kSpec: closest hits over four-wide trees with postponed leaves (travStepsSpec).
template <bool kAny, bool kCount, int kNodes, bool kSpec = false>
__device__ __forceinline__ void persistentTraverse(const SceneView& sc, WaveBuffers& wb, uint32_t n,
                                                   uint32_t* work, int parity, int keys) {
  const uint32_t lane = threadIdx.x & 31u;
  TravCounters cnt{0u, 0u, 0u};
  extern __shared__ int32_t s_stack[];
  std::conditional_t<kAny, LocalStack, ShortStack<kShortStack>> stack;  // left uninitialised
  if constexpr (!kAny) {
    stack.col = s_stack + threadIdx.x;
    stack.stride = blockDim.x;
  }
  TravState st;
  int32_t ray = -1;
  int32_t leaf = kNoLeaf;  // kSpec: the parked BLAS leaf
  bool exhausted = false;
  while (true) {
    const unsigned idle = __ballot_sync(kFull, ray < 0);
    if (!exhausted && __popc(idle) >= kRefill) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(work, static_cast<uint32_t>(__popc(idle)));
      base = __shfl_sync(kFull, base, 0);
      if (base + static_cast<uint32_t>(__popc(idle)) >= n) exhausted = true;
      if (ray < 0) {
        const uint32_t i = base + static_cast<uint32_t>(__popc(idle & ((1u << lane) - 1u)));
        if (i < n) {
          ray = static_cast<int32_t>(i);
          if (kAny) {
            const float4 o = wb.sh_o[i], d = wb.sh_d[i];
            travInit(st, o, d, fminf(d.w, MAXD));
          } else {
            travInit(st, wb.ray_o[parity][i], wb.ray_d[parity][i], MAXD);
          }
        }
      }
    }
    if (__ballot_sync(kFull, ray >= 0) == 0) {
      if (exhausted) break;
      continue;
    }
    bool fin;
    if constexpr (kSpec) {  // every lane of the warp takes part in the leaf votes
      fin = travStepsSpec<kCount, kNodes == kNodesWide4Q>(sc, st, leaf, stack, kStepBudget, cnt,
                                                          wb.status, ray >= 0);
    } else {
      fin = ray >= 0 && travSteps<kAny, kCount, kNodes>(sc, st, stack, kStepBudget, cnt, wb.status);
    }
    if (ray >= 0 && fin) {
      if (kAny) {
        if (st.best.inst < 0) addShadowTerm(wb, static_cast<uint32_t>(ray));
      } else {
        wb.hit[ray] = make_float4(st.best.t, st.best.u, st.best.v, __uint_as_float(st.best.tri));
        wb.hit_inst[ray] = st.best.inst;
        if (keys) writeShadeKey(sc, wb, static_cast<uint32_t>(ray), st.best.inst, keys);
      }
      ray = -1;
    }
  }
  if (kCount) {
    unsigned long long a = cnt.nodes, b = cnt.tris, c = cnt.insts;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(kFull, a, o);
      b += __shfl_down_sync(kFull, b, o);
      c += __shfl_down_sync(kFull, c, o);
    }
    if (lane == 0) {
      atomicAdd(&wb.stats[2], a);
      atomicAdd(&wb.stats[3], b);
      atomicAdd(&wb.stats[4], c);
    }
  }
}

// counts[3] (extend) and counts[4] (shadow) are the work counters; each is
// zeroed by the kernel before its user in stream order (k_gen for depth 0,
// k_shade for the next extend, k_extend for the shadow launch after it).
#ifdef CG_TRAV_MAXNREG  // a measurement switch: another register cap for the closest-hit walk
#define CG_EXTEND_BOUNDS __maxnreg__(CG_TRAV_MAXNREG)
#else
#define CG_EXTEND_BOUNDS __launch_bounds__(256, 4)
#endif
template <bool kCount, int kNodes, bool kSpec = false>
__global__ void CG_EXTEND_BOUNDS k_extend_persistent(SceneView sc, WaveBuffers wb,
                                                              int parity, int keys) {
  const uint32_t n = min(wb.counts[parity], wb.capacity);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    wb.counts[parity ^ 1] = 0u;
    wb.counts[2] = 0u;
    wb.counts[4] = 0u;
    atomicAdd(&wb.stats[0], static_cast<unsigned long long>(n));
  }
  if (keys) beginShadeKeys();
  persistentTraverse<false, kCount, kNodes, kSpec>(sc, wb, n, &wb.counts[3], parity, keys);
  if (keys) finishShadeKeys(wb);
}

template <bool kCount, int kNodes>
__global__ void __launch_bounds__(256, 4) k_shadow_persistent(SceneView sc, WaveBuffers wb) {
  const uint32_t n = min(wb.counts[2], wb.capacity);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&wb.stats[1], static_cast<unsigned long long>(n));
  persistentTraverse<true, kCount, kNodes>(sc, wb, n, &wb.counts[4], 0, 0);
}

// ---- shadow: t-bounded any hit (solveEmission, trace.wesl:91-113) ----------------
template <bool kCount, int kNodes>
__global__ void __launch_bounds__(256, 4) k_shadow(SceneView sc, WaveBuffers wb) {
  const uint32_t n = min(wb.counts[2], wb.capacity);
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) atomicAdd(&wb.stats[1], static_cast<unsigned long long>(n));
  TravCounters cnt{0u, 0u, 0u};
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = tid; i < n; i += stride) {
    const float4 o = wb.sh_o[i];
    const float4 d = wb.sh_d[i];
    // occluded iff the closest hit (< 1e6) is nearer than expected - 1e-3
    const float tmax = fminf(d.w, MAXD);
    HitRec h = trace<true, kCount, kNodes>(sc, o, d, tmax, cnt, wb.status);
    if (h.inst < 0) addShadowTerm(wb, i);
  }
  if (kCount) {
    unsigned long long a = cnt.nodes, b = cnt.tris, c = cnt.insts;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(kFull, a, o);
      b += __shfl_down_sync(kFull, b, o);
      c += __shfl_down_sync(kFull, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&wb.stats[2], a);
      atomicAdd(&wb.stats[3], b);
      atomicAdd(&wb.stats[4], c);
    }
  }
}

// ---- light pdf: sum over every emissive triangle the ray meets -------------------
// (pdf/emission.wesl:120-179).  A BVH over the emissive triangles finds them;
// the terms are added in traversal order rather than buffer order.  Every
// operation is rounded explicitly (no contraction to FMA), so each compiled
// copy of the walk (inside a shading kernel, or in k_light_pdf) returns the
// same bits for the same ray: whether a ray grazing a triangle edge counts
// that triangle must not depend on which kernel asked.
__device__ __forceinline__ float dotRn(V3 a, V3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V3 crossRn(V3 a, V3 b) {
  return V3{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}

__device__ __forceinline__ float triangleHitDist(V3 rp, V3 rd, const DevLightTri& L) {
  const V3 e1 = ld3(L.e1), e2 = ld3(L.e2);
  const V3 pv = crossRn(rd, e2);
  const float det = dotRn(e1, pv);
  if (fabsf(det) <= 1e-3f) return -1.0f;
  const float inv_det = __fdiv_rn(1.0f, det);
  const V3 tv{__fsub_rn(rp.x, L.v0[0]), __fsub_rn(rp.y, L.v0[1]), __fsub_rn(rp.z, L.v0[2])};
  const float bu = __fmul_rn(dotRn(tv, pv), inv_det);
  if (bu < 0.0f || bu > 1.0f) return -1.0f;
  const V3 qv = crossRn(tv, e1);
  const float bv = __fmul_rn(dotRn(rd, qv), inv_det);
  if (bv < 0.0f || __fadd_rn(bu, bv) > 1.0f) return -1.0f;
  const float hd = __fmul_rn(dotRn(e2, qv), inv_det);
  return hd > 1e-3f ? hd : -1.0f;
}

__device__ float lightPdf(const SceneView& sc, V3 pos, V3 next, uint32_t* status) {
  if (!sc.has_lights) return 0.0f;
  const float len = __fsqrt_rn(dotRn(next, next));
  const V3 rd{__fdiv_rn(next.x, len), __fdiv_rn(next.y, len), __fdiv_rn(next.z, len)};
  const float idx = safeInv(rd.x), idy = safeInv(rd.y), idz = safeInv(rd.z);
  const float oix = __fmul_rn(pos.x, idx), oiy = __fmul_rn(pos.y, idy), oiz = __fmul_rn(pos.z, idz);
  int32_t stack[32];
  int sp = 0;
  int32_t node = 0;
  float pdf = 0.0f;
  while (true) {
    while (node >= 0) {
      const float4* np = reinterpret_cast<const float4*>(sc.light_bvh + node);
      const float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
      const int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
      const float a0 = fmaf(n0.x, idx, -oix), a1 = fmaf(n0.y, idx, -oix);
      const float b0 = fmaf(n0.z, idy, -oiy), b1 = fmaf(n0.w, idy, -oiy);
      const float c0 = fmaf(n2.x, idz, -oiz), c1 = fmaf(n2.y, idz, -oiz);
      const float t0min = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), 0.0f));
      const float t0max = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fmaxf(c0, c1));
      const float d0 = fmaf(n1.x, idx, -oix), d1 = fmaf(n1.y, idx, -oix);
      const float e0 = fmaf(n1.z, idy, -oiy), e1 = fmaf(n1.w, idy, -oiy);
      const float f0 = fmaf(n2.z, idz, -oiz), f1 = fmaf(n2.w, idz, -oiz);
      const float t1min = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fmaxf(fminf(f0, f1), 0.0f));
      const float t1max = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fmaxf(f0, f1));
      // a child exists if it is an inner node or a leaf with triangles
      const bool h0 = t0min <= t0max && (n3.x >= 0 || n3.z != 0);
      const bool h1 = t1min <= t1max && (n3.y >= 0 || n3.w != 0);
      if (h0 && h1) {
        if (sp >= 32) {
          atomicOr(status, 1u);
          return pdf;
        }
        stack[sp++] = n3.y;
        node = n3.x;
      } else if (h0) {
        node = n3.x;
      } else if (h1) {
        node = n3.y;
      } else {
        node = sp > 0 ? stack[--sp] : kDone;
      }
    }
    if (node == kDone) break;
    const uint32_t first = static_cast<uint32_t>(~node) >> 3;
    const uint32_t count = static_cast<uint32_t>(~node) & 7u;
    for (uint32_t k = 0; k < count; ++k) {
      const DevLightTri L = sc.light_tri[first + k];
      const float hd = triangleHitDist(pos, rd, L);
      if (hd <= 0.0f) continue;
      const float lp = fabsf(dotRn(ld3(L.n), rd));
      pdf = __fadd_rn(pdf, __fdiv_rn(__fmul_rn(__fmul_rn(L.area_pdf, hd), hd), fmaxf(lp, 1e-3f)));
    }
    node = sp > 0 ? stack[--sp] : kDone;
  }
  return pdf;
}

// ---- environment (environment.wesl:7-25) -----------------------------------------
__device__ __forceinline__ float envRadiance(const SceneView& sc, V3 dir, const SmitsPos& sp) {
  V3 d = normalize(dir);
  float u = atan2f(d.y, d.x) / (2.0f * PI) + 0.5f;
  float v = acosf(wclamp(d.z, -1.0f, 1.0f)) / PI;
  float wu = u - floorf(u);
  float cv = wclamp(1.0f - v, 0.0f, 0.999999f);
  uint32_t x = min(sc.env_w - 1u, u32f(wu * static_cast<float>(sc.env_w)));
  uint32_t y = min(sc.env_h - 1u, u32f(cv * static_cast<float>(sc.env_h)));
  float4 t = __ldg(sc.env + size_t(y) * sc.env_w + x);
  return rgbToRadiance(V3{t.x, t.y, t.z}, sp);
}

enum { M_NONE = 0, M_DIFFUSE = 1, M_SREFL = 2, M_RREFL = 3, M_STRANS = 4, M_RTRANS = 5 };

// balancePdfDenominator (sample.wesl:505-554).  A lobe (or the light) with a
// zero sample count contributes 0 * pdf = 0; its pdf is not evaluated.
// Lobe groups of a shading kernel (kLobes): lobes outside the mask have zero
// sample counts for every ray the kernel takes, so their code is left out.
constexpr int kLobeHit = 1, kLobeDiffuse = 2, kLobeReflect = 4, kLobeTransmit = 8;
constexpr int kLobesAll = kLobeHit | kLobeDiffuse | kLobeReflect | kLobeTransmit;

// The lobes' part of the denominator: the sum before the light term is added.
template <int kLobes = kLobesAll>
__device__ __forceinline__ float balanceSum(V3 curr, V3 next, const Surf& s, const Mat& m,
                                            const Counts& c, int model, float model_pdf) {
  float pd = 0.0f, psr = 0.0f, prr = 0.0f, pst = 0.0f, prt = 0.0f;
  if ((kLobes & kLobeDiffuse) && c.diffuse)
    pd = model == M_DIFFUSE ? model_pdf : diffusePdf(curr, next, s);
  if ((kLobes & kLobeReflect) && c.specular_reflect)
    psr = model == M_SREFL ? model_pdf : specularReflectPdf(curr, next, s);
  if ((kLobes & kLobeReflect) && c.rough_reflect)
    prr = model == M_RREFL ? model_pdf : roughReflectPdf(curr, next, s, m);
  if ((kLobes & kLobeTransmit) && c.specular_transmit)
    pst = model == M_STRANS ? model_pdf : specularTransmitPdf(curr, next, s, m);
  if ((kLobes & kLobeTransmit) && c.rough_transmit)
    prt = model == M_RTRANS ? model_pdf : roughTransmitPdf(curr, next, s, m);
  // rounded explicitly: the deferred light term (k_light_pdf) is added to this
  // value and must give the denominator balanceDenom gives
  float sum = __fmul_rn(static_cast<float>(c.diffuse), pd);
  sum = __fadd_rn(sum, __fmul_rn(static_cast<float>(c.specular_reflect), psr));
  sum = __fadd_rn(sum, __fmul_rn(static_cast<float>(c.rough_reflect), prr));
  sum = __fadd_rn(sum, __fmul_rn(static_cast<float>(c.specular_transmit), pst));
  return __fadd_rn(sum, __fmul_rn(static_cast<float>(c.rough_transmit), prt));
}

template <int kLobes = kLobesAll>
__device__ __forceinline__ float balanceDenom(const SceneView& sc, V3 curr, V3 next, const Surf& s,
                                              const Mat& m, const Counts& c, int model,
                                              float model_pdf, float light_pdf_in,
                                              uint32_t* status) {
  const float sum = balanceSum<kLobes>(curr, next, s, m, c, model, model_pdf);
  float pl = 0.0f;
  if (c.light) pl = light_pdf_in >= 0.0f ? light_pdf_in : lightPdf(sc, s.pos, next, status);
  return fmaxf(__fadd_rn(sum, __fmul_rn(static_cast<float>(c.light), pl)), 1e-6f);
}

// spawnSurfaceRay (spawn_surface_ray.wesl:4-15)
__device__ __forceinline__ V3 spawnOrigin(const Surf& s, V3 next) {
  V3 on = dot(next, s.gn) > 0.0f ? s.gn : -s.gn;
  return s.pos + on * 1e-3f;
}

struct Child {
  V3 o, d;
  float w;
  uint32_t key;
};

// Hero mode, a deferred child (k_light_pdf completes it): bit 1 of its ray_w
// flags says its weight takes the factor kHeroCount (the wavelengths sample
// differently at its parent and the hero goes alone below).
constexpr uint32_t kDeferredKw = 2u;

// Russian roulette (an option beyond the reference, which has none): a child
// spawned at a hit of depth >= FrameConst::roulette survives with
// q = min(1, its path weight t) and then carries t / q.  Returns the factor
// 1 / q, or 0 when the child is dropped; one number from the child's
// roulette stream decides.
__device__ __forceinline__ float rouletteFactor(float t, uint32_t child_key) {
  const float q = fminf(1.0f, t);
  if (!(q < 1.0f)) return 1.0f;
  Rng r;
  seedRng(r, rouletteKey(child_key));
  return randFloat(r) < q ? 1.0f / q : 0.0f;
}

// A lobe's value at a direction (the dist functions of shading/dist/*.wesl).
__device__ __forceinline__ float lobeDist(int model, V3 curr, V3 next, const Surf& s, const Mat& m) {
  switch (model) {
    case M_DIFFUSE: return diffuseDist(curr, next, s, m);
    case M_SREFL: return specularReflectDist(curr, next, s, m);
    case M_RREFL: return roughReflectDist(curr, next, s, m);
    case M_STRANS: return specularTransmitDist(curr, next, s, m);
    case M_RTRANS: return roughTransmitDist(curr, next, s, m);
  }
  return 0.0f;
}

// ---- shade: one tree node per ray ------------------------------------------------
// Places every ray at its key's cursor: shade_perm lists the level's rays
// grouped by key.  A block takes tiles of kScatterTile rays: each warp ranks
// its 512 rays per key in shared memory (one match per 32 rays), the block
// claims its range of every key with one global atomic per key and tile, and
// the rays are written from registers.  (One global atomic per key and warp
// serialised on the 19 cursors and took ~400 us per 8M-ray level.)
constexpr int kScatterBlock = 256, kScatterItems = 16;
constexpr int kScatterWarps = kScatterBlock / 32;
constexpr uint32_t kScatterTile = kScatterBlock * kScatterItems;

__global__ void __launch_bounds__(kScatterBlock) k_shade_scatter(WaveBuffers wb, int parity) {
  __shared__ uint32_t s_cnt[kScatterWarps][kNumKeys];
  __shared__ uint32_t s_off[kScatterWarps][kNumKeys];
  const uint32_t n = min(wb.counts[parity], wb.capacity);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned lower = (1u << lane) - 1u;
  for (uint32_t base = blockIdx.x * kScatterTile; base < n; base += gridDim.x * kScatterTile) {
    for (uint32_t k = threadIdx.x; k < kScatterWarps * kNumKeys; k += kScatterBlock)
      (&s_cnt[0][0])[k] = 0u;
    __syncthreads();
    const uint32_t first = base + warp * (32u * kScatterItems) + lane;
    uint32_t key[kScatterItems], rank[kScatterItems];
#pragma unroll
    for (int r = 0; r < kScatterItems; ++r) {
      const uint32_t i = first + 32u * r;
      const int k = i < n ? wb.shade_key[i] : kNumKeys - 1;  // kNumKeys - 1: no ray
      const unsigned peers = __match_any_sync(kFull, k);
      const int leader = __ffs(peers) - 1;
      uint32_t before = 0;
      if (static_cast<int>(lane) == leader) {
        before = s_cnt[warp][k];
        s_cnt[warp][k] = before + static_cast<uint32_t>(__popc(peers));
      }
      before = __shfl_sync(kFull, before, leader);
      key[r] = static_cast<uint32_t>(k);
      rank[r] = before + static_cast<uint32_t>(__popc(peers & lower));
    }
    __syncthreads();
    if (threadIdx.x < kNumKeys - 1) {
      const uint32_t k = threadIdx.x;
      uint32_t total = 0;
      for (int w = 0; w < kScatterWarps; ++w) {
        s_off[w][k] = total;
        total += s_cnt[w][k];
      }
      const uint32_t at = total ? atomicAdd(&wb.counts[kKeyCursor + k], total) : 0u;
      for (int w = 0; w < kScatterWarps; ++w) s_off[w][k] += at;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kScatterItems; ++r) {
      if (key[r] == kNumKeys - 1) continue;
      const uint32_t at = s_off[warp][key[r]] + rank[r];
      if (at < wb.capacity) wb.shade_perm[at] = first + 32u * r;
    }
    __syncthreads();  // s_cnt / s_off are rewritten by the next tile
  }
}

// kLobes: the lobe group (kLobesAll unless the level is in global shading
// order, where one launch per group takes its keys' contiguous range of the
// permutation: keys [0, 2) misses and hits beyond the depth cut, [2, 10) opaque
// kinds, [10, 18) kinds with transmission; see shadeKeyOf).
// kSort (ShadeSort): kShadeSortBlock — before shading, every block sorts its
// slice of the queue by shading key in shared memory (counting sort);
// kShadeSortGlobal — the level was sorted (keys from the closest-hit kernel,
// permutation from k_shade_scatter) and the kernel takes rays in that order.  Either way a warp shades misses,
// cut hits or one material kind rather than a mix of code paths.
//
// kHero: hero-wavelength mode.  The tree is drawn at the hero wavelength (the
// material, sample counts, directions and balance denominators at it), and
// each ray also carries the path weights of the three other wavelengths: a
// child's weight for wavelength j is the lobe's value at that wavelength over
// the hero's denominator.  The reference's estimator weighs each lobe's
// sample by that lobe alone over the balance denominator (sample.wesl:
// 452-501), so its expectation depends on the counts and pdfs at the
// wavelength; at a hit where they differ across the four wavelengths (a lobe
// heuristic that vanishes at some of them, or a transmission whose refraction
// index varies with the wavelength) the light sample and the subtree carry
// the hero alone with weight 4 — over the four equally likely heroes of one
// wavelength set that is the reference's estimator at each of them.
// Emission is exact per wavelength.
// kLight: the level can draw light samples (false: no ray of the level has a
// light-sample count, so the light sample and the light pdf's code are left out).
// kDefer (with kLight): children leave the light-pdf term of their
// denominators to k_light_pdf (WaveBuffers::defer, and defer_w in hero mode).
template <int kSort, int kLobes, bool kHero, bool kLight = true, bool kDefer = false>
__device__ __forceinline__ void shadeLevel(const SceneView& sc, const FrameConst& fc,
                                           const WaveBuffers& wb, int depth, int parity) {
  stageSmitsTables();
  const uint32_t n = min(wb.counts[parity], wb.capacity);
  // [lo, hi): the queue slice (or, in global order, the permutation range of
  // this launch's keys) the launch takes
  uint32_t lo = 0, hi = n;
  if (kSort == kShadeSortGlobal) {
    // after k_shade_scatter every cursor is the end of its key's range
    constexpr int k0 = kLobes == 0 ? 0 : (kLobes & kLobeTransmit) ? 10 : 2;
    constexpr int k1 = kLobes == 0 ? 2 : (kLobes & kLobeTransmit) ? kNumKeys - 1 : 10;
    lo = k0 == 0 ? 0u : min(wb.counts[kKeyCursor + k0 - 1], n);
    hi = min(wb.counts[kKeyCursor + k1 - 1], n);
  }
  const uint32_t lane = threadIdx.x & 31u;
  const int out = parity ^ 1;
  __shared__ int s_cnt[kNumKeys];
  __shared__ int s_off[kNumKeys];
  __shared__ uint16_t s_order[256];
  const uint32_t cut_depth = max(1u, min(fc.caps.trace_depth, 64u)) - 1u;
  const SampleCaps caps{fc.caps.trace_depth, fc.caps.transport_cap, fc.caps.emission_cap,
                        fc.caps.diffuse_cap, fc.caps.rough_cap};
  // the next extend's work counter, zeroed by the level's first shading launch
  if ((kSort != kShadeSortGlobal || kLobes == 0) && blockIdx.x == 0 && threadIdx.x == 0)
    wb.counts[3] = 0u;
  for (uint32_t bbase = lo + blockIdx.x * blockDim.x; bbase < hi; bbase += gridDim.x * blockDim.x) {
    uint32_t i = bbase + threadIdx.x;
    if (kSort == kShadeSortGlobal) i = i < hi ? wb.shade_perm[i] : n;  // n: no ray
    if (kSort == kShadeSortBlock) {
      const int key = i < n ? shadeKeyOf(sc, wb.hit_inst[i], static_cast<uint32_t>(depth) >= cut_depth)
                            : kNumKeys - 1;
      if (threadIdx.x < kNumKeys) s_cnt[threadIdx.x] = 0;
      __syncthreads();
      const int rank = atomicAdd(&s_cnt[key], 1);
      __syncthreads();
      if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < kNumKeys; ++k) {
          s_off[k] = acc;
          acc += s_cnt[k];
        }
      }
      __syncthreads();
      s_order[s_off[key] + rank] = static_cast<uint16_t>(threadIdx.x);
      __syncthreads();
      i = bbase + s_order[threadIdx.x];
      __syncthreads();  // s_order / s_cnt are rewritten by the next slice
    }
    Child ch[4];
    // hero mode: per child the other wavelengths' weights and the flags (bit 0:
    // the hero alone below)
    float4 chw[kHero ? 4 : 1];
    // kDefer: per child its denominator without the light-pdf term (x; -1:
    // the weight is final) and its lobe value (y); in hero mode also the
    // other wavelengths' lobe values
    float2 cha[kDefer ? 4 : 1];
    float3 chd[kDefer && kHero ? 4 : 1];
    uint32_t nch = 0;
    bool shadow = false;
    float4 sh_o = make_float4(0, 0, 0, 0), sh_d = make_float4(0, 0, 0, 0);
    float4 sh_x = make_float4(0, 0, 0, 0);  // hero mode: the other wavelengths' terms
    V3 dpos{0.0f, 0.0f, 0.0f};  // the hit, for the children's deferred light-pdf terms
    uint32_t slot = 0;
    if (i < n) {
      const float4 o4 = wb.ray_o[parity][i];
      const float4 d4 = wb.ray_d[parity][i];
      slot = wb.ray_slot[parity][i];
      const V3 ro{o4.x, o4.y, o4.z}, rd{d4.x, d4.y, d4.z};
      const float W = o4.w;
      const uint32_t key = __float_as_uint(d4.w);
      const float4 h4 = wb.hit[i];
      const int32_t hinst = wb.hit_inst[i];
      // hero mode: the other wavelengths' weights, and whether the hero goes alone
      float4 Wx = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      bool alone = false;
      float x0 = 0.0f;
      if constexpr (kHero) {
        Wx = wb.ray_w[parity][i];
        alone = (__float_as_uint(Wx.w) & 1u) != 0u;
        x0 = wb.s_lambda[slot];
      }
      const float lambda = kHero ? heroWavelength(x0, 0) : wb.s_lambda[slot];
      const SmitsPos spos = smitsPos(lambda);
      float addL = 0.0f;
      float4 addX = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // hero mode: wavelengths 1..3
      if (hinst < 0) {
        addL = W * envRadiance(sc, rd, spos);
        if constexpr (kHero) {
          if (!alone) {
            addX.x = Wx.x * envRadiance(sc, rd, smitsPos(heroWavelength(x0, 1)));
            addX.y = Wx.y * envRadiance(sc, rd, smitsPos(heroWavelength(x0, 2)));
            addX.z = Wx.z * envRadiance(sc, rd, smitsPos(heroWavelength(x0, 3)));
          }
        }
      } else if ((kLobes & kLobeHit) && static_cast<uint32_t>(depth) < cut_depth) {
        // surface frame of the closest hit (bvh.wesl:102-129, 167-179)
        const uint32_t tri = __float_as_uint(h4.w);
        const float t = h4.x, u = h4.y, v = h4.z;
        const DevInstance* ip = sc.inst + hinst;
        const float4* ipf = reinterpret_cast<const float4*>(ip);
        const float4 r0 = __ldg(ipf), r1 = __ldg(ipf + 1), r2 = __ldg(ipf + 2);
        const uint4 meta = __ldg(reinterpret_cast<const uint4*>(ipf + 3));
        const float inv[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
        const uint4 vi = __ldg(sc.tri_vidx + tri);
        const float4 N0 = __ldg(sc.vnormal + vi.x), N1 = __ldg(sc.vnormal + vi.y),
                     N2 = __ldg(sc.vnormal + vi.z);
        const float4 E1 = __ldg(sc.tris + 3u * tri + 1u), E2 = __ldg(sc.tris + 3u * tri + 2u);
        const float w0 = 1.0f - u - v;
        const V3 ln = normalize(w0 * V3{N0.x, N0.y, N0.z} + u * V3{N1.x, N1.y, N1.z} +
                                v * V3{N2.x, N2.y, N2.z});
        const V3 lgn = normalize(cross(V3{E1.x, E1.y, E1.z}, V3{E2.x, E2.y, E2.z}));
        const V3 wgn = normalize(normalToWorld(inv, lgn));
        const V3 wsn = normalize(normalToWorld(inv, ln));
        Surf s;
        s.pos = ro + t * rd;
        s.gn = wgn;
        s.sn = dot(wsn, wgn) >= 0.0f ? wsn : -wsn;
        const DevMaterial& dmat = sc.mat[meta.y];
        Mat m;
        float4 uv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (dmat.volume & kTexturedBit) {
          // the hit's texture coordinates (bvh.wesl:172-179)
          const float4 a = __ldg(sc.vuv + vi.x), b = __ldg(sc.vuv + vi.y), cc = __ldg(sc.vuv + vi.z);
          uv = make_float4(w0 * a.x + u * b.x + v * cc.x, w0 * a.y + u * b.y + v * cc.y,
                           w0 * a.z + u * b.z + v * cc.z, w0 * a.w + u * b.w + v * cc.w);
          m = decodeTextured(sc, dmat, sc.mattex[meta.y], uv, lambda, spos);
        } else {
          m = decode(dmat, lambda, spos);
        }
        const Counts c = counts(m, kLight && sc.has_lights != 0u, depth, caps);
        // hero mode: the other wavelengths' materials, and whether all four
        // sample alike here (same counts; the same refraction index where a
        // transmission lobe is sampled)
        Mat mx[kHero ? 3 : 1];
        bool uniform = false;
        float kw = 1.0f;
        if constexpr (kHero) {
          uniform = !alone;
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const float lj = heroWavelength(x0, j + 1);
            mx[j] = (dmat.volume & kTexturedBit)
                        ? decodeTextured(sc, dmat, sc.mattex[meta.y], uv, lj, smitsPos(lj))
                        : decode(dmat, lj, smitsPos(lj));
            if (!sameCounts(counts(mx[j], sc.has_lights != 0u, depth, caps), c)) uniform = false;
            if ((c.specular_transmit || c.rough_transmit) && mx[j].ior.re != m.ior.re) uniform = false;
          }
          kw = (uniform || alone) ? 1.0f : static_cast<float>(kHeroCount);
          if (!alone) {
            addX.x = Wx.x * mx[0].emission;
            addX.y = Wx.y * mx[1].emission;
            addX.z = Wx.z * mx[2].emission;
          }
        }
        Rng rng;
        seedRng(rng, key);
        addL = W * m.emission;
        const V3 curr = rd;
        uint32_t ti = 0;  // transport sample index (child key)
        // kDefer: a child whose denominator has a light term leaves it to
        // k_light_pdf (the light-pdf walk then runs in a small kernel at full
        // occupancy, not in this one): it carries the parent's weight, and its
        // lobe value and denominator without the light term go beside it, so
        // the weight is completed as W * (dist / denom) like the others.  The
        // light count is 0
        // or 1 (the emission budget is capped at 1), and roulette, which needs
        // the final weight, is never active on a level launched with kDefer.
        const bool roulette =
            !kDefer && fc.roulette != 0u && static_cast<uint32_t>(depth) >= fc.roulette;
        if constexpr (kDefer) dpos = s.pos;
        auto push = [&](V3 next, int model, float prob, float dist) {
          float denom = 1.0f, a = -1.0f;
          if constexpr (kDefer) {
            a = balanceSum<kLobes>(curr, next, s, m, c, model, prob);
            if (c.light == 0u) {  // nothing to defer: balanceDenom's value
              denom = fmaxf(a, 1e-6f);
              a = -1.0f;
            }
          } else {
            denom = balanceDenom<kLobes>(sc, curr, next, s, m, c, model, prob, -1.0f, wb.status);
          }
          const float coeff = dist / denom;
          const uint32_t ck = childKey(key, ti++);
          if constexpr (kHero) {
            float cw = W * coeff * kw;
            float c1 = 0.0f, c2 = 0.0f, c3 = 0.0f;
            float3 dx = make_float3(0.0f, 0.0f, 0.0f);  // the other wavelengths' lobe values
            if (uniform) {
              dx = make_float3(lobeDist(model, curr, next, s, mx[0]), lobeDist(model, curr, next, s, mx[1]),
                               lobeDist(model, curr, next, s, mx[2]));
              c1 = Wx.x * (dx.x / denom);
              c2 = Wx.y * (dx.y / denom);
              c3 = Wx.z * (dx.z / denom);
            }
            if (roulette) {
              const float tmax = fmaxf(fmaxf(cw, 0.0f), fmaxf(fmaxf(c1, c2), c3));
              if (tmax == 0.0f) return;
              const float rr = rouletteFactor(tmax, ck);
              if (rr == 0.0f) return;
              cw = cw * rr;
              c1 = c1 * rr;
              c2 = c2 * rr;
              c3 = c3 * rr;
            }
            if (cw != 0.0f || c1 != 0.0f || c2 != 0.0f || c3 != 0.0f) {
              uint32_t flags = uniform ? 0u : 1u;
              if constexpr (kDefer) {
                cha[nch] = make_float2(a, dist);
                if (a != -1.0f) {  // completed by k_light_pdf: the parent's weights stay
                  cw = W;
                  c1 = Wx.x;
                  c2 = Wx.y;
                  c3 = Wx.z;
                  chd[nch] = dx;
                  if (kw != 1.0f) flags |= kDeferredKw;
                }
              }
              chw[nch] = make_float4(c1, c2, c3, __uint_as_float(flags));
              ch[nch++] = Child{spawnOrigin(s, next), next, cw, ck};
            }
          } else {
            float cw = W * coeff;
            if (roulette && cw != 0.0f) cw = cw * rouletteFactor(cw, ck);
            if (cw != 0.0f) {
              if constexpr (kDefer) {
                cha[nch] = make_float2(a, dist);
                if (a != -1.0f) cw = W;  // completed by k_light_pdf
              }
              ch[nch++] = Child{spawnOrigin(s, next), next, cw, ck};
            }
          }
        };
        // sampleModels (sample.wesl:301-425) in its lobe order
        if ((kLobes & kLobeDiffuse) && c.diffuse) {  // pdf/diffuse.wesl:7-36
          const V3 macro = orientedNormal(curr, s.sn);
          const float r = sqrtf(randFloat(rng));
          const float angle = 2.0f * PI * randFloat(rng);
          float sa, ca;
          sincosf(angle, &sa, &ca);
          const V3 local{r * ca, r * sa, sqrtf(fmaxf(0.0f, 1.0f - r * r))};
          const V3 next = mul(makeTangentSpace(macro), local);
          push(next, M_DIFFUSE, diffusePdf(curr, next, s), diffuseDist(curr, next, s, m));
        }
        if ((kLobes & kLobeReflect) && c.specular_reflect) {  // pdf/specular_reflection.wesl:7-15
          const V3 next = specularDir(curr, s);
          push(next, M_SREFL, specularReflectPdf(curr, next, s), specularReflectDist(curr, next, s, m));
        }
        if ((kLobes & kLobeReflect) && c.rough_reflect) {  // pdf/rough_reflection.wesl:9-27
          const V3 micro = orientedNormal(curr, sampleNorm(curr, s, m.microfacet_roughness, rng));
          const V3 next = reflect(curr, micro);
          const V3 macro = orientedNormal(curr, s.sn);
          const float prob = dot(next, macro) <= 0.0f
                                 ? 0.0f
                                 : reflectPdf(curr, micro, macro, m.microfacet_roughness);
          push(next, M_RREFL, prob, roughReflectDist(curr, next, s, m));
        }
        if ((kLobes & kLobeTransmit) && c.specular_transmit) {  // pdf/specular_transmission.wesl:9-27
          const V3 next = m.volume ? refract(curr, orientedNormal(curr, s.sn), relIor(s.sn, curr, m).re)
                                   : curr;
          push(next, M_STRANS, specularTransmitPdf(curr, next, s, m),
               specularTransmitDist(curr, next, s, m));
        }
        if ((kLobes & kLobeTransmit) && c.rough_transmit) {  // pdf/rough_transmission.wesl:9-32
          const V3 macro = orientedNormal(curr, s.sn);
          const V3 micro = orientedNormal(curr, sampleNorm(curr, s, m.microfacet_roughness, rng));
          const V3 next = refract(curr, micro, relIorT(relIor(micro, curr, m)));
          float prob;
          if (dot(next, next) <= VNDF_EPS)
            prob = 0.0f;
          else if (dot(next, macro) >= 0.0f)
            prob = 0.0f;
          else
            prob = roughTransmitPdf(curr, next, s, m);
          push(next, M_RTRANS, prob, roughTransmitDist(curr, next, s, m));
        }
        if (c.light) {  // sample.wesl:407-422 with pdf/emission.wesl:32-82
          const uint32_t ne = sc.emissive_count;
          uint32_t bin = static_cast<uint32_t>(randFloat(rng) * static_cast<float>(ne));
          if (bin >= ne) bin = ne - 1u;  // randFloat() can return 1.0
          const float rf = randFloat(rng);
          const DevAlias al = sc.alias[bin];
          const DevEmissivePrim& P = sc.eprim[rf < al.prob ? bin : al.alias];
          const float tsx = randFloat(rng);
          const float tsy = randFloat(rng);
          const float tss = sqrtf(tsx);
          const float bx = 1.0f - tss, by = tss * (1.0f - tsy), bz = tss * tsy;
          const V3 v0 = ld3(P.v0), v1 = ld3(P.v1), v2 = ld3(P.v2);
          const V3 spos3 = bx * v0 + by * v1 + bz * v2;
          const V3 lo = spos3 - s.pos;
          const float dsq = fmaxf(dot(lo, lo), 1e-3f);
          const V3 next = lo / sqrtf(dsq);
          const V3 lnrm = normalize(cross(v1 - v0, v2 - v0));
          const float lp = fabsf(dot(lnrm, -next));
          const float area_pdf = fmaxf(P.weight / P.area, 1e-3f);
          const float sapdf = area_pdf * dsq / fmaxf(lp, 1e-3f);
          if (!(sapdf <= 1e-6f)) {  // addEmissionSample's MIN_SAMPLE_WEIGHT check
            const float radiance = rgbToRadiance(ld3(P.emission), spos);
            const float sproj = fabsf(dot(s.sn, next));
            float ec = diffuseDist(curr, next, s, m) + roughReflectDist(curr, next, s, m);
            if (m.transmission != 0.0f) ec = ec + roughTransmitDist(curr, next, s, m);
            const float denom = balanceDenom<kLobes>(sc, curr, next, s, m, c, M_NONE, -1.0f, sapdf,
                                                     wb.status);
            const float rad = radiance * ec * sproj / denom;
            const float contrib = W * rad * kw;
            float4 cx = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if constexpr (kHero) {
              if (uniform) {
                float cj[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                  const float lj = heroWavelength(x0, j + 1);
                  float ecj = diffuseDist(curr, next, s, mx[j]) + roughReflectDist(curr, next, s, mx[j]);
                  if (mx[j].transmission != 0.0f) ecj = ecj + roughTransmitDist(curr, next, s, mx[j]);
                  cj[j] = rgbToRadiance(ld3(P.emission), smitsPos(lj)) * ecj * sproj / denom;
                }
                cx = make_float4(Wx.x * cj[0], Wx.y * cj[1], Wx.z * cj[2], 0.0f);
              }
            }
            if (contrib != 0.0f || cx.x != 0.0f || cx.y != 0.0f || cx.z != 0.0f) {
              const float expected_dist = sqrtf(dsq);
              const V3 light_pos = s.pos + next * expected_dist;
              const V3 so = spawnOrigin(s, next);
              const float tmax = distance3(so, light_pos) - 1e-3f;
              shadow = true;
              sh_o = make_float4(so.x, so.y, so.z, contrib);
              sh_d = make_float4(next.x, next.y, next.z, tmax);
              sh_x = cx;
            }
          }
        }
      }
      if constexpr (kHero) {
        if (addL != 0.0f || addX.x != 0.0f || addX.y != 0.0f || addX.z != 0.0f)
          atomicAdd(wb.s_L4 + slot, make_float4(addL, addX.x, addX.y, addX.z));
      } else {
        if (addL != 0.0f) atomicAdd(&wb.s_L[slot], addL);
      }
    }
    // ---- warp-aggregated queue appends ----
    uint32_t incl = nch;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= static_cast<uint32_t>(o)) incl += y;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    uint32_t qbase = 0;
    if (lane == 31 && total) qbase = atomicAdd(&wb.counts[out], total);
    qbase = __shfl_sync(kFull, qbase, 31);
    if (total) {
      if (qbase + total > wb.capacity) {
        if (lane == 0) atomicOr(wb.status, 2u);
      } else {
        uint32_t pos = qbase + incl - nch;
        for (uint32_t k = 0; k < nch; ++k, ++pos) {
          wb.ray_o[out][pos] = make_float4(ch[k].o.x, ch[k].o.y, ch[k].o.z, ch[k].w);
          wb.ray_d[out][pos] = make_float4(ch[k].d.x, ch[k].d.y, ch[k].d.z, __uint_as_float(ch[k].key));
          wb.ray_slot[out][pos] = slot;
          if constexpr (kHero) wb.ray_w[out][pos] = chw[k];
          if constexpr (kDefer) {
            wb.defer[pos] = make_float4(dpos.x, dpos.y, dpos.z, cha[k].x);
            wb.defer_dist[pos] = cha[k].y;
            if constexpr (kHero) wb.defer_w[pos] = make_float4(chd[k].x, chd[k].y, chd[k].z, 0.0f);
          }
        }
      }
    }
    const unsigned ballot = __ballot_sync(kFull, shadow);
    if (ballot) {
      uint32_t sbase = 0;
      if (lane == 0) sbase = atomicAdd(&wb.counts[2], static_cast<uint32_t>(__popc(ballot)));
      sbase = __shfl_sync(kFull, sbase, 0);
      if (sbase + __popc(ballot) > wb.capacity) {
        if (lane == 0) atomicOr(wb.status, 2u);
      } else if (shadow) {
        const uint32_t pos = sbase + __popc(ballot & ((1u << lane) - 1u));
        wb.sh_o[pos] = sh_o;
        wb.sh_d[pos] = sh_d;
        wb.sh_slot[pos] = slot;
        if constexpr (kHero) wb.sh_w[pos] = sh_x;
      }
    }
  }
}

// At most 96 registers: five blocks of 128 threads per SM (the lobe groups
// need 90-93 without spills; uncapped they took 98, which left room for four).
// The launches of levels without light samples fit 64 without spills: eight
// blocks instead of seven at their natural 72 registers, shading 84.7 -> 73.7
// ms per 10 icosphere frames and 378 -> 340 ms per 3 instanced frames (a cap of
// 72 for the deferring launches spilled 32 B and gained nothing).
// CG_SHADE_NL_REGS overrides the light-free cap for measurements.
#ifndef CG_SHADE_NL_REGS
#define CG_SHADE_NL_REGS 64
#endif
#ifndef CG_SHADE_DEFER_REGS
#define CG_SHADE_DEFER_REGS 96
#endif
template <int kSort, int kLobes = kLobesAll, bool kLight = true, bool kDefer = false>
__global__ void __maxnreg__(kDefer ? CG_SHADE_DEFER_REGS : kLight ? 96 : CG_SHADE_NL_REGS) k_shade(SceneView sc, FrameConst fc,
                                                                    WaveBuffers wb, int depth,
                                                                    int parity) {
  shadeLevel<kSort, kLobes, false, kLight, kDefer>(sc, fc, wb, depth, parity);
}

// Hero-wavelength mode (level-wide shading order only).  At most 128
// registers: the group with transmission needs 109 without spills (ptxas
// chose 96 with spills when left free).
template <int kLobes, bool kLight = true, bool kDefer = false>
__global__ void __maxnreg__(128) k_shade_hero(SceneView sc, FrameConst fc, WaveBuffers wb,
                                                    int depth, int parity) {
  shadeLevel<kShadeSortGlobal, kLobes, true, kLight, kDefer>(sc, fc, wb, depth, parity);
}

// Completes the weights of the children a light-sampling level deferred
// (WaveBuffers::defer): the light-pdf sum along the child's direction from its
// parent hit (emission.wesl:120-149) joins the rest of the balance-heuristic
// denominator, fmaxf(lobes + light, 1e-6) as balancePdfDenominator
// (sample.wesl:505-554) forms it, and the weight becomes W * (dist / denom)
// as the shading kernel forms it for the other children (W: the stored parent
// weight, dist: the stored lobe value).  One ray per thread, a grid-strided
// loop over the level's queue.
__global__ void __launch_bounds__(256) k_light_pdf(SceneView sc, WaveBuffers wb, int out) {
  const uint32_t n = min(wb.counts[out], wb.capacity);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float4 dp = wb.defer[i];
    if (dp.w == -1.0f) continue;  // not deferred (the lobes' sum is >= 0 or NaN)
    const float4 d4 = wb.ray_d[out][i];
    const float pl = lightPdf(sc, V3{dp.x, dp.y, dp.z}, V3{d4.x, d4.y, d4.z}, wb.status);
    const float denom = fmaxf(__fadd_rn(dp.w, pl), 1e-6f);  // balanceDenom's sum, light count 1
    float* wp = reinterpret_cast<float*>(wb.ray_o[out] + i) + 3;
    float w = *wp * (wb.defer_dist[i] / denom);
    if (wb.hero) {  // the other wavelengths' weights, and the factor kHeroCount
      float4 x = wb.ray_w[out][i];
      const float4 dx = wb.defer_w[i];
      uint32_t flags = __float_as_uint(x.w);
      if (flags & kDeferredKw) w = w * static_cast<float>(kHeroCount);
      flags &= ~kDeferredKw;
      x = make_float4(x.x * (dx.x / denom), x.y * (dx.y / denom), x.z * (dx.z / denom),
                      __uint_as_float(flags));
      wb.ray_w[out][i] = x;
    }
    *wp = w;
  }
}

// ---- resolve: spp loop sum + running mean + sRGB (compute.wesl:41-61) -----------
__global__ void k_resolve(FrameConst fc, WaveBuffers wb, ChunkDesc ch) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ch.pixel_count) return;
  const uint64_t gp = ch.pixel_begin + j;
  const ViewDev& v = fc.views[findViewByPixel(fc, gp)];
  const uint32_t lp = static_cast<uint32_t>(gp - v.pixel_offset);
  const uint32_t pixel = v.pixel_base + lp;
  const uint64_t first = v.sample_offset + uint64_t(lp) * v.spp - ch.sample_begin;
  const float avg = fc.wl_const[1];
  // each sample adds its term / the full frame's spp, so the films of sample
  // ranges that partition a pixel's samples add up to the full frame
  const float spp = static_cast<float>(v.spp_total ? v.spp_total : v.spp);
  V3 acc{0.0f, 0.0f, 0.0f};
  uint32_t dropped = 0;
  for (uint32_t k = 0; k < v.spp; ++k) {
    V3 term;
    if (wb.hero) {
      // four wavelengths, each uniform on [380, 780]: (1/4) sum_j f_j / (1/400)
      const float4 L = wb.s_L4[first + k];
      const float x0 = wb.s_lambda[first + k];
      const float Ls[kHeroCount] = {L.x, L.y, L.z, L.w};
      V3 est{0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int j = 0; j < kHeroCount; ++j) est = est + xyzMatch(heroWavelength(x0, j)) * Ls[j] / avg;
      term = est * 100.0f / spp;
    } else {
      const float L = wb.s_L[first + k];
      const float lambda = wb.s_lambda[first + k];
      const float prob = wb.s_prob[first + k];
      const V3 il = xyzMatch(lambda) * L / avg;
      term = il / prob / spp;
    }
    // a sample whose estimate is not finite adds nothing (and is counted):
    // one NaN would otherwise stay in the pixel's running mean for good
    if (isfinite(term.x) && isfinite(term.y) && isfinite(term.z))
      acc = acc + term;
    else
      ++dropped;
  }
  if (dropped) atomicAdd(&wb.stats[5], static_cast<unsigned long long>(dropped));
  V3 lum{0.0f, 0.0f, 0.0f};
  if (v.frame > 0u) {
    const float4 f = v.film[pixel];
    lum = V3{f.x, f.y, f.z} * (1.0f - v.sample_weight);
  }
  lum = lum + acc * v.sample_weight;
  v.film[pixel] = make_float4(lum.x, lum.y, lum.z, 0.0f);
  if (v.rgba) {
    const V3 lin = xyzToLinearSrgb(lum);
    v.rgba[pixel] = make_uchar4(static_cast<unsigned char>(__float2uint_rn(encodeChannel(lin.x) * 255.0f)),
                                static_cast<unsigned char>(__float2uint_rn(encodeChannel(lin.y) * 255.0f)),
                                static_cast<unsigned char>(__float2uint_rn(encodeChannel(lin.z) * 255.0f)),
                                255);
  }
}

// ---- closest-hit query for parity tests -------------------------------------------
template <int kNodes>
__global__ void k_trace_closest(SceneView sc, const float4* rays, uint32_t n, float4* out_tuv,
                                int4* out_ids, uint32_t* status) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 o = rays[2 * i], d = rays[2 * i + 1];
  TravCounters cnt{0u, 0u, 0u};
  HitRec h = trace<false, false, kNodes>(sc, o, d, MAXD, cnt, status);
  if (h.inst >= 0) {
    const uint32_t orig = __float_as_uint(__ldg(sc.tris + 3u * h.tri).w);
    out_tuv[i] = make_float4(h.t, h.u, h.v, 0.0f);
    out_ids[i] = make_int4(h.inst, static_cast<int>(orig), static_cast<int>(h.tri), 0);
  } else {
    out_tuv[i] = make_float4(MAXD, 0.0f, 0.0f, 0.0f);
    out_ids[i] = make_int4(-1, -1, -1, 0);
  }
}

int gSmCount = 0;

uint32_t gridFor(uint32_t blocks_per_sm) {
  return static_cast<uint32_t>(smCount()) * (blocks_per_sm > 0 ? blocks_per_sm : 1u);
}

}  // namespace

int smCount() {
  if (gSmCount == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&gSmCount, cudaDevAttrMultiProcessorCount, dev);
    if (gSmCount <= 0) gSmCount = 148;
  }
  return gSmCount;
}

void launchWavelengthTree(float* tree, float* consts, cudaStream_t s) {
  k_wavelength_tree<<<(65535 + 255) / 256, 256, 0, s>>>(tree, consts);
}

void launchGen(const FrameConst& fc, const WaveBuffers& wb, const ChunkDesc& ch, cudaStream_t s) {
  const uint32_t n = ch.sample_count > 0 ? ch.sample_count : 1u;
  k_gen<<<(n + 255) / 256, 256, 0, s>>>(fc, wb, ch);
}

// Kernel attributes set once per device before any launch (never inside a
// stream capture).  CG_CARVEOUT (a measurement switch): the shared-memory
// share of the unified L1 / shared memory, in percent, requested for the
// traversal and shading kernels; without it the driver's default.
void configureKernels() {
#ifdef CG_CARVEOUT
  const int pct = CG_CARVEOUT;
  cudaFuncSetAttribute(k_extend_persistent<false, kNodesWide4>,
                       cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  cudaFuncSetAttribute(k_shadow_persistent<false, kNodesWide4>,
                       cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  cudaFuncSetAttribute(k_shade<kShadeSortGlobal, kLobeHit | kLobeDiffuse | kLobeReflect>,
                       cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  cudaFuncSetAttribute(k_shade<kShadeSortGlobal, kLobesAll>,
                       cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  cudaGetLastError();
#endif
}

void launchExtend(const SceneView& sc, const WaveBuffers& wb, int parity, bool counting,
                  const LaunchShape& ls, bool cut, cudaStream_t s) {
  const int keys = ls.shade_sort == kShadeSortGlobal ? (cut ? 2 : 1) : 0;
  const uint32_t block = ls.extend_block;
  if (ls.persistent) {  // one resident grid: 64 registers -> 65536 / (64 * block) blocks per SM
    const uint32_t g = gridFor(std::max(1u, ls.traversal_threads / block));
    const size_t smem = size_t(kShortStack) * block * sizeof(int32_t);
    if (ls.spec && ls.nodes != kNodesBinary) {  // postponed leaves
      const bool q = ls.nodes == kNodesWide4Q;
      if (counting) {
        if (q) k_extend_persistent<true, kNodesWide4Q, true><<<g, block, smem, s>>>(sc, wb, parity, keys);
        else k_extend_persistent<true, kNodesWide4, true><<<g, block, smem, s>>>(sc, wb, parity, keys);
      } else {
        if (q) k_extend_persistent<false, kNodesWide4Q, true><<<g, block, smem, s>>>(sc, wb, parity, keys);
        else k_extend_persistent<false, kNodesWide4, true><<<g, block, smem, s>>>(sc, wb, parity, keys);
      }
      return;
    }
    switch (ls.nodes * 2 + (counting ? 1 : 0)) {
      case kNodesBinary * 2: k_extend_persistent<false, kNodesBinary><<<g, block, smem, s>>>(sc, wb, parity, keys); break;
      case kNodesBinary * 2 + 1: k_extend_persistent<true, kNodesBinary><<<g, block, smem, s>>>(sc, wb, parity, keys); break;
      case kNodesWide4 * 2: k_extend_persistent<false, kNodesWide4><<<g, block, smem, s>>>(sc, wb, parity, keys); break;
      case kNodesWide4 * 2 + 1: k_extend_persistent<true, kNodesWide4><<<g, block, smem, s>>>(sc, wb, parity, keys); break;
      case kNodesWide4Q * 2 + 1: k_extend_persistent<true, kNodesWide4Q><<<g, block, smem, s>>>(sc, wb, parity, keys); break;
      default: k_extend_persistent<false, kNodesWide4Q><<<g, block, smem, s>>>(sc, wb, parity, keys); break;
    }
    return;
  }
  const uint32_t grid = ls.grid_extend ? ls.grid_extend : gridFor(2048u / block);
  switch (ls.nodes * 2 + (counting ? 1 : 0)) {
    case kNodesBinary * 2: k_extend<false, kNodesBinary><<<grid, block, 0, s>>>(sc, wb, parity, keys); break;
    case kNodesBinary * 2 + 1: k_extend<true, kNodesBinary><<<grid, block, 0, s>>>(sc, wb, parity, keys); break;
    case kNodesWide4 * 2: k_extend<false, kNodesWide4><<<grid, block, 0, s>>>(sc, wb, parity, keys); break;
    case kNodesWide4 * 2 + 1: k_extend<true, kNodesWide4><<<grid, block, 0, s>>>(sc, wb, parity, keys); break;
    case kNodesWide4Q * 2 + 1: k_extend<true, kNodesWide4Q><<<grid, block, 0, s>>>(sc, wb, parity, keys); break;
    default: k_extend<false, kNodesWide4Q><<<grid, block, 0, s>>>(sc, wb, parity, keys); break;
  }
}

int launchShade(const SceneView& sc, const FrameConst& fc, const WaveBuffers& wb, int depth,
                int parity, const LaunchShape& ls, cudaStream_t s, bool light) {
  const uint32_t block = ls.shade_block > 256u ? 256u : ls.shade_block;
  const uint32_t grid = ls.grid_shade ? ls.grid_shade : gridFor(1024u / block);
  constexpr int kOpaque = kLobeHit | kLobeDiffuse | kLobeReflect;
  const bool rr = fc.roulette != 0u && static_cast<uint32_t>(depth) >= fc.roulette;
  if (wb.hero) {  // hero-wavelength mode: level-wide order, one launch per lobe group
    k_shade_scatter<<<gridFor(4u), kScatterBlock, 0, s>>>(wb, parity);
    if (light && wb.defer && wb.defer_dist && wb.defer_w && !rr) {  // light-pdf terms in a pass
      k_shade_hero<0><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade_hero<kOpaque, true, true><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade_hero<kLobesAll, true, true><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_light_pdf<<<gridFor(8u), 256, 0, s>>>(sc, wb, parity ^ 1);
      return 5;
    }
    if (light) {
      k_shade_hero<0><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade_hero<kOpaque><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade_hero<kLobesAll><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
    } else {
      k_shade_hero<0, false><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade_hero<kOpaque, false><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade_hero<kLobesAll, false><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
    }
    return 4;
  }
  if (ls.shade_sort == kShadeSortGlobal) {  // keys and counts came with the closest hits
    k_shade_scatter<<<gridFor(4u), kScatterBlock, 0, s>>>(wb, parity);
    // one launch per lobe group, each over its keys' range of the permutation
    // the light-pdf terms in a separate pass (not where roulette needs the
    // final weights)
    if (light && wb.defer && wb.defer_dist && !rr) {
      k_shade<kShadeSortGlobal, 0><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade<kShadeSortGlobal, kOpaque, true, true><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade<kShadeSortGlobal, kLobesAll, true, true><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_light_pdf<<<gridFor(8u), 256, 0, s>>>(sc, wb, parity ^ 1);
      return 5;
    }
    if (light) {
      k_shade<kShadeSortGlobal, 0><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade<kShadeSortGlobal, kOpaque><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade<kShadeSortGlobal, kLobesAll><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
    } else {
      k_shade<kShadeSortGlobal, 0, false><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade<kShadeSortGlobal, kOpaque, false><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
      k_shade<kShadeSortGlobal, kLobesAll, false><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
    }
    return 4;
  }
  if (ls.shade_sort == kShadeSortBlock)
    k_shade<kShadeSortBlock><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
  else
    k_shade<kShadeSortNone><<<grid, block, 0, s>>>(sc, fc, wb, depth, parity);
  return 1;
}

void launchShadow(const SceneView& sc, const WaveBuffers& wb, bool counting,
                  const LaunchShape& ls, cudaStream_t s) {
  const uint32_t block = ls.extend_block;
  if (ls.persistent) {
    const uint32_t g = gridFor(std::max(1u, ls.traversal_threads / block));
    switch (ls.nodes * 2 + (counting ? 1 : 0)) {
      case kNodesBinary * 2: k_shadow_persistent<false, kNodesBinary><<<g, block, 0, s>>>(sc, wb); break;
      case kNodesBinary * 2 + 1: k_shadow_persistent<true, kNodesBinary><<<g, block, 0, s>>>(sc, wb); break;
      case kNodesWide4 * 2: k_shadow_persistent<false, kNodesWide4><<<g, block, 0, s>>>(sc, wb); break;
      case kNodesWide4 * 2 + 1: k_shadow_persistent<true, kNodesWide4><<<g, block, 0, s>>>(sc, wb); break;
      case kNodesWide4Q * 2 + 1: k_shadow_persistent<true, kNodesWide4Q><<<g, block, 0, s>>>(sc, wb); break;
      default: k_shadow_persistent<false, kNodesWide4Q><<<g, block, 0, s>>>(sc, wb); break;
    }
    return;
  }
  const uint32_t grid = ls.grid_extend ? ls.grid_extend : gridFor(2048u / block);
  switch (ls.nodes * 2 + (counting ? 1 : 0)) {
    case kNodesBinary * 2: k_shadow<false, kNodesBinary><<<grid, block, 0, s>>>(sc, wb); break;
    case kNodesBinary * 2 + 1: k_shadow<true, kNodesBinary><<<grid, block, 0, s>>>(sc, wb); break;
    case kNodesWide4 * 2: k_shadow<false, kNodesWide4><<<grid, block, 0, s>>>(sc, wb); break;
    case kNodesWide4 * 2 + 1: k_shadow<true, kNodesWide4><<<grid, block, 0, s>>>(sc, wb); break;
    case kNodesWide4Q * 2 + 1: k_shadow<true, kNodesWide4Q><<<grid, block, 0, s>>>(sc, wb); break;
    default: k_shadow<false, kNodesWide4Q><<<grid, block, 0, s>>>(sc, wb); break;
  }
}

void launchResolve(const FrameConst& fc, const WaveBuffers& wb, const ChunkDesc& ch,
                   cudaStream_t s) {
  const uint32_t n = ch.pixel_count > 0 ? ch.pixel_count : 1u;
  k_resolve<<<(n + 127) / 128, 128, 0, s>>>(fc, wb, ch);
}

// Film readback: the float4 film packed to three floats per pixel, as XYZ or
// converted to linear sRGB (xyz_to_srgb of physics/srgb.wesl:6-10, rounded
// after every product and sum like the host loop it replaces, so no fused
// multiply-adds).
__global__ void k_film_pack(const float4* __restrict__ film, float* __restrict__ out, size_t npx,
                            int rgb) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= npx) return;
  const float4 f = film[i];
  float a = f.x, b = f.y, c = f.z;
  if (rgb) {
    a = __fadd_rn(__fadd_rn(__fmul_rn(2.36461385f, f.x), __fmul_rn(-0.89654057f, f.y)),
                  __fmul_rn(-0.46807328f, f.z));
    b = __fadd_rn(__fadd_rn(__fmul_rn(-0.51516621f, f.x), __fmul_rn(1.4264081f, f.y)),
                  __fmul_rn(0.0887581f, f.z));
    c = __fadd_rn(__fadd_rn(__fmul_rn(0.0052037f, f.x), __fmul_rn(-0.01440816f, f.y)),
                  __fmul_rn(1.00920446f, f.z));
  }
  out[3 * i] = a;
  out[3 * i + 1] = b;
  out[3 * i + 2] = c;
}

__global__ void k_film_rgba8(const float4* __restrict__ film, uchar4* __restrict__ rgba, size_t npx) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= npx) return;
  const float4 f = film[i];
  const V3 lin = xyzToLinearSrgb(V3{f.x, f.y, f.z});
  rgba[i] = make_uchar4(static_cast<unsigned char>(__float2uint_rn(encodeChannel(lin.x) * 255.0f)),
                        static_cast<unsigned char>(__float2uint_rn(encodeChannel(lin.y) * 255.0f)),
                        static_cast<unsigned char>(__float2uint_rn(encodeChannel(lin.z) * 255.0f)),
                        255);
}

void launchFilmRgba8(const float4* film, uchar4* rgba, size_t npx, cudaStream_t s) {
  if (npx == 0) return;
  k_film_rgba8<<<static_cast<unsigned>((npx + 255) / 256), 256, 0, s>>>(film, rgba, npx);
}

void launchFilmPack(const float4* film, float* out, size_t npx, bool rgb, cudaStream_t s) {
  if (npx == 0) return;
  k_film_pack<<<static_cast<unsigned>((npx + 255) / 256), 256, 0, s>>>(film, out, npx, rgb ? 1 : 0);
}

void launchTraceClosest(const SceneView& sc, const float4* rays, uint32_t n, float4* out_tuv,
                        int4* out_ids, uint32_t* status, int nodes, cudaStream_t s) {
  if (n == 0) return;
  const uint32_t g = (n + 127) / 128;
  if (nodes == kNodesBinary)
    k_trace_closest<kNodesBinary><<<g, 128, 0, s>>>(sc, rays, n, out_tuv, out_ids, status);
  else if (nodes == kNodesWide4)
    k_trace_closest<kNodesWide4><<<g, 128, 0, s>>>(sc, rays, n, out_tuv, out_ids, status);
  else
    k_trace_closest<kNodesWide4Q><<<g, 128, 0, s>>>(sc, rays, n, out_tuv, out_ids, status);
}

}  // namespace cg
