// cg_traverse.cuh — two-level BVH traversal on sm_100a.
//
// Closest hit (rayTraverseTlas / rayTraverseBlas, structural/bvh.wesl:52-186)
// and t-bounded any hit (the shadow test of trace.wesl:91-113) over the
// BvhNode layout of cg_types.h.  Unlike the reference, which walks every
// overlapping node, boxes beyond the current closest hit are skipped and the
// nearer child is visited first; the closest hit is the same except for
// exact ties.  The ray->instance transform and Möller–Trumbore
// (bvh.wesl:84-88, 188-221) use explicitly rounded intrinsics in the
// reference's operation order, so t, u, v are bit-identical to it.
#ifndef CG_TRAVERSE_CUH_
#define CG_TRAVERSE_CUH_

#include <climits>
#include <cstdint>

#include "cg_types.h"

namespace cg {
namespace dev {

#define XM(a, b) __fmul_rn((a), (b))
#define XA(a, b) __fadd_rn((a), (b))
#define XS(a, b) __fsub_rn((a), (b))

constexpr int kStackSize = 64;
constexpr int32_t kToTlas = INT_MIN;      // marker: return to the TLAS
constexpr int32_t kDone = INT_MIN + 1;    // empty stack

struct TravCounters {
  uint32_t nodes, tris, insts;
};

struct HitRec {
  float t, u, v;
  int32_t inst;   // -1: miss
  uint32_t tri;   // global triangle slot
};

__device__ __forceinline__ float safeInv(float d) {
  return 1.0f / (fabsf(d) > 1e-20f ? d : copysignf(1e-20f, d));
}

// Möller–Trumbore on precomputed v0 / e1 = v1 - v0 / e2 = v2 - v0.
__device__ __forceinline__ bool intersectTri(float ox, float oy, float oz, float dx, float dy,
                                             float dz, float4 a, float4 b, float4 c, float& t,
                                             float& u, float& v) {
  // h = cross(dir, e2)
  const float hx = XS(XM(dy, c.z), XM(c.y, dz));
  const float hy = XS(XM(dz, c.x), XM(c.z, dx));
  const float hz = XS(XM(dx, c.y), XM(c.x, dy));
  const float det = XA(XA(XM(b.x, hx), XM(b.y, hy)), XM(b.z, hz));
  if (det > -1e-6f && det < 1e-6f) return false;
  const float f = __fdiv_rn(1.0f, det);
  const float sx = XS(ox, a.x), sy = XS(oy, a.y), sz = XS(oz, a.z);
  u = XM(f, XA(XA(XM(sx, hx), XM(sy, hy)), XM(sz, hz)));
  if (u < 0.0f || u > 1.0f) return false;
  // q = cross(s, e1)
  const float qx = XS(XM(sy, b.z), XM(b.y, sz));
  const float qy = XS(XM(sz, b.x), XM(b.z, sx));
  const float qz = XS(XM(sx, b.y), XM(b.x, sy));
  v = XM(f, XA(XA(XM(dx, qx), XM(dy, qy)), XM(dz, qz)));
  if (v < 0.0f || XA(u, v) > 1.0f) return false;
  t = XM(f, XA(XA(XM(c.x, qx), XM(c.y, qy)), XM(c.z, qz)));
  return t > 1e-6f;
}

// Ray -> instance space, ((m0 x + m1 y) + m2 z) + m3 w, rounded per op.
__device__ __forceinline__ void toLocal(const float* m, float ox, float oy, float oz, float dx,
                                        float dy, float dz, float& lox, float& loy, float& loz,
                                        float& ldx, float& ldy, float& ldz) {
  lox = XA(XA(XA(XM(m[0], ox), XM(m[1], oy)), XM(m[2], oz)), m[3]);
  loy = XA(XA(XA(XM(m[4], ox), XM(m[5], oy)), XM(m[6], oz)), m[7]);
  loz = XA(XA(XA(XM(m[8], ox), XM(m[9], oy)), XM(m[10], oz)), m[11]);
  ldx = XA(XA(XM(m[0], dx), XM(m[1], dy)), XM(m[2], dz));
  ldy = XA(XA(XM(m[4], dx), XM(m[5], dy)), XM(m[6], dz));
  ldz = XA(XA(XM(m[8], dx), XM(m[9], dy)), XM(m[10], dz));
}

// kAny: stop at the first hit with t < tmax (returns inst >= 0 if one).
// kCount: accumulate node / triangle / instance counters.
template <bool kAny, bool kCount>
__device__ __forceinline__ HitRec traceRay(const SceneView& sc, float wox, float woy, float woz,
                                           float wdx, float wdy, float wdz, float tmax,
                                           TravCounters& cnt, uint32_t* status) {
  HitRec best{tmax, 0.0f, 0.0f, -1, 0u};
  if (!sc.has_tlas) return best;
  int32_t stack[kStackSize];
  int sp = 0;
  const BvhNode* nodes = sc.tlas;
  bool in_blas = false;
  int32_t cur_inst = -1;
  float ox = wox, oy = woy, oz = woz, dx = wdx, dy = wdy, dz = wdz;
  float idx = safeInv(dx), idy = safeInv(dy), idz = safeInv(dz);
  float oix = ox * idx, oiy = oy * idy, oiz = oz * idz;
  int32_t node = 0;
  while (true) {
    while (node >= 0) {
      const float4* np = reinterpret_cast<const float4*>(nodes + node);
      const float4 n0 = __ldg(np);
      const float4 n1 = __ldg(np + 1);
      const float4 n2 = __ldg(np + 2);
      const int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
      if (kCount) ++cnt.nodes;
      const float a0 = fmaf(n0.x, idx, -oix), a1 = fmaf(n0.y, idx, -oix);
      const float b0 = fmaf(n0.z, idy, -oiy), b1 = fmaf(n0.w, idy, -oiy);
      const float c0 = fmaf(n2.x, idz, -oiz), c1 = fmaf(n2.y, idz, -oiz);
      const float t0min = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), 0.0f));
      const float t0max = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), best.t));
      const float d0 = fmaf(n1.x, idx, -oix), d1 = fmaf(n1.y, idx, -oix);
      const float e0 = fmaf(n1.z, idy, -oiy), e1 = fmaf(n1.w, idy, -oiy);
      const float f0 = fmaf(n2.z, idz, -oiz), f1 = fmaf(n2.w, idz, -oiz);
      const float t1min = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fmaxf(fminf(f0, f1), 0.0f));
      const float t1max = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fminf(fmaxf(f0, f1), best.t));
      const bool h0 = t0min <= t0max;
      const bool h1 = t1min <= t1max;
      if (h0 && h1) {
        int32_t near = n3.x, far = n3.y;
        if (t1min < t0min) {
          near = n3.y;
          far = n3.x;
        }
        if (sp >= kStackSize) {
          atomicOr(status, 1u);
          return HitRec{tmax, 0.0f, 0.0f, -1, 0u};
        }
        stack[sp++] = far;
        node = near;
      } else if (h0) {
        node = n3.x;
      } else if (h1) {
        node = n3.y;
      } else {
        node = sp > 0 ? stack[--sp] : kDone;
      }
    }
    if (node == kDone) break;
    if (node == kToTlas) {
      nodes = sc.tlas;
      in_blas = false;
      ox = wox; oy = woy; oz = woz;
      dx = wdx; dy = wdy; dz = wdz;
      idx = safeInv(dx); idy = safeInv(dy); idz = safeInv(dz);
      oix = ox * idx; oiy = oy * idy; oiz = oz * idz;
      node = sp > 0 ? stack[--sp] : kDone;
      continue;
    }
    const uint32_t first = static_cast<uint32_t>(~node) >> 3;
    const uint32_t count = static_cast<uint32_t>(~node) & 7u;
    if (!in_blas) {
      if (count == 0u) {
        node = sp > 0 ? stack[--sp] : kDone;
        continue;
      }
      // instance leaf: enter its BLAS in local space
      const DevInstance* ip = sc.inst + first;
      const float4* ipf = reinterpret_cast<const float4*>(ip);
      const float4 r0 = __ldg(ipf), r1 = __ldg(ipf + 1), r2 = __ldg(ipf + 2);
      const uint4 meta = __ldg(reinterpret_cast<const uint4*>(ipf + 3));
      const float m[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
      if (kCount) ++cnt.insts;
      toLocal(m, wox, woy, woz, wdx, wdy, wdz, ox, oy, oz, dx, dy, dz);
      idx = safeInv(dx); idy = safeInv(dy); idz = safeInv(dz);
      oix = ox * idx; oiy = oy * idy; oiz = oz * idz;
      if (sp >= kStackSize) {
        atomicOr(status, 1u);
        return HitRec{tmax, 0.0f, 0.0f, -1, 0u};
      }
      stack[sp++] = kToTlas;
      nodes = sc.blas;
      in_blas = true;
      cur_inst = static_cast<int32_t>(first);
      node = static_cast<int32_t>(meta.x);  // blas_root
      continue;
    }
    for (uint32_t k = 0; k < count; ++k) {
      const float4* tp = sc.tris + 3u * (first + k);
      const float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
      if (kCount) ++cnt.tris;
      float t, u, v;
      if (intersectTri(ox, oy, oz, dx, dy, dz, ta, tb, tc, t, u, v) && t < best.t) {
        best.t = t;
        best.u = u;
        best.v = v;
        best.inst = cur_inst;
        best.tri = first + k;
        if (kAny) return best;
      }
    }
    node = sp > 0 ? stack[--sp] : kDone;
  }
  return best;
}

__device__ __forceinline__ void cswap(float& ka, int32_t& la, float& kb, int32_t& lb) {
  if (kb < ka) {
    const float tk = ka;
    ka = kb;
    kb = tk;
    const int32_t tl = la;
    la = lb;
    lb = tl;
  }
}


// Byte c of w as a float (exact): the byte under the exponent of 2^23, minus 2^23.
__device__ __forceinline__ float byteToFloat(uint32_t w, uint32_t c) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | c)) - 8388608.0f;
}

// The two four-wide node formats: full-precision child slabs, or 8-bit
// offsets from the node origin (decoded to world-space bounds that contain
// the full-precision ones: fmaf rounds q * scale + origin to nearest, and the
// exact value is already outside the child's box).  fetch() returns, per
// axis, the near and far bound of each child for a ray whose inverse
// direction has the given signs (near = lo where the inverse direction is
// >= 0): the slab distances then need no min/max per axis.  With FMA rounding
// monotonic in the bound, near <= far along the ray, so the entry and exit
// distances equal min/max of the two slab planes bit for bit.
template <bool kQuant>
struct Wide;

template <>
struct Wide<false> {
  using Node = Bvh4Node;
  static __device__ __forceinline__ const Node* tlas(const SceneView& sc) { return sc.tlas4; }
  static __device__ __forceinline__ const Node* blas(const SceneView& sc) { return sc.blas4; }
  static __device__ __forceinline__ int4 fetch(const Node* n, bool negx, bool negy, bool negz,
                                               float nx[4], float fx[4], float ny[4], float fy[4],
                                               float nz[4], float fz[4]) {
    const float4* np = reinterpret_cast<const float4*>(n);
    // float4 rows: lo.x, hi.x, lo.y, hi.y, lo.z, hi.z
    const float4 a = __ldg(np + (negx ? 1 : 0)), b = __ldg(np + (negx ? 0 : 1));
    const float4 c = __ldg(np + (negy ? 3 : 2)), d = __ldg(np + (negy ? 2 : 3));
    const float4 e = __ldg(np + (negz ? 5 : 4)), f = __ldg(np + (negz ? 4 : 5));
    nx[0] = a.x; nx[1] = a.y; nx[2] = a.z; nx[3] = a.w;
    fx[0] = b.x; fx[1] = b.y; fx[2] = b.z; fx[3] = b.w;
    ny[0] = c.x; ny[1] = c.y; ny[2] = c.z; ny[3] = c.w;
    fy[0] = d.x; fy[1] = d.y; fy[2] = d.z; fy[3] = d.w;
    nz[0] = e.x; nz[1] = e.y; nz[2] = e.z; nz[3] = e.w;
    fz[0] = f.x; fz[1] = f.y; fz[2] = f.z; fz[3] = f.w;
    return __ldg(reinterpret_cast<const int4*>(np + 6));
  }
};

template <>
struct Wide<true> {
  using Node = Bvh4QNode;
  static __device__ __forceinline__ const Node* tlas(const SceneView& sc) { return sc.tlas4q; }
  static __device__ __forceinline__ const Node* blas(const SceneView& sc) { return sc.blas4q; }
  static __device__ __forceinline__ int4 fetch(const Node* n, bool negx, bool negy, bool negz,
                                               float nx[4], float fx[4], float ny[4], float fy[4],
                                               float nz[4], float fz[4]) {
    const float4* np = reinterpret_cast<const float4*>(n);
    const float4 h = __ldg(np);
    const uint4 qa = __ldg(reinterpret_cast<const uint4*>(np + 1));  // lo.x hi.x lo.y hi.y
    const uint4 qb = __ldg(reinterpret_cast<const uint4*>(np + 2));  // lo.z hi.z
    const uint32_t sb = __float_as_uint(h.w);
    const float sx = __uint_as_float((sb & 0xffu) << 23);
    const float sy = __uint_as_float(((sb >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((sb >> 16) & 0xffu) << 23);
    const uint32_t wnx = negx ? qa.y : qa.x, wfx = negx ? qa.x : qa.y;
    const uint32_t wny = negy ? qa.w : qa.z, wfy = negy ? qa.z : qa.w;
    const uint32_t wnz = negz ? qb.y : qb.x, wfz = negz ? qb.x : qb.y;
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
      nx[c] = fmaf(byteToFloat(wnx, c), sx, h.x);
      fx[c] = fmaf(byteToFloat(wfx, c), sx, h.x);
      ny[c] = fmaf(byteToFloat(wny, c), sy, h.y);
      fy[c] = fmaf(byteToFloat(wfy, c), sy, h.y);
      nz[c] = fmaf(byteToFloat(wnz, c), sz, h.z);
      fz[c] = fmaf(byteToFloat(wfz, c), sz, h.z);
    }
    return __ldg(reinterpret_cast<const int4*>(np + 3));
  }
};

// Traversal state of one ray, advanced a bounded number of steps at a time so
// a warp can refill lanes whose ray finished (persistent threads with
// dynamic fetch): the closest-hit walk of traceRay, resumable.
struct TravState {
  float wox, woy, woz, wdx, wdy, wdz;  // world ray
  float ox, oy, oz, dx, dy, dz;        // ray in the current (world or instance) space
  float idx, idy, idz, oix, oiy, oiz;
  int32_t node;
  int32_t sp;
  int32_t cur_inst;                    // -1 in the TLAS
  HitRec best;
};

__device__ __forceinline__ void travInit(TravState& s, float4 o, float4 d, float tmax) {
  s.wox = s.ox = o.x; s.woy = s.oy = o.y; s.woz = s.oz = o.z;
  s.wdx = s.dx = d.x; s.wdy = s.dy = d.y; s.wdz = s.dz = d.z;
  s.idx = safeInv(s.dx); s.idy = safeInv(s.dy); s.idz = safeInv(s.dz);
  s.oix = s.ox * s.idx; s.oiy = s.oy * s.idy; s.oiz = s.oz * s.idz;
  s.node = 0;
  s.sp = 0;
  s.cur_inst = -1;
  s.best = HitRec{tmax, 0.0f, 0.0f, -1, 0u};
}

// Back from an instance to the TLAS: the world ray and its slab terms.
__device__ __forceinline__ void restoreWorld(TravState& s) {
  s.cur_inst = -1;
  s.ox = s.wox; s.oy = s.woy; s.oz = s.woz;
  s.dx = s.wdx; s.dy = s.wdy; s.dz = s.wdz;
  s.idx = safeInv(s.dx); s.idy = safeInv(s.dy); s.idz = safeInv(s.dz);
  s.oix = s.ox * s.idx; s.oiy = s.oy * s.idy; s.oiz = s.oz * s.idz;
}

// Traversal stacks of the resumable walk.  LocalStack: all entries in local
// memory.  ShortStack: the first kShort entries live in
// shared memory, one column per thread (entry i of thread t at i * stride + t,
// so a warp's accesses hit 32 different banks at any depths), the rest in
// local memory.  Most walks stay within the shared part, so pushes and pops do
// not compete with node fetches for L1 and L2.
struct LocalStack {
  int32_t e[kStackSize];
  __device__ __forceinline__ int32_t get(int i) const { return e[i]; }
  __device__ __forceinline__ void set(int i, int32_t v) { e[i] = v; }
};

template <int kShort>
struct ShortStack {
  int32_t* col;      // this thread's column of the block's shared stack
  uint32_t stride;   // threads per block
  int32_t spill[kStackSize - kShort];
  __device__ __forceinline__ int32_t get(int i) const {
    return i < kShort ? col[i * stride] : spill[i - kShort];
  }
  __device__ __forceinline__ void set(int i, int32_t v) {
    if (i < kShort)
      col[i * stride] = v;
    else
      spill[i - kShort] = v;
  }
};

// Runs at most `budget` steps (a node visit, a leaf, or a return to the
// TLAS); returns true when the ray is finished (s.best holds its hit; with
// kAny the first hit below s.best.t finishes it).
template <bool kAny, bool kCount, int kNodes, class Stack>
__device__ __forceinline__ bool travSteps(const SceneView& sc, TravState& s, Stack& stack,
                                          int budget, TravCounters& cnt, uint32_t* status) {
  for (int step = 0; step < budget; ++step) {
    const int32_t node = s.node;
    if (kNodes != kNodesBinary && node >= 0) {  // a four-wide node (traceRay4's inner step)
      using W = Wide<kNodes == kNodesWide4Q>;
      const typename W::Node* nodes = s.cur_inst < 0 ? W::tlas(sc) : W::blas(sc);
      float nxs[4], fxs[4], nys[4], fys[4], nzs[4], fzs[4];
      const int4 ch = W::fetch(nodes + node, s.idx < 0.0f, s.idy < 0.0f, s.idz < 0.0f, nxs, fxs,
                               nys, fys, nzs, fzs);
      if (kCount) ++cnt.nodes;
      float k[4];
      const int32_t links[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float a0 = fmaf(nxs[c], s.idx, -s.oix), a1 = fmaf(fxs[c], s.idx, -s.oix);
        const float b0 = fmaf(nys[c], s.idy, -s.oiy), b1 = fmaf(fys[c], s.idy, -s.oiy);
        const float c0 = fmaf(nzs[c], s.idz, -s.oiz), c1 = fmaf(fzs[c], s.idz, -s.oiz);
        const float tmin = fmaxf(fmaxf(a0, b0), fmaxf(c0, 0.0f));
        const float tmx = fminf(fminf(a1, b1), fminf(c1, s.best.t));
        const bool hit = kNodes == kNodesWide4Q ? (tmin <= tmx && links[c] != kEmptyLink)
                                                : tmin <= tmx;
        k[c] = hit ? tmin : INFINITY;
      }
      int32_t l0 = ch.x, l1 = ch.y, l2 = ch.z, l3 = ch.w;
      float k0 = k[0], k1 = k[1], k2 = k[2], k3 = k[3];
      cswap(k0, l0, k1, l1);
      cswap(k2, l2, k3, l3);
      cswap(k0, l0, k2, l2);
      cswap(k1, l1, k3, l3);
      cswap(k1, l1, k2, l2);
      if (k0 == INFINITY) {
        s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
        continue;
      }
      const int pushes = (k1 != INFINITY) + (k2 != INFINITY) + (k3 != INFINITY);
      if (s.sp + pushes > kStackSize) {
        atomicOr(status, 1u);
        s.best = HitRec{s.best.t, 0.0f, 0.0f, -1, 0u};
        return true;
      }
      if (k3 != INFINITY) stack.set(s.sp++, l3);
      if (k2 != INFINITY) stack.set(s.sp++, l2);
      if (k1 != INFINITY) stack.set(s.sp++, l1);
      s.node = l0;
      continue;
    }
    if (node >= 0) {
      const BvhNode* nodes = s.cur_inst < 0 ? sc.tlas : sc.blas;
      const float4* np = reinterpret_cast<const float4*>(nodes + node);
      const float4 n0 = __ldg(np);
      const float4 n1 = __ldg(np + 1);
      const float4 n2 = __ldg(np + 2);
      const int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
      if (kCount) ++cnt.nodes;
      const float a0 = fmaf(n0.x, s.idx, -s.oix), a1 = fmaf(n0.y, s.idx, -s.oix);
      const float b0 = fmaf(n0.z, s.idy, -s.oiy), b1 = fmaf(n0.w, s.idy, -s.oiy);
      const float c0 = fmaf(n2.x, s.idz, -s.oiz), c1 = fmaf(n2.y, s.idz, -s.oiz);
      const float t0min = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), 0.0f));
      const float t0max = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), s.best.t));
      const float d0 = fmaf(n1.x, s.idx, -s.oix), d1 = fmaf(n1.y, s.idx, -s.oix);
      const float e0 = fmaf(n1.z, s.idy, -s.oiy), e1 = fmaf(n1.w, s.idy, -s.oiy);
      const float f0 = fmaf(n2.z, s.idz, -s.oiz), f1 = fmaf(n2.w, s.idz, -s.oiz);
      const float t1min = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fmaxf(fminf(f0, f1), 0.0f));
      const float t1max = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fminf(fmaxf(f0, f1), s.best.t));
      const bool h0 = t0min <= t0max;
      const bool h1 = t1min <= t1max;
      if (h0 && h1) {
        int32_t near = n3.x, far = n3.y;
        if (t1min < t0min) {
          near = n3.y;
          far = n3.x;
        }
        if (s.sp >= kStackSize) {
          atomicOr(status, 1u);
          s.best = HitRec{s.best.t, 0.0f, 0.0f, -1, 0u};
          return true;
        }
        stack.set(s.sp++, far);
        s.node = near;
      } else if (h0) {
        s.node = n3.x;
      } else if (h1) {
        s.node = n3.y;
      } else {
        s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
      }
      continue;
    }
    if (node == kDone) return true;
    if (node == kToTlas) {
      restoreWorld(s);
      s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
      continue;
    }
    const uint32_t first = static_cast<uint32_t>(~node) >> 3;
    const uint32_t count = static_cast<uint32_t>(~node) & 7u;
    if (s.cur_inst < 0) {
      if (count == 0u) {
        s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
        continue;
      }
      const float4* ipf = reinterpret_cast<const float4*>(sc.inst + first);
      const float4 r0 = __ldg(ipf), r1 = __ldg(ipf + 1), r2 = __ldg(ipf + 2);
      const uint4 meta = __ldg(reinterpret_cast<const uint4*>(ipf + 3));
      const float m[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
      if (kCount) ++cnt.insts;
      toLocal(m, s.wox, s.woy, s.woz, s.wdx, s.wdy, s.wdz, s.ox, s.oy, s.oz, s.dx, s.dy, s.dz);
      s.idx = safeInv(s.dx); s.idy = safeInv(s.dy); s.idz = safeInv(s.dz);
      s.oix = s.ox * s.idx; s.oiy = s.oy * s.idy; s.oiz = s.oz * s.idz;
      if (s.sp >= kStackSize) {
        atomicOr(status, 1u);
        s.best = HitRec{s.best.t, 0.0f, 0.0f, -1, 0u};
        return true;
      }
      stack.set(s.sp++, kToTlas);
      s.cur_inst = static_cast<int32_t>(first);
      // blas_root (binary) or blas4_root (four-wide)
      s.node = static_cast<int32_t>(kNodes == kNodesBinary ? meta.x : meta.w);
      continue;
    }
    for (uint32_t k = 0; k < count; ++k) {
      const float4* tp = sc.tris + 3u * (first + k);
      const float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
      if (kCount) ++cnt.tris;
      float t, u, v;
      if (intersectTri(s.ox, s.oy, s.oz, s.dx, s.dy, s.dz, ta, tb, tc, t, u, v) && t < s.best.t) {
        s.best.t = t;
        s.best.u = u;
        s.best.v = v;
        s.best.inst = s.cur_inst;
        s.best.tri = first + k;
        if (kAny) return true;
      }
    }
    s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
  }
  return false;
}

// The closest-hit walk of travSteps over four-wide trees with postponed
// leaves ("speculative traversal", Aila & Laine 2009): a lane that reaches a
// BLAS leaf parks it and goes on with its next inner node; the parked
// triangles are tested when no lane of the warp still walks inner nodes
// without a parked leaf, so the node visits and the triangle tests each run
// with most lanes of the warp instead of alternating between lanes.  A lane
// that reaches a second leaf, the end of its instance (return to the TLAS) or
// the end of its walk while a leaf is parked waits for the flush.  Every lane
// of the warp calls it together (`active` false for idle lanes); returns true
// when the lane's ray is finished.  Hits are those of travSteps: every
// overlapping node is still visited or bounded by a closest hit found so far
// (the bound is only looser while a leaf is parked).
constexpr int32_t kNoLeaf = INT_MIN + 2;
// Parked leaves that start a flush.  Waiting for every lane (the flush only
// once no lane walks inner nodes without a parked leaf) left lanes that met a
// second leaf idle: closest-hit time per 10 icosphere frames 224.5 ms against
// 205.7 / 204.6 / 207.4 / 212.3 ms with a flush at 4 / 8 / 12 / 16 parked lanes
// (instanced scene, 3 frames: 3225 against 2235 / 2254 / 2325 / 2434 ms).
#ifndef CG_FLUSH_LANES
#define CG_FLUSH_LANES 8
#endif
constexpr int kFlushLanes = CG_FLUSH_LANES;

template <bool kCount, bool kQuant, class Stack>
__device__ __forceinline__ bool travStepsSpec(const SceneView& sc, TravState& s, int32_t& leaf,
                                              Stack& stack, int budget, TravCounters& cnt,
                                              uint32_t* status, bool active) {
  using W = Wide<kQuant>;
  bool finished = false;
  for (int step = 0; step < budget; ++step) {
    if (active && !finished) {
      int32_t node = s.node;
      if (node >= 0) {  // one inner node visit
        const typename W::Node* nodes = s.cur_inst < 0 ? W::tlas(sc) : W::blas(sc);
        float nxs[4], fxs[4], nys[4], fys[4], nzs[4], fzs[4];
        const int4 ch = W::fetch(nodes + node, s.idx < 0.0f, s.idy < 0.0f, s.idz < 0.0f, nxs, fxs,
                                 nys, fys, nzs, fzs);
        if (kCount) ++cnt.nodes;
        float k[4];
        const int32_t links[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float a0 = fmaf(nxs[c], s.idx, -s.oix), a1 = fmaf(fxs[c], s.idx, -s.oix);
          const float b0 = fmaf(nys[c], s.idy, -s.oiy), b1 = fmaf(fys[c], s.idy, -s.oiy);
          const float c0 = fmaf(nzs[c], s.idz, -s.oiz), c1 = fmaf(fzs[c], s.idz, -s.oiz);
          const float tmin = fmaxf(fmaxf(a0, b0), fmaxf(c0, 0.0f));
          const float tmx = fminf(fminf(a1, b1), fminf(c1, s.best.t));
          const bool hit = kQuant ? (tmin <= tmx && links[c] != kEmptyLink) : tmin <= tmx;
          k[c] = hit ? tmin : INFINITY;
        }
        int32_t l0 = ch.x, l1 = ch.y, l2 = ch.z, l3 = ch.w;
        float k0 = k[0], k1 = k[1], k2 = k[2], k3 = k[3];
        cswap(k0, l0, k1, l1);
        cswap(k2, l2, k3, l3);
        cswap(k0, l0, k2, l2);
        cswap(k1, l1, k3, l3);
        cswap(k1, l1, k2, l2);
        if (k0 == INFINITY) {
          s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
        } else {
          const int pushes = (k1 != INFINITY) + (k2 != INFINITY) + (k3 != INFINITY);
          if (s.sp + pushes > kStackSize) {
            atomicOr(status, 1u);
            s.best = HitRec{s.best.t, 0.0f, 0.0f, -1, 0u};
            s.node = kDone;
            leaf = kNoLeaf;
            finished = true;
          } else {
            if (k3 != INFINITY) stack.set(s.sp++, l3);
            if (k2 != INFINITY) stack.set(s.sp++, l2);
            if (k1 != INFINITY) stack.set(s.sp++, l1);
            s.node = l0;
          }
        }
      } else if (node != kDone && node != kToTlas) {
        const uint32_t first = static_cast<uint32_t>(~node) >> 3;
        const uint32_t count = static_cast<uint32_t>(~node) & 7u;
        if (s.cur_inst >= 0) {  // a BLAS leaf: park it if the slot is free
          if (leaf == kNoLeaf) {
            leaf = node;
            s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
          }
        } else if (count == 0u) {
          s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
        } else {  // a TLAS leaf: enter the instance's BLAS in its space
          const float4* ipf = reinterpret_cast<const float4*>(sc.inst + first);
          const float4 r0 = __ldg(ipf), r1 = __ldg(ipf + 1), r2 = __ldg(ipf + 2);
          const uint4 meta = __ldg(reinterpret_cast<const uint4*>(ipf + 3));
          const float m[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
          if (kCount) ++cnt.insts;
          toLocal(m, s.wox, s.woy, s.woz, s.wdx, s.wdy, s.wdz, s.ox, s.oy, s.oz, s.dx, s.dy, s.dz);
          s.idx = safeInv(s.dx); s.idy = safeInv(s.dy); s.idz = safeInv(s.dz);
          s.oix = s.ox * s.idx; s.oiy = s.oy * s.idy; s.oiz = s.oz * s.idz;
          if (s.sp >= kStackSize) {
            atomicOr(status, 1u);
            s.best = HitRec{s.best.t, 0.0f, 0.0f, -1, 0u};
            s.node = kDone;
            finished = true;
          } else {
            stack.set(s.sp++, kToTlas);
            s.cur_inst = static_cast<int32_t>(first);
            s.node = static_cast<int32_t>(meta.w);  // blas4_root
          }
        }
      } else if (leaf == kNoLeaf) {  // the end of an instance or of the walk
        if (node == kDone) {
          finished = true;
        } else {
          restoreWorld(s);
          s.node = s.sp > 0 ? stack.get(--s.sp) : kDone;
        }
      }
    }
    // flush the parked leaves once kFlushLanes lanes hold one, or once no lane
    // walks inner nodes without one
    const bool parked = active && leaf != kNoLeaf;
    const bool walking = active && !finished && leaf == kNoLeaf && s.node >= 0;
    const unsigned want = __ballot_sync(0xffffffffu, parked);
    const bool flush = want && (__popc(want) >= kFlushLanes || !__any_sync(0xffffffffu, walking));
    if (flush && parked) {
      const uint32_t first = static_cast<uint32_t>(~leaf) >> 3;
      const uint32_t count = static_cast<uint32_t>(~leaf) & 7u;
      for (uint32_t kk = 0; kk < count; ++kk) {
        const float4* tp = sc.tris + 3u * (first + kk);
        const float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
        if (kCount) ++cnt.tris;
        float t, u, v;
        if (intersectTri(s.ox, s.oy, s.oz, s.dx, s.dy, s.dz, ta, tb, tc, t, u, v) &&
            t < s.best.t) {
          s.best.t = t;
          s.best.u = u;
          s.best.v = v;
          s.best.inst = s.cur_inst;
          s.best.tri = first + kk;
        }
      }
      leaf = kNoLeaf;
    }
    if (__all_sync(0xffffffffu, !active || finished)) break;
  }
  return active && finished;
}

// The same closest / any hit over Bvh4Node trees: one node visit tests four
// boxes (six independent 128-bit slab loads), the hit children are ordered
// by entry distance, the nearest is visited next and the others pushed.
// Triangle and instance handling is that of traceRay (bit-identical hits).
template <bool kAny, bool kCount, bool kQuant = false>
__device__ __forceinline__ HitRec traceRay4(const SceneView& sc, float wox, float woy, float woz,
                                            float wdx, float wdy, float wdz, float tmax,
                                            TravCounters& cnt, uint32_t* status) {
  using W = Wide<kQuant>;
  HitRec best{tmax, 0.0f, 0.0f, -1, 0u};
  if (!sc.has_tlas) return best;
  int32_t stack[kStackSize];
  int sp = 0;
  const typename W::Node* nodes = W::tlas(sc);
  bool in_blas = false;
  int32_t cur_inst = -1;
  float ox = wox, oy = woy, oz = woz, dx = wdx, dy = wdy, dz = wdz;
  float idx = safeInv(dx), idy = safeInv(dy), idz = safeInv(dz);
  float oix = ox * idx, oiy = oy * idy, oiz = oz * idz;
  int32_t node = 0;
  while (true) {
    while (node >= 0) {
      float nxs[4], fxs[4], nys[4], fys[4], nzs[4], fzs[4];
      const int4 ch = W::fetch(nodes + node, idx < 0.0f, idy < 0.0f, idz < 0.0f, nxs, fxs, nys, fys,
                               nzs, fzs);
      if (kCount) ++cnt.nodes;
      float k[4];
      const int32_t links[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float a0 = fmaf(nxs[c], idx, -oix), a1 = fmaf(fxs[c], idx, -oix);
        const float b0 = fmaf(nys[c], idy, -oiy), b1 = fmaf(fys[c], idy, -oiy);
        const float c0 = fmaf(nzs[c], idz, -oiz), c1 = fmaf(fzs[c], idz, -oiz);
        const float tmin = fmaxf(fmaxf(a0, b0), fmaxf(c0, 0.0f));
        const float tmx = fminf(fminf(a1, b1), fminf(c1, best.t));
        // absent children: a point box at 1e30 (full precision) or the link (quantised)
        const bool hit = kQuant ? (tmin <= tmx && links[c] != kEmptyLink) : tmin <= tmx;
        k[c] = hit ? tmin : INFINITY;
      }
      int32_t l0 = ch.x, l1 = ch.y, l2 = ch.z, l3 = ch.w;
      float k0 = k[0], k1 = k[1], k2 = k[2], k3 = k[3];
      // sort the four (distance, link) pairs, misses (+inf) last
      cswap(k0, l0, k1, l1);
      cswap(k2, l2, k3, l3);
      cswap(k0, l0, k2, l2);
      cswap(k1, l1, k3, l3);
      cswap(k1, l1, k2, l2);
      if (k0 == INFINITY) {
        node = sp > 0 ? stack[--sp] : kDone;
        continue;
      }
      const int pushes = (k1 != INFINITY) + (k2 != INFINITY) + (k3 != INFINITY);
      if (sp + pushes > kStackSize) {
        atomicOr(status, 1u);
        return HitRec{tmax, 0.0f, 0.0f, -1, 0u};
      }
      if (k3 != INFINITY) stack[sp++] = l3;
      if (k2 != INFINITY) stack[sp++] = l2;
      if (k1 != INFINITY) stack[sp++] = l1;
      node = l0;
    }
    if (node == kDone) break;
    if (node == kToTlas) {
      nodes = W::tlas(sc);
      in_blas = false;
      ox = wox; oy = woy; oz = woz;
      dx = wdx; dy = wdy; dz = wdz;
      idx = safeInv(dx); idy = safeInv(dy); idz = safeInv(dz);
      oix = ox * idx; oiy = oy * idy; oiz = oz * idz;
      node = sp > 0 ? stack[--sp] : kDone;
      continue;
    }
    const uint32_t first = static_cast<uint32_t>(~node) >> 3;
    const uint32_t count = static_cast<uint32_t>(~node) & 7u;
    if (!in_blas) {
      if (count == 0u) {
        node = sp > 0 ? stack[--sp] : kDone;
        continue;
      }
      const float4* ipf = reinterpret_cast<const float4*>(sc.inst + first);
      const float4 r0 = __ldg(ipf), r1 = __ldg(ipf + 1), r2 = __ldg(ipf + 2);
      const uint4 meta = __ldg(reinterpret_cast<const uint4*>(ipf + 3));
      const float m[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
      if (kCount) ++cnt.insts;
      toLocal(m, wox, woy, woz, wdx, wdy, wdz, ox, oy, oz, dx, dy, dz);
      idx = safeInv(dx); idy = safeInv(dy); idz = safeInv(dz);
      oix = ox * idx; oiy = oy * idy; oiz = oz * idz;
      if (sp >= kStackSize) {
        atomicOr(status, 1u);
        return HitRec{tmax, 0.0f, 0.0f, -1, 0u};
      }
      stack[sp++] = kToTlas;
      nodes = W::blas(sc);
      in_blas = true;
      cur_inst = static_cast<int32_t>(first);
      node = static_cast<int32_t>(meta.w);  // blas4_root
      continue;
    }
    for (uint32_t kk = 0; kk < count; ++kk) {
      const float4* tp = sc.tris + 3u * (first + kk);
      const float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
      if (kCount) ++cnt.tris;
      float t, u, v;
      if (intersectTri(ox, oy, oz, dx, dy, dz, ta, tb, tc, t, u, v) && t < best.t) {
        best.t = t;
        best.u = u;
        best.v = v;
        best.inst = cur_inst;
        best.tri = first + kk;
        if (kAny) return best;
      }
    }
    node = sp > 0 ? stack[--sp] : kDone;
  }
  return best;
}

}  // namespace dev
}  // namespace cg

#endif
