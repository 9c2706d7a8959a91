// cg_bvh_device.cu — binned-SAH BVH build on the GPU (the split structure
// that cg_bvh.cpp's emission turns into BvhNode arrays).
//
// Level-synchronous: one launch per tree level, one CTA per node of the
// level.  A CTA reduces its node's box and centroid box, bins the centroids
// on each axis (16 bins, shared-memory atomics), evaluates the surface-area
// cost of every bin boundary, and partitions its primitive range stably
// around the best one, writing the two children for the next level.  Every
// decision uses the host builder's rule and float arithmetic (cg_bvh.cpp,
// Builder::split): the same bin of each centroid, the same sweep order and
// rounding of the costs (no contraction), the same leaf test.  Min/max
// reductions and bin counts are exact in any order, so a node splits into
// the same two primitive sets as on the host; only the order inside a range
// differs (std::partition is not stable), which changes nothing but the
// all-centroids-equal fallback that halves a node by position.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "cg_bvh.h"

namespace cg {
namespace {

constexpr uint32_t kBins = 16;
constexpr uint32_t kBlock = 256;

struct Work {
  int32_t node;
  uint32_t begin, end, depth;
};

struct DevOpt {
  uint32_t max_leaf;
  float traversal_cost, intersect_cost;
};

// Floats as ints whose signed order is the float order (no NaNs).
__device__ __forceinline__ int ordInt(float f) {
  const int b = __float_as_int(f);
  return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float ordFloat(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

// boxArea (cg_bvh.cpp) without contraction: 2 * (dx*dy + dy*dz + dz*dx)
__device__ __forceinline__ float areaRn(float lx, float ly, float lz, float hx, float hy, float hz) {
  const float dx = __fsub_rn(hx, lx), dy = __fsub_rn(hy, ly), dz = __fsub_rn(hz, lz);
  if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
  const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
  return __fmul_rn(2.0f, s);
}

__device__ __forceinline__ float warpMin(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warpMax(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide min (lo[0..5]) / max (hi[0..5]) of 6 + 6 values; result in s_out[12].
__device__ void blockBounds(float v[12], float* s_warp /*[kBlock/32][12]*/, float* s_out) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const float r = k < 6 ? warpMin(v[k]) : warpMax(v[k]);
    if (lane == 0) s_warp[warp * 12 + k] = r;
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    const int k = static_cast<int>(threadIdx.x);
    float r = s_warp[k];
    for (uint32_t w = 1; w < blockDim.x / 32u; ++w)
      r = k < 6 ? fminf(r, s_warp[w * 12 + k]) : fmaxf(r, s_warp[w * 12 + k]);
    s_out[k] = r;
  }
  __syncthreads();
}

__device__ __forceinline__ uint32_t binOf(float c, float lo, float scale) {
  uint32_t k = static_cast<uint32_t>(__fmul_rn(__fsub_rn(c, lo), scale));
  return k >= kBins ? kBins - 1u : k;
}

__global__ void __launch_bounds__(kBlock, 2) k_build_level(
    const float* __restrict__ boxes, const float* __restrict__ centers, uint32_t* order,
    uint32_t* order_tmp, const Work* __restrict__ in, Work* out, uint32_t* n_out, BvhTmpNode* tmp,
    uint32_t* n_tmp, uint32_t* max_depth, DevOpt opt) {
  const Work w = in[blockIdx.x];
  const uint32_t n = w.end - w.begin;
  __shared__ float s_warp[(kBlock / 32) * 12];
  __shared__ float s_bnd[12];   // box lo, centroid lo, box hi, centroid hi
  __shared__ int s_bin_lo[3][kBins][3], s_bin_hi[3][kBins][3];
  __shared__ uint32_t s_bin_cnt[3][kBins];
  __shared__ int s_axis;
  __shared__ uint32_t s_bin, s_mid, s_leaf;
  __shared__ uint32_t s_scan[kBlock / 32];
  if (threadIdx.x == 0) atomicMax(max_depth, w.depth);

  // ---- node box and centroid box ----
  float v[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    v[k] = INFINITY;
    v[6 + k] = -INFINITY;
  }
  for (uint32_t i = w.begin + threadIdx.x; i < w.end; i += blockDim.x) {
    const uint32_t p = order[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      v[a] = fminf(v[a], boxes[6 * p + a]);
      v[6 + a] = fmaxf(v[6 + a], boxes[6 * p + 3 + a]);
      v[3 + a] = fminf(v[3 + a], centers[3 * p + a]);
      v[9 + a] = fmaxf(v[9 + a], centers[3 * p + a]);
    }
  }
  blockBounds(v, s_warp, s_bnd);
  const float blo[3] = {s_bnd[0], s_bnd[1], s_bnd[2]}, bhi[3] = {s_bnd[6], s_bnd[7], s_bnd[8]};
  const float clo[3] = {s_bnd[3], s_bnd[4], s_bnd[5]}, chi[3] = {s_bnd[9], s_bnd[10], s_bnd[11]};
  if (threadIdx.x == 0) {
    BvhTmpNode& t = tmp[w.node];
    for (int a = 0; a < 3; ++a) {
      t.box.lo[a] = blo[a];
      t.box.hi[a] = bhi[a];
    }
  }
  float scale[3];
  bool live[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float ext = __fsub_rn(chi[a], clo[a]);
    live[a] = ext > 0.0f;
    scale[a] = live[a] ? __fdiv_rn(static_cast<float>(kBins), ext) : 0.0f;
  }

  // ---- bins ----
  if (n > 1) {
    for (uint32_t k = threadIdx.x; k < 3 * kBins; k += blockDim.x) {
      const uint32_t a = k / kBins, b = k % kBins;
      for (int c = 0; c < 3; ++c) {
        s_bin_lo[a][b][c] = ordInt(INFINITY);
        s_bin_hi[a][b][c] = ordInt(-INFINITY);
      }
      s_bin_cnt[a][b] = 0u;
    }
    __syncthreads();
    for (uint32_t i = w.begin + threadIdx.x; i < w.end; i += blockDim.x) {
      const uint32_t p = order[i];
      float lo[3], hi[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = boxes[6 * p + c];
        hi[c] = boxes[6 * p + 3 + c];
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (!live[a]) continue;
        const uint32_t b = binOf(centers[3 * p + a], clo[a], scale[a]);
        for (int c = 0; c < 3; ++c) {
          atomicMin(&s_bin_lo[a][b][c], ordInt(lo[c]));
          atomicMax(&s_bin_hi[a][b][c], ordInt(hi[c]));
        }
        atomicAdd(&s_bin_cnt[a][b], 1u);
      }
    }
    __syncthreads();
  }

  // ---- the host's split rule (Builder::split), one thread ----
  if (threadIdx.x == 0) {
    uint32_t leaf = 0, mid = w.end;
    int best_axis = -1;
    uint32_t best_bin = 0;
    if (n <= 1) {
      leaf = 1;
    } else {
      float best_cost = INFINITY;
      for (int a = 0; a < 3; ++a) {
        if (!live[a]) continue;
        float r_area[kBins];
        uint32_t r_cnt[kBins];
        float al[3] = {INFINITY, INFINITY, INFINITY}, ah[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t cnt = 0;
        for (uint32_t k = kBins - 1; k > 0; --k) {
          for (int c = 0; c < 3; ++c) {
            al[c] = fminf(al[c], ordFloat(s_bin_lo[a][k][c]));
            ah[c] = fmaxf(ah[c], ordFloat(s_bin_hi[a][k][c]));
          }
          cnt += s_bin_cnt[a][k];
          r_area[k] = areaRn(al[0], al[1], al[2], ah[0], ah[1], ah[2]);
          r_cnt[k] = cnt;
        }
        for (int c = 0; c < 3; ++c) {
          al[c] = INFINITY;
          ah[c] = -INFINITY;
        }
        cnt = 0;
        for (uint32_t k = 0; k + 1 < kBins; ++k) {
          for (int c = 0; c < 3; ++c) {
            al[c] = fminf(al[c], ordFloat(s_bin_lo[a][k][c]));
            ah[c] = fmaxf(ah[c], ordFloat(s_bin_hi[a][k][c]));
          }
          cnt += s_bin_cnt[a][k];
          if (cnt == 0 || r_cnt[k + 1] == 0) continue;
          const float cst =
              __fadd_rn(__fmul_rn(areaRn(al[0], al[1], al[2], ah[0], ah[1], ah[2]),
                                  static_cast<float>(cnt)),
                        __fmul_rn(r_area[k + 1], static_cast<float>(r_cnt[k + 1])));
          if (cst < best_cost) {
            best_cost = cst;
            best_axis = a;
            best_bin = k;
          }
        }
      }
      const float parent_area = areaRn(blo[0], blo[1], blo[2], bhi[0], bhi[1], bhi[2]);
      const float leaf_cost = __fmul_rn(static_cast<float>(n), opt.intersect_cost);
      const float split_cost =
          parent_area > 0.0f
              ? __fadd_rn(opt.traversal_cost,
                          __fdiv_rn(__fmul_rn(opt.intersect_cost, best_cost), parent_area))
              : INFINITY;
      if (best_axis < 0) {
        if (n <= opt.max_leaf)
          leaf = 1;
        else
          mid = w.begin + n / 2;  // all centroids coincide: halve by position
      } else if (n <= opt.max_leaf && leaf_cost <= split_cost) {
        leaf = 1;
      } else {
        uint32_t nl = 0;
        for (uint32_t k = 0; k <= best_bin; ++k) nl += s_bin_cnt[best_axis][k];
        mid = w.begin + nl;
      }
    }
    s_axis = best_axis;
    s_bin = best_bin;
    s_mid = mid;
    s_leaf = leaf;
  }
  __syncthreads();
  const uint32_t mid = s_mid;
  if (s_leaf) {
    if (threadIdx.x == 0) {
      tmp[w.node].first = w.begin;
      tmp[w.node].count = n;
    }
    return;
  }

  // ---- stable partition around (axis, bin) through order_tmp ----
  const int axis = s_axis;
  if (axis >= 0) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t left_base = w.begin, right_base = mid;
    for (uint32_t c0 = w.begin; c0 < w.end; c0 += blockDim.x) {
      const uint32_t i = c0 + threadIdx.x;
      uint32_t p = 0;
      bool is_left = false;
      if (i < w.end) {
        p = order[i];
        is_left = binOf(centers[3 * p + axis], clo[axis], scale[axis]) <= s_bin;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, is_left);
      if (lane == 0) s_scan[warp] = static_cast<uint32_t>(__popc(bal));
      __syncthreads();
      uint32_t before = 0, total = 0;
      for (uint32_t k = 0; k < blockDim.x / 32u; ++k) {
        if (k < warp) before += s_scan[k];
        total += s_scan[k];
      }
      const uint32_t lrank = before + static_cast<uint32_t>(__popc(bal & ((1u << lane) - 1u)));
      if (i < w.end) {
        const uint32_t chunk_pos = i - c0;  // position within this chunk
        if (is_left)
          order_tmp[left_base + lrank] = p;
        else
          order_tmp[right_base + (chunk_pos - lrank)] = p;
      }
      const uint32_t chunk_n = min(blockDim.x, w.end - c0);
      left_base += total;
      right_base += chunk_n - total;
      __syncthreads();  // s_scan is rewritten by the next chunk
    }
    __syncthreads();
    for (uint32_t i = w.begin + threadIdx.x; i < w.end; i += blockDim.x) order[i] = order_tmp[i];
  }
  if (threadIdx.x == 0) {
    const uint32_t l = atomicAdd(n_tmp, 2u);
    tmp[w.node].left = static_cast<int32_t>(l);
    tmp[w.node].right = static_cast<int32_t>(l + 1);
    tmp[l] = BvhTmpNode{};
    tmp[l + 1] = BvhTmpNode{};
    const uint32_t o = atomicAdd(n_out, 2u);
    out[o] = Work{static_cast<int32_t>(l), w.begin, mid, w.depth + 1};
    out[o + 1] = Work{static_cast<int32_t>(l + 1), mid, w.end, w.depth + 1};
  }
}

__global__ void k_centers(const float* __restrict__ boxes, float* centers, uint32_t* order,
                          uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int a = 0; a < 3; ++a)
    centers[3 * i + a] = __fmul_rn(0.5f, __fadd_rn(boxes[6 * i + a], boxes[6 * i + 3 + a]));
  order[i] = i;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

bool check(cudaError_t e, const char* what, std::string& err) {
  if (e == cudaSuccess) return true;
  cudaGetLastError();
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

}  // namespace

bool buildBvhTmpDevice(const std::vector<Box>& boxes, const BvhBuildOptions& opt,
                       std::vector<BvhTmpNode>& tmp, std::vector<uint32_t>& order_local,
                       uint32_t* depth_out, std::string& err) {
  const uint32_t N = static_cast<uint32_t>(boxes.size());
  if (N == 0 || opt.bins != kBins) {
    err = "device build needs primitives and 16 bins";
    return false;
  }
  const size_t max_nodes = 2 * size_t(N);
  const size_t bytes_boxes = sizeof(Box) * N, bytes_c = 12 * size_t(N), bytes_o = 4 * size_t(N);
  const size_t bytes_tmp = sizeof(BvhTmpNode) * max_nodes, bytes_work = sizeof(Work) * size_t(N);
  size_t offs[9], total = 0;
  const size_t sizes[9] = {bytes_boxes, bytes_c, bytes_o, bytes_o, bytes_tmp,
                           bytes_work,  bytes_work, 16, 16};
  for (int k = 0; k < 9; ++k) {
    offs[k] = total;
    total += (sizes[k] + 255) & ~size_t(255);
  }
  DevBuf buf;
  if (!check(cudaMalloc(&buf.p, total), "cudaMalloc (device BVH build)", err)) return false;
  char* base = static_cast<char*>(buf.p);
  float* d_boxes = reinterpret_cast<float*>(base + offs[0]);
  float* d_centers = reinterpret_cast<float*>(base + offs[1]);
  uint32_t* d_order = reinterpret_cast<uint32_t*>(base + offs[2]);
  uint32_t* d_order_tmp = reinterpret_cast<uint32_t*>(base + offs[3]);
  BvhTmpNode* d_tmp = reinterpret_cast<BvhTmpNode*>(base + offs[4]);
  Work* d_work[2] = {reinterpret_cast<Work*>(base + offs[5]), reinterpret_cast<Work*>(base + offs[6])};
  uint32_t* d_cnt = reinterpret_cast<uint32_t*>(base + offs[7]);  // [0] next level, [1] nodes, [2] depth
  cudaStream_t s = nullptr;
  if (!check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate", err)) return false;
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{s};
  if (!check(cudaMemcpyAsync(d_boxes, boxes.data(), bytes_boxes, cudaMemcpyHostToDevice, s),
             "cudaMemcpyAsync", err))
    return false;
  k_centers<<<(N + 255) / 256, 256, 0, s>>>(d_boxes, d_centers, d_order, N);
  const BvhTmpNode root{};
  const Work first{0, 0u, N, 1u};
  const uint32_t init_cnt[4] = {0u, 1u, 0u, 0u};
  if (!check(cudaMemcpyAsync(d_tmp, &root, sizeof(root), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync", err) ||
      !check(cudaMemcpyAsync(d_work[0], &first, sizeof(first), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync", err) ||
      !check(cudaMemcpyAsync(d_cnt, init_cnt, sizeof(init_cnt), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync", err))
    return false;
  const DevOpt dopt{opt.max_leaf, opt.traversal_cost, opt.intersect_cost};
  uint32_t level_n = 1;
  int cur = 0;
  // a tree over N primitives has at most N levels; each level doubles at most
  for (uint32_t level = 0; level_n > 0 && level <= N; ++level) {
    if (!check(cudaMemsetAsync(d_cnt, 0, 4, s), "cudaMemsetAsync", err)) return false;
    k_build_level<<<level_n, kBlock, 0, s>>>(d_boxes, d_centers, d_order, d_order_tmp, d_work[cur],
                                             d_work[cur ^ 1], d_cnt, d_tmp, d_cnt + 1, d_cnt + 2, dopt);
    if (!check(cudaGetLastError(), "k_build_level", err)) return false;
    uint32_t next = 0;
    if (!check(cudaMemcpyAsync(&next, d_cnt, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync", err) ||
        !check(cudaStreamSynchronize(s), "k_build_level", err))
      return false;
    if (next > N) {
      err = "device BVH build: level overflow";
      return false;
    }
    level_n = next;
    cur ^= 1;
  }
  uint32_t counts[3] = {0u, 0u, 0u};
  if (!check(cudaMemcpyAsync(counts, d_cnt, sizeof(counts), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync", err) ||
      !check(cudaStreamSynchronize(s), "cudaStreamSynchronize", err))
    return false;
  const uint32_t n_nodes = counts[1];
  if (n_nodes == 0 || n_nodes > max_nodes) {
    err = "device BVH build: bad node count";
    return false;
  }
  tmp.resize(n_nodes);
  order_local.resize(N);
  if (!check(cudaMemcpyAsync(tmp.data(), d_tmp, sizeof(BvhTmpNode) * n_nodes, cudaMemcpyDeviceToHost, s),
             "cudaMemcpyAsync", err) ||
      !check(cudaMemcpyAsync(order_local.data(), d_order, bytes_o, cudaMemcpyDeviceToHost, s),
             "cudaMemcpyAsync", err) ||
      !check(cudaStreamSynchronize(s), "cudaStreamSynchronize", err))
    return false;
  if (depth_out) *depth_out = counts[2];
  return true;
}

}  // namespace cg
