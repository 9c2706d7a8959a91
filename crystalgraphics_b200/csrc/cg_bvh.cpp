// cg_bvh.cpp — binned-SAH BVH builder for the device BvhNode layout.
#include "cg_bvh.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace cg {
namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();
constexpr uint32_t kMaxBins = 64;

inline void boxReset(Box& b) {
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = kInf;
    b.hi[a] = -kInf;
  }
}
inline void boxGrow(Box& b, const Box& o) {
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = std::min(b.lo[a], o.lo[a]);
    b.hi[a] = std::max(b.hi[a], o.hi[a]);
  }
}
inline void boxGrowPt(Box& b, const float* p) {
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = std::min(b.lo[a], p[a]);
    b.hi[a] = std::max(b.hi[a], p[a]);
  }
}
inline float boxArea(const Box& b) {
  float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
  if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

using TmpNode = BvhTmpNode;

struct Builder {
  const std::vector<Box>& boxes;
  const BvhBuildOptions& opt;
  std::vector<float> centers;  // 3 per primitive
  std::vector<uint32_t>& order;
  uint32_t order_base;
  std::vector<TmpNode> tmp;
  uint32_t max_depth = 0;

  Builder(const std::vector<Box>& b, const BvhBuildOptions& o, std::vector<uint32_t>& ord)
      : boxes(b), opt(o), order(ord), order_base(static_cast<uint32_t>(ord.size())) {}

  // Splits order[begin, end) in place; returns the split position or `end`
  // to make a leaf.
  uint32_t split(uint32_t begin, uint32_t end, const Box& bounds) {
    const uint32_t n = end - begin;
    if (n <= 1) return end;
    Box cb;
    boxReset(cb);
    for (uint32_t i = begin; i < end; ++i) boxGrowPt(cb, &centers[3 * order[i]]);
    const uint32_t B = std::min<uint32_t>(std::max<uint32_t>(opt.bins, 2u), kMaxBins);
    float best_cost = kInf;
    int best_axis = -1;
    uint32_t best_bin = 0;
    Box bin_box[kMaxBins];
    uint32_t bin_cnt[kMaxBins];
    float right_area[kMaxBins];
    uint32_t right_cnt[kMaxBins];
    for (int a = 0; a < 3; ++a) {
      float ext = cb.hi[a] - cb.lo[a];
      if (!(ext > 0.0f)) continue;
      float scale = static_cast<float>(B) / ext;
      for (uint32_t k = 0; k < B; ++k) {
        boxReset(bin_box[k]);
        bin_cnt[k] = 0;
      }
      for (uint32_t i = begin; i < end; ++i) {
        uint32_t p = order[i];
        uint32_t k = static_cast<uint32_t>((centers[3 * p + a] - cb.lo[a]) * scale);
        if (k >= B) k = B - 1;
        boxGrow(bin_box[k], boxes[p]);
        ++bin_cnt[k];
      }
      Box acc;
      boxReset(acc);
      uint32_t cnt = 0;
      for (uint32_t k = B - 1; k > 0; --k) {
        boxGrow(acc, bin_box[k]);
        cnt += bin_cnt[k];
        right_area[k] = boxArea(acc);
        right_cnt[k] = cnt;
      }
      boxReset(acc);
      cnt = 0;
      for (uint32_t k = 0; k + 1 < B; ++k) {
        boxGrow(acc, bin_box[k]);
        cnt += bin_cnt[k];
        if (cnt == 0 || right_cnt[k + 1] == 0) continue;
        float c = boxArea(acc) * static_cast<float>(cnt) +
                  right_area[k + 1] * static_cast<float>(right_cnt[k + 1]);
        if (c < best_cost) {
          best_cost = c;
          best_axis = a;
          best_bin = k;
        }
      }
    }
    float parent_area = boxArea(bounds);
    float leaf_cost = static_cast<float>(n) * opt.intersect_cost;
    float split_cost = parent_area > 0.0f
                           ? opt.traversal_cost + opt.intersect_cost * best_cost / parent_area
                           : kInf;
    if (best_axis < 0) {
      // all centroids coincide: median split by index if the node is too big
      if (n <= opt.max_leaf) return end;
      return begin + n / 2;
    }
    if (n <= opt.max_leaf && leaf_cost <= split_cost) return end;
    const int a = best_axis;
    const float scale = static_cast<float>(B) / (cb.hi[a] - cb.lo[a]);  // as when binning
    auto mid = std::partition(order.begin() + begin, order.begin() + end, [&](uint32_t p) {
      uint32_t k = static_cast<uint32_t>((centers[3 * p + a] - cb.lo[a]) * scale);
      if (k >= B) k = B - 1;
      return k <= best_bin;
    });
    uint32_t m = static_cast<uint32_t>(mid - order.begin());
    if (m == begin || m == end) m = begin + n / 2;
    return m;
  }

  void run() {
    const uint32_t N = static_cast<uint32_t>(boxes.size());
    centers.resize(3 * size_t(N));
    for (uint32_t i = 0; i < N; ++i)
      for (int a = 0; a < 3; ++a) centers[3 * i + a] = 0.5f * (boxes[i].lo[a] + boxes[i].hi[a]);
    for (uint32_t i = 0; i < N; ++i) order.push_back(i);
    tmp.reserve(2 * size_t(N) + 1);
    struct Work {
      int32_t node;
      uint32_t begin, end, depth;
    };
    std::vector<Work> stack;
    tmp.emplace_back();
    stack.push_back({0, order_base, order_base + N, 1});
    while (!stack.empty()) {
      Work w = stack.back();
      stack.pop_back();
      max_depth = std::max(max_depth, w.depth);
      Box bounds;
      boxReset(bounds);
      for (uint32_t i = w.begin; i < w.end; ++i) boxGrow(bounds, boxes[order[i]]);
      tmp[w.node].box = bounds;
      // split works on local order indices; order[] holds local primitive ids
      uint32_t m = (w.end - w.begin <= 1) ? w.end : split(w.begin, w.end, bounds);
      if (m == w.end) {
        tmp[w.node].first = w.begin;
        tmp[w.node].count = w.end - w.begin;
        continue;
      }
      int32_t l = static_cast<int32_t>(tmp.size());
      tmp.emplace_back();
      tmp.emplace_back();
      tmp[w.node].left = l;
      tmp[w.node].right = l + 1;
      stack.push_back({l + 1, m, w.end, w.depth + 1});
      stack.push_back({l, w.begin, m, w.depth + 1});
    }
  }
};

void setChild(BvhNode& n, int which, const Box& b, int32_t link, uint32_t cnt) {
  if (which == 0) {
    n.c0lx = b.lo[0]; n.c0hx = b.hi[0]; n.c0ly = b.lo[1]; n.c0hy = b.hi[1];
    n.c0lz = b.lo[2]; n.c0hz = b.hi[2];
    n.child0 = link;
    n.cnt0 = cnt;
  } else {
    n.c1lx = b.lo[0]; n.c1hx = b.hi[0]; n.c1ly = b.lo[1]; n.c1hy = b.hi[1];
    n.c1lz = b.lo[2]; n.c1hz = b.hi[2];
    n.child1 = link;
    n.cnt1 = cnt;
  }
}

}  // namespace

void padBox(Box& b) {
  for (int a = 0; a < 3; ++a) {
    float m = std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a]));
    float pad = m * 1.0e-5f + 1.0e-5f;
    b.lo[a] -= pad;
    b.hi[a] += pad;
  }
}

namespace {

struct Child4 {
  Box box;
  int32_t link;
};

// A node's children (at most four while collapsing), without allocation.
struct Kids {
  Child4 c[4];
  size_t size = 0;
  void push(const Child4& k) { c[size++] = k; }
  void erase(size_t i) {
    for (size_t k = i; k + 1 < size; ++k) c[k] = c[k + 1];
    --size;
  }
};

void childrenOf(const BvhNode& n, Kids& out) {
  const Child4 c0{{{n.c0lx, n.c0ly, n.c0lz}, {n.c0hx, n.c0hy, n.c0hz}}, n.child0};
  const Child4 c1{{{n.c1lx, n.c1ly, n.c1lz}, {n.c1hx, n.c1hy, n.c1hz}}, n.child1};
  // an absent child is a leaf of zero primitives
  if (c0.link >= 0 || leafCount(c0.link) != 0) out.push(c0);
  if (c1.link >= 0 || leafCount(c1.link) != 0) out.push(c1);
}

uint32_t collapse(const std::vector<BvhNode>& b2, uint32_t n2, std::vector<Bvh4Node>& out) {
  const uint32_t idx = static_cast<uint32_t>(out.size());
  out.emplace_back();
  Kids kids;
  childrenOf(b2[n2], kids);
  while (kids.size < 4) {
    int best = -1;
    float best_area = -1.0f;
    for (size_t k = 0; k < kids.size; ++k) {
      if (kids.c[k].link < 0) continue;
      const float a = boxArea(kids.c[k].box);
      if (a > best_area) {
        best_area = a;
        best = static_cast<int>(k);
      }
    }
    if (best < 0) break;
    Kids sub;
    childrenOf(b2[kids.c[best].link], sub);
    if (kids.size - 1 + sub.size > 4) break;
    kids.erase(static_cast<size_t>(best));
    for (size_t k = 0; k < sub.size; ++k) kids.push(sub.c[k]);
  }
  int32_t links[4];
  for (size_t k = 0; k < 4; ++k) {
    if (k < kids.size)
      links[k] = kids.c[k].link >= 0 ? static_cast<int32_t>(collapse(b2, kids.c[k].link, out))
                                     : kids.c[k].link;
    else
      links[k] = kEmptyLink;
  }
  Bvh4Node& n = out[idx];
  for (int k = 0; k < 4; ++k) {
    const bool has = static_cast<size_t>(k) < kids.size;
    n.lox[k] = has ? kids.c[k].box.lo[0] : 1e30f;
    n.loy[k] = has ? kids.c[k].box.lo[1] : 1e30f;
    n.loz[k] = has ? kids.c[k].box.lo[2] : 1e30f;
    n.hix[k] = has ? kids.c[k].box.hi[0] : 1e30f;
    n.hiy[k] = has ? kids.c[k].box.hi[1] : 1e30f;
    n.hiz[k] = has ? kids.c[k].box.hi[2] : 1e30f;
    n.child[k] = links[k];
    n._pad[k] = 0;
  }
  return idx;
}

}  // namespace

uint32_t collapseBvh4(const std::vector<BvhNode>& bvh2, uint32_t root2, std::vector<Bvh4Node>& out) {
  return collapse(bvh2, root2, out);
}

void quantizeBvh4(const std::vector<Bvh4Node>& in, std::vector<Bvh4QNode>& out) {
  out.resize(in.size());
  for (size_t i = 0; i < in.size(); ++i) {
    const Bvh4Node& n = in[i];
    Bvh4QNode q{};
    const float* lo[3] = {n.lox, n.loy, n.loz};
    const float* hi[3] = {n.hix, n.hiy, n.hiz};
    float org[3] = {0.0f, 0.0f, 0.0f};
    int exps[3] = {0, 0, 0};
    uint32_t qlo[3] = {0u, 0u, 0u}, qhi[3] = {0u, 0u, 0u};
    for (int a = 0; a < 3; ++a) {
      float mn = std::numeric_limits<float>::infinity(), mx = -mn;
      for (int c = 0; c < 4; ++c) {
        if (n.child[c] == kEmptyLink) continue;
        mn = std::min(mn, lo[a][c]);
        mx = std::max(mx, hi[a][c]);
      }
      if (!(mn <= mx)) mn = mx = 0.0f;  // no children
      org[a] = mn;
      // smallest power of two s with 255 * s >= extent (s >= 2^-126)
      const double ext = static_cast<double>(mx) - static_cast<double>(mn);
      int k = -126;
      if (ext > 0.0) {
        k = static_cast<int>(std::ceil(std::log2(ext / 255.0)));
        while (k > -126 && std::ldexp(255.0, k - 1) >= ext) --k;
        while (std::ldexp(255.0, k) < ext) ++k;
        k = std::max(k, -126);
      }
      exps[a] = k;
      const double s = std::ldexp(1.0, k);
      for (int c = 0; c < 4; ++c) {
        if (n.child[c] == kEmptyLink) continue;
        // outward rounding: org + ql * s <= lo and org + qh * s >= hi exactly,
        // and a float rounding of either stays on the same side
        const double fl = std::floor((static_cast<double>(lo[a][c]) - mn) / s);
        const double ch = std::ceil((static_cast<double>(hi[a][c]) - mn) / s);
        const uint32_t ql = static_cast<uint32_t>(std::clamp(fl, 0.0, 255.0));
        const uint32_t qh = static_cast<uint32_t>(std::clamp(ch, 0.0, 255.0));
        qlo[a] |= ql << (8 * c);
        qhi[a] |= qh << (8 * c);
      }
    }
    q.ox = org[0];
    q.oy = org[1];
    q.oz = org[2];
    q.scale_bits = static_cast<uint32_t>(exps[0] + 127) | (static_cast<uint32_t>(exps[1] + 127) << 8) |
                   (static_cast<uint32_t>(exps[2] + 127) << 16);
    q.qlox = qlo[0];
    q.qhix = qhi[0];
    q.qloy = qlo[1];
    q.qhiy = qhi[1];
    q.qloz = qlo[2];
    q.qhiz = qhi[2];
    for (int c = 0; c < 4; ++c) q.child[c] = n.child[c];
    out[i] = q;
  }
}

namespace {
std::atomic<int> g_build_mode{kBuildAuto};
thread_local BvhBuildStats tl_build_stats;

bool deviceAvailable() {
  static const bool ok = [] {
    int n = 0;
    const bool has = cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
    cudaGetLastError();
    return has;
  }();
  return ok;
}
}  // namespace

void setBvhBuildMode(int mode) { g_build_mode.store(mode); }
int bvhBuildMode() { return g_build_mode.load(); }
void resetBvhBuildStats() { tl_build_stats = BvhBuildStats{}; }
BvhBuildStats bvhBuildStats() { return tl_build_stats; }

uint32_t buildBvh(const std::vector<Box>& boxes, const BvhBuildOptions& opt, uint32_t prim_base,
                  std::vector<BvhNode>& nodes, std::vector<uint32_t>& order,
                  uint32_t* depth_out) {
  const uint32_t base = static_cast<uint32_t>(nodes.size());
  const size_t order_base = order.size();
  const auto t0 = std::chrono::steady_clock::now();
  Builder b(boxes, opt, order);
  const int mode = g_build_mode.load();
  const bool device = !boxes.empty() && opt.bins == 16 &&
                      (mode == kBuildDevice ||
                       (mode == kBuildAuto && boxes.size() >= kDeviceBuildMinPrims &&
                        deviceAvailable()));
  bool built = false;
  if (device) {
    std::vector<uint32_t> local;
    std::string err;
    uint32_t depth = 0;
    if (buildBvhTmpDevice(boxes, opt, b.tmp, local, &depth, err)) {
      for (TmpNode& t : b.tmp)
        if (t.left < 0) t.first += static_cast<uint32_t>(order_base);
      order.insert(order.end(), local.begin(), local.end());
      b.max_depth = depth;
      built = true;
      ++tl_build_stats.device_builds;
    } else if (mode == kBuildDevice) {
      throw std::runtime_error(err);
    }
  }
  if (!built && !boxes.empty()) {
    b.tmp.clear();
    b.run();
    ++tl_build_stats.host_builds;
  }
  tl_build_stats.seconds +=
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (depth_out) *depth_out = b.max_depth;
  // Emit: every inner TmpNode becomes one BvhNode; DFS order keeps siblings'
  // subtrees contiguous.  A root that is a leaf gets a node with one child.
  // An absent child gets a point box at 1e30: slab tests reorder bounds, so an
  // inverted box would still be entered; a box that far is entered only
  // beyond any t the traversal accepts (hits are below 1e6).
  Box empty;
  for (int a = 0; a < 3; ++a) {
    empty.lo[a] = 1e30f;
    empty.hi[a] = 1e30f;
  }
  auto leafLink = [&](const TmpNode& t) {
    // order[] entries from order_base are local ids; leaves index order[]
    return leafLinkOf(prim_base + (t.first - static_cast<uint32_t>(order_base)), t.count);
  };
  if (boxes.empty()) {
    BvhNode n{};
    setChild(n, 0, empty, leafLinkOf(prim_base, 0), 0);
    setChild(n, 1, empty, leafLinkOf(prim_base, 0), 0);
    nodes.push_back(n);
    return base;
  }
  std::vector<int32_t> out_index(b.tmp.size(), -1);
  // assign output indices in DFS preorder over inner nodes
  std::vector<int32_t> st{0};
  uint32_t next = base;
  std::vector<int32_t> inner_order;
  while (!st.empty()) {
    int32_t t = st.back();
    st.pop_back();
    if (b.tmp[t].left < 0) continue;
    out_index[t] = static_cast<int32_t>(next++);
    inner_order.push_back(t);
    st.push_back(b.tmp[t].right);
    st.push_back(b.tmp[t].left);
  }
  if (inner_order.empty()) {  // root is a leaf
    BvhNode n{};
    Box bx = b.tmp[0].box;
    padBox(bx);
    setChild(n, 0, bx, leafLink(b.tmp[0]), b.tmp[0].count);
    setChild(n, 1, empty, kEmptyLink, 0);
    nodes.push_back(n);
    return base;
  }
  nodes.resize(next);
  for (int32_t t : inner_order) {
    BvhNode n{};
    for (int c = 0; c < 2; ++c) {
      const TmpNode& ch = b.tmp[c == 0 ? b.tmp[t].left : b.tmp[t].right];
      int32_t ci = c == 0 ? b.tmp[t].left : b.tmp[t].right;
      Box bx = ch.box;
      padBox(bx);
      if (ch.left >= 0)
        setChild(n, c, bx, out_index[ci], 0);
      else
        setChild(n, c, bx, leafLink(ch), ch.count);
    }
    nodes[out_index[t]] = n;
  }
  return base;
}

}  // namespace cg
