// cg_bvh.h — host BVH builder (binned SAH) emitting the device BvhNode layout.
//
// The reference builds median-split BVH2s with one triangle pair per leaf
// (src/pathtracing/blas.h:112-194) and a median-split TLAS
// (src/pathtracing/tlas.h:98-140).  The closest hit does not depend on the
// tree (only exact ties can resolve differently), so this backend builds
// surface-area-heuristic trees instead, which visit fewer nodes per ray.
#ifndef CG_BVH_H_
#define CG_BVH_H_

#include <cstdint>
#include <string>
#include <vector>

#include "cg_types.h"

namespace cg {

struct Box {
  float lo[3], hi[3];
};

struct BvhBuildOptions {
  uint32_t max_leaf = 4;      // primitives per leaf at most
  uint32_t bins = 16;         // SAH bins per axis
  float traversal_cost = 1.0f;
  float intersect_cost = 1.0f;
};

// Builds a BVH over `boxes`.  Appends nodes to `nodes` (child indices are
// absolute, offset by nodes.size() at entry) and returns the root index.
// `order` receives the primitive permutation: leaf ranges index `order`,
// offset by `prim_base` (the caller's global primitive offset).  The split
// structure comes from the GPU (buildBvhTmpDevice) or the host builder, as
// the build mode selects.
uint32_t buildBvh(const std::vector<Box>& boxes, const BvhBuildOptions& opt,
                  uint32_t prim_base, std::vector<BvhNode>& nodes,
                  std::vector<uint32_t>& order, uint32_t* depth_out = nullptr);

// The split structure a builder produces before emission: node 0 is the
// root; an inner node has two children (indices into the same array), a leaf
// the range [first, first + count) of the primitive permutation.
struct BvhTmpNode {
  Box box;
  int32_t left = -1, right = -1;
  uint32_t first = 0, count = 0;
};

// Binned-SAH build on the current CUDA device with the host builder's split
// rule; `order_local` receives the permutation of 0-based primitive ids and
// leaf ranges index it from 0.  Returns false (with `err`) on a CUDA error.
bool buildBvhTmpDevice(const std::vector<Box>& boxes, const BvhBuildOptions& opt,
                       std::vector<BvhTmpNode>& tmp, std::vector<uint32_t>& order_local,
                       uint32_t* depth_out, std::string& err);

// Where buildBvh builds: kBuildAuto = on the GPU for trees of at least
// kDeviceBuildMinPrims primitives when a CUDA device is present, else on the
// host; kBuildHost / kBuildDevice force one (a failed device build then makes
// buildBvh throw std::runtime_error).
enum BvhBuildMode : int { kBuildAuto = 0, kBuildHost = 1, kBuildDevice = 2 };
constexpr uint32_t kDeviceBuildMinPrims = 16384;
void setBvhBuildMode(int mode);
int bvhBuildMode();
// Statistics of the calling thread's builds since the last reset: host and
// device builds and the seconds they took.
struct BvhBuildStats {
  uint32_t host_builds = 0, device_builds = 0;
  double seconds = 0.0;
};
void resetBvhBuildStats();
BvhBuildStats bvhBuildStats();

// Leaf links: ~((first << 3) | count), count <= 7 (so the values INT_MIN and
// INT_MIN + 1, i.e. count 7 and 6 with first = 2^28 - 1, never occur and
// serve as traversal markers).  first < 2^28.
inline int32_t leafLinkOf(uint32_t first, uint32_t count) {
  return static_cast<int32_t>(~((first << 3) | count));
}
inline uint32_t leafFirst(int32_t link) { return static_cast<uint32_t>(~link) >> 3; }
inline uint32_t leafCount(int32_t link) { return static_cast<uint32_t>(~link) & 7u; }

// Enlarges a box by a small margin so slab tests computed with rounding
// never reject a primitive that lies on the box boundary.
void padBox(Box& b);

// Collapses the BVH2 subtree at `root2` of `bvh2` into four-wide nodes
// appended to `out` (each node takes up to four descendants, expanding the
// inner child of largest surface area first); returns the new root's index.
// Leaf links are kept as they are.
uint32_t collapseBvh4(const std::vector<BvhNode>& bvh2, uint32_t root2, std::vector<Bvh4Node>& out);

// Quantises every node of a four-wide tree into Bvh4QNode (same indices and
// links): per node the union of its children's boxes gives the origin, each
// axis a power-of-two scale with 255 steps covering the extent, and the
// child bounds are rounded outwards to those steps.
void quantizeBvh4(const std::vector<Bvh4Node>& in, std::vector<Bvh4QNode>& out);

}  // namespace cg

#endif
