// cg_types.h — device data layout of the B200 path-tracing backend, shared by
// host packing (cg_scene.cpp) and the kernels (cg_kernels.cu).
//
// Everything the traversal reads is 16-byte aligned and fetched with 128-bit
// loads:
//   BvhNode      64 B  two child boxes + child links (binary BVH, both
//                      children tested per visit)
//   triangle     48 B  v0 | e1 | e2 (Möller–Trumbore operands, precomputed
//                      on the host with the same float subtraction the
//                      reference does per test, so t/u/v are bit-identical)
//   DevInstance  64 B  world->local rows + BLAS root + material
// Shading-only data (vertex normals, materials) is touched once per hit.
#ifndef CG_TYPES_H_
#define CG_TYPES_H_

#include <cstdint>

#ifdef __CUDACC__
#define CG_HD __host__ __device__
#else
#define CG_HD
#endif

namespace cg {

// One binary BVH node; children are described in the node itself.
// child >= 0: inner node index; child < 0: leaf, ~child = first primitive,
// count in cnt.  An absent child has a point box at 1e30 and count 0.
struct alignas(16) BvhNode {
  float c0lx, c0hx, c0ly, c0hy;  // child 0: x and y slabs
  float c1lx, c1hx, c1ly, c1hy;  // child 1: x and y slabs
  float c0lz, c0hz, c1lz, c1hz;  // z slabs of both children
  int32_t child0, child1;
  uint32_t cnt0, cnt1;
};
static_assert(sizeof(BvhNode) == 64, "BvhNode is 64 bytes");

// Link of an absent four-wide child (a leaf of zero primitives).
constexpr int32_t kEmptyLink = -1;

// Node format the traversal walks.
enum NodeFormat : int {
  kNodesBinary = 0,  // BvhNode, two children
  kNodesWide4 = 1,   // Bvh4Node, four children with full-precision boxes
  kNodesWide4Q = 2,  // Bvh4QNode, four children with 8-bit boxes
};

// Four-wide node: the slabs of four children, structure-of-arrays so each
// axis bound is one 128-bit load; links as in BvhNode (leaf count in the low
// 3 bits of ~link).  An absent child has link kEmptyLink and a point box at
// 1e30.  Collapsed from the SAH BVH2, it halves the dependent node fetches of
// a ray.
struct alignas(16) Bvh4Node {
  float lox[4], hix[4], loy[4], hiy[4], loz[4], hiz[4];
  int32_t child[4];
  uint32_t _pad[4];
};
static_assert(sizeof(Bvh4Node) == 128, "Bvh4Node is 128 bytes");

// Compressed four-wide node (64 B, four 128-bit loads per visit instead of
// eight): the node's box origin, one power-of-two scale per axis, and the
// four child boxes as 8-bit offsets in units of that scale, rounded outwards
// (child lo = origin + qlo * scale <= the child's box, hi likewise >=), so a
// quantised box always contains the full-precision one.  Same indices and
// links as the Bvh4Node array it is built from; an absent child
// (kEmptyLink) is skipped by its link, not by its box.
struct alignas(16) Bvh4QNode {
  float ox, oy, oz;
  uint32_t scale_bits;    // biased float exponents of the x, y, z scales (bytes 0..2)
  uint32_t qlox, qhix, qloy, qhiy;  // byte c = child c
  uint32_t qloz, qhiz, _pad0, _pad1;
  int32_t child[4];
};
static_assert(sizeof(Bvh4QNode) == 64, "Bvh4QNode is 64 bytes");

struct alignas(16) DevInstance {
  float inv[12];        // row-major world -> local (3x4)
  uint32_t blas_root;   // node index of the mesh BLAS root (BVH2)
  uint32_t material;
  uint32_t tri_base;    // first triangle of the mesh in the global arrays
  uint32_t blas4_root;  // node index of the mesh BLAS root (BVH4)
};
static_assert(sizeof(DevInstance) == 64, "DevInstance is 64 bytes");

// Pre-decoded material (the fields shading/material.wesl:19-53 reads, with
// the clamps and max(emissive * strength, 0) that do not depend on the
// wavelength already applied).
struct alignas(16) DevMaterial {
  float base[3];
  float metallic;         // clamp(metallic, 0, 1)
  float emission[3];      // max(emissive_factor * emissive_strength, 0)
  float roughness;        // clamp(roughness, 0, 1)
  float ior;
  float dispersion;
  float transmission;     // clamp(transmission, 0, 1)
  uint32_t volume;        // bit 0: thickness_factor > 0; bits 8..11: shading kind
};
// Shading kind of a material: which lobe code paths a hit on it can take
// (bit 0 diffuse, bit 1 specular, bit 2 rough, bit 3 transmission).  Hits are
// grouped by kind before shading so a warp runs one path.
constexpr uint32_t kKindShift = 8u;
// volume bit 1: the material samples at least one texture (DevMatTex holds them)
constexpr uint32_t kTexturedBit = 2u;
static_assert(sizeof(DevMaterial) == 48, "DevMaterial is 48 bytes");

// Texture references of a material (read only when DevMaterial has
// kTexturedBit): the layer of each texture decode() samples (-1 = none), in
// the order base color, metallic-roughness, emissive, transmission; bit k of
// uv1_bits selects TEXCOORD_1 for texture k; and the unclamped factors the
// texels multiply (material.wesl:181-262).
struct alignas(16) DevMatTex {
  int32_t layer[4];
  uint32_t uv1_bits;
  float metallic, roughness, transmission;  // factors before the clamp
  float emissive[3];                        // emissive_factor
  float emissive_strength;
};
static_assert(sizeof(DevMatTex) == 48, "DevMatTex is 48 bytes");

// Emissive triangle for the light-pdf sum (pdf/emission.wesl:120-179):
// v0, e1, e2, the normalised light normal and max(weight / area, 1e-3).
struct alignas(16) DevLightTri {
  float v0[3];
  float area_pdf;
  float e1[3];
  float _p1;
  float e2[3];
  float _p2;
  float n[3];
  float _p3;
};
static_assert(sizeof(DevLightTri) == 64, "DevLightTri is 64 bytes");

// Mirror of cg_emissive_prim / EmissivePrim (80 B).
struct alignas(16) DevEmissivePrim {
  float v0[3], _p0;
  float v1[3], _p1;
  float v2[3], _p2;
  float emission[3];
  float area;
  float weight;
  float _pad[3];
};
static_assert(sizeof(DevEmissivePrim) == 80, "DevEmissivePrim is 80 bytes");

struct DevAlias {
  uint32_t alias;
  float prob;
};

// Device pointers of an uploaded scene (passed to kernels by value).
struct SceneView {
  const BvhNode* tlas;         // TLAS nodes (root 0); leaves hold instances
  const BvhNode* blas;         // all BLAS nodes
  const Bvh4Node* tlas4;       // the same trees, four-wide (root 0)
  const Bvh4Node* blas4;
  const Bvh4QNode* tlas4q;     // the four-wide trees with 8-bit child boxes
  const Bvh4QNode* blas4q;
  const float4* tris;          // 3 float4 per triangle: (v0, orig id bits) (e1) (e2)
  const uint4* tri_vidx;       // vertex indices per triangle (i0, i1, i2, _)
  const float4* vnormal;       // vertex normals
  const DevInstance* inst;
  const DevMaterial* mat;
  const DevEmissivePrim* eprim;
  const DevAlias* alias;
  const BvhNode* light_bvh;    // over DevLightTri
  const DevLightTri* light_tri;
  const float4* env;           // env_w * env_h texels
  const DevMatTex* mattex;     // per material (textured materials only read it)
  const uchar4* tex;           // tex_layers x tex_h x tex_w RGBA8 texels
  const float4* vuv;           // per vertex: TEXCOORD_0.xy, TEXCOORD_1.xy (textured scenes)
  uint32_t tex_w, tex_h, tex_layers, _tex_pad;
  uint32_t env_w, env_h;
  uint32_t emissive_count;
  uint32_t instance_count;
  uint32_t has_tlas;
  uint32_t has_lights;
};

}  // namespace cg

#endif
