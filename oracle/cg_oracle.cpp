/*
 * cg_oracle.cpp — CPU oracle for the View() path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see cg_oracle.h).  A restatement of
 * ray847/CrystalGraphics' host scene packing (src/pathtracing/ headers) and WGSL
 * estimator (src/wgpu/shader/compute.wesl and the compute/ modules), compiled with
 * -ffp-contract=off.  Citations are file:line in the reference project.
 */
#include "cg_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <chrono>
#include <thread>
#include <vector>

#include "cg_oracle_math.h"
#include "cg_oracle_spectral.h"

namespace oracle {
namespace {

// ---------------------------------------------------------------------------
// Scene containers (src/scene_impl.h:24-93, src/pathtracing/*.h)
// ---------------------------------------------------------------------------
struct BLASNode {        // blas.h:15-28
  V3 lb, ub;
  uint32_t child = 0, triangle_count = 0;
};
struct TLASNode {        // tlas.h:17-30
  V3 lb{std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
        std::numeric_limits<float>::max()};
  V3 ub{std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
        std::numeric_limits<float>::lowest()};
  uint32_t child = 0, instance_idx = 0;
};
struct Instance {        // instance.h:9-17; inv is row-major 3x4 (world -> local)
  float inv[12];
  float fwd[12];
  uint32_t blas_root_idx, material_idx;
};
struct AABB {            // aabb.h:14-54 (ub defaults to numeric_limits<float>::min())
  V3 lb{std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
        std::numeric_limits<float>::max()};
  V3 ub{std::numeric_limits<float>::min(), std::numeric_limits<float>::min(),
        std::numeric_limits<float>::min()};
  void merge(V3 v) {
    lb = vmin(lb, v);
    ub = vmax(ub, v);
  }
  V3 center() const { return (lb + ub) * 0.5f; }
  V3 range() const { return ub - lb; }
};
inline float axis(V3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct Material {        // the fields shading/material.wesl:19-53 reads
  V3 base_color;
  V3 emissive;
  float emissive_strength, metallic, roughness, ior, dispersion, transmission, thickness;
  // MaterialTextureInfo index (-1 none) and tex_coord of the four textures
  // decode samples: base color, metallic-roughness, emissive, transmission
  int32_t tex[4];
  uint32_t tex_coord[4];
};

}  // namespace
}  // namespace oracle

struct oracle_scene_s {
  // the material texture array (WriteMaterialTextures, src/wgpu/resource.cpp:
  // 471-546): RGBA8 texels, every texture resized to the largest width/height
  std::vector<uint8_t> tex;
  uint32_t tex_w = 1, tex_h = 1;
  std::vector<cg_texture> tex_desc;             // the decoded images as given
  std::vector<std::vector<uint8_t>> tex_data;   // copies of their texels
  std::vector<cg_vertex> vertices;
  std::vector<uint32_t> indices;
  std::vector<cg_mesh> meshes;
  std::vector<cg_instance> inst_desc;
  std::vector<oracle::Material> materials;
  // BLAS, one tree per mesh (the reference builds one per instance with the
  // same algorithm; identical meshes give identical trees).
  std::vector<oracle::BLASNode> bnodes;
  std::vector<std::array<uint32_t, 3>> bindex;   // Index (blas.h:30-32)
  std::vector<uint32_t> borig;                     // original triangle index
  std::vector<uint32_t> mesh_root;
  std::vector<oracle::TLASNode> tnodes;
  std::vector<oracle::Instance> insts;
  std::vector<cg_emissive_prim> eprims;
  std::vector<cg_alias_entry> alias;
  float total_weight = 0.0f;
  uint32_t env_w = 0, env_h = 0;
  std::vector<float> env;
  // single-threaded seconds of each host packing stage of the create call:
  // BLAS builds, TLAS build, emissive buffer, alias table
  double pack_s[4] = {0, 0, 0, 0};
};

namespace oracle {
namespace {

// ---- transforms ---------------------------------------------------------------
// world_from_local is row-major 3x4.  The inverse is computed in double and
// rounded to float (the reference uses glm::inverse, tlas.h:62; CrystalSpatial
// and glm are absent, so this convention is the backend's and is shared by
// the oracle and the library).
void invertAffine(const float* m, float* out) {
  double a[3][3], t[3];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) a[i][j] = m[i * 4 + j];
    t[i] = m[i * 4 + 3];
  }
  double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
  double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
  double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
  double inv[3][3];
  inv[0][0] = c00 / det;
  inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
  inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
  inv[1][0] = c01 / det;
  inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
  inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
  inv[2][0] = c02 / det;
  inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
  inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
  for (int i = 0; i < 3; ++i) {
    double ti = -(inv[i][0] * t[0] + inv[i][1] * t[1] + inv[i][2] * t[2]);
    for (int j = 0; j < 3; ++j) out[i * 4 + j] = static_cast<float>(inv[i][j]);
    out[i * 4 + 3] = static_cast<float>(ti);
  }
}
// glm mat4 * vec4(p, 1) (glm type_mat4x4.inl): (m0 x + m1 y) + (m2 z + m3 w).
V3 transformPoint(const float* m, V3 p) {
  V3 r;
  float* rr = &r.x;
  for (int i = 0; i < 3; ++i) {
    float add0 = m[i * 4 + 0] * p.x + m[i * 4 + 1] * p.y;
    float add1 = m[i * 4 + 2] * p.z + m[i * 4 + 3] * 1.0f;
    rr[i] = add0 + add1;
  }
  return r;
}
// The traversal's ray -> local transform (bvh.wesl:84-88), order fixed as
// ((m0 x + m1 y) + m2 z) + m3 w; the CUDA kernels use the same order.
V3 localPoint(const float* m, V3 p) {
  return {((m[0] * p.x + m[1] * p.y) + m[2] * p.z) + m[3],
          ((m[4] * p.x + m[5] * p.y) + m[6] * p.z) + m[7],
          ((m[8] * p.x + m[9] * p.y) + m[10] * p.z) + m[11]};
}
V3 localDir(const float* m, V3 d) {
  return {(m[0] * d.x + m[1] * d.y) + m[2] * d.z, (m[4] * d.x + m[5] * d.y) + m[6] * d.z,
          (m[8] * d.x + m[9] * d.y) + m[10] * d.z};
}
// transpose(inv_trans) * vec4(n, 0) (bvh.wesl:110-111).
V3 normalToWorld(const float* m, V3 n) {
  return {(m[0] * n.x + m[4] * n.y) + m[8] * n.z, (m[1] * n.x + m[5] * n.y) + m[9] * n.z,
          (m[2] * n.x + m[6] * n.y) + m[10] * n.z};
}

inline V3 pos(const cg_vertex& v) { return {v.position[0], v.position[1], v.position[2]}; }
inline V3 nrm(const cg_vertex& v) { return {v.normal[0], v.normal[1], v.normal[2]}; }

// ---- BLAS (src/pathtracing/blas.h:36-194) -------------------------------------
struct TriangleInfo {
  V3 center;
  uint32_t index;
};

void blasBuildTree(oracle_scene_s& s, uint32_t node_idx, uint32_t l, uint32_t r,
                   std::vector<TriangleInfo>& info, const cg_mesh& mesh, uint32_t tri_offset) {
  BLASNode& node = s.bnodes[node_idx];
  node.lb = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
             std::numeric_limits<float>::max()};
  node.ub = {std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
             std::numeric_limits<float>::lowest()};
  for (uint32_t i = l; i < r; ++i) {
    uint32_t o = mesh.index_offset + info[i].index * 3;
    V3 v0 = pos(s.vertices[s.indices[o]]), v1 = pos(s.vertices[s.indices[o + 1]]),
       v2 = pos(s.vertices[s.indices[o + 2]]);
    node.lb = vmin(node.lb, vmin(vmin(v0, v1), v2));
    node.ub = vmax(node.ub, vmax(vmax(v0, v1), v2));
  }
  V3 pad{0.001f, 0.001f, 0.001f};
  node.lb = node.lb - pad;
  node.ub = node.ub + pad;
  uint32_t count = r - l;
  if (count <= 2) {
    node.child = tri_offset + l;
    node.triangle_count = count;
    return;
  }
  AABB cb;
  cb.lb = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
           std::numeric_limits<float>::max()};
  cb.ub = {std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
           std::numeric_limits<float>::lowest()};
  for (uint32_t i = l; i < r; ++i) cb.merge(info[i].center);
  V3 range = cb.range();
  int split = 0;
  if (range.y > range.x) split = 1;
  if (range.z > axis(range, split)) split = 2;
  uint32_t mid = l + (r - l) / 2;
  std::nth_element(info.begin() + l, info.begin() + mid, info.begin() + r,
                   [=](const TriangleInfo& a, const TriangleInfo& b) {
                     return axis(a.center, split) < axis(b.center, split);
                   });
  s.bnodes[node_idx].child = static_cast<uint32_t>(s.bnodes.size());
  s.bnodes[node_idx].triangle_count = 0;
  uint32_t left = s.bnodes[node_idx].child;
  s.bnodes.emplace_back();
  s.bnodes.emplace_back();
  blasBuildTree(s, left, l, mid, info, mesh, tri_offset);
  blasBuildTree(s, left + 1, mid, r, info, mesh, tri_offset);
}

void blasBuildMesh(oracle_scene_s& s, const cg_mesh& mesh) {
  uint32_t tri_count = mesh.index_count / 3;
  std::vector<TriangleInfo> info(tri_count);
  for (uint32_t t = 0; t < tri_count; ++t) {
    uint32_t o = mesh.index_offset + t * 3;
    V3 v0 = pos(s.vertices[s.indices[o]]), v1 = pos(s.vertices[s.indices[o + 1]]),
       v2 = pos(s.vertices[s.indices[o + 2]]);
    info[t] = TriangleInfo{(v0 + v1 + v2) / 3.0f, t};
  }
  s.mesh_root.push_back(static_cast<uint32_t>(s.bnodes.size()));
  s.bnodes.emplace_back();
  uint32_t tri_offset = static_cast<uint32_t>(s.bindex.size());
  blasBuildTree(s, static_cast<uint32_t>(s.bnodes.size() - 1), 0, tri_count, info, mesh,
                tri_offset);
  for (const auto& ti : info) {
    uint32_t o = mesh.index_offset + ti.index * 3;
    s.bindex.push_back({s.indices[o], s.indices[o + 1], s.indices[o + 2]});
    s.borig.push_back(ti.index);
  }
}

// ---- TLAS (src/pathtracing/tlas.h:34-140) ---------------------------------------
struct BoundedPrimitive {
  AABB aabb;
  V3 center;
  uint32_t prim_idx;
};

void tlasBuild(oracle_scene_s& s, uint32_t node_idx, uint32_t l, uint32_t r,
               std::vector<BoundedPrimitive>& bm) {
  TLASNode& node = s.tnodes[node_idx];
  for (uint32_t i = l; i < r; ++i) {
    node.lb = vmin(node.lb, bm[i].aabb.lb);
    node.ub = vmax(node.ub, bm[i].aabb.ub);
  }
  V3 pad{0.001f, 0.001f, 0.001f};
  node.lb = node.lb - pad;
  node.ub = node.ub + pad;
  uint32_t count = r - l;
  if (count <= 1) {
    node.instance_idx = bm[l].prim_idx;
    node.child = 0;
    return;
  }
  AABB cb;  // default AABB: ub starts at numeric_limits<float>::min() (aabb.h:17-21)
  for (uint32_t i = l; i < r; ++i) cb.merge(bm[i].center);
  V3 range = cb.range();
  int split = 0;
  if (range.y > range.x) split = 1;
  if (range.z > axis(range, split)) split = 2;
  uint32_t mid = l + (r - l) / 2;
  std::nth_element(bm.begin() + l, bm.begin() + mid, bm.begin() + r,
                   [=](const BoundedPrimitive& x, const BoundedPrimitive& y) {
                     return axis(x.center, split) < axis(y.center, split);
                   });
  s.tnodes[node_idx].child = static_cast<uint32_t>(s.tnodes.size());
  s.tnodes[node_idx].instance_idx = 0;
  uint32_t lc = s.tnodes[node_idx].child;
  s.tnodes.emplace_back();
  s.tnodes.emplace_back();
  tlasBuild(s, lc, l, mid, bm);
  tlasBuild(s, lc + 1, mid, r, bm);
}

// trans_aabb (tlas.h:38-55): matrix[j][i] is row i, column j of world_from_local.
AABB transAabb(const AABB& a, const float* m) {
  V3 lb{m[3], m[7], m[11]};
  V3 ub = lb;
  float* plb = &lb.x;
  float* pub = &ub.x;
  const float* alb = &a.lb.x;
  const float* aub = &a.ub.x;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      float x = m[i * 4 + j] * alb[j];
      float y = m[i * 4 + j] * aub[j];
      if (x < y) {
        plb[i] += x;
        pub[i] += y;
      } else {
        plb[i] += y;
        pub[i] += x;
      }
    }
  }
  AABB out;
  out.lb = lb;
  out.ub = ub;
  return out;
}

// ---- emissive buffer (src/pathtracing/emissive_buffer.h:44-100) ------------------
float luminanceRgb(V3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }

// WrapCoord (emissive_buffer.h:191-204)
float wrapCoord(float coord, int32_t wrap) {
  if (wrap == 33071) return std::clamp(coord, 0.0f, 0.999999f);
  if (wrap == 33648) {
    float wrapped = coord - std::floor(coord);
    const auto tile = static_cast<int32_t>(std::floor(coord));
    if (tile % 2 != 0) wrapped = 1.0f - wrapped;
    return std::clamp(wrapped, 0.0f, 0.999999f);
  }
  float wrapped = coord - std::floor(coord);
  return std::clamp(wrapped, 0.0f, 0.999999f);
}

// EmissiveTextureFactor / TriangleUv / SampleTexture (emissive_buffer.h:138-189):
// nearest texel of the original image at the triangle's mean UV.
V3 emissiveTextureFactor(const oracle_scene_s& s, const Material& m, const cg_vertex& v0,
                         const cg_vertex& v1, const cg_vertex& v2) {
  if (m.tex[2] < 0) return V3{1.0f, 1.0f, 1.0f};
  const size_t idx = static_cast<size_t>(m.tex[2]);
  if (idx >= s.tex_desc.size()) return V3{1.0f, 1.0f, 1.0f};
  const cg_texture& t = s.tex_desc[idx];
  const bool one = m.tex_coord[2] == 1u;
  const float* a = one ? v0.tex_coord1 : v0.tex_coord0;
  const float* b = one ? v1.tex_coord1 : v1.tex_coord0;
  const float* c = one ? v2.tex_coord1 : v2.tex_coord0;
  float u = ((a[0] + b[0]) + c[0]) / 3.0f, v = ((a[1] + b[1]) + c[1]) / 3.0f;
  u = wrapCoord(u, t.wrap_s);
  v = wrapCoord(v, t.wrap_t);
  const uint32_t x = std::min(t.width - 1, static_cast<uint32_t>(u * static_cast<float>(t.width)));
  const uint32_t y = std::min(t.height - 1, static_cast<uint32_t>(v * static_cast<float>(t.height)));
  const uint8_t* px = s.tex_data[idx].data() + (size_t(y) * t.width + x) * 4;
  return V3{static_cast<float>(px[0]) / 255.0f, static_cast<float>(px[1]) / 255.0f,
            static_cast<float>(px[2]) / 255.0f};
}

void buildEmissive(oracle_scene_s& s) {
  for (size_t p = 0; p < s.inst_desc.size(); ++p) {
    const cg_instance& inst = s.inst_desc[p];
    if (inst.material >= s.materials.size()) continue;
    const Material& m = s.materials[inst.material];
    V3 base = vmax(m.emissive * m.emissive_strength, V3{0.0f, 0.0f, 0.0f});
    if (luminanceRgb(base) <= 0.0f) continue;
    const cg_mesh& mesh = s.meshes[inst.mesh];
    for (uint32_t i = 0; i + 2 < mesh.index_count; i += 3) {
      uint32_t o = mesh.index_offset + i;
      V3 p0 = transformPoint(inst.world_from_local, pos(s.vertices[s.indices[o]]));
      V3 p1 = transformPoint(inst.world_from_local, pos(s.vertices[s.indices[o + 1]]));
      V3 p2 = transformPoint(inst.world_from_local, pos(s.vertices[s.indices[o + 2]]));
      // glm::length(cross) * 0.5 with glm::dot = (x + y) + z.
      V3 c = cross(p1 - p0, p2 - p0);
      float area = std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z) * 0.5f;
      if (area <= 0.0f) continue;
      const cg_vertex& va = s.vertices[s.indices[o]];
      const cg_vertex& vb = s.vertices[s.indices[o + 1]];
      const cg_vertex& vc = s.vertices[s.indices[o + 2]];
      V3 f = emissiveTextureFactor(s, m, va, vb, vc);
      V3 emission = V3{base.x * f.x, base.y * f.y, base.z * f.z};
      float w = luminanceRgb(emission);
      if (w <= 0.0f) continue;
      cg_emissive_prim e;
      std::memset(&e, 0, sizeof(e));
      e.v0[0] = p0.x; e.v0[1] = p0.y; e.v0[2] = p0.z;
      e.v1[0] = p1.x; e.v1[1] = p1.y; e.v1[2] = p1.z;
      e.v2[0] = p2.x; e.v2[1] = p2.y; e.v2[2] = p2.z;
      e.emission[0] = emission.x; e.emission[1] = emission.y; e.emission[2] = emission.z;
      e.area = area;
      e.weight = area * w;
      s.eprims.push_back(e);
      s.total_weight += e.weight;
    }
  }
  if (s.total_weight > 0.0f)
    for (auto& e : s.eprims) e.weight /= s.total_weight;
}

// ---- alias table (src/pathtracing/alias_table.h:24-70) ---------------------------
void aliasBuild(const double* weights, uint32_t count, cg_alias_entry* entries) {
  for (uint32_t i = 0; i < count; ++i) entries[i] = cg_alias_entry{0u, 0.0f};
  if (count == 0) return;
  std::vector<double> p(count);
  for (uint32_t i = 0; i < count; ++i) p[i] = std::max(0.0, weights[i]);
  double total = 0.0;
  for (uint32_t i = 0; i < count; ++i) total += p[i];
  if (total <= 0.0) return;
  std::vector<uint32_t> large, small;
  for (uint32_t i = 0; i < count; ++i) {
    p[i] = p[i] / total * count;
    if (p[i] >= 1.0)
      large.push_back(i);
    else
      small.push_back(i);
  }
  while (!large.empty() && !small.empty()) {
    uint32_t i = small.back(), j = large.back();
    small.pop_back();
    large.pop_back();
    entries[i].prob = static_cast<float>(p[i]);
    entries[i].alias = j;
    p[j] -= 1.0 - static_cast<double>(entries[i].prob);
    if (p[j] < 1.0)
      small.push_back(j);
    else
      large.push_back(j);
  }
  while (!large.empty()) {
    uint32_t i = large.back();
    large.pop_back();
    entries[i].prob = 1.0f;
    entries[i].alias = i;
  }
  while (!small.empty()) {
    uint32_t i = small.back();
    small.pop_back();
    entries[i].prob = 1.0f;
    entries[i].alias = i;
  }
}

// ---------------------------------------------------------------------------
// Traversal (structural/bvh.wesl:52-221, math/geometric.wesl:5-26)
// ---------------------------------------------------------------------------
struct Ray {
  V3 pos, dir;
};

inline V3 dirInv(V3 d) {
  V3 s{d.x == 0.0f ? 1e-7f : d.x, d.y == 0.0f ? 1e-7f : d.y, d.z == 0.0f ? 1e-7f : d.z};
  return V3{1.0f / s.x, 1.0f / s.y, 1.0f / s.z};
}
// rayIntersectAABB (geometric.wesl:13-26); tmax_limit only in prune mode.
inline bool rayIntersectAABB(const Ray& ray, V3 lb, V3 ub, float tmax_limit) {
  V3 inv = dirInv(ray.dir);
  V3 t0 = (lb - ray.pos) * inv;
  V3 t1 = (ub - ray.pos) * inv;
  V3 tmin = vmin(t0, t1), tmax = vmax(t0, t1);
  float tn = wmax(wmax(tmin.x, tmin.y), tmin.z);
  float tf = wmin(wmin(tmax.x, tmax.y), tmax.z);
  return tf >= tn && tf > 0.0f && tn <= tmax_limit;
}
struct TriHit {
  float t, u, v;
};
// rayIntersectTriangle (bvh.wesl:188-221).
inline TriHit rayIntersectTriangle(const Ray& ray, V3 v0, V3 v1, V3 v2) {
  const float EPS = 1e-6f;
  V3 e1 = v1 - v0, e2 = v2 - v0;
  V3 h = cross(ray.dir, e2);
  float a = dot(e1, h);
  if (a > -EPS && a < EPS) return {-1.0f, 0.0f, 0.0f};
  float f = 1.0f / a;
  V3 s = ray.pos - v0;
  float u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return {-1.0f, 0.0f, 0.0f};
  V3 q = cross(s, e1);
  float v = f * dot(ray.dir, q);
  if (v < 0.0f || u + v > 1.0f) return {-1.0f, 0.0f, 0.0f};
  float t = f * dot(e2, q);
  if (t > EPS) return {t, u, v};
  return {-1.0f, 0.0f, 0.0f};
}

struct Counters {
  uint64_t extend = 0, shadow = 0, nodes = 0, tris = 0, nonfinite = 0;
};

struct ClosestHit {
  bool hit = false;
  float t = MAXD, u = 0.0f, v = 0.0f;
  int32_t instance = -1, triangle = -1;
  uint32_t tri_slot = 0;  // index into bindex
  float t2 = MAXD;        // second-best distinct hit (tie detection)
};

// rayTraverseBlas (bvh.wesl:131-186).  best_t: the global best in prune mode.
void traverseBlas(const oracle_scene_s& s, const Ray& ray, uint32_t root, float& closest_t,
                  float& cu, float& cv, uint32_t& slot, float& t2, bool prune,
                  Counters& cnt) {
  uint32_t stack[64];
  int top = 0;
  stack[0] = root;
  while (top >= 0) {
    uint32_t ni = stack[top--];
    const BLASNode& node = s.bnodes[ni];
    ++cnt.nodes;
    if (rayIntersectAABB(ray, node.lb, node.ub, prune ? closest_t : INFINITY)) {
      if (node.triangle_count == 0u) {
        stack[++top] = node.child;
        stack[++top] = node.child + 1u;
      } else {
        for (uint32_t i = 0; i < node.triangle_count; ++i) {
          uint32_t ts = node.child + i;
          const auto& idx = s.bindex[ts];
          ++cnt.tris;
          TriHit h = rayIntersectTriangle(ray, pos(s.vertices[idx[0]]), pos(s.vertices[idx[1]]),
                                          pos(s.vertices[idx[2]]));
          if (h.t > 0.0f && h.t < closest_t) {
            t2 = closest_t;
            closest_t = h.t;
            cu = h.u;
            cv = h.v;
            slot = ts;
          } else if (h.t > 0.0f && h.t < t2) {
            t2 = h.t;
          }
        }
      }
    }
  }
}

// rayTraverseTlas (bvh.wesl:52-130): closest hit over all instances.
ClosestHit traverse(const oracle_scene_s& s, const Ray& ray, bool prune, Counters& cnt) {
  ClosestHit best;
  if (s.tnodes.empty()) return best;
  uint32_t stack[64];
  int top = 0;
  stack[0] = 0;
  float dis = MAXD;
  while (top >= 0) {
    uint32_t ni = stack[top--];
    const TLASNode& node = s.tnodes[ni];
    if (rayIntersectAABB(ray, node.lb, node.ub, prune ? dis : INFINITY)) {
      if (node.child != 0u) {
        stack[++top] = node.child;
        stack[++top] = node.child + 1u;
      } else {
        const Instance& inst = s.insts[node.instance_idx];
        Ray local{localPoint(inst.inv, ray.pos), localDir(inst.inv, ray.dir)};
        float ct = prune ? dis : MAXD, cu = 0.0f, cv = 0.0f, t2 = MAXD;
        uint32_t slot = 0xffffffffu;
        traverseBlas(s, local, inst.blas_root_idx, ct, cu, cv, slot, t2, prune, cnt);
        // second-best tracking across instances
        if (slot != 0xffffffffu && ct < dis) {
          best.t2 = std::min(std::min(best.t2, dis), t2);
          dis = ct;
          best.hit = true;
          best.t = ct;
          best.u = cu;
          best.v = cv;
          best.instance = static_cast<int32_t>(node.instance_idx);
          best.tri_slot = slot;
          best.triangle = static_cast<int32_t>(s.borig[slot]);
        } else {
          if (slot != 0xffffffffu) best.t2 = std::min(best.t2, ct);
          best.t2 = std::min(best.t2, t2);
        }
      }
    }
  }
  if (dis >= MAXD) best = ClosestHit{};
  return best;
}

// ---------------------------------------------------------------------------
// Shading (structural/types.wesl, shading/**)
// ---------------------------------------------------------------------------
struct SurfacePos {     // structural/types.wesl:8-14
  V3 pos, shading_norm, geometry_norm;
  uint32_t material_idx;
  float uv[2][2];        // TEXCOORD_0, TEXCOORD_1 at the hit
};
struct HitInfo {
  bool hit;
  float dist;
  SurfacePos sp;
};

// rayHit: closest hit plus the surface frame (bvh.wesl:102-129, 167-179).
HitInfo rayHit(const oracle_scene_s& s, const Ray& ray, bool prune, Counters& cnt) {
  ClosestHit h = traverse(s, ray, prune, cnt);
  HitInfo out{};
  if (!h.hit) {
    out.hit = false;
    out.dist = MAXD;
    return out;
  }
  const auto& idx = s.bindex[h.tri_slot];
  const cg_vertex &a = s.vertices[idx[0]], &b = s.vertices[idx[1]], &c = s.vertices[idx[2]];
  float w0 = 1.0f - h.u - h.v;
  V3 ln = normalize(w0 * nrm(a) + h.u * nrm(b) + h.v * nrm(c));
  V3 lgn = normalize(cross(pos(b) - pos(a), pos(c) - pos(a)));
  const Instance& inst = s.insts[h.instance];
  V3 wgn = normalize(normalToWorld(inst.inv, lgn));
  V3 wsn = normalize(normalToWorld(inst.inv, ln));
  out.hit = true;
  out.dist = h.t;
  out.sp.pos = ray.pos + h.t * ray.dir;
  out.sp.shading_norm = dot(wsn, wgn) >= 0.0f ? wsn : -wsn;
  out.sp.geometry_norm = wgn;
  out.sp.material_idx = inst.material_idx;
  // uv0 = w0 * uv00 + u * uv01 + v * uv02, likewise uv1 (bvh.wesl:172-179)
  for (int k = 0; k < 2; ++k) {
    out.sp.uv[0][k] = (w0 * a.tex_coord0[k] + h.u * b.tex_coord0[k]) + h.v * c.tex_coord0[k];
    out.sp.uv[1][k] = (w0 * a.tex_coord1[k] + h.u * b.tex_coord1[k]) + h.v * c.tex_coord1[k];
  }
  return out;
}

struct IOR {
  float re, im;
};
struct MatEval {         // Material (material.wesl:60-67)
  float diffuse_reflectance, microfacet_roughness;
  IOR ior;
  float transmission;
  bool volumn_transmission;
  float emission;
};

// textureSampleLevel(material_textures, sampler, uv, layer, 0.0) with linear
// filtering and clamp to edge (src/wgpu/resource.cpp:133-142) on the RGBA8Unorm
// array: texel centres at (i + 0.5) / size, bilinear weights in float.  x and
// y are clamped to [-1, size] first (every tap beyond is the edge texel).  The
// GPU's texture units quantise the weights (to 1/256 on NVIDIA hardware); this
// backend and its kernels use float weights (a documented deviation).
struct Texel {
  float r, g, b, a;
};
Texel sampleTexture(const oracle_scene_s& s, int32_t layer, float u, float v) {
  const float W = static_cast<float>(s.tex_w), H = static_cast<float>(s.tex_h);
  const float x = std::fmin(std::fmax(u * W - 0.5f, -1.0f), W);
  const float y = std::fmin(std::fmax(v * H - 0.5f, -1.0f), H);
  const float fx = std::floor(x), fy = std::floor(y);
  const float ax = x - fx, ay = y - fy;
  const int wmax = static_cast<int>(s.tex_w) - 1, hmax = static_cast<int>(s.tex_h) - 1;
  const int x0 = std::clamp(static_cast<int>(fx), 0, wmax), x1 = std::clamp(static_cast<int>(fx) + 1, 0, wmax);
  const int y0 = std::clamp(static_cast<int>(fy), 0, hmax), y1 = std::clamp(static_cast<int>(fy) + 1, 0, hmax);
  const uint8_t* L = s.tex.data() + size_t(layer) * s.tex_w * s.tex_h * 4;
  auto at = [&](int x, int y, int c) {
    return static_cast<float>(L[(size_t(y) * s.tex_w + x) * 4 + c]) / 255.0f;
  };
  const float bx = 1.0f - ax, by = 1.0f - ay;
  float out[4];
  for (int c = 0; c < 4; ++c) {
    const float top = at(x0, y0, c) * bx + at(x1, y0, c) * ax;
    const float bot = at(x0, y1, c) * bx + at(x1, y1, c) * ax;
    out[c] = top * by + bot * ay;
  }
  return Texel{out[0], out[1], out[2], out[3]};
}

// decode (material.wesl:19-53) with the texture getters (material.wesl:181-262).
MatEval decode(const oracle_scene_s& s, const Material& m, const float (&uv)[2][2], float w) {
  auto texel = [&](int k) {
    const uint32_t set = m.tex_coord[k] == 1u ? 1u : 0u;  // textureUv
    return sampleTexture(s, m.tex[k], uv[set][0], uv[set][1]);
  };
  V3 base = m.base_color;
  if (m.tex[0] >= 0) {
    const Texel t = texel(0);
    base = V3{base.x * t.r, base.y * t.g, base.z * t.b};
  }
  float reflectance = rgbToWavelengthReflectance(base, w);
  float roughness_f = m.roughness, metallic_f = m.metallic, transmission_f = m.transmission;
  if (m.tex[1] >= 0) {
    const Texel t = texel(1);
    roughness_f = roughness_f * t.g;
    metallic_f = metallic_f * t.b;
  }
  if (m.tex[3] >= 0) transmission_f = transmission_f * texel(3).r;
  float roughness = wclamp(roughness_f, 0.0f, 1.0f);
  float metallic = wclamp(metallic_f, 0.0f, 1.0f);
  float transmission = wclamp(transmission_f, 0.0f, 1.0f);
  float raw_ior = m.ior;
  float real_ior = raw_ior;
  if (metallic == 0.0f && transmission > 0.0f) {
    // dispersedIor (material.wesl:80-97)
    if (!(m.dispersion <= 0.0f)) {
      float inv_abbe = m.dispersion / 20.0f;
      real_ior = wmax(raw_ior + (raw_ior - 1.0f) * inv_abbe * (523655.0f / (w * w) - 1.5168f), 1.0f);
    }
  }
  // imaginaryIorFromReflectance (material.wesl:99-110)
  float im = std::sqrt(wclamp((4.0f * real_ior) / (1.0f - reflectance) -
                                  std::pow(real_ior + 1.0f, 2.0f),
                              0.0f, 10.0f));
  V3 strength = m.emissive;
  if (m.tex[2] >= 0) {
    const Texel t = texel(2);
    strength = V3{strength.x * t.r, strength.y * t.g, strength.z * t.b};
  }
  V3 raw_emission = vmax(strength * m.emissive_strength, V3{0.0f, 0.0f, 0.0f});
  MatEval e;
  e.diffuse_reflectance = (1.0f - metallic) * (1.0f - transmission) * reflectance;
  e.microfacet_roughness = roughness * roughness;
  e.ior = IOR{real_ior, metallic * im};
  e.transmission = transmission;
  e.volumn_transmission = m.thickness > 0.0f;
  e.emission = rgbToWavelengthReflectance(raw_emission, w);
  return e;
}

// shading/util.wesl:4-81
inline V3 orientedNormal(V3 curr, V3 n) { return dot(curr, n) > 0.0f ? -n : n; }
inline IOR invIor(IOR i) {
  float ns = i.re * i.re + i.im * i.im;
  return IOR{i.re / ns, -i.im / ns};
}
inline IOR relIor(V3 sn, V3 curr, const MatEval& m) {
  if (dot(sn, curr) < 0.0f) return invIor(m.ior);
  return m.ior;
}
inline float complexFresnelReflectance(float cosine, IOR mi) {
  float re = mi.re, im = mi.im;
  float real_sq = re * re, im_sq = im * im, cos_sq = cosine * cosine;
  float ns = real_sq + im_sq;
  float trc = 2.0f * re * cosine;
  float perp = (ns - trc + cos_sq) / wmax(ns + trc + cos_sq, 1e-6f);
  float par = (ns * cos_sq - trc + 1.0f) / wmax(ns * cos_sq + trc + 1.0f, 1e-6f);
  return wclamp(0.5f * (perp + par), 0.0f, 1.0f);
}
inline float fresnelReflectance(V3 curr, V3 normal, IOR rel) {
  float ic = wclamp(dot(-curr, normal), 0.0f, 1.0f);
  if (std::fabs(rel.im) > 1e-6f) return complexFresnelReflectance(ic, rel);
  float r = rel.re;
  float tss = r * r * wmax(0.0f, 1.0f - ic * ic);
  if (tss >= 1.0f) return 1.0f;
  float tc = std::sqrt(wmax(0.0f, 1.0f - tss));
  float perp = (r * ic - tc) / (r * ic + tc);
  float par = (ic - r * tc) / (ic + r * tc);
  return wclamp(0.5f * (perp * perp + par * par), 0.0f, 1.0f);
}

// spawn_surface_ray.wesl:4-15
inline Ray spawnSurfaceRay(const SurfacePos& sp, V3 next) {
  V3 on = dot(next, sp.geometry_norm) > 0.0f ? sp.geometry_norm : -sp.geometry_norm;
  return Ray{sp.pos + on * 1e-3f, next};
}

// ---- GGX helpers (pdf/rough_*.wesl, dist/rough_*.wesl) -------------------------
constexpr float VNDF_EPS = 1e-6f;
inline float ggxNormDist(V3 micro, V3 macro, float alpha) {
  float nc = wclamp(dot(micro, macro), 0.0f, 1.0f);
  float nts = wmax(0.0f, 1.0f - nc * nc) / wmax(nc * nc, VNDF_EPS);
  float denom = PI * std::pow(nc, 4.0f) * std::pow(alpha + nts, 2.0f);
  return alpha / wmax(denom, VNDF_EPS);
}
inline float ggxMaskUniDir(float angle, float alpha) {
  return 1.0f / (1.0f + (std::sqrt(1.0f + alpha * std::tan(angle) * std::tan(angle)) - 1.0f) / 2.0f);
}
inline float ggxMaskBiDir(float a1, float a2, float alpha) {
  return 1.0f / (1.0f + (std::sqrt(1.0f + alpha * std::tan(a1) * std::tan(a1)) - 1.0f) / 2.0f +
                 (std::sqrt(1.0f + alpha * std::tan(a2) * std::tan(a2)) - 1.0f) / 2.0f);
}
// sampleNorm (pdf/rough_reflection.wesl:52-103, identical in rough_transmission)
V3 sampleNorm(V3 curr, const SurfacePos& sp, const MatEval& m, Rng& rng) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  M3 ts = makeTangentSpace(macro);
  V3 view = -curr;
  V3 lc = normalize(mulT(ts, view));
  float alpha = m.microfacet_roughness;
  V3 st = normalize(V3{alpha * lc.x, alpha * lc.y, wmax(lc.z, VNDF_EPS)});
  float tl2 = st.x * st.x + st.y * st.y;
  V3 tx = tl2 > VNDF_EPS ? V3{-st.y, st.x, 0.0f} / std::sqrt(wmax(tl2, VNDF_EPS))
                         : V3{1.0f, 0.0f, 0.0f};
  V3 ty = cross(st, tx);
  float radius = std::sqrt(randFloat(rng));
  float angle = 2.0f * PI * randFloat(rng);
  float px = radius * std::cos(angle);
  float py = radius * std::sin(angle);
  float vis = 0.5f * (1.0f + st.z);
  py = mix(std::sqrt(wmax(0.0f, 1.0f - px * px)), py, vis);
  V3 lsm = px * tx + py * ty + std::sqrt(wmax(0.0f, 1.0f - px * px - py * py)) * st;
  V3 lm = normalize(V3{alpha * lsm.x, alpha * lsm.y, wmax(lsm.z, VNDF_EPS)});
  return normalize(mul(ts, lm));
}

// reflectPdf (pdf/rough_reflection.wesl:105-118)
inline float reflectPdf(V3 curr, V3 micro, V3 macro, float alpha) {
  float cmp = wmax(dot(-curr, macro), VNDF_EPS);
  float cmi = wmax(dot(-curr, micro), VNDF_EPS);
  float vnp = ggxNormDist(micro, macro, alpha) * ggxMaskUniDir(std::acos(cmp), alpha) * cmi / cmp;
  return vnp / (4.0f * cmi);
}
inline float relativeIorT(IOR i) { return wmax(i.re, VNDF_EPS); }
inline float transmissionIor(IOR i) { return 1.0f / relativeIorT(i); }
// transmitPdf (pdf/rough_transmission.wesl:129-152)
inline float transmitPdf(V3 curr, V3 micro, V3 macro, V3 next, float tior, float alpha) {
  float cmp = wmax(dot(-curr, macro), VNDF_EPS);
  float cmi = wmax(dot(-curr, micro), VNDF_EPS);
  float vnp = ggxNormDist(micro, macro, alpha) * ggxMaskUniDir(std::acos(cmp), alpha) * cmi / cmp;
  float nmi = dot(next, micro);
  float denom = nmi + cmi / tior;
  return vnp * cmi / wmax(denom * denom, VNDF_EPS);
}

// ---- lobe pdfs (shading/pdf/*.wesl) ----------------------------------------------
inline float diffusePdf(V3 curr, V3 next, const SurfacePos& sp) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  return wmax(dot(next, macro), 0.0f) / PI;
}
inline V3 specularDir(V3 curr, const SurfacePos& sp) {
  return reflect(curr, orientedNormal(curr, sp.shading_norm));
}
inline float specularReflectPdf(V3 curr, V3 next, const SurfacePos& sp) {
  V3 e = specularDir(curr, sp);
  return dot(next - e, next - e) <= 1e-6f ? 1.0f : 0.0f;
}
inline float roughReflectPdf(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  if (dot(next, macro) <= 0.0f) return 0.0f;
  V3 mu = next - curr;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 micro = orientedNormal(curr, normalize(mu));
  return reflectPdf(curr, micro, macro, m.microfacet_roughness);
}
inline V3 refractDir(V3 sn, V3 curr, IOR rel) {
  V3 n = orientedNormal(curr, sn);
  return refract(curr, n, rel.re);
}
inline V3 specularTransmissionDir(V3 curr, const SurfacePos& sp, const MatEval& m) {
  if (m.volumn_transmission) {
    IOR rel = relIor(sp.shading_norm, curr, m);
    return refractDir(sp.shading_norm, curr, rel);
  }
  return curr;
}
inline float specularTransmitPdf(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 e = specularTransmissionDir(curr, sp, m);
  return (dot(e, e) > 1e-6f && dot(next - e, next - e) <= 1e-6f) ? 1.0f : 0.0f;
}
inline float roughTransmitPdf(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  if (dot(next, macro) >= 0.0f) return 0.0f;
  IOR mri = relIor(macro, curr, m);
  float mriv = relativeIorT(mri);
  V3 mu = mriv * curr - next;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 micro = orientedNormal(curr, normalize(mu));
  IOR rel = relIor(micro, curr, m);
  return transmitPdf(curr, micro, macro, next, transmissionIor(rel), m.microfacet_roughness);
}

// ---- BSDF values (shading/dist/*.wesl) ---------------------------------------------
inline float diffuseDist(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  float np = wmax(dot(next, macro), 0.0f);
  return m.diffuse_reflectance * np / PI;
}
inline float specularReflectDist(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  V3 e = reflect(curr, macro);
  float d = dot(next - e, next - e) <= 1e-6f ? 1.0f : 0.0f;
  IOR rel = relIor(sp.shading_norm, curr, m);
  return fresnelReflectance(curr, macro, rel) * d;
}
inline float roughReflectDist(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  float np = wmax(dot(next, macro), 0.0f);
  if (np <= 0.0f) return 0.0f;
  V3 mu = next - curr;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 raw = normalize(mu);
  V3 micro = orientedNormal(curr, raw);
  IOR rel = relIor(raw, curr, m);
  float alpha = m.microfacet_roughness;
  float cmp = wmax(dot(-curr, macro), VNDF_EPS);
  float nmp = wmax(dot(next, macro), VNDF_EPS);
  float rd = ggxNormDist(micro, macro, alpha) * ggxMaskBiDir(std::acos(cmp), std::acos(nmp), alpha) /
             (4.0f * cmp * nmp);
  return fresnelReflectance(curr, micro, rel) * rd * np;
}
inline float specularTransmitDist(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  V3 e = specularTransmissionDir(curr, sp, m);
  float d = dot(next - e, next - e) <= 1e-6f ? 1.0f : 0.0f;
  IOR rel = relIor(sp.shading_norm, curr, m);
  return m.transmission * (1.0f - fresnelReflectance(curr, macro, rel)) * d;
}
inline float roughTransmitDist(V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  V3 macro = orientedNormal(curr, sp.shading_norm);
  if (dot(next, macro) >= 0.0f) return 0.0f;
  float np = wmax(dot(-next, macro), 0.0f);
  IOR mri = relIor(macro, curr, m);
  float mriv = relativeIorT(mri);
  V3 mu = mriv * curr - next;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 raw = normalize(mu);
  V3 micro = orientedNormal(curr, raw);
  IOR rel = relIor(raw, curr, m);
  float tior = transmissionIor(rel);
  float alpha = m.microfacet_roughness;
  // transmitDist (dist/rough_transmission.wesl:236-265)
  float cmp = wmax(dot(-curr, macro), VNDF_EPS);
  float nmp = wmax(dot(-next, macro), VNDF_EPS);
  float cmi = wmax(dot(-curr, micro), VNDF_EPS);
  float nmi = dot(next, micro);
  float denom = nmi + cmi / tior;
  float td = m.transmission * ggxNormDist(micro, macro, alpha) *
             ggxMaskBiDir(std::acos(cmp), std::acos(nmp), alpha) * std::fabs(cmi * nmi) /
             wmax(cmp * nmp * denom * denom, VNDF_EPS);
  return (1.0f - fresnelReflectance(curr, micro, rel)) * td * np;
}

// ---- emission (shading/pdf/emission.wesl) -----------------------------------------
constexpr float EPDF_EPS = 1e-3f;
inline V3 ev(const float* p) { return {p[0], p[1], p[2]}; }

float triangleHitDist(V3 rp, V3 rd, const cg_emissive_prim& prim) {
  V3 v0 = ev(prim.v0), v1 = ev(prim.v1), v2 = ev(prim.v2);
  V3 e1 = v1 - v0, e2 = v2 - v0;
  V3 pv = cross(rd, e2);
  float det = dot(e1, pv);
  if (std::fabs(det) <= EPDF_EPS) return -1.0f;
  float inv_det = 1.0f / det;
  V3 tv = rp - v0;
  float bu = dot(tv, pv) * inv_det;
  if (bu < 0.0f || bu > 1.0f) return -1.0f;
  V3 qv = cross(tv, e1);
  float bv = dot(rd, qv) * inv_det;
  if (bv < 0.0f || bu + bv > 1.0f) return -1.0f;
  float hd = dot(e2, qv) * inv_det;
  return hd > EPDF_EPS ? hd : -1.0f;
}
// dist (pdf/emission.wesl:120-149): sum over every emissive prim the ray meets.
float lightPdf(const oracle_scene_s& s, V3 next, const SurfacePos& sp) {
  if (s.alias.empty()) return 0.0f;
  float pdf = 0.0f;
  V3 rd = normalize(next);
  for (const auto& prim : s.eprims) {
    float hd = triangleHitDist(sp.pos, rd, prim);
    if (hd <= 0.0f) continue;
    V3 v0 = ev(prim.v0), v1 = ev(prim.v1), v2 = ev(prim.v2);
    V3 ln = normalize(cross(v1 - v0, v2 - v0));
    float lp = std::fabs(dot(ln, -rd));
    float area_pdf = wmax(prim.weight / prim.area, EPDF_EPS);
    pdf += area_pdf * hd * hd / wmax(lp, EPDF_EPS);
  }
  return pdf;
}
struct EmissionDraw {
  V3 next;
  float prob, radiance, expected_dist;
  uint32_t prim;  // the emissive primitive drawn
};
// sample (pdf/emission.wesl:32-82) with sampleEmissivePrim (:181-191); a bin
// of u32(1.0 * N) is clamped to N - 1 (WGSL robust access).
EmissionDraw emissionSample(const oracle_scene_s& s, float w, const SurfacePos& sp, Rng& rng) {
  if (s.alias.empty()) return {V3{0, 0, 0}, 0.0f, 0.0f, 0.0f, 0u};
  uint32_t n = static_cast<uint32_t>(s.alias.size());
  uint32_t bin = static_cast<uint32_t>(randFloat(rng) * static_cast<float>(n));
  if (bin >= n) bin = n - 1u;
  float rf = randFloat(rng);
  uint32_t pi = rf < s.alias[bin].prob ? bin : s.alias[bin].alias;
  const cg_emissive_prim& prim = s.eprims[pi];
  float tsx = randFloat(rng);
  float tsy = randFloat(rng);
  float tss = std::sqrt(tsx);
  V3 bary{1.0f - tss, tss * (1.0f - tsy), tss * tsy};
  V3 v0 = ev(prim.v0), v1 = ev(prim.v1), v2 = ev(prim.v2);
  V3 spos = bary.x * v0 + bary.y * v1 + bary.z * v2;
  V3 lo = spos - sp.pos;
  float dsq = wmax(dot(lo, lo), EPDF_EPS);
  V3 next = lo / std::sqrt(dsq);
  V3 ln = normalize(cross(v1 - v0, v2 - v0));
  float lp = std::fabs(dot(ln, -next));
  float area_pdf = wmax(prim.weight / prim.area, EPDF_EPS);
  float sapdf = area_pdf * dsq / wmax(lp, EPDF_EPS);
  return {next, sapdf, rgbToWavelengthRadiance(ev(prim.emission), w), std::sqrt(dsq), pi};
}

// ---- sample counts (shading/sample.wesl:151-299, lod.wesl) -------------------------
struct Conf {
  uint32_t trace_depth, transport_cap, emission_cap, diffuse_cap, rough_cap;
};
struct Counts {
  uint32_t diffuse = 0, specular_reflect = 0, rough_reflect = 0, specular_transmit = 0,
           rough_transmit = 0, light = 0;
};
inline float normalReflectance(const MatEval& m) {
  float lo = m.ior.re - 1.0f, hi = m.ior.re + 1.0f, im2 = m.ior.im * m.ior.im;
  return wclamp((lo * lo + im2) / wmax(hi * hi + im2, 1e-6f), 0.0f, 1.0f);
}
inline uint32_t u32f(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967295.0f) return 0xffffffffu;
  return static_cast<uint32_t>(x);
}
inline uint32_t scaledCount(float h, float scale, uint32_t maxc) {
  if (h <= 1e-6f) return 0u;
  return std::min(std::max(1u, u32f(h * scale)), maxc);
}
Counts counts(const MatEval& m, bool can_sample_light, int depth, const Conf& c) {
  float diffuse_h = m.diffuse_reflectance;
  float refl_h = normalReflectance(m);
  float trans_h = m.transmission;
  float sr = m.microfacet_roughness == 0.0f ? refl_h : 0.0f;
  float rr = m.microfacet_roughness > 0.0f ? refl_h : 0.0f;
  float st = (trans_h > 1e-6f && m.microfacet_roughness == 0.0f) ? trans_h : 0.0f;
  float rt = (trans_h > 1e-6f && m.microfacet_roughness > 0.0f) ? trans_h : 0.0f;
  float light_h = can_sample_light ? 1.0f : 0.0f;
  int32_t maxd = static_cast<int32_t>(c.trace_depth);
  float heur = static_cast<float>(maxd - depth) / static_cast<float>(maxd);
  uint32_t ta = u32f(heur * static_cast<float>(std::min(c.transport_cap, 4u)));
  uint32_t ea = u32f(heur * static_cast<float>(std::min(c.emission_cap, 1u)));
  Counts out;
  float hsum = diffuse_h + sr + rr + st + rt;
  if (!(ta == 0u || hsum <= 1e-6f)) {
    float scale = static_cast<float>(ta) / hsum;
    Counts sc;
    sc.diffuse = scaledCount(diffuse_h, scale, std::min(c.diffuse_cap, 1u));
    sc.specular_reflect = scaledCount(sr, scale, 1u);
    sc.rough_reflect = scaledCount(rr, scale, std::min(c.rough_cap, 1u));
    sc.specular_transmit = scaledCount(st, scale, 1u);
    sc.rough_transmit = scaledCount(rt, scale, std::min(c.rough_cap, 1u));
    uint32_t rem = ta;
    out.diffuse = std::min(sc.diffuse, rem);
    rem -= out.diffuse;
    out.specular_reflect = std::min(sc.specular_reflect, rem);
    rem -= out.specular_reflect;
    out.rough_reflect = std::min(sc.rough_reflect, rem);
    rem -= out.rough_reflect;
    out.specular_transmit = std::min(sc.specular_transmit, rem);
    rem -= out.specular_transmit;
    out.rough_transmit = std::min(sc.rough_transmit, rem);
  }
  out.light = (light_h > 1e-6f && ea > 0u) ? std::max(1u, ea) : 0u;
  return out;
}

enum { M_NONE = 0, M_DIFFUSE = 1, M_SREFL = 2, M_RREFL = 3, M_STRANS = 4, M_RTRANS = 5 };

// balancePdfDenominator (sample.wesl:505-554); every lobe pdf is evaluated.
float balanceDenominator(const oracle_scene_s& s, V3 curr, V3 next, const SurfacePos& sp,
                         const MatEval& m, const Counts& c, int model, float model_pdf,
                         float light_pdf_in) {
  float pd = model == M_DIFFUSE ? model_pdf : diffusePdf(curr, next, sp);
  float psr = model == M_SREFL ? model_pdf : specularReflectPdf(curr, next, sp);
  float prr = model == M_RREFL ? model_pdf : roughReflectPdf(curr, next, sp, m);
  float pst = model == M_STRANS ? model_pdf : specularTransmitPdf(curr, next, sp, m);
  float prt = model == M_RTRANS ? model_pdf : roughTransmitPdf(curr, next, sp, m);
  float pl = light_pdf_in >= 0.0f ? light_pdf_in : lightPdf(s, next, sp);
  return wmax(static_cast<float>(c.diffuse) * pd + static_cast<float>(c.specular_reflect) * psr +
                  static_cast<float>(c.rough_reflect) * prr +
                  static_cast<float>(c.specular_transmit) * pst +
                  static_cast<float>(c.rough_transmit) * prt + static_cast<float>(c.light) * pl,
              1e-6f);
}

struct TransportSample {
  V3 dir;
  float coeff;
  int model;    // the lobe that drew it
  float denom;  // its balance-heuristic denominator
};
struct EmissionSampleOut {
  V3 dir;
  float radiance, expected_dist;
  uint32_t prim;      // the emissive primitive drawn
  float sproj, denom; // |cos| at the surface, balance-heuristic denominator
};
struct Sample {
  uint32_t transport_count = 0, emission_count = 0;
  TransportSample ts[4];
  EmissionSampleOut es[1];
};

// sampleModels (sample.wesl:301-425) with the lobe samplers of pdf/*.wesl.
Sample sampleModels(const oracle_scene_s& s, V3 curr, float w, const SurfacePos& sp,
                    const MatEval& m, const Counts& c, Rng& rng) {
  Sample res;
  auto add = [&](V3 dir, int model, float prob, float dist) {
    float denom = balanceDenominator(s, curr, dir, sp, m, c, model, prob, -1.0f);
    res.ts[res.transport_count++] = TransportSample{dir, dist / denom, model, denom};
  };
  for (uint32_t i = 0; i < c.diffuse; ++i) {  // pdf/diffuse.wesl:7-36
    V3 macro = orientedNormal(curr, sp.shading_norm);
    float r = std::sqrt(randFloat(rng));
    float angle = 2.0f * PI * randFloat(rng);
    V3 local{r * std::cos(angle), r * std::sin(angle), std::sqrt(wmax(0.0f, 1.0f - r * r))};
    V3 next = mul(makeTangentSpace(macro), local);
    add(next, M_DIFFUSE, diffusePdf(curr, next, sp), diffuseDist(curr, next, sp, m));
  }
  for (uint32_t i = 0; i < c.specular_reflect; ++i) {  // pdf/specular_reflection.wesl:7-15
    V3 next = specularDir(curr, sp);
    add(next, M_SREFL, specularReflectPdf(curr, next, sp), specularReflectDist(curr, next, sp, m));
  }
  for (uint32_t i = 0; i < c.rough_reflect; ++i) {  // pdf/rough_reflection.wesl:9-27
    V3 micro = orientedNormal(curr, sampleNorm(curr, sp, m, rng));
    V3 next = reflect(curr, micro);
    V3 macro = orientedNormal(curr, sp.shading_norm);
    float prob = dot(next, macro) <= 0.0f ? 0.0f
                                          : reflectPdf(curr, micro, macro, m.microfacet_roughness);
    add(next, M_RREFL, prob, roughReflectDist(curr, next, sp, m));
  }
  for (uint32_t i = 0; i < c.specular_transmit; ++i) {  // pdf/specular_transmission.wesl:9-27
    V3 next = m.volumn_transmission ? refractDir(sp.shading_norm, curr, relIor(sp.shading_norm, curr, m))
                                    : curr;
    add(next, M_STRANS, specularTransmitPdf(curr, next, sp, m),
        specularTransmitDist(curr, next, sp, m));
  }
  for (uint32_t i = 0; i < c.rough_transmit; ++i) {  // pdf/rough_transmission.wesl:9-32
    V3 macro = orientedNormal(curr, sp.shading_norm);
    V3 micro = orientedNormal(curr, sampleNorm(curr, sp, m, rng));
    IOR rel = relIor(micro, curr, m);
    V3 next = refract(curr, micro, relativeIorT(rel));
    float prob;
    if (dot(next, next) <= VNDF_EPS)
      prob = 0.0f;
    else if (dot(next, macro) >= 0.0f)
      prob = 0.0f;
    else
      prob = roughTransmitPdf(curr, next, sp, m);
    add(next, M_RTRANS, prob, roughTransmitDist(curr, next, sp, m));
  }
  for (uint32_t i = 0; i < c.light; ++i) {  // sample.wesl:407-422, 437-470
    EmissionDraw d = emissionSample(s, w, sp, rng);
    if (d.prob <= 1e-6f) continue;
    float sproj = std::fabs(dot(sp.shading_norm, d.next));
    float ec = diffuseDist(curr, d.next, sp, m) + roughReflectDist(curr, d.next, sp, m) +
               roughTransmitDist(curr, d.next, sp, m);
    float denom = balanceDenominator(s, curr, d.next, sp, m, c, M_NONE, -1.0f, d.prob);
    float rad = d.radiance * ec * sproj / denom;
    res.es[res.emission_count++] =
        EmissionSampleOut{d.next, rad, d.expected_dist, d.prim, sproj, denom};
  }
  return res;
}

// ---- environment (environment.wesl:7-25) -------------------------------------------
float envRadiance(const oracle_scene_s& s, V3 dir, float w) {
  V3 d = normalize(dir);
  float u = std::atan2(d.y, d.x) / (2.0f * PI) + 0.5f;
  float v = std::acos(wclamp(d.z, -1.0f, 1.0f)) / PI;
  float wu = u - std::floor(u);
  float cv = wclamp(1.0f - v, 0.0f, 0.999999f);
  uint32_t x = std::min(s.env_w - 1u, u32f(wu * static_cast<float>(s.env_w)));
  uint32_t y = std::min(s.env_h - 1u, u32f(cv * static_cast<float>(s.env_h)));
  const float* t = &s.env[(static_cast<size_t>(y) * s.env_w + x) * 4];
  return rgbToWavelengthRadiance(V3{t[0], t[1], t[2]}, w);
}

// ---- the estimator (trace.wesl:22-113, shading.wesl:30-53) ---------------------------
struct TraceCtx {
  const oracle_scene_s* s;
  Conf conf;
  bool prune;
  bool keyed;
  Rng* seq;  // reference mode: the pixel stream
  Counters cnt;
  uint32_t roulette = 0;  // Russian roulette from this hit depth on (0 = off, as the reference)
};

// Russian roulette (an option beyond the reference, which has none): a child
// spawned at a hit of depth >= the start survives with q = min(1, its path
// weight t) and then carries t / q; one uniform number decides, from the
// child's roulette stream (keyed) or the pixel stream right before the child
// is traced (reference order).  Returns the factor 1 / q, or 0 if the child
// is dropped.
float roulette(TraceCtx& tc, float t, uint32_t child_key) {
  const float q = wmin(1.0f, t);
  if (!(q < 1.0f)) return 1.0f;
  float u;
  if (tc.keyed) {
    Rng r;
    seedRng(r, rouletteKey(child_key));
    u = randFloat(r);
  } else {
    u = randFloat(*tc.seq);
  }
  return u < q ? 1.0f / q : 0.0f;
}

float trace(TraceCtx& tc, const Ray& ray, float w, int depth, uint32_t key, float thr) {
  const oracle_scene_s& s = *tc.s;
  ++tc.cnt.extend;
  HitInfo hi = rayHit(s, ray, tc.prune, tc.cnt);
  if (!hi.hit) return envRadiance(s, ray.dir, w);
  uint32_t trace_depth = std::max(1u, std::min(tc.conf.trace_depth, 64u));
  if (depth >= static_cast<int>(tc.conf.trace_depth) ||
      static_cast<uint32_t>(depth) >= trace_depth - 1u)
    return 0.0f;
  Rng node_rng;
  Rng* rng = tc.seq;
  if (tc.keyed) {
    seedRng(node_rng, key);
    rng = &node_rng;
  }
  const Material& mat = s.materials[hi.sp.material_idx];
  MatEval m = decode(s, mat, hi.sp.uv, w);
  Counts c = counts(m, !s.alias.empty(), depth, tc.conf);
  Sample smp = sampleModels(s, ray.dir, w, hi.sp, m, c, *rng);
  float emission = m.emission;
  // solveEmission (trace.wesl:91-113)
  for (uint32_t i = 0; i < smp.emission_count; ++i) {
    const auto& es = smp.es[i];
    V3 light_pos = hi.sp.pos + es.dir * es.expected_dist;
    Ray shadow = spawnSurfaceRay(hi.sp, es.dir);
    float expected = distance(shadow.pos, light_pos);
    ++tc.cnt.shadow;
    HitInfo sh = rayHit(s, shadow, tc.prune, tc.cnt);
    if (sh.hit && sh.dist < (expected - 1e-3f)) smp.es[i].radiance = 0.0f;
  }
  float child_l[4] = {0, 0, 0, 0};
  for (uint32_t i = 0; i < smp.transport_count; ++i) {
    const float t = thr * smp.ts[i].coeff;
    const uint32_t ck = tc.keyed ? childKey(key, i) : 0u;
    float rr = 1.0f;
    if (tc.roulette != 0u && static_cast<uint32_t>(depth) >= tc.roulette) {
      if (t == 0.0f) continue;  // adds exactly 0: not traced, no number drawn (as the kernels)
      rr = roulette(tc, t, ck);
      if (rr == 0.0f) continue;
    }
    Ray child = spawnSurfaceRay(hi.sp, smp.ts[i].dir);
    child_l[i] = rr * trace(tc, child, w, depth + 1, ck, t * rr);
  }
  // backwardPass = emission + collect (collect.wesl:4-17)
  float rad = 0.0f;
  for (uint32_t i = 0; i < smp.transport_count; ++i) rad += smp.ts[i].coeff * child_l[i];
  for (uint32_t i = 0; i < smp.emission_count; ++i) rad += smp.es[i].radiance;
  return emission + rad;
}

// ---- hero-wavelength mode -------------------------------------------------------
// The same sample tree, drawn at the hero wavelength w[0] (material, sample
// counts, directions and balance-heuristic denominators), carries the
// radiance of all four wavelengths: a child's coefficient for wavelength j is
// the lobe's value at w[j] over the hero's denominator.  The reference's
// estimator weighs each lobe's sample by that lobe alone over the balance
// denominator (sample.wesl:452-501), so its expected value depends on the
// sample counts and pdfs at the wavelength; where they are the same at all
// four wavelengths, the hero's tree gives each wavelength the reference's
// expectation.  At a hit where they are not (a lobe whose heuristic vanishes
// at some of the four, e.g. a reflectance of 0 in the Smits table's deep-red
// gap, or a transmission whose refraction index varies with the wavelength),
// the light sample and the subtree carry the hero alone with weight 4: over
// the four equally likely heroes of the same wavelength set that is the
// reference's estimator at each of them.  Emission is exact per wavelength.
struct L4 {
  float v[HERO_COUNT];
};

float lobeDist(int model, V3 curr, V3 next, const SurfacePos& sp, const MatEval& m) {
  switch (model) {
    case M_DIFFUSE: return diffuseDist(curr, next, sp, m);
    case M_SREFL: return specularReflectDist(curr, next, sp, m);
    case M_RREFL: return roughReflectDist(curr, next, sp, m);
    case M_STRANS: return specularTransmitDist(curr, next, sp, m);
    case M_RTRANS: return roughTransmitDist(curr, next, sp, m);
  }
  return 0.0f;
}

bool sameCounts(const Counts& a, const Counts& b) {
  return a.diffuse == b.diffuse && a.specular_reflect == b.specular_reflect &&
         a.rough_reflect == b.rough_reflect && a.specular_transmit == b.specular_transmit &&
         a.rough_transmit == b.rough_transmit && a.light == b.light;
}

L4 traceHero(TraceCtx& tc, const Ray& ray, const float (&w)[HERO_COUNT], int depth, uint32_t key,
             bool hero_only, const float (&thr)[HERO_COUNT]) {
  const oracle_scene_s& s = *tc.s;
  L4 out{};
  ++tc.cnt.extend;
  HitInfo hi = rayHit(s, ray, tc.prune, tc.cnt);
  if (!hi.hit) {
    for (int j = 0; j < HERO_COUNT; ++j)
      out.v[j] = (j == 0 || !hero_only) ? envRadiance(s, ray.dir, w[j]) : 0.0f;
    return out;
  }
  uint32_t trace_depth = std::max(1u, std::min(tc.conf.trace_depth, 64u));
  if (depth >= static_cast<int>(tc.conf.trace_depth) ||
      static_cast<uint32_t>(depth) >= trace_depth - 1u)
    return out;
  Rng node_rng;
  Rng* rng = tc.seq;
  if (tc.keyed) {
    seedRng(node_rng, key);
    rng = &node_rng;
  }
  const Material& mat = s.materials[hi.sp.material_idx];
  MatEval m[HERO_COUNT];
  for (int j = 0; j < HERO_COUNT; ++j) m[j] = decode(s, mat, hi.sp.uv, w[j]);
  Counts c = counts(m[0], !s.alias.empty(), depth, tc.conf);
  Sample smp = sampleModels(s, ray.dir, w[0], hi.sp, m[0], c, *rng);
  // the four wavelengths share the hero's counts and pdfs here
  bool uniform = !hero_only;
  for (int j = 1; j < HERO_COUNT && uniform; ++j) {
    uniform = sameCounts(counts(m[j], !s.alias.empty(), depth, tc.conf), c);
    if ((c.specular_transmit || c.rough_transmit) && m[j].ior.re != m[0].ior.re) uniform = false;
  }
  const float k = (uniform || hero_only) ? 1.0f : static_cast<float>(HERO_COUNT);
  for (int j = 0; j < HERO_COUNT; ++j)
    out.v[j] = (j == 0 || !hero_only) ? m[j].emission : 0.0f;
  for (uint32_t i = 0; i < smp.emission_count; ++i) {
    const auto& es = smp.es[i];
    V3 light_pos = hi.sp.pos + es.dir * es.expected_dist;
    Ray shadow = spawnSurfaceRay(hi.sp, es.dir);
    float expected = distance(shadow.pos, light_pos);
    ++tc.cnt.shadow;
    HitInfo sh = rayHit(s, shadow, tc.prune, tc.cnt);
    if (sh.hit && sh.dist < (expected - 1e-3f)) continue;
    // es.radiance is the hero's whole light-sample term already
    out.v[0] += k * es.radiance;
    if (!uniform) continue;
    const cg_emissive_prim& prim = s.eprims[es.prim];
    for (int j = 1; j < HERO_COUNT; ++j) {
      float radiance = rgbToWavelengthRadiance(ev(prim.emission), w[j]);
      float ec = diffuseDist(ray.dir, es.dir, hi.sp, m[j]) +
                 roughReflectDist(ray.dir, es.dir, hi.sp, m[j]) +
                 roughTransmitDist(ray.dir, es.dir, hi.sp, m[j]);
      out.v[j] += radiance * ec * es.sproj / es.denom;
    }
  }
  for (uint32_t i = 0; i < smp.transport_count; ++i) {
    const TransportSample& t = smp.ts[i];
    float cj[HERO_COUNT] = {t.coeff * k, 0.0f, 0.0f, 0.0f};  // the child's coefficients
    if (uniform)
      for (int j = 1; j < HERO_COUNT; ++j)
        cj[j] = lobeDist(t.model, ray.dir, t.dir, hi.sp, m[j]) / t.denom;
    float ct[HERO_COUNT];  // the child's path weights
    float tmax = 0.0f;
    for (int j = 0; j < HERO_COUNT; ++j) {
      ct[j] = j == 0 ? thr[0] * t.coeff * k : thr[j] * cj[j];
      tmax = wmax(tmax, ct[j]);
    }
    const uint32_t ck = tc.keyed ? childKey(key, i) : 0u;
    float rr = 1.0f;
    if (tc.roulette != 0u && static_cast<uint32_t>(depth) >= tc.roulette) {
      if (tmax == 0.0f) continue;
      rr = roulette(tc, tmax, ck);
      if (rr == 0.0f) continue;
    }
    for (int j = 0; j < HERO_COUNT; ++j) ct[j] = ct[j] * rr;
    Ray child = spawnSurfaceRay(hi.sp, t.dir);
    L4 cl = traceHero(tc, child, w, depth + 1, ck, !uniform, ct);
    out.v[0] += cj[0] * rr * cl.v[0];
    if (!uniform) continue;
    for (int j = 1; j < HERO_COUNT; ++j) out.v[j] += cj[j] * rr * cl.v[j];
  }
  return out;
}

// cameraRay (compute.wesl:64-79)
Ray cameraRay(const cg_camera& cam, uint32_t px, uint32_t py, uint32_t W, uint32_t H) {
  float cx = static_cast<float>(px) / static_cast<float>(W) * 2.0f - 1.0f;
  float cy = static_cast<float>(py) / static_cast<float>(H) * 2.0f - 1.0f;
  V3 dir{cam.direction[0], cam.direction[1], cam.direction[2]};
  V3 dx = normalize(cross(dir, V3{0.0f, 0.0f, 1.0f})) * cam.viewport[0];
  V3 dy = normalize(cross(dir, dx)) * cam.viewport[1];
  return Ray{V3{cam.position[0], cam.position[1], cam.position[2]},
             normalize(dir + cx * dx + cy * dy)};
}

}  // namespace
}  // namespace oracle

using namespace oracle;

namespace {
unsigned pickThreads(uint32_t t) {
  if (t) return t;
  unsigned h = std::thread::hardware_concurrency();
  return h ? h : 1u;
}

template <class F>
void parallelFor(uint32_t n, unsigned threads, F&& f) {
  std::atomic<uint32_t> next{0};
  const uint32_t grain = 64;
  auto worker = [&](unsigned tid) {
    for (;;) {
      uint32_t b = next.fetch_add(grain);
      if (b >= n) break;
      uint32_t e = std::min(n, b + grain);
      for (uint32_t i = b; i < e; ++i) f(tid, i);
    }
  };
  if (threads <= 1) {
    worker(0);
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t) pool.emplace_back(worker, t);
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

oracle_scene_t oracle_scene_create(const cg_scene_desc* d) {
  if (!d) return nullptr;
  auto* s = new oracle_scene_s();
  s->vertices.assign(d->vertices, d->vertices + d->vertex_count);
  s->indices.assign(d->indices, d->indices + d->index_count);
  s->meshes.assign(d->meshes, d->meshes + d->mesh_count);
  s->inst_desc.assign(d->instances, d->instances + d->instance_count);
  for (uint32_t i = 0; i < d->material_count; ++i) {
    const cg_material& m = d->materials[i];
    oracle::Material om;
    om.base_color = {m.base_color_factor[0], m.base_color_factor[1], m.base_color_factor[2]};
    om.emissive = {m.emissive_factor[0], m.emissive_factor[1], m.emissive_factor[2]};
    om.emissive_strength = m.emissive_strength;
    om.metallic = m.metallic_factor;
    om.roughness = m.roughness_factor;
    om.ior = m.ior;
    om.dispersion = m.dispersion;
    om.transmission = m.transmission_factor;
    om.thickness = m.thickness_factor;
    const int32_t tex[4] = {m.base_color_texture, m.metallic_roughness_texture, m.emissive_texture,
                            m.transmission_texture};
    for (int k = 0; k < 4; ++k) {
      om.tex[k] = tex[k];
      om.tex_coord[k] = (m.texcoord_sets >> k) & 1u;
    }
    s->materials.push_back(om);
  }
  for (uint32_t t = 0; t < d->texture_count; ++t) {
    const cg_texture& tx = d->textures[t];
    s->tex_desc.push_back(tx);
    s->tex_data.emplace_back(tx.rgba8, tx.rgba8 + size_t(tx.width) * tx.height * 4);
    s->tex_w = std::max(s->tex_w, tx.width);
    s->tex_h = std::max(s->tex_h, tx.height);
  }
  if (d->texture_count) {
    // ResizeRgba8Nearest (src/wgpu/resource.cpp:52-75) into one layer per texture
    const size_t layer = size_t(s->tex_w) * s->tex_h * 4;
    s->tex.resize(layer * d->texture_count);
    for (uint32_t t = 0; t < d->texture_count; ++t) {
      const cg_texture& tx = s->tex_desc[t];
      const uint8_t* src = s->tex_data[t].data();
      for (uint32_t y = 0; y < s->tex_h; ++y) {
        const uint32_t sy = std::min(tx.height - 1,
                                     static_cast<uint32_t>((uint64_t(y) * tx.height) / s->tex_h));
        for (uint32_t x = 0; x < s->tex_w; ++x) {
          const uint32_t sx = std::min(tx.width - 1,
                                       static_cast<uint32_t>((uint64_t(x) * tx.width) / s->tex_w));
          std::memcpy(&s->tex[t * layer + (size_t(y) * s->tex_w + x) * 4],
                      src + (size_t(sy) * tx.width + sx) * 4, 4);
        }
      }
    }
  }
  using Clock = std::chrono::steady_clock;
  auto seconds = [](Clock::time_point a) {
    return std::chrono::duration<double>(Clock::now() - a).count();
  };
  auto t0 = Clock::now();
  for (const auto& mesh : s->meshes) blasBuildMesh(*s, mesh);
  s->pack_s[0] = seconds(t0);
  t0 = Clock::now();
  // TLAS over instances in scene order (tlas.h:34-77)
  std::vector<BoundedPrimitive> bp;
  for (size_t i = 0; i < s->inst_desc.size(); ++i) {
    const cg_instance& ci = s->inst_desc[i];
    oracle::Instance inst;
    std::memcpy(inst.fwd, ci.world_from_local, sizeof(inst.fwd));
    invertAffine(ci.world_from_local, inst.inv);
    inst.blas_root_idx = s->mesh_root[ci.mesh];
    inst.material_idx = ci.material;
    s->insts.push_back(inst);
    AABB local;
    const cg_mesh& mesh = s->meshes[ci.mesh];
    for (uint32_t v = mesh.vertex_offset; v < mesh.vertex_offset + mesh.vertex_count; ++v)
      local.merge(pos(s->vertices[v]));
    BoundedPrimitive b;
    b.aabb = transAabb(local, ci.world_from_local);
    b.center = b.aabb.center();
    b.prim_idx = static_cast<uint32_t>(i);
    bp.push_back(b);
  }
  if (!bp.empty()) {
    s->tnodes.emplace_back();
    tlasBuild(*s, 0, 0, static_cast<uint32_t>(bp.size()), bp);
  }
  s->pack_s[1] = seconds(t0);
  t0 = Clock::now();
  buildEmissive(*s);
  s->pack_s[2] = seconds(t0);
  t0 = Clock::now();
  std::vector<double> w;
  for (const auto& e : s->eprims) w.push_back(static_cast<double>(e.weight));
  s->alias.resize(w.size());
  aliasBuild(w.data(), static_cast<uint32_t>(w.size()), s->alias.data());
  s->pack_s[3] = seconds(t0);
  // environment (scene_data.h:57-98)
  if (d->env_rgba32f && d->env_width && d->env_height) {
    s->env_w = d->env_width;
    s->env_h = d->env_height;
    s->env.assign(d->env_rgba32f, d->env_rgba32f + size_t(s->env_w) * s->env_h * 4);
  } else {
    s->env_w = 512;
    s->env_h = 256;
    s->env.resize(size_t(512) * 256 * 4);
    for (uint32_t y = 0; y < 256; ++y) {
      float t = static_cast<float>(y) / static_cast<float>(255);
      float c[3] = {mix(0.7f, 0.05f, t), mix(0.8f, 0.05f, t), mix(1.0f, 0.06f, t)};
      for (uint32_t x = 0; x < 512; ++x) {
        float* p = &s->env[(size_t(y) * 512 + x) * 4];
        p[0] = c[0];
        p[1] = c[1];
        p[2] = c[2];
        p[3] = 1.0f;
      }
    }
  }
  return s;
}

void oracle_scene_destroy(oracle_scene_t s) { delete s; }

int oracle_scene_pack_seconds(oracle_scene_t s, double* out) {
  if (!s || !out) return -1;
  std::memcpy(out, s->pack_s, sizeof(s->pack_s));
  return 0;
}

uint32_t oracle_emissive_count(oracle_scene_t s) {
  return s ? static_cast<uint32_t>(s->eprims.size()) : 0u;
}

int oracle_emissive(oracle_scene_t s, cg_emissive_prim* prims, cg_alias_entry* alias,
                    float* total) {
  if (!s) return -1;
  if (prims) std::memcpy(prims, s->eprims.data(), s->eprims.size() * sizeof(cg_emissive_prim));
  if (alias) std::memcpy(alias, s->alias.data(), s->alias.size() * sizeof(cg_alias_entry));
  if (total) *total = s->total_weight;
  return 0;
}

int oracle_alias_build(const double* weights, uint32_t count, cg_alias_entry* out) {
  if (count && (!weights || !out)) return -1;
  aliasBuild(weights, count, out);
  return 0;
}

int oracle_trace_closest(oracle_scene_t s, const float* rays, uint32_t n, cg_hit* hits, float* t2,
                         int threads) {
  if (!s || (n && (!rays || !hits))) return -1;
  parallelFor(n, pickThreads(threads > 0 ? static_cast<uint32_t>(threads) : 0u),
              [&](unsigned, uint32_t i) {
                const float* r = rays + size_t(i) * 8;
                Ray ray{V3{r[0], r[1], r[2]}, V3{r[4], r[5], r[6]}};
                Counters cnt;
                ClosestHit h = traverse(*s, ray, false, cnt);
                cg_hit out{};
                if (h.hit) {
                  out.t = h.t;
                  out.u = h.u;
                  out.v = h.v;
                  out.instance = h.instance;
                  out.triangle = h.triangle;
                } else {
                  out.t = MAXD;
                  out.instance = -1;
                  out.triangle = -1;
                }
                hits[i] = out;
                if (t2) t2[i] = h.t2;
              });
  return 0;
}

int oracle_render(oracle_scene_t s, const oracle_render_args* a, float* film, uint32_t* seeds,
                  uint64_t* stats) {
  if (!s || !a || !film) return -1;
  const uint32_t W = a->conf.render_width, H = a->conf.render_height;
  if (W == 0 || H == 0) return -1;
  if (a->rng_mode == ORACLE_RNG_REFERENCE && !seeds) return -1;
  Conf conf;
  conf.trace_depth = std::clamp(a->conf.trace_depth, 1u, 64u);
  conf.transport_cap = a->conf.max_transport_sample_count;
  conf.emission_cap = a->conf.max_emission_sample_count;
  conf.diffuse_cap = a->conf.max_diffuse_sample_count;
  conf.rough_cap = a->conf.max_rough_sample_count;
  const uint32_t spp = a->conf.sample_count;
  const uint32_t pb = a->pixel_begin;
  const uint32_t pe = a->pixel_end ? std::min(a->pixel_end, W * H) : W * H;
  if (pb >= pe) return 0;
  unsigned threads = pickThreads(a->threads);
  std::vector<Counters> per(threads);
  parallelFor(pe - pb, threads, [&](unsigned tid, uint32_t k) {
    uint32_t pix = pb + k;
    uint32_t px = pix % W, py = pix / W;
    Ray ray = cameraRay(a->camera, px, py, W, H);
    float sample_weight = 1.0f / static_cast<float>(a->iter_count + 1u);
    V3 lum{0.0f, 0.0f, 0.0f};
    uint32_t rand_seed = px + py * W;
    float* f = film + size_t(pix) * 3;
    if (a->iter_count > 0u) {
      lum = V3{f[0], f[1], f[2]} * (1.0f - sample_weight);
      if (a->rng_mode == ORACLE_RNG_REFERENCE) rand_seed = seeds[pix];
    }
    TraceCtx tc;
    tc.s = s;
    tc.conf = conf;
    tc.prune = a->prune != 0;
    tc.keyed = a->rng_mode == ORACLE_RNG_KEYED;
    tc.roulette = a->roulette;
    Rng seq;
    seedRng(seq, rand_seed);
    tc.seq = &seq;
    // render (render.wesl:7-18)
    V3 acc{0.0f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < spp; ++i) {
      float u = 0.0f;
      uint32_t key = 0;
      if (tc.keyed) {
        key = sampleKey(a->seed, a->iter_count, pix, i);
        Rng wr;
        seedRng(wr, wavelengthKey(key));
        u = randFloat(wr);
      } else {
        u = randFloat(seq);
      }
      V3 term;
      if (a->spectral == ORACLE_SPECTRAL_HERO) {
        float w[HERO_COUNT];
        heroWavelengths(u, w);
        const float one[HERO_COUNT] = {1.0f, 1.0f, 1.0f, 1.0f};
        const L4 L = traceHero(tc, ray, w, 0, key, false, one);
        V3 est{0.0f, 0.0f, 0.0f};
        for (int j = 0; j < HERO_COUNT; ++j) est = est + illuminate(w[j], L.v[j]);
        term = est * (HERO_SPAN / HERO_COUNT) / static_cast<float>(spp);
      } else {
        const WavelengthSample ws = sampleWavelengthCdf(u);
        float L = trace(tc, ray, ws.wavelength, 0, key, 1.0f);
        term = illuminate(ws.wavelength, L) / ws.prob / static_cast<float>(spp);
      }
      // the library's film policy: a sample whose estimate is not finite adds
      // nothing (the reference's running mean would keep the NaN for good)
      if (std::isfinite(term.x) && std::isfinite(term.y) && std::isfinite(term.z))
        acc = acc + term;
      else
        ++per[tid].nonfinite;
    }
    lum = lum + acc * sample_weight;
    f[0] = lum.x;
    f[1] = lum.y;
    f[2] = lum.z;
    if (a->rng_mode == ORACLE_RNG_REFERENCE) seeds[pix] = randUInt(seq);
    per[tid].extend += tc.cnt.extend;
    per[tid].shadow += tc.cnt.shadow;
    per[tid].nodes += tc.cnt.nodes;
    per[tid].tris += tc.cnt.tris;
  });
  if (stats) {
    Counters t;
    for (const auto& c : per) {
      t.extend += c.extend;
      t.shadow += c.shadow;
      t.nodes += c.nodes;
      t.tris += c.tris;
      t.nonfinite += c.nonfinite;
    }
    stats[0] = t.extend;
    stats[1] = t.shadow;
    stats[2] = t.nodes;
    stats[3] = t.tris;
    stats[4] = t.nonfinite;
  }
  return 0;
}

float oracle_sample_wavelength(float u, float* prob) {
  WavelengthSample ws = sampleWavelengthCdf(u);
  if (prob) *prob = ws.prob;
  return ws.wavelength;
}
void oracle_xyz_match(float w, float* xyz) {
  V3 m = xyzMatch(w);
  xyz[0] = m.x;
  xyz[1] = m.y;
  xyz[2] = m.z;
}
float oracle_rgb_to_reflectance(const float* rgb, float w) {
  return rgbToWavelengthReflectance(V3{rgb[0], rgb[1], rgb[2]}, w);
}
float oracle_rgb_to_radiance(const float* rgb, float w) {
  return rgbToWavelengthRadiance(V3{rgb[0], rgb[1], rgb[2]}, w);
}
void oracle_xyz_to_srgb(const float* xyz, float* rgb) {
  V3 r = luminanceToSrgb(V3{xyz[0], xyz[1], xyz[2]});
  rgb[0] = r.x;
  rgb[1] = r.y;
  rgb[2] = r.z;
}
uint32_t oracle_rng_sequence(uint32_t seed, uint32_t n, float* out) {
  Rng r;
  seedRng(r, seed);
  for (uint32_t i = 0; i < n; ++i) out[i] = randFloat(r);
  return r.s;
}
uint32_t oracle_sample_key(uint32_t seed, uint32_t frame, uint32_t pixel, uint32_t sample) {
  return sampleKey(seed, frame, pixel, sample);
}

}  // extern "C"
