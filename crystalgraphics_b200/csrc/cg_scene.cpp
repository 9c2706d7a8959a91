// cg_scene.cpp — host scene packing for the CUDA backend.
//
// Compiled with -ffp-contract=off: the emissive buffer, its weights and the
// inverse instance transforms must round exactly as the host code they
// restate (src/pathtracing/emissive_buffer.h:44-100, tlas.h:56-73).
#include "cg_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "cg_bvh.h"

namespace cg {
namespace {

struct F3 {
  float x, y, z;
};
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 cross3(F3 a, F3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline F3 vpos(const cg_vertex& v) { return {v.position[0], v.position[1], v.position[2]}; }

// glm mat4 * vec4(p, 1): (m0 x + m1 y) + (m2 z + m3 w)  (emissive_buffer.h:134-137)
F3 transformPoint(const float* m, F3 p) {
  float r[3];
  const float q[3] = {p.x, p.y, p.z};
  for (int i = 0; i < 3; ++i) {
    float add0 = m[i * 4 + 0] * q[0] + m[i * 4 + 1] * q[1];
    float add1 = m[i * 4 + 2] * q[2] + m[i * 4 + 3] * 1.0f;
    r[i] = add0 + add1;
  }
  return {r[0], r[1], r[2]};
}

float luminance(F3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }

bool textured(const cg_material& m) {
  return m.base_color_texture >= 0 || m.metallic_roughness_texture >= 0 || m.emissive_texture >= 0 ||
         m.transmission_texture >= 0;
}

// ResizeRgba8Nearest (src/wgpu/resource.cpp:52-75): the source texel of each
// target texel by integer scaling; texels packed as uint32 (r | g<<8 | b<<16 | a<<24).
void resizeNearest(const cg_texture& t, uint32_t w, uint32_t h, uint32_t* out) {
  for (uint32_t y = 0; y < h; ++y) {
    const uint32_t sy = std::min(t.height - 1, static_cast<uint32_t>((uint64_t(y) * t.height) / h));
    for (uint32_t x = 0; x < w; ++x) {
      const uint32_t sx = std::min(t.width - 1, static_cast<uint32_t>((uint64_t(x) * t.width) / w));
      std::memcpy(out + size_t(y) * w + x, t.rgba8 + (size_t(sy) * t.width + sx) * 4, 4);
    }
  }
}

// WrapCoord (emissive_buffer.h:191-204): glTF clamp to edge (33071), mirrored
// repeat (33648), else repeat; the result is clamped below 1.
float wrapCoord(float c, int32_t wrap) {
  if (wrap == 33071) return std::clamp(c, 0.0f, 0.999999f);
  if (wrap == 33648) {
    float wrapped = c - std::floor(c);
    const auto tile = static_cast<int32_t>(std::floor(c));
    if (tile % 2 != 0) wrapped = 1.0f - wrapped;
    return std::clamp(wrapped, 0.0f, 0.999999f);
  }
  const float wrapped = c - std::floor(c);
  return std::clamp(wrapped, 0.0f, 0.999999f);
}

// EmissiveTextureFactor (emissive_buffer.h:138-189): the emissive texture's
// texel (nearest, glTF wrap modes, original image) at the triangle's mean UV;
// (1, 1, 1) without an emissive texture.
F3 emissiveTextureFactor(const cg_scene_desc* d, const cg_material& m, const cg_vertex& v0,
                         const cg_vertex& v1, const cg_vertex& v2) {
  if (m.emissive_texture < 0 || static_cast<uint32_t>(m.emissive_texture) >= d->texture_count)
    return F3{1.0f, 1.0f, 1.0f};
  const cg_texture& t = d->textures[m.emissive_texture];
  const bool set1 = (m.texcoord_sets >> 2) & 1u;
  const float* a = set1 ? v0.tex_coord1 : v0.tex_coord0;
  const float* b = set1 ? v1.tex_coord1 : v1.tex_coord0;
  const float* c = set1 ? v2.tex_coord1 : v2.tex_coord0;
  const float u = wrapCoord(((a[0] + b[0]) + c[0]) / 3.0f, t.wrap_s);
  const float v = wrapCoord(((a[1] + b[1]) + c[1]) / 3.0f, t.wrap_t);
  const uint32_t x = std::min(t.width - 1, static_cast<uint32_t>(u * static_cast<float>(t.width)));
  const uint32_t y = std::min(t.height - 1, static_cast<uint32_t>(v * static_cast<float>(t.height)));
  const uint8_t* px = t.rgba8 + (size_t(y) * t.width + x) * 4;
  return F3{static_cast<float>(px[0]) / 255.0f, static_cast<float>(px[1]) / 255.0f,
            static_cast<float>(px[2]) / 255.0f};
}

// A cut of a mesh's BVH2 of at most `target` boxes (the inner node of largest
// surface area is replaced by its two children first).  Their union contains
// every triangle, and transformed corner by corner they bound a rotated
// instance far tighter than the corners of the mesh's single box.
void bvhCut(const std::vector<BvhNode>& nodes, uint32_t root, size_t target, std::vector<Box>& out) {
  struct Item {
    Box box;
    int32_t link;
  };
  auto kids = [&](int32_t n, std::vector<Item>& v) {
    const BvhNode& b = nodes[static_cast<size_t>(n)];
    const Item c0{{{b.c0lx, b.c0ly, b.c0lz}, {b.c0hx, b.c0hy, b.c0hz}}, b.child0};
    const Item c1{{{b.c1lx, b.c1ly, b.c1lz}, {b.c1hx, b.c1hy, b.c1hz}}, b.child1};
    if (c0.link >= 0 || leafCount(c0.link) != 0) v.push_back(c0);
    if (c1.link >= 0 || leafCount(c1.link) != 0) v.push_back(c1);
  };
  auto area = [](const Box& b) {
    const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return x * y + y * z + z * x;
  };
  std::vector<Item> items;
  kids(static_cast<int32_t>(root), items);
  while (items.size() < target) {
    int best = -1;
    float best_area = -1.0f;
    for (size_t k = 0; k < items.size(); ++k) {
      if (items[k].link < 0) continue;
      const float a = area(items[k].box);
      if (a > best_area) {
        best_area = a;
        best = static_cast<int>(k);
      }
    }
    if (best < 0) break;
    const int32_t n = items[best].link;
    items.erase(items.begin() + best);
    kids(n, items);
  }
  out.clear();
  for (const Item& it : items) out.push_back(it.box);
}

}  // namespace

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

void buildAliasTable(const double* weights, uint32_t count, cg_alias_entry* entries) {
  for (uint32_t i = 0; i < count; ++i) entries[i] = cg_alias_entry{0u, 0.0f};
  if (count == 0) return;
  std::vector<double> p(count);
  double total = 0.0;
  for (uint32_t i = 0; i < count; ++i) p[i] = std::max(0.0, weights[i]);
  for (uint32_t i = 0; i < count; ++i) total += p[i];
  if (total <= 0.0) return;
  std::vector<uint32_t> small, large;
  small.reserve(count);
  large.reserve(count);
  for (uint32_t i = 0; i < count; ++i) {
    p[i] = p[i] / total * count;
    (p[i] >= 1.0 ? large : small).push_back(i);
  }
  while (!large.empty() && !small.empty()) {
    const uint32_t s = small.back(), l = large.back();
    small.pop_back();
    large.pop_back();
    entries[s].prob = static_cast<float>(p[s]);
    entries[s].alias = l;
    p[l] -= 1.0 - static_cast<double>(entries[s].prob);
    (p[l] < 1.0 ? small : large).push_back(l);
  }
  for (auto* list : {&large, &small}) {
    while (!list->empty()) {
      const uint32_t i = list->back();
      list->pop_back();
      entries[i].prob = 1.0f;
      entries[i].alias = i;
    }
  }
}

int packScene(const cg_scene_desc* d, HostScene& s, std::string& err) {
  if (!d) {
    err = "scene description is null";
    return CG_E_INVALID;
  }
  if ((d->vertex_count && !d->vertices) || (d->index_count && !d->indices) ||
      (d->mesh_count && !d->meshes) || (d->instance_count && !d->instances) ||
      (d->material_count && !d->materials)) {
    err = "scene description has a null array with a nonzero count";
    return CG_E_INVALID;
  }
  // ---- validation -------------------------------------------------------
  for (uint32_t m = 0; m < d->mesh_count; ++m) {
    const cg_mesh& mesh = d->meshes[m];
    if (uint64_t(mesh.index_offset) + mesh.index_count > d->index_count) {
      err = "mesh " + std::to_string(m) + " index range exceeds the index buffer";
      return CG_E_INVALID;
    }
    if (uint64_t(mesh.vertex_offset) + mesh.vertex_count > d->vertex_count) {
      err = "mesh " + std::to_string(m) + " vertex range exceeds the vertex buffer";
      return CG_E_INVALID;
    }
    for (uint32_t i = 0; i < mesh.index_count; ++i) {
      if (d->indices[mesh.index_offset + i] >= d->vertex_count) {
        err = "mesh " + std::to_string(m) + " has an index beyond the vertex buffer";
        return CG_E_INVALID;
      }
    }
  }
  for (uint32_t i = 0; i < d->instance_count; ++i) {
    const cg_instance& in = d->instances[i];
    if (in.mesh >= d->mesh_count || in.material >= d->material_count) {
      err = "instance " + std::to_string(i) + " names a missing mesh or material";
      return CG_E_INVALID;
    }
    for (float f : in.world_from_local)
      if (!std::isfinite(f)) {
        err = "instance " + std::to_string(i) + " has a non-finite transform";
        return CG_E_INVALID;
      }
  }
  if (d->texture_count && !d->textures) {
    err = "scene description has a null texture array with a nonzero count";
    return CG_E_INVALID;
  }
  for (uint32_t t = 0; t < d->texture_count; ++t) {
    const cg_texture& tx = d->textures[t];
    if (tx.width == 0 || tx.height == 0 || !tx.rgba8) {
      err = "texture " + std::to_string(t) + " has no image data";
      return CG_E_INVALID;
    }
  }
  for (uint32_t i = 0; i < d->material_count; ++i) {
    const cg_material& m = d->materials[i];
    for (int32_t t : {m.base_color_texture, m.metallic_roughness_texture, m.emissive_texture,
                      m.transmission_texture})
      if (t < -1 || t >= static_cast<int64_t>(d->texture_count)) {
        err = "material " + std::to_string(i) + " names a missing texture";
        return CG_E_INVALID;
      }
  }
  if (d->env_rgba32f && (d->env_width == 0 || d->env_height == 0)) {
    err = "environment texture has a zero dimension";
    return CG_E_INVALID;
  }

  // ---- vertices ---------------------------------------------------------
  s.vnormal.resize(size_t(d->vertex_count) * 4);
  for (uint32_t v = 0; v < d->vertex_count; ++v) {
    for (int k = 0; k < 3; ++k) s.vnormal[size_t(v) * 4 + k] = d->vertices[v].normal[k];
    s.vnormal[size_t(v) * 4 + 3] = 0.0f;
  }
  bool any_textured = false;
  for (uint32_t i = 0; i < d->material_count; ++i) any_textured = any_textured || textured(d->materials[i]);
  if (any_textured) {
    s.vuv.resize(size_t(d->vertex_count) * 4);
    for (uint32_t v = 0; v < d->vertex_count; ++v) {
      const cg_vertex& vx = d->vertices[v];
      const float uv[4] = {vx.tex_coord0[0], vx.tex_coord0[1], vx.tex_coord1[0], vx.tex_coord1[1]};
      std::memcpy(&s.vuv[size_t(v) * 4], uv, sizeof(uv));
    }
  }
  // ---- material texture array (WriteMaterialTextures, src/wgpu/resource.cpp:471-546):
  // every texture resized (nearest) to the largest width and height, one layer each
  if (d->texture_count) {
    s.tex_w = 1;
    s.tex_h = 1;
    for (uint32_t t = 0; t < d->texture_count; ++t) {
      s.tex_w = std::max(s.tex_w, d->textures[t].width);
      s.tex_h = std::max(s.tex_h, d->textures[t].height);
    }
    s.tex_layers = d->texture_count;
    s.tex.resize(size_t(s.tex_w) * s.tex_h * s.tex_layers);
    for (uint32_t t = 0; t < d->texture_count; ++t)
      resizeNearest(d->textures[t], s.tex_w, s.tex_h, s.tex.data() + size_t(t) * s.tex_w * s.tex_h);
  }

  // ---- one BLAS per mesh ------------------------------------------------------
  s.mesh_count = d->mesh_count;
  std::vector<uint32_t> mesh_root(d->mesh_count), mesh_root4(d->mesh_count),
      mesh_tri_base(d->mesh_count);
  std::vector<Box> mesh_bounds(d->mesh_count);
  BvhBuildOptions blas_opt;
  blas_opt.max_leaf = 4;
  std::vector<uint32_t> order;
  for (uint32_t m = 0; m < d->mesh_count; ++m) {
    const cg_mesh& mesh = d->meshes[m];
    const uint32_t nt = mesh.index_count / 3;
    std::vector<Box> boxes(nt);
    Box mb;
    for (int a = 0; a < 3; ++a) {
      mb.lo[a] = std::numeric_limits<float>::infinity();
      mb.hi[a] = -std::numeric_limits<float>::infinity();
    }
    for (uint32_t t = 0; t < nt; ++t) {
      const uint32_t* ix = d->indices + mesh.index_offset + 3 * t;
      Box& b = boxes[t];
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::numeric_limits<float>::infinity();
        b.hi[a] = -std::numeric_limits<float>::infinity();
      }
      for (int k = 0; k < 3; ++k) {
        const float* p = d->vertices[ix[k]].position;
        for (int a = 0; a < 3; ++a) {
          b.lo[a] = std::min(b.lo[a], p[a]);
          b.hi[a] = std::max(b.hi[a], p[a]);
          mb.lo[a] = std::min(mb.lo[a], p[a]);
          mb.hi[a] = std::max(mb.hi[a], p[a]);
        }
      }
    }
    mesh_bounds[m] = mb;
    const uint32_t tri_base = static_cast<uint32_t>(s.tri_vidx.size() / 4);
    mesh_tri_base[m] = tri_base;
    order.clear();
    uint32_t depth = 0;
    mesh_root[m] = buildBvh(boxes, blas_opt, tri_base, s.blas, order, &depth);
    mesh_root4[m] = collapseBvh4(s.blas, mesh_root[m], s.blas4);
    s.blas_depth = std::max(s.blas_depth, depth);
    for (uint32_t k = 0; k < nt; ++k) {
      const uint32_t t = order[k];
      const uint32_t* ix = d->indices + mesh.index_offset + 3 * t;
      F3 v0 = vpos(d->vertices[ix[0]]), v1 = vpos(d->vertices[ix[1]]), v2 = vpos(d->vertices[ix[2]]);
      F3 e1 = sub(v1, v0), e2 = sub(v2, v0);  // the subtractions of bvh.wesl:189-190
      float idbits;
      std::memcpy(&idbits, &t, 4);
      const float rec[12] = {v0.x, v0.y, v0.z, idbits, e1.x, e1.y, e1.z, 0.0f,
                             e2.x, e2.y, e2.z, 0.0f};
      s.tris.insert(s.tris.end(), rec, rec + 12);
      const uint32_t vi[4] = {ix[0], ix[1], ix[2], t};
      s.tri_vidx.insert(s.tri_vidx.end(), vi, vi + 4);
    }
  }
  s.triangle_count = static_cast<uint32_t>(s.tri_vidx.size() / 4);

  // ---- materials ------------------------------------------------------------------
  auto clamp01 = [](float x) { return std::fmin(std::fmax(x, 0.0f), 1.0f); };
  s.max_lobes = 0;
  for (uint32_t i = 0; i < d->material_count; ++i) {
    const cg_material& m = d->materials[i];
    DevMaterial dm{};
    for (int k = 0; k < 3; ++k) {
      dm.base[k] = m.base_color_factor[k];
      dm.emission[k] = std::fmax(m.emissive_factor[k] * m.emissive_strength, 0.0f);
    }
    dm.metallic = clamp01(m.metallic_factor);
    dm.roughness = clamp01(m.roughness_factor);
    dm.ior = m.ior;
    dm.dispersion = m.dispersion;
    dm.transmission = clamp01(m.transmission_factor);
    dm.volume = m.thickness_factor > 0.0f ? 1u : 0u;
    DevMatTex mt{};
    mt.layer[0] = m.base_color_texture;
    mt.layer[1] = m.metallic_roughness_texture;
    mt.layer[2] = m.emissive_texture;
    mt.layer[3] = m.transmission_texture;
    mt.uv1_bits = m.texcoord_sets & 15u;
    mt.metallic = m.metallic_factor;
    mt.roughness = m.roughness_factor;
    mt.transmission = m.transmission_factor;
    for (int k = 0; k < 3; ++k) mt.emissive[k] = m.emissive_factor[k];
    mt.emissive_strength = m.emissive_strength;
    s.mattex.push_back(mt);
    const bool tx = textured(m);
    if (tx) dm.volume |= kTexturedBit;
    // the lobes a hit can sample; a texture can lower metallic, transmission and
    // roughness below their factors, so textured channels count every lobe
    const bool mr_tex = m.metallic_roughness_texture >= 0, tr_tex = m.transmission_texture >= 0;
    const bool diffuse = mr_tex || tr_tex || (1.0f - dm.metallic) * (1.0f - dm.transmission) > 0.0f;
    const bool transmit = dm.transmission > 1e-6f;
    {
      uint32_t kind = 0;
      if (diffuse) kind |= 1u;
      kind |= mr_tex ? 6u : (dm.roughness == 0.0f ? 2u : 4u);
      if (transmit) kind |= 8u;
      dm.volume |= kind << kKindShift;
    }
    s.mat.push_back(dm);
    uint32_t lobes = 1;  // a reflection lobe
    if (diffuse) ++lobes;
    if (transmit) ++lobes;
    s.max_lobes = std::max(s.max_lobes, lobes);
  }

  // ---- instances and the TLAS ---------------------------------------------------------
  std::vector<std::vector<Box>> mesh_cut(d->mesh_count);
  for (uint32_t m = 0; m < d->mesh_count; ++m)
    if (mesh_bounds[m].lo[0] <= mesh_bounds[m].hi[0]) bvhCut(s.blas, mesh_root[m], 64, mesh_cut[m]);
  std::vector<Box> inst_boxes(d->instance_count);
  for (uint32_t i = 0; i < d->instance_count; ++i) {
    const cg_instance& ci = d->instances[i];
    DevInstance di{};
    invertAffine(ci.world_from_local, di.inv);
    di.blas_root = mesh_root[ci.mesh];
    di.material = ci.material;
    di.tri_base = mesh_tri_base[ci.mesh];
    di.blas4_root = mesh_root4[ci.mesh];
    s.inst.push_back(di);
    // world box: the corners of the mesh's BVH cut boxes, transformed in
    // double and widened by one float step
    const Box& mb = mesh_bounds[ci.mesh];
    Box wb;
    for (int a = 0; a < 3; ++a) {
      wb.lo[a] = std::numeric_limits<float>::infinity();
      wb.hi[a] = -std::numeric_limits<float>::infinity();
    }
    if (mb.lo[0] <= mb.hi[0]) {
      for (const Box& cb : mesh_cut[ci.mesh]) {
        for (int c = 0; c < 8; ++c) {
          double p[3] = {(c & 1) ? cb.hi[0] : cb.lo[0], (c & 2) ? cb.hi[1] : cb.lo[1],
                         (c & 4) ? cb.hi[2] : cb.lo[2]};
          for (int a = 0; a < 3; ++a) {
            const float* r = ci.world_from_local + 4 * a;
            double w =
                double(r[0]) * p[0] + double(r[1]) * p[1] + double(r[2]) * p[2] + double(r[3]);
            wb.lo[a] = std::min(wb.lo[a], std::nextafter(static_cast<float>(w), -INFINITY));
            wb.hi[a] = std::max(wb.hi[a], std::nextafter(static_cast<float>(w), INFINITY));
          }
        }
      }
    } else {
      for (int a = 0; a < 3; ++a) {
        wb.lo[a] = 1.0f;
        wb.hi[a] = -1.0f;
      }
    }
    inst_boxes[i] = wb;
  }
  {
    BvhBuildOptions opt;
    opt.max_leaf = 1;
    std::vector<uint32_t> tlas_order;
    uint32_t depth = 0;
    buildBvh(inst_boxes, opt, 0, s.tlas, tlas_order, &depth);
    s.tlas_depth = depth;
    // TLAS leaves index tlas_order -> instance; store instance ids directly
    for (BvhNode& n : s.tlas) {
      if (n.child0 < 0 && n.cnt0) n.child0 = leafLinkOf(tlas_order[leafFirst(n.child0)], 1);
      if (n.child1 < 0 && n.cnt1) n.child1 = leafLinkOf(tlas_order[leafFirst(n.child1)], 1);
    }
    collapseBvh4(s.tlas, 0, s.tlas4);  // root 0
  }
  quantizeBvh4(s.tlas4, s.tlas4q);
  quantizeBvh4(s.blas4, s.blas4q);

  // ---- emissive buffer (emissive_buffer.h:44-100) --------------------------------------
  for (uint32_t p = 0; p < d->instance_count; ++p) {
    const cg_instance& inst = d->instances[p];
    const DevMaterial& m = s.mat[inst.material];
    F3 base{m.emission[0], m.emission[1], m.emission[2]};
    if (luminance(base) <= 0.0f) continue;
    const cg_mesh& mesh = d->meshes[inst.mesh];
    for (uint32_t i = 0; i + 2 < mesh.index_count; i += 3) {
      const uint32_t* ix = d->indices + mesh.index_offset + i;
      F3 p0 = transformPoint(inst.world_from_local, vpos(d->vertices[ix[0]]));
      F3 p1 = transformPoint(inst.world_from_local, vpos(d->vertices[ix[1]]));
      F3 p2 = transformPoint(inst.world_from_local, vpos(d->vertices[ix[2]]));
      F3 c = cross3(sub(p1, p0), sub(p2, p0));
      float area = std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z) * 0.5f;
      if (area <= 0.0f) continue;
      const F3 f = emissiveTextureFactor(d, d->materials[inst.material], d->vertices[ix[0]],
                                         d->vertices[ix[1]], d->vertices[ix[2]]);
      const F3 emission{base.x * f.x, base.y * f.y, base.z * f.z};
      float w = luminance(emission);
      if (w <= 0.0f) continue;
      DevEmissivePrim e{};
      e.v0[0] = p0.x; e.v0[1] = p0.y; e.v0[2] = p0.z;
      e.v1[0] = p1.x; e.v1[1] = p1.y; e.v1[2] = p1.z;
      e.v2[0] = p2.x; e.v2[1] = p2.y; e.v2[2] = p2.z;
      e.emission[0] = emission.x; e.emission[1] = emission.y; e.emission[2] = emission.z;
      e.area = area;
      e.weight = area * w;
      s.eprim.push_back(e);
      s.total_weight += e.weight;
    }
  }
  if (s.total_weight > 0.0f)
    for (auto& e : s.eprim) e.weight /= s.total_weight;
  {
    std::vector<double> w(s.eprim.size());
    for (size_t i = 0; i < w.size(); ++i) w[i] = static_cast<double>(s.eprim[i].weight);
    std::vector<cg_alias_entry> a(w.size());
    buildAliasTable(w.data(), static_cast<uint32_t>(w.size()), a.data());
    s.alias.resize(a.size());
    for (size_t i = 0; i < a.size(); ++i) s.alias[i] = DevAlias{a[i].alias, a[i].prob};
  }

  // ---- light BVH for the light-pdf sum (pdf/emission.wesl:120-149) ------------------------
  {
    std::vector<Box> boxes(s.eprim.size());
    for (size_t i = 0; i < s.eprim.size(); ++i) {
      const DevEmissivePrim& e = s.eprim[i];
      Box& b = boxes[i];
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(std::min(e.v0[a], e.v1[a]), e.v2[a]);
        b.hi[a] = std::max(std::max(e.v0[a], e.v1[a]), e.v2[a]);
      }
    }
    BvhBuildOptions opt;
    opt.max_leaf = 4;
    std::vector<uint32_t> lorder;
    buildBvh(boxes, opt, 0, s.light_bvh, lorder);
    for (uint32_t k = 0; k < lorder.size(); ++k) {
      const DevEmissivePrim& e = s.eprim[lorder[k]];
      DevLightTri lt{};
      F3 v0{e.v0[0], e.v0[1], e.v0[2]}, v1{e.v1[0], e.v1[1], e.v1[2]}, v2{e.v2[0], e.v2[1], e.v2[2]};
      F3 e1 = sub(v1, v0), e2 = sub(v2, v0);
      F3 n = cross3(e1, e2);
      float len = std::sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
      lt.v0[0] = v0.x; lt.v0[1] = v0.y; lt.v0[2] = v0.z;
      lt.e1[0] = e1.x; lt.e1[1] = e1.y; lt.e1[2] = e1.z;
      lt.e2[0] = e2.x; lt.e2[1] = e2.y; lt.e2[2] = e2.z;
      lt.n[0] = n.x / len; lt.n[1] = n.y / len; lt.n[2] = n.z / len;
      lt.area_pdf = std::fmax(e.weight / e.area, 1e-3f);
      s.ltri.push_back(lt);
    }
  }

  // ---- environment (scene_data.h:57-98) ---------------------------------------------------
  if (d->env_rgba32f) {
    s.env_w = d->env_width;
    s.env_h = d->env_height;
    s.env.assign(d->env_rgba32f, d->env_rgba32f + size_t(s.env_w) * s.env_h * 4);
  } else {
    s.env_w = 512;
    s.env_h = 256;
    s.env.resize(size_t(512) * 256 * 4);
    for (uint32_t y = 0; y < 256; ++y) {
      float t = static_cast<float>(y) / static_cast<float>(255);
      float c[3] = {0.7f * (1.0f - t) + 0.05f * t, 0.8f * (1.0f - t) + 0.05f * t,
                    1.0f * (1.0f - t) + 0.06f * t};
      for (uint32_t x = 0; x < 512; ++x) {
        float* p = &s.env[(size_t(y) * 512 + x) * 4];
        p[0] = c[0];
        p[1] = c[1];
        p[2] = c[2];
        p[3] = 1.0f;
      }
    }
  }
  return CG_OK;
}

}  // namespace cg
