// cg_scene.h — host scene packing (LoadScene's work) for the CUDA backend.
//
// Replaces SceneData (src/pathtracing/scene_data.h:38-54), which the
// reference rebuilds on every View(): the BVHs, the emissive buffer, its
// alias table and the environment are built once here and uploaded.
#ifndef CG_SCENE_H_
#define CG_SCENE_H_

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cg_cuda.h"
#include "cg_types.h"

namespace cg {

struct HostScene {
  std::vector<BvhNode> tlas, blas, light_bvh;
  std::vector<Bvh4Node> tlas4, blas4;  // the TLAS and BLAS collapsed four-wide
  std::vector<Bvh4QNode> tlas4q, blas4q;  // the same, child boxes quantised to 8 bits
  std::vector<float> tris;          // 12 floats per triangle (3 x float4)
  std::vector<uint32_t> tri_vidx;   // 4 per triangle
  std::vector<float> vnormal;       // 4 per vertex
  std::vector<DevInstance> inst;
  std::vector<DevMaterial> mat;
  std::vector<DevEmissivePrim> eprim;
  std::vector<DevAlias> alias;
  std::vector<DevLightTri> ltri;
  std::vector<float> env;           // 4 per texel
  std::vector<DevMatTex> mattex;    // per material
  std::vector<uint32_t> tex;        // RGBA8 texels of the texture array (layer-major)
  std::vector<float> vuv;           // 4 per vertex, when a material is textured
  uint32_t tex_w = 1, tex_h = 1, tex_layers = 0;
  uint32_t env_w = 0, env_h = 0;
  float total_weight = 0.0f;
  uint32_t mesh_count = 0, triangle_count = 0, blas_depth = 0, tlas_depth = 0;
  uint32_t max_lobes = 0;           // most BSDF lobes any material can sample at once
};

// Validates `desc` and packs it.  Returns CG_OK or CG_E_INVALID with `err`.
int packScene(const cg_scene_desc* desc, HostScene& out, std::string& err);

// Vose alias table with LIFO small/large work lists, built in double
// (the construction of src/pathtracing/alias_table.h:24-70).
void buildAliasTable(const double* weights, uint32_t count, cg_alias_entry* out);

// Inverse of a row-major 3x4 affine matrix, computed in double and rounded.
void invertAffine(const float* m, float* out);

}  // namespace cg

#endif
