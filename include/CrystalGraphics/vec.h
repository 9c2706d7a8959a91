// Vector types of the public API.  The reference uses glm::vec2 / glm::vec3
// (camera.h:4-5); when glm is on the include path the same types are used,
// otherwise layout-identical plain structs (12 and 8 bytes, aligned by the
// members that hold them exactly as the reference's Camera aligns glm).
#ifndef CRYSTALGRAPHICS_VEC_H_
#define CRYSTALGRAPHICS_VEC_H_

#if __has_include(<glm/ext/vector_float3.hpp>)
#include <glm/ext/vector_float2.hpp>
#include <glm/ext/vector_float3.hpp>
namespace crystal::graphics {
using Vec2 = glm::vec2;
using Vec3 = glm::vec3;
}  // namespace crystal::graphics
#else
namespace crystal::graphics {
struct Vec3 {
  float x = 0.0f, y = 0.0f, z = 0.0f;
};
struct Vec2 {
  float x = 0.0f, y = 0.0f;
};
}  // namespace crystal::graphics
#endif

#endif
