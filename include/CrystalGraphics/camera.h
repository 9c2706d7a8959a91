// crystal::graphics::Camera — the reference's layout (camera.h:9-13):
// position, direction, viewport half-extents; 48 bytes.
#ifndef CRYSTALGRAPHICS_CAMERA_H_
#define CRYSTALGRAPHICS_CAMERA_H_

#include "vec.h"

namespace crystal::graphics {

struct Camera {
  alignas(16) Vec3 position{0, 0, 0};
  alignas(16) Vec3 direction{1, 0, 0};
  alignas(8) Vec2 viewport{0.5, 0.5};
};

static_assert(sizeof(Camera) == 48, "Camera keeps the reference's 48-byte layout");

}  // namespace crystal::graphics

#endif
