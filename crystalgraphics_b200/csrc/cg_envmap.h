// cg_envmap.h — environment maps from image-based lights (cg_envmap.cpp).
#ifndef CG_ENVMAP_H_
#define CG_ENVMAP_H_

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace cg {

// Decodes a Radiance RGBE (.hdr) image into linear RGBA32F (alpha 1, top
// row first): header "#?RADIANCE" or "#?RGBE", FORMAT=32-bit_rle_rgbe,
// resolution "-Y height +X width", flat or run-length-encoded scanlines.
bool decodeRadianceHdr(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                       std::vector<float>& rgba, std::string& err);

// Decodes an image to linear RGBA32F as the reference's DecodeImageRgba32f
// does: Radiance HDR as is, PNG and JPEG through their 8-bit RGBA with the
// colour channels raised to the power 2.2 and alpha scaled to [0, 1].
bool decodeImageRgba32f(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                        std::vector<float>& rgba, std::string& err);

// The lat-long environment (4w x 2h RGBA32F, alpha 1) of six w x h RGBA32F
// cube faces (order +-X, +-Y, +-Z as the image-based light lists them) seen
// through the light's rotation quaternion (x, y, z, w).
void cubeToLatLong(const float* const faces[6], uint32_t face_width, uint32_t face_height,
                   const float rotation[4], std::vector<float>& out);

}  // namespace cg

#endif
