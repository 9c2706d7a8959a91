// cg_png.h — PNG decoding to RGBA8 (cg_png.cpp).
#ifndef CG_PNG_H_
#define CG_PNG_H_

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace cg {

// Decodes a PNG file image into `rgba` (width * height * 4 bytes, top row
// first).  Returns false with `err` for anything else (JPEG included) or a
// corrupt file.
bool decodePng(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
               std::vector<uint8_t>& rgba, std::string& err);

}  // namespace cg

#endif
