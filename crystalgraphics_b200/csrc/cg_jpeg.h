// cg_jpeg.h — JPEG decoding to RGBA8 (cg_jpeg.cpp).
#ifndef CG_JPEG_H_
#define CG_JPEG_H_

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace cg {

// Decodes a JPEG (JFIF / Exif) image into `rgba` (width * height * 4 bytes,
// top row first, alpha 255): Huffman-coded baseline, extended sequential and
// progressive 8-bit images with one (grey) or three (YCbCr, or RGB per an
// Adobe marker) components, any sampling factors, restart intervals.  Returns
// false with `err` for anything else (arithmetic coding, lossless, 12-bit,
// CMYK) or a corrupt stream.
bool decodeJpeg(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                std::vector<uint8_t>& rgba, std::string& err);

// A glTF image (PNG or JPEG, told apart by their signatures) to RGBA8: the
// reference's DecodeImageRgba8 (src/image_decode.cpp:12-45).
bool decodeImageRgba8(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                      std::vector<uint8_t>& rgba, std::string& err);

}  // namespace cg

#endif
