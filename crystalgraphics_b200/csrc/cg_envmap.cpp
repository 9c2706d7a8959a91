// cg_envmap.cpp — the environment texture of a glTF image-based light.
//
// The reference loads EXT_lights_image_based's first specular cube (six
// images) and resamples it into the lat-long RGBA32F environment the shader
// reads (src/scene.cpp:541-625, LoadImageBasedEnvironmentTexture /
// CubeToEnvironmentTexture), decoding the faces with stb_image's float loader
// (src/image_decode.cpp:51-88).  stb_image is not available here, so the two
// formats are decoded by this file (Radiance HDR) and cg_png.cpp /
// cg_jpeg.cpp (PNG, JPEG), and stb's 8-bit-to-float rule is restated.
#include "cg_envmap.h"

#include <cmath>
#include <cstdio>
#include <cstring>

#include "cg_jpeg.h"

namespace cg {
namespace {

// One header line (without its newline); false at the end of the data.
bool headerLine(const uint8_t* data, size_t size, size_t& pos, std::string& line) {
  if (pos >= size) return false;
  line.clear();
  while (pos < size && data[pos] != '\n') line.push_back(static_cast<char>(data[pos++]));
  if (pos < size) ++pos;  // the newline
  return true;
}

// RGBE -> linear float (mantissa * 2^(exponent - 136); exponent 0 is black).
void rgbeToFloat(const uint8_t e[4], float* out) {
  if (e[3] == 0) {
    out[0] = out[1] = out[2] = 0.0f;
  } else {
    const float f = std::ldexp(1.0f, static_cast<int>(e[3]) - (128 + 8));
    out[0] = static_cast<float>(e[0]) * f;
    out[1] = static_cast<float>(e[1]) * f;
    out[2] = static_cast<float>(e[2]) * f;
  }
  out[3] = 1.0f;
}

}  // namespace

bool decodeRadianceHdr(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                       std::vector<float>& rgba, std::string& err) {
  size_t pos = 0;
  std::string line;
  if (!headerLine(data, size, pos, line) || (line != "#?RADIANCE" && line != "#?RGBE")) {
    err = "not a Radiance HDR image";
    return false;
  }
  bool format_ok = false;
  while (true) {
    if (!headerLine(data, size, pos, line)) {
      err = "truncated HDR header";
      return false;
    }
    if (line.empty()) break;
    if (line == "FORMAT=32-bit_rle_rgbe") format_ok = true;
  }
  if (!format_ok) {
    err = "unsupported HDR format (only 32-bit_rle_rgbe)";
    return false;
  }
  if (!headerLine(data, size, pos, line)) {
    err = "missing HDR resolution line";
    return false;
  }
  long h = 0, w = 0;
  char tail = 0;
  if (std::sscanf(line.c_str(), "-Y %ld +X %ld%c", &h, &w, &tail) != 2 || h <= 0 || w <= 0 ||
      h > (1 << 15) || w > (1 << 15)) {
    err = "unsupported HDR resolution line (only \"-Y height +X width\")";
    return false;
  }
  width = static_cast<uint32_t>(w);
  height = static_cast<uint32_t>(h);
  rgba.assign(size_t(width) * height * 4, 0.0f);
  std::vector<uint8_t> scan(size_t(width) * 4);
  for (uint32_t y = 0; y < height; ++y) {
    float* row = rgba.data() + size_t(y) * width * 4;
    // a run-length-encoded scanline starts with 2, 2, then the width
    const bool rle = width >= 8 && width < 32768 && pos + 4 <= size && data[pos] == 2 &&
                     data[pos + 1] == 2 && (data[pos + 2] & 0x80) == 0;
    if (!rle) {
      if (pos + size_t(width) * 4 > size) {
        err = "truncated HDR pixels";
        return false;
      }
      for (uint32_t x = 0; x < width; ++x) rgbeToFloat(data + pos + size_t(x) * 4, row + x * 4);
      pos += size_t(width) * 4;
      continue;
    }
    if ((uint32_t(data[pos + 2]) << 8 | data[pos + 3]) != width) {
      err = "HDR scanline width mismatch";
      return false;
    }
    pos += 4;
    for (int c = 0; c < 4; ++c) {  // each component's bytes, run-length encoded
      uint32_t x = 0;
      while (x < width) {
        if (pos >= size) {
          err = "truncated HDR scanline";
          return false;
        }
        uint32_t count = data[pos++];
        if (count > 128) {  // a run of one value
          count -= 128;
          if (count > width - x || pos >= size) {
            err = "bad HDR run";
            return false;
          }
          const uint8_t v = data[pos++];
          for (uint32_t k = 0; k < count; ++k) scan[size_t(x++) * 4 + c] = v;
        } else {  // `count` literal values
          if (count == 0 || count > width - x || pos + count > size) {
            err = "bad HDR literal run";
            return false;
          }
          for (uint32_t k = 0; k < count; ++k) scan[size_t(x++) * 4 + c] = data[pos++];
        }
      }
    }
    for (uint32_t x = 0; x < width; ++x) rgbeToFloat(scan.data() + size_t(x) * 4, row + x * 4);
  }
  return true;
}

bool decodeImageRgba32f(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                        std::vector<float>& rgba, std::string& err) {
  if (size >= 2 && data[0] == '#' && data[1] == '?')
    return decodeRadianceHdr(data, size, width, height, rgba, err);
  std::vector<uint8_t> px;
  if (!decodeImageRgba8(data, size, width, height, px, err)) return false;
  // stb_image's LDR -> float (stbi__ldr_to_hdr with its default gamma 2.2 and
  // scale 1): colour channels (c / 255)^2.2, alpha c / 255.  The reference
  // compiles stb in a C++ file, where pow(float, float) is the float overload.
  rgba.resize(px.size());
  for (size_t i = 0; i < px.size(); ++i) {
    const float c = static_cast<float>(px[i]) / 255.0f;
    rgba[i] = (i & 3u) == 3u ? c : std::pow(c, 2.2f) * 1.0f;
  }
  return true;
}

namespace {

struct F3 {
  float x, y, z;
};
F3 cross3(F3 a, F3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}

// Rotation of `d` by the quaternion (x, y, z, w), normalised first
// (RotateVector, scene.cpp:524-535): d + w t + q x t with t = 2 q x d.
F3 rotateByQuaternion(const float q[4], F3 d) {
  F3 im{q[0], q[1], q[2]};
  float re = q[3];
  const float norm = im.x * im.x + im.y * im.y + im.z * im.z + re * re;
  if (norm <= 0.0f) return d;
  const float len = std::sqrt(norm);
  im = {im.x / len, im.y / len, im.z / len};
  re = re / len;
  const F3 c = cross3(im, d);
  const F3 t{2.0f * c.x, 2.0f * c.y, 2.0f * c.z};
  const F3 u = cross3(im, t);
  return {d.x + re * t.x + u.x, d.y + re * t.y + u.y, d.z + re * t.z + u.z};
}

// Nearest texel of a face at (s, t) in [0, 1] (ImageTexel, scene.cpp:460-476).
const float* faceTexel(const float* face, uint32_t w, uint32_t h, float s, float t) {
  s = std::fmin(std::fmax(s, 0.0f), 1.0f);
  t = std::fmin(std::fmax(t, 0.0f), 1.0f);
  uint32_t x = static_cast<uint32_t>(s * static_cast<float>(w));
  uint32_t y = static_cast<uint32_t>(t * static_cast<float>(h));
  if (x > w - 1) x = w - 1;
  if (y > h - 1) y = h - 1;
  return face + (size_t(y) * w + x) * 4;
}

// The face a direction leaves the cube through and the texel it meets there
// (SampleCube, scene.cpp:478-518): the dominant axis picks the face (ties
// favour x, then y), each face has its own (s, t) parameterisation, and the
// image is read at (1 - s, 1 - t).
const float* cubeTexel(const float* const faces[6], uint32_t w, uint32_t h, F3 d) {
  const float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
  int face;
  float s, t;
  if (ax >= ay && ax >= az) {
    face = d.x >= 0.0f ? 1 : 0;
    s = ((d.x >= 0.0f ? -d.z : d.z) / ax + 1.0f) * 0.5f;
    t = (-d.y / ax + 1.0f) * 0.5f;
  } else if (ay >= az) {
    face = d.y >= 0.0f ? 2 : 3;
    s = (d.x / ay + 1.0f) * 0.5f;
    t = ((d.y >= 0.0f ? d.z : -d.z) / ay + 1.0f) * 0.5f;
  } else {
    face = d.z >= 0.0f ? 4 : 5;
    s = ((d.z >= 0.0f ? d.x : -d.x) / az + 1.0f) * 0.5f;
    t = (1.0f - d.y / az) * 0.5f;
  }
  return faceTexel(faces[face], w, h, 1.0f - s, 1.0f - t);
}

}  // namespace

void cubeToLatLong(const float* const faces[6], uint32_t face_width, uint32_t face_height,
                   const float rotation[4], std::vector<float>& out) {
  constexpr float kPi = 3.14159265358979323846f;
  const uint32_t W = face_width * 4, H = face_height * 2;
  out.assign(size_t(W) * H * 4, 0.0f);
  const float inverse[4] = {-rotation[0], -rotation[1], -rotation[2], rotation[3]};
  for (uint32_t y = 0; y < H; ++y) {
    const float v = (static_cast<float>(y) + 0.5f) / static_cast<float>(H);
    const float theta = v * kPi;
    const float sin_theta = std::sin(theta);
    const float z = std::cos(theta);
    for (uint32_t x = 0; x < W; ++x) {
      const float u = (static_cast<float>(x) + 0.5f) / static_cast<float>(W);
      const float phi = (u - 0.5f) * 2.0f * kPi;
      // engine direction (z up) -> glTF (y up): (x, -z, y); then into the
      // image's frame through the inverse of the light's rotation
      const F3 engine{std::cos(phi) * sin_theta, std::sin(phi) * sin_theta, z};
      const F3 gltf{engine.x, -engine.z, engine.y};
      const float* c = cubeTexel(faces, face_width, face_height, rotateByQuaternion(inverse, gltf));
      float* o = out.data() + (size_t(y) * W + x) * 4;
      o[0] = c[0];
      o[1] = c[1];
      o[2] = c[2];
      o[3] = 1.0f;
    }
  }
}

}  // namespace cg
