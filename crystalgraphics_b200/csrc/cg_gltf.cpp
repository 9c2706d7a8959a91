// cg_gltf.cpp — glTF 2.0 loader for LoadScene(path).
//
// The reference loads glTF through cgltf v1.14 (src/scene.cpp:829-1003; the
// library is fetched at build time by lib/cgltf/CMakeLists.txt), which is not
// available here, so this is a self-contained reader of the subset the path
// tracer consumes, with the reference's conventions:
//   - material 0 is the default material, glTF material i becomes i + 1, a
//     primitive without a material uses 0 (scene.cpp:869-872, 952-956);
//   - the default material is glTF's defaults (scene.cpp:659-690);
//   - POSITION / NORMAL / TEXCOORD_0 / TEXCOORD_1 and indices per primitive,
//     indices made absolute (scene.cpp:876-967); a primitive without indices
//     contributes no triangles;
//   - one instance per (node, mesh primitive) in depth-first node order,
//     node matrix or TRS (scene.cpp:972-995);
//   - the y-up glTF world is rotated by +90 degrees about x to z-up
//     (scene.cpp:1000).
// Supported: .gltf with external .bin or base64 data URIs, and .glb.
//   - sparse accessors read as zeros, as cgltf's per-element readers return
//     them (see readAccessor).
// Material extensions read: KHR_materials_emissive_strength, _ior,
// _transmission, _volume (thickness), _dispersion; the four textures the
// shader samples; EXT_lights_image_based (the environment).
#include <array>
#include <cmath>
#include <cstring>
#include <utility>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cg_cuda.h"
#include "cg_api_internal.h"

#include "cg_envmap.h"
#include "cg_jpeg.h"
#include "cg_png.h"

namespace cg {
namespace {

// ---- minimal JSON -----------------------------------------------------------
struct Json {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double n = 0.0;
  std::string s;
  std::vector<Json> a;
  std::map<std::string, Json> o;

  const Json* get(const std::string& k) const {
    if (kind != Obj) return nullptr;
    auto it = o.find(k);
    return it == o.end() ? nullptr : &it->second;
  }
  double num(const std::string& k, double def) const {
    const Json* j = get(k);
    return (j && j->kind == Num) ? j->n : def;
  }
  // The number truncated to an integer, clamped to +-2^53 (exact in a
  // double) so that the conversion is defined and a sum of two cannot overflow.
  int64_t asInt() const {
    constexpr double kLim = 9007199254740992.0;
    return static_cast<int64_t>(std::fmax(-kLim, std::fmin(n, kLim)));
  }
  int64_t integer(const std::string& k, int64_t def) const {
    const Json* j = get(k);
    return j && j->kind == Num ? j->asInt() : def;
  }
};

// [off, off + len) lies inside [0, limit).
bool within(int64_t off, int64_t len, size_t limit) {
  return off >= 0 && len >= 0 && uint64_t(off) <= limit && uint64_t(len) <= limit - uint64_t(off);
}

struct Parser {
  const char* p;
  const char* end;
  std::string err;
  int depth = 0;  // open arrays and objects; bounded so that recursion cannot exhaust the stack
  static constexpr int kMaxDepth = 256;

  void ws() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  bool parse(Json& out) {
    ws();
    if (p >= end) return fail("unexpected end");
    char c = *p;
    if (c == '{' || c == '[') {
      if (++depth > kMaxDepth) return fail("JSON nested too deeply");
      const bool ok = c == '{' ? object(out) : array(out);
      --depth;
      return ok;
    }
    if (c == '"') {
      out.kind = Json::Str;
      return string(out.s);
    }
    if (c == 't' || c == 'f' || c == 'n') return literal(out);
    return number(out);
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m;
    return false;
  }
  bool literal(Json& out) {
    auto match = [&](const char* w) {
      size_t n = std::strlen(w);
      if (size_t(end - p) >= n && std::strncmp(p, w, n) == 0) {
        p += n;
        return true;
      }
      return false;
    };
    if (match("true")) {
      out.kind = Json::Bool;
      out.b = true;
      return true;
    }
    if (match("false")) {
      out.kind = Json::Bool;
      out.b = false;
      return true;
    }
    if (match("null")) {
      out.kind = Json::Null;
      return true;
    }
    return fail("bad literal");
  }
  bool number(Json& out) {
    // the JSON number grammar's characters, copied so that strtod cannot read
    // past the end of the text (a GLB's JSON chunk is not NUL-terminated)
    char buf[64];
    size_t n = 0;
    while (p + n < end && n < sizeof(buf) - 1 && std::strchr("0123456789+-.eE", p[n]) && p[n]) {
      buf[n] = p[n];
      ++n;
    }
    buf[n] = '\0';
    char* e = nullptr;
    out.n = std::strtod(buf, &e);
    if (e == buf) return fail("bad number");
    p += e - buf;
    out.kind = Json::Num;
    return true;
  }
  bool string(std::string& s) {
    ++p;  // opening quote
    while (p < end && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= end) return fail("bad escape");
        char c = *p++;
        switch (c) {
          case 'n': s += '\n'; break;
          case 't': s += '\t'; break;
          case 'r': s += '\r'; break;
          case 'b': s += '\b'; break;
          case 'f': s += '\f'; break;
          case 'u': {
            if (end - p < 4) return fail("bad unicode escape");
            unsigned v = 0;
            for (int k = 0; k < 4; ++k, ++p) {
              const char h = *p;
              const int d = h >= '0' && h <= '9' ? h - '0' : h >= 'a' && h <= 'f' ? h - 'a' + 10
                          : h >= 'A' && h <= 'F' ? h - 'A' + 10 : -1;
              if (d < 0) return fail("bad unicode escape");
              v = v * 16 + unsigned(d);
            }
            if (v < 0x80) {
              s += static_cast<char>(v);
            } else if (v < 0x800) {
              s += static_cast<char>(0xC0 | (v >> 6));
              s += static_cast<char>(0x80 | (v & 0x3F));
            } else {
              s += static_cast<char>(0xE0 | (v >> 12));
              s += static_cast<char>(0x80 | ((v >> 6) & 0x3F));
              s += static_cast<char>(0x80 | (v & 0x3F));
            }
            break;
          }
          default: s += c;
        }
      } else {
        s += *p++;
      }
    }
    if (p >= end) return fail("unterminated string");
    ++p;
    return true;
  }
  bool array(Json& out) {
    out.kind = Json::Arr;
    ++p;
    ws();
    if (p < end && *p == ']') {
      ++p;
      return true;
    }
    while (true) {
      out.a.emplace_back();
      if (!parse(out.a.back())) return false;
      ws();
      if (p < end && *p == ',') {
        ++p;
        continue;
      }
      if (p < end && *p == ']') {
        ++p;
        return true;
      }
      return fail("expected , or ]");
    }
  }
  bool object(Json& out) {
    out.kind = Json::Obj;
    ++p;
    ws();
    if (p < end && *p == '}') {
      ++p;
      return true;
    }
    while (true) {
      ws();
      if (p >= end || *p != '"') return fail("expected key");
      std::string key;
      if (!string(key)) return false;
      ws();
      if (p >= end || *p != ':') return fail("expected :");
      ++p;
      if (!parse(out.o[key])) return false;
      ws();
      if (p < end && *p == ',') {
        ++p;
        continue;
      }
      if (p < end && *p == '}') {
        ++p;
        return true;
      }
      return fail("expected , or }");
    }
  }
};

std::vector<uint8_t> base64(const std::string& in) {
  auto val = [](char c) -> int {
    if (c >= 'A' && c <= 'Z') return c - 'A';
    if (c >= 'a' && c <= 'z') return c - 'a' + 26;
    if (c >= '0' && c <= '9') return c - '0' + 52;
    if (c == '+') return 62;
    if (c == '/') return 63;
    return -1;
  };
  std::vector<uint8_t> out;
  uint32_t acc = 0;
  int bits = 0;
  for (char c : in) {
    int v = val(c);
    if (v < 0) continue;
    acc = (acc << 6) | static_cast<uint32_t>(v);
    bits += 6;
    if (bits >= 8) {
      bits -= 8;
      out.push_back(static_cast<uint8_t>((acc >> bits) & 0xFF));
    }
  }
  return out;
}

// column-major 4x4 helpers (glTF convention)
struct M4 {
  double m[16];  // column-major
};
M4 identity() {
  M4 r{};
  for (int i = 0; i < 4; ++i) r.m[i * 5] = 1.0;
  return r;
}
M4 mul(const M4& a, const M4& b) {
  M4 r{};
  for (int c = 0; c < 4; ++c)
    for (int rr = 0; rr < 4; ++rr) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a.m[k * 4 + rr] * b.m[c * 4 + k];
      r.m[c * 4 + rr] = s;
    }
  return r;
}

struct Loader {
  Json doc;
  std::vector<std::vector<uint8_t>> buffers;
  std::string dir;
  std::string err;

  std::vector<cg_vertex> vertices;
  std::vector<uint32_t> indices;
  std::vector<cg_mesh> meshes;  // one per distinct primitive geometry
  // glTF mesh -> its primitives as (cg_mesh id, material index)
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> mesh_prims;
  // primitives that name the same accessors share one cg_mesh (and BLAS)
  std::map<std::array<int64_t, 5>, uint32_t> geometry_ids;
  std::vector<cg_instance> instances;
  std::vector<cg_material> materials;
  // decoded images (RGBA8) and one cg_texture per glTF texture pointing into them
  std::vector<std::vector<uint8_t>> image_rgba;
  std::vector<std::array<uint32_t, 2>> image_size;
  std::vector<cg_texture> textures;
  // the environment of an image-based light (lat-long RGBA32F), if any
  std::vector<float> env;
  uint32_t env_w = 0, env_h = 0;

  bool fail(const std::string& m) {
    if (err.empty()) err = m;
    return false;
  }

  bool loadBuffers(const std::vector<uint8_t>* glb_bin) {
    const Json* bs = doc.get("buffers");
    if (!bs) return true;
    for (size_t i = 0; i < bs->a.size(); ++i) {
      const Json& b = bs->a[i];
      const Json* uri = b.get("uri");
      if (!uri) {
        if (!glb_bin) return fail("buffer without uri outside a .glb");
        buffers.push_back(*glb_bin);
        continue;
      }
      const std::string& u = uri->s;
      if (u.rfind("data:", 0) == 0) {
        size_t comma = u.find(',');
        if (comma == std::string::npos) return fail("bad data uri");
        buffers.push_back(base64(u.substr(comma + 1)));
        continue;
      }
      std::ifstream f(dir + "/" + u, std::ios::binary);
      if (!f) return fail("cannot open buffer " + u);
      buffers.emplace_back((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    }
    return true;
  }

  // Elements allowed in an accessor without a bufferView (all zeros): 2^26,
  // far above any mesh's vertex count (a 1.3M-triangle sphere has 0.66M), so
  // that a damaged count fails instead of allocating gigabytes of zeros.
  static constexpr size_t kMaxZeroAccessor = size_t(1) << 26;

  // Reads accessor `idx` as `comps` floats per element (or as indices).
  bool readAccessor(int64_t idx, int comps, std::vector<double>& out, size_t& count) {
    const Json* acc = doc.get("accessors");
    if (!acc || idx < 0 || size_t(idx) >= acc->a.size()) return fail("bad accessor index");
    const Json& a = acc->a[idx];
    const int64_t n = a.integer("count", 0);
    if (n < 0 || n > int64_t(UINT32_MAX)) return fail("invalid accessor count");
    count = static_cast<size_t>(n);
    const int64_t ctype = a.integer("componentType", 5126);
    const bool normalized = a.get("normalized") && a.get("normalized")->b;
    const std::string type = a.get("type") ? a.get("type")->s : "SCALAR";
    int ncomp = type == "SCALAR" ? 1 : type == "VEC2" ? 2 : type == "VEC3" ? 3 : type == "VEC4" ? 4 : 0;
    if (ncomp == 0) return fail("unsupported accessor type " + type);
    int csize = (ctype == 5120 || ctype == 5121) ? 1 : (ctype == 5122 || ctype == 5123) ? 2 : 4;
    const size_t elem = size_t(ncomp * csize);
    const uint8_t* src = nullptr;
    size_t stride = elem;
    if (a.get("bufferView")) {
      const Json* bvs = doc.get("bufferViews");
      const int64_t bvi = a.integer("bufferView", -1);
      if (!bvs || bvi < 0 || size_t(bvi) >= bvs->a.size()) return fail("bad bufferView");
      const Json& bv = bvs->a[bvi];
      const int64_t bi = bv.integer("buffer", -1);
      if (bi < 0 || size_t(bi) >= buffers.size()) return fail("bad buffer index");
      const std::vector<uint8_t>& buf = buffers[bi];
      // the view inside its buffer and the accessor inside its view, the
      // checks cgltf_validate makes (before anything is allocated for it)
      const int64_t vo = bv.integer("byteOffset", 0), vl = bv.integer("byteLength", 0);
      const int64_t ao = a.integer("byteOffset", 0), bs = bv.integer("byteStride", 0);
      if (!within(vo, vl, buf.size())) return fail("bufferView exceeds its buffer");
      if (bs < 0 || bs > 252) return fail("invalid byteStride");
      if (bs) stride = size_t(bs);
      if (count && !within(ao, int64_t((count - 1) * stride + elem), size_t(vl)))
        return fail("accessor exceeds its buffer");
      src = buf.data() + size_t(vo + ao);
    } else if (count > kMaxZeroAccessor) {
      return fail("accessor without a bufferView has too many elements");
    }
    if (const Json* sp = a.get("sparse")) {
      // cgltf v1.14 (the reference's glTF library) validates the sparse
      // block, but its cgltf_accessor_read_float / cgltf_accessor_read_index
      // return without reading an element of a sparse accessor, so every
      // element of one reaches the reference's vertices and indices as the
      // zero they were resized to (src/scene.cpp:900-945).
      if (!checkSparse(*sp, count, elem)) return false;
      src = nullptr;
    }
    out.assign(count * comps, 0.0);
    if (!src) return true;  // all zeros
    for (size_t e = 0; e < count; ++e) {
      const uint8_t* el = src + e * stride;
      for (int c = 0; c < std::min(ncomp, comps); ++c) {
        const uint8_t* q = el + c * csize;
        double v = 0;
        switch (ctype) {
          case 5126: { float f; std::memcpy(&f, q, 4); v = f; break; }
          case 5125: { uint32_t u; std::memcpy(&u, q, 4); v = u; break; }
          // normalized integers divide in float, as cgltf does
          case 5123: { uint16_t u; std::memcpy(&u, q, 2); v = normalized ? u / 65535.0f : u; break; }
          case 5121: { uint8_t u = *q; v = normalized ? u / 255.0f : u; break; }
          case 5122: { int16_t s; std::memcpy(&s, q, 2); v = normalized ? std::max(s / 32767.0f, -1.0f) : s; break; }
          case 5120: { int8_t s = static_cast<int8_t>(*q); v = normalized ? std::max(s / 127.0f, -1.0f) : s; break; }
          default: return fail("unsupported component type");
        }
        out[e * comps + c] = v;
      }
    }
    return true;
  }

  // The sparse block of an accessor with `count` elements of `elem_bytes`:
  // its indices (unsigned, each below `count`) and values must lie in their
  // buffer views, the checks cgltf_validate makes.
  bool checkSparse(const Json& sp, size_t count, size_t elem_bytes) {
    const int64_t n = sp.integer("count", 0);
    const Json* ix = sp.get("indices");
    const Json* vs = sp.get("values");
    if (n < 1 || size_t(n) > count || !ix || !vs) return fail("invalid sparse accessor");
    const int64_t ct = ix->integer("componentType", 0);
    const size_t isz = ct == 5121 ? 1 : ct == 5123 ? 2 : ct == 5125 ? 4 : 0;
    if (!isz) return fail("invalid sparse accessor index type");
    const uint8_t* idx = viewBytes(ix->integer("bufferView", -1), ix->integer("byteOffset", 0), size_t(n) * isz);
    if (!idx || !viewBytes(vs->integer("bufferView", -1), vs->integer("byteOffset", 0), size_t(n) * elem_bytes))
      return fail("sparse accessor data exceeds its buffer view");
    for (int64_t k = 0; k < n; ++k) {
      uint32_t v = 0;
      std::memcpy(&v, idx + size_t(k) * isz, isz);  // little-endian
      if (size_t(v) >= count) return fail("invalid sparse accessor index");
    }
    return true;
  }

  // `size` bytes at `offset` in buffer view `bvi`, or null when they do not
  // lie inside the view and its buffer.
  const uint8_t* viewBytes(int64_t bvi, int64_t offset, size_t size) {
    const Json* bvs = doc.get("bufferViews");
    if (!bvs || bvi < 0 || size_t(bvi) >= bvs->a.size() || offset < 0) return nullptr;
    const Json& bv = bvs->a[bvi];
    const int64_t bi = bv.integer("buffer", -1);
    if (bi < 0 || size_t(bi) >= buffers.size()) return nullptr;
    const int64_t vo = bv.integer("byteOffset", 0), vl = bv.integer("byteLength", 0);
    if (!within(vo, vl, buffers[bi].size()) || !within(offset, int64_t(size), size_t(vl))) return nullptr;
    return buffers[bi].data() + size_t(vo + offset);
  }

  int32_t textureIndex(const Json* info) {
    if (!info) return -1;
    return static_cast<int32_t>(info->integer("index", -1));
  }
  // bit `slot` of texcoord_sets: textureInfo.texCoord == 1 (textureUv, material.wesl:174-179)
  static uint32_t texCoordBit(const Json* info, int slot) {
    return info && info->integer("texCoord", 0) == 1 ? (1u << slot) : 0u;
  }

  // Bytes of an image: a data URI, a file next to the glTF, or a bufferView.
  bool imageBytes(const Json& img, std::vector<uint8_t>& out) {
    if (const Json* uri = img.get("uri")) {
      const std::string& u = uri->s;
      if (u.rfind("data:", 0) == 0) {
        const size_t comma = u.find(',');
        if (comma == std::string::npos) return fail("bad image data uri");
        out = base64(u.substr(comma + 1));
        return true;
      }
      std::ifstream f(dir + "/" + u, std::ios::binary);
      if (!f) return fail("cannot open image " + u);
      out.assign((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
      return true;
    }
    const Json* bvs = doc.get("bufferViews");
    const int64_t bvi = img.integer("bufferView", -1);
    if (!bvs || bvi < 0 || size_t(bvi) >= bvs->a.size()) return fail("image without uri or bufferView");
    const Json& bv = bvs->a[bvi];
    const int64_t bi = bv.integer("buffer", -1);
    if (bi < 0 || size_t(bi) >= buffers.size()) return fail("bad buffer index");
    const int64_t off = bv.integer("byteOffset", 0), len = bv.integer("byteLength", 0);
    if (!within(off, len, buffers[bi].size())) return fail("image bufferView exceeds its buffer");
    out.assign(buffers[bi].begin() + off, buffers[bi].begin() + off + len);
    return true;
  }

  // Every glTF texture: its source image decoded to RGBA8 (the reference's
  // DecodeImageRgba8 with stb) and its sampler's wrap modes (default repeat).
  bool loadTextures() {
    const Json* ts = doc.get("textures");
    if (!ts) return true;
    const Json* imgs = doc.get("images");
    const Json* samplers = doc.get("samplers");
    const size_t nimg = imgs ? imgs->a.size() : 0;
    image_rgba.assign(nimg, {});
    image_size.assign(nimg, {0u, 0u});
    for (size_t t = 0; t < ts->a.size(); ++t) {
      const Json& tj = ts->a[t];
      const int64_t src = tj.integer("source", -1);
      if (src < 0 || size_t(src) >= nimg)
        return fail("texture " + std::to_string(t) + " has no image source");
      if (image_rgba[src].empty()) {
        std::vector<uint8_t> bytes;
        if (!imageBytes(imgs->a[src], bytes)) return false;
        std::string e;
        uint32_t w = 0, h = 0;
        if (!decodeImageRgba8(bytes.data(), bytes.size(), w, h, image_rgba[src], e))
          return fail("image " + std::to_string(src) + ": " + e);
        image_size[src] = {w, h};
      }
      cg_texture tx{};
      tx.width = image_size[src][0];
      tx.height = image_size[src][1];
      tx.rgba8 = image_rgba[src].data();
      tx.wrap_s = tx.wrap_t = 10497;
      const int64_t si = tj.integer("sampler", -1);
      if (samplers && si >= 0 && size_t(si) < samplers->a.size()) {
        tx.wrap_s = static_cast<int32_t>(samplers->a[si].integer("wrapS", 10497));
        tx.wrap_t = static_cast<int32_t>(samplers->a[si].integer("wrapT", 10497));
      }
      textures.push_back(tx);
    }
    return true;
  }

  // EXT_lights_image_based: the first specular cube (six images, the first
  // mip level) and the first rotation, resampled to the lat-long environment
  // (LoadImageBasedEnvironmentTexture, src/scene.cpp:588-625; the reference
  // finds both by searching the extension's JSON text for the first
  // "specularImages" and "rotation" keys).  No light, no complete image set:
  // no environment (the fallback sky is used).
  bool loadImageBasedLight() {
    const Json* ext = doc.get("extensions");
    const Json* ibl = ext ? ext->get("EXT_lights_image_based") : nullptr;
    const Json* lights = ibl ? ibl->get("lights") : nullptr;
    if (!lights || lights->kind != Json::Arr) return true;
    const Json* set = nullptr;
    float rotation[4] = {0.0f, 0.0f, 0.0f, 1.0f};
    bool have_rotation = false;
    for (const Json& l : lights->a) {
      const Json* si = l.get("specularImages");
      if (!set && si && si->kind == Json::Arr && !si->a.empty() && si->a[0].kind == Json::Arr &&
          si->a[0].a.size() >= 6)
        set = &si->a[0];
      const Json* r = l.get("rotation");
      if (!have_rotation && r && r->kind == Json::Arr && r->a.size() == 4) {
        for (int k = 0; k < 4; ++k) rotation[k] = static_cast<float>(r->a[k].n);
        have_rotation = true;
      }
    }
    if (!set) return true;
    const Json* imgs = doc.get("images");
    const size_t nimg = imgs ? imgs->a.size() : 0;
    std::vector<float> faces[6];
    uint32_t fw = 0, fh = 0;
    for (int i = 0; i < 6; ++i) {
      const Json& e = set->a[i];
      if (e.kind != Json::Num || e.n < 0 || e.n != static_cast<double>(e.asInt()))
        return true;  // not an image index: the reference reads no image set
      const size_t index = static_cast<size_t>(e.n);
      if (index >= nimg) return fail("Image based light references an invalid image.");
      std::vector<uint8_t> bytes;
      if (!imageBytes(imgs->a[index], bytes)) return false;
      uint32_t w = 0, h = 0;
      std::string err;
      if (!decodeImageRgba32f(bytes.data(), bytes.size(), w, h, faces[i], err))
        return fail("image " + std::to_string(index) + ": " + err);
      if (w == 0 || h == 0) return fail("Image based light has an empty cube face.");
      if (i > 0 && (w != fw || h != fh))
        return fail("Image based light cube faces do not share one size.");
      fw = w;
      fh = h;
    }
    const float* fp[6];
    for (int i = 0; i < 6; ++i) fp[i] = faces[i].data();
    cubeToLatLong(fp, fw, fh, rotation, env);
    env_w = fw * 4;
    env_h = fh * 2;
    return true;
  }

  void loadMaterials() {
    auto def = [] {
      cg_material m{};
      for (int k = 0; k < 4; ++k) m.base_color_factor[k] = 1.0f;
      m.emissive_strength = 1.0f;
      m.metallic_factor = 1.0f;
      m.roughness_factor = 1.0f;
      m.ior = 1.5f;
      m.base_color_texture = m.metallic_roughness_texture = m.emissive_texture =
          m.transmission_texture = -1;
      return m;
    };
    materials.push_back(def());
    const Json* ms = doc.get("materials");
    if (!ms) return;
    for (const Json& mj : ms->a) {
      cg_material m = def();
      if (const Json* pbr = mj.get("pbrMetallicRoughness")) {
        if (const Json* bc = pbr->get("baseColorFactor"))
          for (size_t k = 0; k < 4 && k < bc->a.size(); ++k)
            m.base_color_factor[k] = static_cast<float>(bc->a[k].n);
        m.metallic_factor = static_cast<float>(pbr->num("metallicFactor", 1.0));
        m.roughness_factor = static_cast<float>(pbr->num("roughnessFactor", 1.0));
        m.base_color_texture = textureIndex(pbr->get("baseColorTexture"));
        m.metallic_roughness_texture = textureIndex(pbr->get("metallicRoughnessTexture"));
        m.texcoord_sets |= texCoordBit(pbr->get("baseColorTexture"), 0) |
                           texCoordBit(pbr->get("metallicRoughnessTexture"), 1);
      }
      if (const Json* ef = mj.get("emissiveFactor"))
        for (size_t k = 0; k < 3 && k < ef->a.size(); ++k)
          m.emissive_factor[k] = static_cast<float>(ef->a[k].n);
      m.emissive_texture = textureIndex(mj.get("emissiveTexture"));
      m.texcoord_sets |= texCoordBit(mj.get("emissiveTexture"), 2);
      if (const Json* ext = mj.get("extensions")) {
        if (const Json* e = ext->get("KHR_materials_emissive_strength"))
          m.emissive_strength = static_cast<float>(e->num("emissiveStrength", 1.0));
        if (const Json* e = ext->get("KHR_materials_ior"))
          m.ior = static_cast<float>(e->num("ior", 1.5));
        if (const Json* e = ext->get("KHR_materials_dispersion"))
          m.dispersion = static_cast<float>(e->num("dispersion", 0.0));
        if (const Json* e = ext->get("KHR_materials_transmission")) {
          m.transmission_factor = static_cast<float>(e->num("transmissionFactor", 0.0));
          m.transmission_texture = textureIndex(e->get("transmissionTexture"));
          m.texcoord_sets |= texCoordBit(e->get("transmissionTexture"), 3);
        }
        if (const Json* e = ext->get("KHR_materials_volume"))
          m.thickness_factor = static_cast<float>(e->num("thicknessFactor", 0.0));
      }
      materials.push_back(m);
    }
  }

  bool loadMeshes() {
    const Json* ms = doc.get("meshes");
    if (!ms) return true;
    for (const Json& mesh : ms->a) {
      mesh_prims.emplace_back();
      const Json* prims = mesh.get("primitives");
      if (!prims) continue;
      for (const Json& pr : prims->a) {
        if (pr.integer("mode", 4) != 4) return fail("only triangle primitives are supported");
        const Json* attrs = pr.get("attributes");
        if (!attrs || !attrs->get("POSITION")) return fail("primitive without POSITION");
        const int64_t mat = pr.integer("material", -1);
        const uint32_t mat_idx = mat >= 0 ? static_cast<uint32_t>(mat + 1) : 0u;
        const std::array<int64_t, 5> key = {attrs->integer("POSITION", -1), attrs->integer("NORMAL", -1),
                                            attrs->integer("TEXCOORD_0", -1),
                                            attrs->integer("TEXCOORD_1", -1), pr.integer("indices", -1)};
        auto seen = geometry_ids.find(key);
        if (seen != geometry_ids.end()) {
          mesh_prims.back().push_back({seen->second, mat_idx});
          continue;
        }
        std::vector<double> pos, nrm, uv0, uv1, idx;
        size_t nv = 0, n2 = 0;
        if (!readAccessor(attrs->integer("POSITION", -1), 3, pos, nv)) return false;
        const uint32_t voff = static_cast<uint32_t>(vertices.size());
        vertices.resize(vertices.size() + nv);
        auto fill = [&](const char* name, int comps, int which) -> bool {
          if (!attrs->get(name)) return true;
          std::vector<double> d;
          if (!readAccessor(attrs->integer(name, -1), comps, d, n2)) return false;
          for (size_t v = 0; v < std::min(nv, n2); ++v) {
            cg_vertex& vx = vertices[voff + v];
            float* dst = which == 0 ? vx.normal : which == 1 ? vx.tex_coord0 : vx.tex_coord1;
            for (int c = 0; c < comps; ++c) dst[c] = static_cast<float>(d[v * comps + c]);
          }
          return true;
        };
        for (size_t v = 0; v < nv; ++v)
          for (int c = 0; c < 3; ++c) vertices[voff + v].position[c] = static_cast<float>(pos[v * 3 + c]);
        if (!fill("NORMAL", 3, 0) || !fill("TEXCOORD_0", 2, 1) || !fill("TEXCOORD_1", 2, 2))
          return false;
        const uint32_t ioff = static_cast<uint32_t>(indices.size());
        size_t ni = 0;
        if (pr.get("indices")) {
          if (!readAccessor(pr.integer("indices", -1), 1, idx, ni)) return false;
          for (size_t k = 0; k < ni; ++k) {
            const double iv = idx[k];
            if (iv < 0 || iv >= double(nv)) return fail("index out of range in a primitive");
            indices.push_back(static_cast<uint32_t>(iv) + voff);
          }
        }
        cg_mesh m{voff, static_cast<uint32_t>(nv), ioff, static_cast<uint32_t>(ni)};
        const uint32_t id = static_cast<uint32_t>(meshes.size());
        geometry_ids[key] = id;
        mesh_prims.back().push_back({id, mat_idx});
        meshes.push_back(m);
      }
    }
    return true;
  }

  M4 nodeTransform(const Json& n) {
    if (const Json* mj = n.get("matrix")) {
      M4 r = identity();
      for (size_t k = 0; k < 16 && k < mj->a.size(); ++k) r.m[k] = mj->a[k].n;
      return r;
    }
    double t[3] = {0, 0, 0}, q[4] = {0, 0, 0, 1}, s[3] = {1, 1, 1};
    if (const Json* tj = n.get("translation"))
      for (size_t k = 0; k < 3 && k < tj->a.size(); ++k) t[k] = tj->a[k].n;
    if (const Json* rj = n.get("rotation"))
      for (size_t k = 0; k < 4 && k < rj->a.size(); ++k) q[k] = rj->a[k].n;
    if (const Json* sj = n.get("scale"))
      for (size_t k = 0; k < 3 && k < sj->a.size(); ++k) s[k] = sj->a[k].n;
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)},
                            {2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)},
                            {2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)}};
    M4 r = identity();
    for (int c = 0; c < 3; ++c)
      for (int rr = 0; rr < 3; ++rr) r.m[c * 4 + rr] = R[rr][c] * s[c];
    for (int rr = 0; rr < 3; ++rr) r.m[12 + rr] = t[rr];
    return r;
  }

  // Every node has at most one parent and the parent links form no loop, as
  // cgltf v1.14 checks while it parses and validates a file (the reference
  // loads through cgltf_parse_file and cgltf_validate, src/scene.cpp:838-850).
  // It also keeps the walk below linear in the number of nodes: a node shared
  // by two parents at every level would otherwise multiply the paths.
  bool checkHierarchy() {
    const Json* ns = doc.get("nodes");
    if (!ns) return true;
    const size_t n = ns->a.size();
    std::vector<int64_t> parent(n, -1);
    for (size_t i = 0; i < n; ++i)
      if (const Json* ch = ns->a[i].get("children"))
        for (const Json& c : ch->a) {
          const int64_t k = c.asInt();
          if (k < 0 || size_t(k) >= n) return fail("bad node index");
          if (parent[k] >= 0) return fail("node " + std::to_string(k) + " has two parents");
          parent[k] = int64_t(i);
        }
    // 0 = not seen, 1 = on the chain being followed, 2 = reaches a root
    std::vector<uint8_t> state(n, 0);
    std::vector<int64_t> chain;
    for (size_t i = 0; i < n; ++i) {
      chain.clear();
      int64_t k = int64_t(i);
      while (k >= 0 && state[k] == 0) {
        state[k] = 1;
        chain.push_back(k);
        k = parent[k];
      }
      if (k >= 0 && state[k] == 1) return fail("node hierarchy has a cycle");
      for (int64_t c : chain) state[c] = 2;
    }
    return true;
  }

  bool walk(int64_t node, const M4& parent, int depth) {
    const Json* ns = doc.get("nodes");
    if (!ns || node < 0 || size_t(node) >= ns->a.size()) return fail("bad node index");
    if (depth > 256) return fail("node hierarchy too deep (cycle?)");
    const Json& n = ns->a[node];
    const M4 world = mul(parent, nodeTransform(n));
    const int64_t mesh = n.integer("mesh", -1);
    if (mesh >= 0) {
      if (size_t(mesh) >= mesh_prims.size()) return fail("bad mesh index");
      for (const auto& [geom, mat] : mesh_prims[mesh]) {
        cg_instance in{};
        for (int rr = 0; rr < 3; ++rr)
          for (int c = 0; c < 4; ++c) in.world_from_local[rr * 4 + c] = static_cast<float>(world.m[c * 4 + rr]);
        in.mesh = geom;
        in.material = mat < materials.size() ? mat : 0u;
        instances.push_back(in);
      }
    }
    if (const Json* ch = n.get("children"))
      for (const Json& c : ch->a)
        if (!walk(c.asInt(), world, depth + 1)) return false;
    return true;
  }

  bool load(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return fail("cannot open " + path);
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t slash = path.find_last_of('/');
    dir = slash == std::string::npos ? "." : path.substr(0, slash);
    std::string json;
    std::vector<uint8_t> bin;
    bool glb = bytes.size() >= 12 && std::memcmp(bytes.data(), "glTF", 4) == 0;
    if (glb) {
      size_t off = 12;
      while (off + 8 <= bytes.size()) {
        uint32_t len, type;
        std::memcpy(&len, &bytes[off], 4);
        std::memcpy(&type, &bytes[off + 4], 4);
        if (off + 8 + len > bytes.size()) return fail("truncated .glb chunk");
        if (type == 0x4E4F534Au) json.assign(reinterpret_cast<char*>(&bytes[off + 8]), len);
        if (type == 0x004E4942u) bin.assign(bytes.begin() + off + 8, bytes.begin() + off + 8 + len);
        off += 8 + len;
      }
    } else {
      json.assign(bytes.begin(), bytes.end());
    }
    Parser p{json.data(), json.data() + json.size(), {}};
    if (!p.parse(doc)) return fail("invalid JSON: " + p.err);
    if (!loadBuffers(glb ? &bin : nullptr)) return false;
    if (!loadTextures()) return false;
    if (!loadImageBasedLight()) return false;
    loadMaterials();
    if (!loadMeshes()) return false;
    // root: Rx(+90 deg), glTF y-up -> z-up (scene.cpp:1000)
    M4 root = identity();
    root.m[5] = 0.0;   // column 1: (0, 0, 1)
    root.m[6] = 1.0;
    root.m[9] = -1.0;  // column 2: (0, -1, 0)
    root.m[10] = 0.0;
    if (!checkHierarchy()) return false;
    const Json* scenes = doc.get("scenes");
    int64_t sc = doc.integer("scene", 0);
    if (scenes && !scenes->a.empty()) {
      if (sc < 0 || size_t(sc) >= scenes->a.size()) sc = 0;
      if (const Json* nodes = scenes->a[sc].get("nodes"))
        for (const Json& n : nodes->a)
          if (!walk(n.asInt(), root, 0)) return false;
    }
    return true;
  }
};

}  // namespace
}  // namespace cg

using namespace cg;

extern "C" CG_API int cg_gltf_parse(const char* path, cg_scene_desc* out, void** storage) {
  return guarded([&]() -> int {
    if (!path || !out || !storage) return fail(CG_E_INVALID, "null argument");
    *storage = nullptr;
    auto L = std::make_unique<Loader>();
    if (!L->load(path)) return fail(CG_E_INVALID, std::string(path) + ": " + L->err);
    cg_scene_desc d{};
    d.vertices = L->vertices.data();
    d.vertex_count = static_cast<uint32_t>(L->vertices.size());
    d.indices = L->indices.data();
    d.index_count = static_cast<uint32_t>(L->indices.size());
    d.meshes = L->meshes.data();
    d.mesh_count = static_cast<uint32_t>(L->meshes.size());
    d.instances = L->instances.data();
    d.instance_count = static_cast<uint32_t>(L->instances.size());
    d.materials = L->materials.data();
    d.material_count = static_cast<uint32_t>(L->materials.size());
    d.textures = L->textures.data();
    d.texture_count = static_cast<uint32_t>(L->textures.size());
    if (!L->env.empty()) {
      d.env_rgba32f = L->env.data();
      d.env_width = L->env_w;
      d.env_height = L->env_h;
    }
    *out = d;
    *storage = L.release();
    return CG_OK;
  });
}

extern "C" CG_API int cg_png_decode(const uint8_t* data, size_t size, uint32_t* width,
                                     uint32_t* height, uint8_t* rgba_out) {
  return guarded([&]() -> int {
    if (!data || !width || !height) return fail(CG_E_INVALID, "null argument");
    std::vector<uint8_t> rgba;
    std::string err;
    uint32_t w = 0, h = 0;
    if (!decodePng(data, size, w, h, rgba, err)) return fail(CG_E_INVALID, err);
    *width = w;
    *height = h;
    if (rgba_out) std::memcpy(rgba_out, rgba.data(), rgba.size());
    return CG_OK;
  });
}

extern "C" CG_API int cg_jpeg_decode(const uint8_t* data, size_t size, uint32_t* width,
                                    uint32_t* height, uint8_t* rgba_out) {
  return guarded([&]() -> int {
    if (!data || !width || !height) return fail(CG_E_INVALID, "null argument");
    std::vector<uint8_t> px;
    std::string e;
    uint32_t w = 0, h = 0;
    if (!decodeJpeg(data, size, w, h, px, e)) return fail(CG_E_INVALID, e);
    *width = w;
    *height = h;
    if (rgba_out) std::memcpy(rgba_out, px.data(), px.size());
    return CG_OK;
  });
}

extern "C" CG_API int cg_hdr_decode(const uint8_t* data, size_t size, uint32_t* width,
                                   uint32_t* height, float* rgba_out) {
  return guarded([&]() -> int {
    if (!data || !width || !height) return fail(CG_E_INVALID, "null argument");
    std::vector<float> px;
    std::string e;
    uint32_t w = 0, h = 0;
    if (!decodeRadianceHdr(data, size, w, h, px, e)) return fail(CG_E_INVALID, e);
    *width = w;
    *height = h;
    if (rgba_out) std::memcpy(rgba_out, px.data(), px.size() * sizeof(float));
    return CG_OK;
  });
}

extern "C" CG_API int cg_env_from_cube(const float* faces, uint32_t face_width,
                                      uint32_t face_height, const float* rotation, float* env_out) {
  return guarded([&]() -> int {
    if (!faces || !rotation || !env_out) return fail(CG_E_INVALID, "null argument");
    if (face_width == 0 || face_height == 0 || face_width > (1u << 14) || face_height > (1u << 14))
      return fail(CG_E_INVALID, "cube face size must be in [1, 16384]");
    const size_t face = size_t(face_width) * face_height * 4;
    const float* fp[6];
    for (int i = 0; i < 6; ++i) fp[i] = faces + i * face;
    std::vector<float> out;
    cubeToLatLong(fp, face_width, face_height, rotation, out);
    std::memcpy(env_out, out.data(), out.size() * sizeof(float));
    return CG_OK;
  });
}

extern "C" CG_API int cg_gltf_free(void* storage) {
  delete static_cast<Loader*>(storage);
  return CG_OK;
}

extern "C" CG_API int cg_scene_load_gltf(const char* path, cg_scene_t* out) {
  return guarded([&]() -> int {
    if (!path || !out) return fail(CG_E_INVALID, "null argument");
    *out = nullptr;
    cg_scene_desc d{};
    void* storage = nullptr;
    int rc = cg_gltf_parse(path, &d, &storage);
    if (rc != CG_OK) return rc;
    rc = cg_scene_create(&d, out);
    cg_gltf_free(storage);
    return rc;
  });
}
