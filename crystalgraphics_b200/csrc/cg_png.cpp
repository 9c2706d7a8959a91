// cg_png.cpp — PNG decoding to RGBA8 for glTF material images.
//
// The reference decodes texture images with stb_image (src/image_decode.cpp,
// stbi_load_from_memory with 4 channels requested).  stb is not part of this
// tree, so PNG — the lossless format glTF files carry — is decoded here:
// zlib/DEFLATE (RFC 1950/1951: stored, fixed- and dynamic-Huffman blocks),
// the five scanline filters, Adam7 interlacing, and every colour type at
// bit depths 1-16 (16-bit samples keep their high byte, as stb does when
// 8 bits per channel are requested; palette and grey expand to RGBA, a tRNS
// chunk gives alpha).  JPEG and other formats are rejected with an error.
#include "cg_png.h"

#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>

namespace cg {
namespace {

// ---- DEFLATE --------------------------------------------------------------------
struct BitReader {
  const uint8_t* p;
  size_t n, pos = 0;
  uint32_t bitbuf = 0;
  int bitcnt = 0;
  bool overrun = false;
  uint32_t bits(int k) {  // k <= 24
    while (bitcnt < k) {
      uint32_t b = 0;
      if (pos < n)
        b = p[pos++];
      else
        overrun = true;
      bitbuf |= b << bitcnt;
      bitcnt += 8;
    }
    const uint32_t v = bitbuf & ((1u << k) - 1u);
    bitbuf >>= k;
    bitcnt -= k;
    return v;
  }
  void alignByte() {
    bitbuf >>= (bitcnt & 7);
    bitcnt -= (bitcnt & 7);
  }
};

// Canonical Huffman code: symbols sorted by code length, counts per length.
struct Huffman {
  std::array<uint16_t, 16> count{};
  std::array<uint16_t, 320> symbol{};
  bool build(const uint8_t* lengths, int n) {
    count.fill(0);
    for (int i = 0; i < n; ++i) ++count[lengths[i]];
    count[0] = 0;
    int left = 1;
    for (int len = 1; len < 16; ++len) {
      left <<= 1;
      left -= count[len];
      if (left < 0) return false;  // over-subscribed
    }
    std::array<uint16_t, 16> offs{};
    for (int len = 1; len < 15; ++len) offs[len + 1] = offs[len] + count[len];
    for (int i = 0; i < n; ++i)
      if (lengths[i]) symbol[offs[lengths[i]]++] = static_cast<uint16_t>(i);
    return true;
  }
  // Decodes one symbol reading the code bit by bit (codes are stored MSB first).
  int decode(BitReader& br) const {
    int code = 0, first = 0, index = 0;
    for (int len = 1; len < 16; ++len) {
      code |= static_cast<int>(br.bits(1));
      const int c = count[len];
      if (code - c < first) return symbol[index + (code - first)];
      index += c;
      first += c;
      first <<= 1;
      code <<= 1;
      if (br.overrun) return -1;
    }
    return -1;
  }
};

constexpr uint16_t kLenBase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                   31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
constexpr uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                   2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
constexpr uint16_t kDistBase[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                    33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                    1025, 1537, 2049, 3073, 4097, 6145,  8193,  12289, 16385, 24577};
constexpr uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                    6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

bool inflateBlock(BitReader& br, const Huffman& lit, const Huffman& dist, std::vector<uint8_t>& out,
                  size_t limit, std::string& err) {
  while (true) {
    const int sym = lit.decode(br);
    if (sym < 0) return (err = "corrupt deflate stream (literal code)"), false;
    if (sym < 256) {
      if (out.size() >= limit) return (err = "image data larger than its header says"), false;
      out.push_back(static_cast<uint8_t>(sym));
    } else if (sym == 256) {
      return true;
    } else {
      const int li = sym - 257;
      if (li >= 29) return (err = "corrupt deflate stream (length code)"), false;
      const size_t len = kLenBase[li] + br.bits(kLenExtra[li]);
      const int ds = dist.decode(br);
      if (ds < 0 || ds >= 30) return (err = "corrupt deflate stream (distance code)"), false;
      const size_t d = kDistBase[ds] + br.bits(kDistExtra[ds]);
      if (d > out.size()) return (err = "corrupt deflate stream (distance too far)"), false;
      if (out.size() + len > limit) return (err = "image data larger than its header says"), false;
      const size_t from = out.size() - d;
      for (size_t k = 0; k < len; ++k) out.push_back(out[from + k]);
    }
    if (br.overrun) return (err = "truncated deflate stream"), false;
  }
}

bool inflateZlib(const uint8_t* p, size_t n, std::vector<uint8_t>& out, size_t limit, std::string& err) {
  if (n < 2) return (err = "truncated zlib stream"), false;
  if ((p[0] & 15) != 8 || ((p[0] << 8) | p[1]) % 31 != 0 || (p[1] & 32))
    return (err = "unsupported zlib header"), false;
  BitReader br{p + 2, n - 2};
  bool last = false;
  while (!last) {
    last = br.bits(1) != 0;
    const uint32_t type = br.bits(2);
    if (type == 0) {
      br.alignByte();
      br.bitbuf = 0;
      br.bitcnt = 0;
      if (br.pos + 4 > br.n) return (err = "truncated stored block"), false;
      const uint32_t len = br.p[br.pos] | (br.p[br.pos + 1] << 8);
      const uint32_t nlen = br.p[br.pos + 2] | (br.p[br.pos + 3] << 8);
      br.pos += 4;
      if ((len ^ 0xffffu) != nlen) return (err = "corrupt stored block"), false;
      if (br.pos + len > br.n || out.size() + len > limit) return (err = "truncated stored block"), false;
      out.insert(out.end(), br.p + br.pos, br.p + br.pos + len);
      br.pos += len;
    } else if (type == 1) {
      uint8_t l[288];
      for (int i = 0; i < 144; ++i) l[i] = 8;
      for (int i = 144; i < 256; ++i) l[i] = 9;
      for (int i = 256; i < 280; ++i) l[i] = 7;
      for (int i = 280; i < 288; ++i) l[i] = 8;
      uint8_t dl[30];
      for (int i = 0; i < 30; ++i) dl[i] = 5;
      Huffman lit, dist;
      lit.build(l, 288);
      dist.build(dl, 30);
      if (!inflateBlock(br, lit, dist, out, limit, err)) return false;
    } else if (type == 2) {
      const int hlit = static_cast<int>(br.bits(5)) + 257, hdist = static_cast<int>(br.bits(5)) + 1;
      const int hclen = static_cast<int>(br.bits(4)) + 4;
      static constexpr uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
      uint8_t cl[19] = {};
      for (int i = 0; i < hclen; ++i) cl[order[i]] = static_cast<uint8_t>(br.bits(3));
      Huffman clh;
      if (!clh.build(cl, 19)) return (err = "corrupt code-length code"), false;
      uint8_t lens[320] = {};
      int i = 0;
      while (i < hlit + hdist) {
        const int sym = clh.decode(br);
        if (sym < 0) return (err = "corrupt code lengths"), false;
        if (sym < 16) {
          lens[i++] = static_cast<uint8_t>(sym);
        } else {
          int rep = 0;
          uint8_t val = 0;
          if (sym == 16) {
            if (i == 0) return (err = "corrupt code lengths (repeat)"), false;
            val = lens[i - 1];
            rep = 3 + static_cast<int>(br.bits(2));
          } else if (sym == 17) {
            rep = 3 + static_cast<int>(br.bits(3));
          } else {
            rep = 11 + static_cast<int>(br.bits(7));
          }
          if (i + rep > hlit + hdist) return (err = "corrupt code lengths (overflow)"), false;
          while (rep--) lens[i++] = val;
        }
      }
      Huffman lit, dist;
      if (!lit.build(lens, hlit) || !dist.build(lens + hlit, hdist))
        return (err = "corrupt Huffman code"), false;
      if (!inflateBlock(br, lit, dist, out, limit, err)) return false;
    } else {
      return (err = "invalid deflate block type"), false;
    }
    if (br.overrun) return (err = "truncated deflate stream"), false;
  }
  return true;
}

// ---- PNG -------------------------------------------------------------------------
uint32_t be32(const uint8_t* p) {
  return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3];
}

int paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  if (pb <= pc) return b;
  return c;
}

// Undoes the scanline filters of one (sub)image in place; raw holds rows of
// 1 + stride bytes.  bpp = bytes per complete pixel (at least 1).
bool unfilter(uint8_t* raw, uint32_t rows, size_t stride, size_t bpp, std::string& err) {
  std::vector<uint8_t> prev(stride, 0);
  for (uint32_t y = 0; y < rows; ++y) {
    uint8_t* row = raw + size_t(y) * (stride + 1);
    const uint8_t f = row[0];
    uint8_t* cur = row + 1;
    for (size_t x = 0; x < stride; ++x) {
      const int a = x >= bpp ? cur[x - bpp] : 0, b = prev[x], c = x >= bpp ? prev[x - bpp] : 0;
      int v = cur[x];
      switch (f) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) / 2; break;
        case 4: v += paeth(a, b, c); break;
        default: return (err = "invalid PNG filter type"), false;
      }
      cur[x] = static_cast<uint8_t>(v);
    }
    std::memcpy(prev.data(), cur, stride);
  }
  return true;
}

}  // namespace

bool decodePng(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
               std::vector<uint8_t>& rgba, std::string& err) {
  static constexpr uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (size < 8 || std::memcmp(data, sig, 8) != 0) {
    if (size >= 3 && data[0] == 0xFF && data[1] == 0xD8 && data[2] == 0xFF)
      err = "JPEG images are not supported (only PNG)";
    else
      err = "not a PNG image";
    return false;
  }
  uint32_t depth = 0, ctype = 0, interlace = 0;
  width = height = 0;
  std::vector<uint8_t> idat, palette, trns;
  size_t pos = 8;
  bool have_ihdr = false;
  while (pos + 12 <= size) {
    const uint32_t len = be32(data + pos);
    const uint8_t* type = data + pos + 4;
    if (len > size - pos - 12) return (err = "truncated PNG chunk"), false;
    const uint8_t* body = data + pos + 8;
    if (!std::memcmp(type, "IHDR", 4)) {
      if (len < 13) return (err = "bad IHDR"), false;
      width = be32(body);
      height = be32(body + 4);
      depth = body[8];
      ctype = body[9];
      interlace = body[12];
      if (body[10] != 0 || body[11] != 0 || interlace > 1) return (err = "unsupported PNG method"), false;
      have_ihdr = true;
    } else if (!std::memcmp(type, "PLTE", 4)) {
      palette.assign(body, body + len);
    } else if (!std::memcmp(type, "tRNS", 4)) {
      trns.assign(body, body + len);
    } else if (!std::memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), body, body + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      break;
    }
    pos += size_t(len) + 12;
  }
  if (!have_ihdr || width == 0 || height == 0) return (err = "PNG without a valid IHDR"), false;
  if (uint64_t(width) * height > (uint64_t(1) << 28)) return (err = "PNG image too large"), false;
  int channels = 0;
  switch (ctype) {
    case 0: channels = 1; break;
    case 2: channels = 3; break;
    case 3: channels = 1; break;
    case 4: channels = 2; break;
    case 6: channels = 4; break;
    default: return (err = "invalid PNG colour type"), false;
  }
  const bool depth_ok = (ctype == 0 && (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)) ||
                        (ctype == 3 && (depth == 1 || depth == 2 || depth == 4 || depth == 8)) ||
                        ((ctype == 2 || ctype == 4 || ctype == 6) && (depth == 8 || depth == 16));
  if (!depth_ok) return (err = "invalid PNG bit depth"), false;
  if (ctype == 3 && palette.empty()) return (err = "palette PNG without PLTE"), false;
  const size_t bits_pp = size_t(channels) * depth;
  const size_t bpp = std::max<size_t>(1, bits_pp / 8);
  // the sub-images (one, or Adam7's seven passes)
  struct Pass {
    uint32_t x0, y0, dx, dy;
  };
  const Pass adam7[7] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                         {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
  const Pass whole[1] = {{0, 0, 1, 1}};
  const Pass* passes = interlace ? adam7 : whole;
  const int npass = interlace ? 7 : 1;
  size_t expect = 0;
  for (int p = 0; p < npass; ++p) {
    const uint32_t pw = (width - passes[p].x0 + passes[p].dx - 1) / passes[p].dx;
    const uint32_t ph = (height - passes[p].y0 + passes[p].dy - 1) / passes[p].dy;
    if (passes[p].x0 >= width || passes[p].y0 >= height || pw == 0 || ph == 0) continue;
    expect += size_t(ph) * (1 + (size_t(pw) * bits_pp + 7) / 8);
  }
  std::vector<uint8_t> raw;
  raw.reserve(expect);
  if (!inflateZlib(idat.data(), idat.size(), raw, expect, err)) return false;
  if (raw.size() != expect) return (err = "PNG image data has the wrong size"), false;
  rgba.assign(size_t(width) * height * 4, 0);
  size_t off = 0;
  for (int p = 0; p < npass; ++p) {
    if (passes[p].x0 >= width || passes[p].y0 >= height) continue;
    const uint32_t pw = (width - passes[p].x0 + passes[p].dx - 1) / passes[p].dx;
    const uint32_t ph = (height - passes[p].y0 + passes[p].dy - 1) / passes[p].dy;
    if (pw == 0 || ph == 0) continue;
    const size_t stride = (size_t(pw) * bits_pp + 7) / 8;
    uint8_t* sub = raw.data() + off;
    if (!unfilter(sub, ph, stride, bpp, err)) return false;
    for (uint32_t y = 0; y < ph; ++y) {
      const uint8_t* row = sub + size_t(y) * (stride + 1) + 1;
      for (uint32_t x = 0; x < pw; ++x) {
        // sample c of pixel x, scaled to 8 bits (16-bit: the high byte)
        auto sample = [&](int c) -> uint32_t {
          if (depth == 8) return row[size_t(x) * channels + c];
          if (depth == 16) return row[(size_t(x) * channels + c) * 2];
          const size_t bit = size_t(x) * depth;
          const uint32_t v = (row[bit / 8] >> (8 - depth - (bit % 8))) & ((1u << depth) - 1u);
          return v;
        };
        auto raw16 = [&](int c) -> uint32_t {
          const uint8_t* q = row + (size_t(x) * channels + c) * 2;
          return (uint32_t(q[0]) << 8) | q[1];
        };
        uint8_t* o = rgba.data() + (size_t(passes[p].y0 + y * passes[p].dy) * width +
                                    passes[p].x0 + x * passes[p].dx) * 4;
        if (ctype == 3) {
          const uint32_t idx = sample(0);
          if (size_t(idx) * 3 + 2 >= palette.size()) return (err = "PNG palette index out of range"), false;
          o[0] = palette[idx * 3];
          o[1] = palette[idx * 3 + 1];
          o[2] = palette[idx * 3 + 2];
          o[3] = idx < trns.size() ? trns[idx] : 255;
        } else if (ctype == 0 || ctype == 4) {
          uint32_t g = sample(0);
          bool transparent = false;
          if (ctype == 0 && trns.size() >= 2) {
            const uint32_t key = (uint32_t(trns[0]) << 8) | trns[1];
            transparent = (depth == 16 ? raw16(0) : g) == key;
          }
          if (depth < 8) g = g * 255u / ((1u << depth) - 1u);
          o[0] = o[1] = o[2] = static_cast<uint8_t>(g);
          o[3] = ctype == 4 ? static_cast<uint8_t>(sample(1)) : (transparent ? 0 : 255);
        } else {
          o[0] = static_cast<uint8_t>(sample(0));
          o[1] = static_cast<uint8_t>(sample(1));
          o[2] = static_cast<uint8_t>(sample(2));
          if (ctype == 6) {
            o[3] = static_cast<uint8_t>(sample(3));
          } else {
            bool transparent = false;
            if (trns.size() >= 6) {
              transparent = true;
              for (int c = 0; c < 3; ++c) {
                const uint32_t key = (uint32_t(trns[2 * c]) << 8) | trns[2 * c + 1];
                const uint32_t v = depth == 16 ? raw16(c) : sample(c);
                transparent = transparent && v == key;
              }
            }
            o[3] = transparent ? 0 : 255;
          }
        }
      }
    }
    off += size_t(ph) * (stride + 1);
  }
  return true;
}

}  // namespace cg
