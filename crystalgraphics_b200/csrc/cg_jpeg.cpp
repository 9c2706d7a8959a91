// cg_jpeg.cpp — JPEG decoding (ITU-T T.81 | ISO/IEC 10918-1) for glTF images.
//
// The reference decodes glTF images with stb_image (src/image_decode.cpp),
// which is not available here; this decoder follows the standard.  Every
// scan's coefficients are kept per block (sequential scans fill them, the
// progressive scans of Annex G refine them), then each block is dequantised
// and transformed with a separable float IDCT, chroma planes are upsampled
// to full size (the usual triangle filter for 2x1 and 2x2 subsampling,
// replication otherwise) and YCbCr is converted to RGB with the JFIF
// equations.  Sample values can differ from stb_image's or libjpeg's by a
// level or two (IDCT and conversion rounding).
#include "cg_jpeg.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "cg_png.h"

namespace cg {
namespace {

// zig-zag index -> natural (row-major) index of an 8x8 block (T.81 Figure A.6)
constexpr uint8_t kNatural[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
    41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
    30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Canonical Huffman table (T.81 Annex C, decoding per F.2.2.3) with a lookup
// of every code up to 9 bits.
struct Huffman {
  bool defined = false;
  uint8_t vals[256] = {};
  int maxcode[17] = {};
  int valptr[17] = {};
  int mincode[17] = {};
  uint16_t fast[512] = {};  // (length << 8) | value; 0: longer code

  bool build(const uint8_t counts[16], const uint8_t* values, int nvals) {
    std::memcpy(vals, values, static_cast<size_t>(nvals));
    std::memset(fast, 0, sizeof(fast));
    int code = 0, k = 0;
    for (int len = 1; len <= 16; ++len) {
      const int n = counts[len - 1];
      valptr[len] = k;
      mincode[len] = code;
      for (int i = 0; i < n; ++i, ++code, ++k) {
        if (code >= (1 << len)) return false;  // over-subscribed lengths
        if (len <= 9) {
          const int shift = 9 - len;
          for (int f = code << shift; f < ((code + 1) << shift); ++f)
            fast[f] = static_cast<uint16_t>(len << 8 | vals[k]);
        }
      }
      maxcode[len] = n ? code - 1 : -1;
      code <<= 1;
    }
    defined = true;
    return true;
  }
};

// Bits of an entropy-coded segment: stuffed 0xFF 0x00 pairs read as 0xFF; at
// a marker the reader stops (pos stays on it) and supplies zero bits.
struct BitReader {
  const uint8_t* data = nullptr;
  size_t size = 0, pos = 0;
  uint32_t acc = 0;
  int nbits = 0;
  bool at_marker = false;

  void fill() {
    while (nbits <= 24) {
      uint32_t byte = 0;
      if (!at_marker && pos < size) {
        byte = data[pos];
        if (byte == 0xFF) {
          const uint8_t next = pos + 1 < size ? data[pos + 1] : 0xD9;
          if (next == 0x00) {
            pos += 2;
          } else {
            at_marker = true;
            byte = 0;
          }
        } else {
          ++pos;
        }
      }
      acc |= byte << (24 - nbits);
      nbits += 8;
    }
  }
  uint32_t bits(int n) {
    if (n == 0) return 0;
    if (nbits < n) fill();
    const uint32_t v = acc >> (32 - n);
    acc <<= n;
    nbits -= n;
    return v;
  }
  int bit() { return static_cast<int>(bits(1)); }
  // T.81 F.2.2.1 EXTEND of RECEIVE(s)
  int receiveExtend(int s) {
    if (s == 0) return 0;
    const int v = static_cast<int>(bits(s));
    return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v;
  }
  int decode(const Huffman& h) {
    if (nbits < 9) fill();
    const uint16_t f = h.fast[acc >> 23];
    if (f) {
      acc <<= (f >> 8);
      nbits -= (f >> 8);
      return f & 0xFF;
    }
    int code = 0;
    for (int len = 1; len <= 16; ++len) {
      code = (code << 1) | bit();
      if (h.maxcode[len] >= 0 && code <= h.maxcode[len])
        return h.vals[h.valptr[len] + code - h.mincode[len]];
    }
    return -1;
  }
  void restart() {
    acc = 0;
    nbits = 0;
    at_marker = false;
  }
};

struct Component {
  int id = 0, h = 1, v = 1, tq = 0;
  int bw = 0, bh = 0;    // block grid allocated (whole MCUs)
  int cbw = 0, cbh = 0;  // blocks covering the component's samples
  int dc_tab = 0, ac_tab = 0, dc_pred = 0;
  std::vector<int16_t> coef;  // bw * bh blocks of 64, natural order
};

struct Decoder {
  const uint8_t* data;
  size_t size;
  std::string& err;
  uint16_t quant[4][64] = {};  // natural order
  Huffman dc[4], ac[4];
  int restart_interval = 0;
  bool progressive = false, have_frame = false;
  int adobe_transform = -1;
  uint32_t width = 0, height = 0;
  int hmax = 1, vmax = 1, mcux = 0, mcuy = 0;
  std::vector<Component> comps;
  int eobrun = 0;

  bool fail(const char* m) {
    err = m;
    return false;
  }

  bool segment(size_t& pos, size_t& len) {
    if (pos + 2 > size) return fail("truncated JPEG segment");
    len = size_t(data[pos]) << 8 | data[pos + 1];
    if (len < 2 || pos + len > size) return fail("bad JPEG segment length");
    return true;
  }

  bool readDqt(size_t p, size_t end) {
    while (p < end) {
      const int pq = data[p] >> 4, tq = data[p] & 15;
      ++p;
      if (tq > 3 || pq > 1) return fail("bad JPEG quantisation table");
      if (p + 64 * (pq + 1) > end) return fail("truncated JPEG quantisation table");
      for (int k = 0; k < 64; ++k) {
        const uint16_t q = pq ? static_cast<uint16_t>(data[p + 2 * k] << 8 | data[p + 2 * k + 1])
                              : data[p + k];
        quant[tq][kNatural[k]] = q;
      }
      p += 64 * (pq + 1);
    }
    return true;
  }

  bool readDht(size_t p, size_t end) {
    while (p < end) {
      if (p + 17 > end) return fail("truncated JPEG Huffman table");
      const int tc = data[p] >> 4, th = data[p] & 15;
      if (tc > 1 || th > 3) return fail("bad JPEG Huffman table");
      uint8_t counts[16];
      int n = 0;
      for (int i = 0; i < 16; ++i) n += counts[i] = data[p + 1 + i];
      if (n > 256 || p + 17 + n > end) return fail("bad JPEG Huffman table");
      Huffman& h = tc ? ac[th] : dc[th];
      if (!h.build(counts, data + p + 17, n)) return fail("bad JPEG Huffman table");
      p += 17 + n;
    }
    return true;
  }

  bool readSof(size_t p, size_t end, uint8_t marker) {
    if (have_frame) return fail("more than one JPEG frame");
    if (end - p < 6) return fail("truncated JPEG frame header");
    if (data[p] != 8) return fail("only 8-bit JPEG images are supported");
    height = uint32_t(data[p + 1]) << 8 | data[p + 2];
    width = uint32_t(data[p + 3]) << 8 | data[p + 4];
    const int nf = data[p + 5];
    if (height == 0) return fail("JPEG images with a DNL height are not supported");
    if (width == 0) return fail("JPEG image of zero width");
    if (uint64_t(width) * height > (uint64_t(1) << 28)) return fail("JPEG image too large");
    if (nf != 1 && nf != 3) return fail("only grey and three-component JPEG images are supported");
    if (end - p < size_t(6 + 3 * nf)) return fail("truncated JPEG frame header");
    progressive = marker == 0xC2;
    comps.resize(nf);
    for (int i = 0; i < nf; ++i) {
      Component& c = comps[i];
      c.id = data[p + 6 + 3 * i];
      c.h = data[p + 7 + 3 * i] >> 4;
      c.v = data[p + 7 + 3 * i] & 15;
      c.tq = data[p + 8 + 3 * i];
      if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3)
        return fail("bad JPEG component parameters");
      hmax = std::max(hmax, c.h);
      vmax = std::max(vmax, c.v);
    }
    mcux = static_cast<int>((width + 8 * hmax - 1) / (8 * hmax));
    mcuy = static_cast<int>((height + 8 * vmax - 1) / (8 * vmax));
    for (Component& c : comps) {
      c.bw = mcux * c.h;
      c.bh = mcuy * c.v;
      const uint32_t cw = (width * c.h + hmax - 1) / hmax, ch = (height * c.v + vmax - 1) / vmax;
      c.cbw = static_cast<int>((cw + 7) / 8);
      c.cbh = static_cast<int>((ch + 7) / 8);
      c.coef.assign(size_t(c.bw) * c.bh * 64, 0);
    }
    have_frame = true;
    return true;
  }

  // ---- one block of a scan (T.81 F.2.2 sequential, G.1.2 progressive) ----
  bool blockSequential(BitReader& br, Component& c, int16_t* b) {
    const int t = br.decode(dc[c.dc_tab]);
    if (t < 0 || t > 16) return fail("corrupt JPEG data");
    c.dc_pred += br.receiveExtend(t);
    b[0] = static_cast<int16_t>(c.dc_pred);
    for (int k = 1; k < 64;) {
      const int rs = br.decode(ac[c.ac_tab]);
      if (rs < 0) return fail("corrupt JPEG data");
      const int r = rs >> 4, s = rs & 15;
      if (s == 0) {
        if (r != 15) break;  // end of block
        k += 16;
        continue;
      }
      k += r;
      if (k > 63) return fail("corrupt JPEG data");
      b[kNatural[k++]] = static_cast<int16_t>(br.receiveExtend(s));
    }
    return true;
  }

  bool blockDcFirst(BitReader& br, Component& c, int16_t* b, int al) {
    const int t = br.decode(dc[c.dc_tab]);
    if (t < 0 || t > 16) return fail("corrupt JPEG data");
    c.dc_pred += br.receiveExtend(t);
    b[0] = static_cast<int16_t>(c.dc_pred * (1 << al));
    return true;
  }

  void blockDcRefine(BitReader& br, int16_t* b, int al) {
    if (br.bit()) b[0] = static_cast<int16_t>(b[0] | (1 << al));
  }

  bool blockAcFirst(BitReader& br, Component& c, int16_t* b, int ss, int se, int al) {
    if (eobrun > 0) {
      --eobrun;
      return true;
    }
    for (int k = ss; k <= se;) {
      const int rs = br.decode(ac[c.ac_tab]);
      if (rs < 0) return fail("corrupt JPEG data");
      const int r = rs >> 4, s = rs & 15;
      if (s == 0) {
        if (r < 15) {  // EOBn: this and the next 2^r - 1 + bits blocks end here
          eobrun = (1 << r) - 1;
          if (r) eobrun += static_cast<int>(br.bits(r));
          break;
        }
        k += 16;
        continue;
      }
      k += r;
      if (k > 63) return fail("corrupt JPEG data");
      b[kNatural[k++]] = static_cast<int16_t>(br.receiveExtend(s) * (1 << al));
    }
    return true;
  }

  bool blockAcRefine(BitReader& br, Component& c, int16_t* b, int ss, int se, int al) {
    const int p1 = 1 << al, m1 = -(1 << al);
    int k = ss;
    auto refine = [&](int16_t& coef) {  // a correction bit of an already nonzero coefficient
      if (br.bit() && (coef & p1) == 0) coef = static_cast<int16_t>(coef + (coef >= 0 ? p1 : m1));
    };
    if (eobrun <= 0) {
      while (k <= se) {
        const int rs = br.decode(ac[c.ac_tab]);
        if (rs < 0) return fail("corrupt JPEG data");
        int r = rs >> 4;
        const int s = rs & 15;
        int value = 0;
        if (s == 0) {
          if (r < 15) {
            eobrun = 1 << r;
            if (r) eobrun += static_cast<int>(br.bits(r));
            break;
          }
          // r == 15: sixteen zero coefficients (nonzero ones in between are refined)
        } else {
          if (s != 1) return fail("corrupt JPEG data");
          value = br.bit() ? p1 : m1;
        }
        // skip r zero coefficients (refining the nonzero ones met on the way)
        // and place `value` at the next zero one
        while (k <= se) {
          int16_t& coef = b[kNatural[k]];
          ++k;
          if (coef != 0) {
            refine(coef);
          } else {
            if (r == 0) {
              if (value) coef = static_cast<int16_t>(value);
              break;
            }
            --r;
          }
        }
      }
    }
    if (eobrun > 0) {  // the rest of the band only refines nonzero coefficients
      for (; k <= se; ++k) {
        int16_t& coef = b[kNatural[k]];
        if (coef != 0) refine(coef);
      }
      --eobrun;
    }
    return true;
  }

  // ---- a scan: its header and entropy-coded data; `pos` ends on the next marker ----
  bool readScan(size_t p, size_t end, size_t& pos) {
    if (!have_frame) return fail("JPEG scan before the frame header");
    const int ns = data[p];
    if (ns < 1 || ns > 4 || end - p < size_t(4 + 2 * ns)) return fail("bad JPEG scan header");
    Component* sc[4] = {};
    for (int i = 0; i < ns; ++i) {
      const int cid = data[p + 1 + 2 * i], tabs = data[p + 2 + 2 * i];
      for (Component& c : comps)
        if (c.id == cid) sc[i] = &c;
      if (!sc[i]) return fail("JPEG scan names a missing component");
      sc[i]->dc_tab = tabs >> 4;
      sc[i]->ac_tab = tabs & 15;
      if (sc[i]->dc_tab > 3 || sc[i]->ac_tab > 3) return fail("bad JPEG scan header");
    }
    const int ss = data[p + 1 + 2 * ns], se = data[p + 2 + 2 * ns];
    const int ah = data[p + 3 + 2 * ns] >> 4, al = data[p + 3 + 2 * ns] & 15;
    if (progressive) {
      if (ss > se || se > 63 || (ss == 0 && se != 0) || (ss > 0 && ns != 1) || al > 13)
        return fail("bad JPEG progressive scan");
    } else if (ss != 0 || se != 63 || ah != 0 || al != 0) {
      return fail("bad JPEG sequential scan");
    }
    // the tables this scan decodes with
    for (int i = 0; i < ns; ++i) {
      const bool need_dc = !progressive || (ss == 0 && ah == 0);
      const bool need_ac = !progressive || ss > 0;
      if (need_dc && !dc[sc[i]->dc_tab].defined) return fail("JPEG scan uses an undefined table");
      if (need_ac && !ac[sc[i]->ac_tab].defined) return fail("JPEG scan uses an undefined table");
    }
    BitReader br;
    br.data = data;
    br.size = size;
    br.pos = end;
    for (int i = 0; i < ns; ++i) sc[i]->dc_pred = 0;
    eobrun = 0;

    auto decodeBlock = [&](Component& c, int bx, int by) {
      int16_t* b = c.coef.data() + (size_t(by) * c.bw + bx) * 64;
      if (!progressive) return blockSequential(br, c, b);
      if (ss == 0) {
        if (ah == 0) return blockDcFirst(br, c, b, al);
        blockDcRefine(br, b, al);
        return true;
      }
      return ah == 0 ? blockAcFirst(br, c, b, ss, se, al) : blockAcRefine(br, c, b, ss, se, al);
    };
    const bool single = ns == 1;
    const int units_x = single ? sc[0]->cbw : mcux, units_y = single ? sc[0]->cbh : mcuy;
    const long total = long(units_x) * units_y;
    for (long u = 0; u < total; ++u) {
      if (restart_interval && u > 0 && u % restart_interval == 0) {
        // the restart marker ends the interval: predictors and EOB runs restart
        size_t q = br.pos;
        while (q + 1 < size && !(data[q] == 0xFF && data[q + 1] >= 0xD0 && data[q + 1] <= 0xD7))
          ++q;
        if (q + 1 >= size) return fail("missing JPEG restart marker");
        br.pos = q + 2;
        br.restart();
        for (int i = 0; i < ns; ++i) sc[i]->dc_pred = 0;
        eobrun = 0;
      }
      const int ux = static_cast<int>(u % units_x), uy = static_cast<int>(u / units_x);
      if (single) {
        if (!decodeBlock(*sc[0], ux, uy)) return false;
        continue;
      }
      for (int i = 0; i < ns; ++i)
        for (int v = 0; v < sc[i]->v; ++v)
          for (int h = 0; h < sc[i]->h; ++h)
            if (!decodeBlock(*sc[i], ux * sc[i]->h + h, uy * sc[i]->v + v)) return false;
    }
    // the next marker (skipping any restart marker and padding after the data)
    size_t q = br.pos;
    while (q + 1 < size && !(data[q] == 0xFF && data[q + 1] != 0 && data[q + 1] != 0xFF &&
                             !(data[q + 1] >= 0xD0 && data[q + 1] <= 0xD7)))
      ++q;
    pos = q;
    return true;
  }

  // ---- blocks -> samples -> RGBA ----
  // floor(h) clamped to 0..255, exactly as std::floor gives it, without the
  // library call that x86-64's baseline instruction set needs for std::floor.
  // h is bounded first: a damaged stream's coefficients can take a sum far
  // outside the int range (and fmax/fmin take a NaN to a bound).
  static uint8_t floorToByte(float h) {
    h = std::fmin(std::fmax(h, -1.0f), 256.0f);
    int i = static_cast<int>(h);
    i -= static_cast<float>(i) > h;
    return static_cast<uint8_t>(std::clamp(i, 0, 255));
  }

  void idct(const int16_t* b, const uint16_t* q, uint8_t* out, int stride) {
    // ctab[x][u] = C(u) / 2 * cos((2x + 1) u pi / 16), C(0) = 1 / sqrt(2); a
    // function-local static is initialised once even when threads decode at
    // the same time
    struct CosTable {
      float v[8][8];
    };
    static const CosTable tab = [] {
      CosTable t{};
      for (int x = 0; x < 8; ++x)
        for (int u = 0; u < 8; ++u)
          t.v[x][u] = static_cast<float>((u == 0 ? std::sqrt(0.5) : 1.0) * 0.5 *
                                         std::cos((2 * x + 1) * u * M_PI / 16.0));
      return t;
    }();
    const auto& ctab = tab.v;
    float f[64], rows[64];
    for (int i = 0; i < 64; ++i) f[i] = static_cast<float>(b[i]) * static_cast<float>(q[i]);
    for (int v = 0; v < 8; ++v)
      for (int x = 0; x < 8; ++x) {
        float s = 0.0f;
        for (int u = 0; u < 8; ++u) s += ctab[x][u] * f[v * 8 + u];
        rows[v * 8 + x] = s;
      }
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) {
        float s = 0.0f;
        for (int v = 0; v < 8; ++v) s += ctab[y][v] * rows[v * 8 + x];
        out[y * stride + x] = floorToByte(s + 128.5f);
      }
  }

  // A component's samples at full image size.
  std::vector<uint8_t> fullPlane(const Component& c) {
    const int stride = c.bw * 8;
    std::vector<uint8_t> plane(size_t(stride) * c.bh * 8);
    for (int by = 0; by < c.bh; ++by)
      for (int bx = 0; bx < c.bw; ++bx)
        idct(c.coef.data() + (size_t(by) * c.bw + bx) * 64, quant[c.tq],
             plane.data() + size_t(by) * 8 * stride + bx * 8, stride);
    const int W = static_cast<int>(width), H = static_cast<int>(height);
    if (c.h == hmax && c.v == vmax) {
      std::vector<uint8_t> out(size_t(W) * H);
      for (int y = 0; y < H; ++y) std::memcpy(&out[size_t(y) * W], &plane[size_t(y) * stride], W);
      return out;
    }
    std::vector<uint8_t> out(size_t(W) * H);
    const int cw = (W * c.h + hmax - 1) / hmax, ch = (H * c.v + vmax - 1) / vmax;
    auto in = [&](int x, int y) -> int {
      return plane[size_t(std::clamp(y, 0, ch - 1)) * stride + std::clamp(x, 0, cw - 1)];
    };
    if (hmax == 2 * c.h && (vmax == c.v || vmax == 2 * c.v)) {
      // triangle filter: each output sample weighs its nearer input sample 3/4
      // and the next one 1/4, per axis
      const bool v2 = vmax == 2 * c.v;
      for (int y = 0; y < H; ++y) {
        const int iy = v2 ? y / 2 : y;
        const int ny = v2 ? (y % 2 == 0 ? iy - 1 : iy + 1) : iy;
        for (int x = 0; x < W; ++x) {
          const int ix = x / 2, nx = x % 2 == 0 ? ix - 1 : ix + 1;
          int val;
          if (v2) {  // column sums 3 * near row + far row, then the same across
            const int here = 3 * in(ix, iy) + in(ix, ny);
            const bool edge = (x % 2 == 0 && ix == 0) || (x % 2 == 1 && ix == cw - 1);
            const int there = edge ? here : 3 * in(nx, iy) + in(nx, ny);
            val = (3 * here + there + (x % 2 == 0 ? 8 : 7)) >> 4;
          } else {
            const bool edge = (x % 2 == 0 && ix == 0) || (x % 2 == 1 && ix == cw - 1);
            val = edge ? in(ix, iy) : (3 * in(ix, iy) + in(nx, iy) + (x % 2 == 0 ? 1 : 2)) >> 2;
          }
          out[size_t(y) * W + x] = static_cast<uint8_t>(val);
        }
      }
      return out;
    }
    for (int y = 0; y < H; ++y)  // other ratios: the covering sample
      for (int x = 0; x < W; ++x)
        out[size_t(y) * W + x] = static_cast<uint8_t>(in(x * c.h / hmax, y * c.v / vmax));
    return out;
  }

  void toRgba(std::vector<uint8_t>& rgba) {
    const size_t n = size_t(width) * height;
    rgba.assign(n * 4, 255);
    if (comps.size() == 1) {
      const std::vector<uint8_t> g = fullPlane(comps[0]);
      for (size_t i = 0; i < n; ++i) rgba[4 * i] = rgba[4 * i + 1] = rgba[4 * i + 2] = g[i];
      return;
    }
    const std::vector<uint8_t> a = fullPlane(comps[0]), b = fullPlane(comps[1]),
                               c = fullPlane(comps[2]);
    // RGB when an Adobe marker says so or the component ids spell R, G, B
    const bool rgb = adobe_transform == 0 ||
                     (adobe_transform < 0 && comps[0].id == 'R' && comps[1].id == 'G' &&
                      comps[2].id == 'B');
    for (size_t i = 0; i < n; ++i) {
      if (rgb) {
        rgba[4 * i] = a[i];
        rgba[4 * i + 1] = b[i];
        rgba[4 * i + 2] = c[i];
        continue;
      }
      const float y = a[i], cb = b[i] - 128.0f, cr = c[i] - 128.0f;  // JFIF YCbCr
      const float r = y + 1.402f * cr, g = y - 0.344136f * cb - 0.714136f * cr, bl = y + 1.772f * cb;
      rgba[4 * i] = floorToByte(r + 0.5f);
      rgba[4 * i + 1] = floorToByte(g + 0.5f);
      rgba[4 * i + 2] = floorToByte(bl + 0.5f);
    }
  }

  bool run(uint32_t& w, uint32_t& h, std::vector<uint8_t>& rgba) {
    if (size < 4 || data[0] != 0xFF || data[1] != 0xD8) return fail("not a JPEG image");
    size_t pos = 2;
    bool scanned = false;
    while (true) {
      while (pos < size && data[pos] != 0xFF) ++pos;  // tolerate junk between segments
      while (pos < size && data[pos] == 0xFF) ++pos;  // fill bytes
      if (pos >= size) break;                         // no EOI: decode what arrived
      const uint8_t m = data[pos++];
      if (m == 0xD9) break;                                  // EOI
      if (m == 0xD8 || (m >= 0xD0 && m <= 0xD7)) continue;  // SOI, stray RSTn
      size_t len = 0;
      if (!segment(pos, len)) return false;
      const size_t p = pos + 2, end = pos + len;
      switch (m) {
        case 0xC0:
        case 0xC1:
        case 0xC2:
          if (!readSof(p, end, m)) return false;
          break;
        case 0xC4:
          if (!readDht(p, end)) return false;
          break;
        case 0xDB:
          if (!readDqt(p, end)) return false;
          break;
        case 0xDD:
          if (len < 4) return fail("bad JPEG restart interval");
          restart_interval = data[p] << 8 | data[p + 1];
          break;
        case 0xDA: {
          if (!readScan(p, end, pos)) return false;
          scanned = true;
          continue;  // pos is on the next marker
        }
        case 0xEE:  // APP14 "Adobe": its transform flag says RGB (0) or YCbCr (1)
          if (len >= 14 && std::memcmp(data + p, "Adobe", 5) == 0) adobe_transform = data[p + 11];
          break;
        default:
          if ((m >= 0xC3 && m <= 0xCF) && m != 0xC4 && m != 0xC8 && m != 0xCC)
            return fail("unsupported JPEG coding (lossless, hierarchical or arithmetic)");
          break;  // APPn, COM and others: skipped
      }
      pos = end;
    }
    if (!have_frame || !scanned) return fail("JPEG image without frame or scan");
    toRgba(rgba);
    w = width;
    h = height;
    return true;
  }
};

}  // namespace

bool decodeJpeg(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                std::vector<uint8_t>& rgba, std::string& err) {
  Decoder d{data, size, err};
  return d.run(width, height, rgba);
}

bool decodeImageRgba8(const uint8_t* data, size_t size, uint32_t& width, uint32_t& height,
                      std::vector<uint8_t>& rgba, std::string& err) {
  if (size >= 3 && data[0] == 0xFF && data[1] == 0xD8 && data[2] == 0xFF)
    return decodeJpeg(data, size, width, height, rgba, err);
  return decodePng(data, size, width, height, rgba, err);
}

}  // namespace cg
