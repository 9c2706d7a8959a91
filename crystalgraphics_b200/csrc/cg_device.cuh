// cg_device.cuh — device functions of the spectral path tracer (sm_100a).
//
// A CUDA restatement of the reference's WGSL modules
// (src/wgpu/shader/compute/**) for the wavefront kernels in cg_kernels.cu.
// Expression order follows the WGSL source; nvcc may contract a*b+c into FMA
// here, except in the intersection code (cg_traverse.cuh), which uses
// explicitly rounded intrinsics so hit distances are bit-identical to the
// reference's arithmetic.  min/max/clamp use fminf/fmaxf (NaN operands are
// dropped), the documented semantics of the NaN produced by the reference's
// Smits lookup for wavelengths in [686, 720) nm (shading/smits.wesl:3-28).
#ifndef CG_DEVICE_CUH_
#define CG_DEVICE_CUH_

#include <cstdint>

#include "cg_types.h"

namespace cg {
namespace dev {

// ---- float3 helpers ------------------------------------------------------
struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ V3 normalize(V3 a) {
  float l = sqrtf(dot(a, a));
  return a / l;
}
__device__ __forceinline__ float distance3(V3 a, V3 b) {
  V3 d = a - b;
  return sqrtf(dot(d, d));
}
__device__ __forceinline__ float wclamp(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}
__device__ __forceinline__ float wmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 reflect(V3 e1, V3 e2) { return e1 - (2.0f * dot(e2, e1)) * e2; }
__device__ __forceinline__ V3 refract(V3 e1, V3 e2, float e3) {
  float d = dot(e2, e1);
  float k = 1.0f - e3 * e3 * (1.0f - d * d);
  if (k < 0.0f) return {0.0f, 0.0f, 0.0f};
  return e3 * e1 - (e3 * d + sqrtf(k)) * e2;
}
struct M3 {
  V3 c0, c1, c2;
};
__device__ __forceinline__ V3 mul(const M3& m, V3 v) { return (m.c0 * v.x + m.c1 * v.y) + m.c2 * v.z; }
__device__ __forceinline__ V3 mulT(const M3& m, V3 v) { return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }

constexpr float PI = 3.1415926535f;   // math/constant.wesl:1
constexpr float MAXD = 1e6f;          // math/constant.wesl:2

// math/geometric.wesl:28-33
__device__ __forceinline__ M3 makeTangentSpace(V3 n) {
  V3 helper = (fabsf(n.x) > 0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
  V3 tangent = normalize(cross(helper, n));
  V3 bitangent = cross(n, tangent);
  return M3{tangent, bitangent, n};
}

// ---- RNG (math/rng.wesl:1-22) and keyed streams ------------------------------
struct Rng {
  uint32_t s;
};
__device__ __forceinline__ void stepRng(Rng& r) {
  r.s = r.s * 747796405u + 2891336453u;
  uint32_t word = ((r.s >> ((r.s >> 28u) + 4u)) ^ r.s) * 277803737u;
  r.s = (word >> 22u) ^ word;
}
__device__ __forceinline__ void seedRng(Rng& r, uint32_t seed) {
  r.s = seed;
  stepRng(r);
}
__device__ __forceinline__ float randFloat(Rng& r) {
  stepRng(r);
  return __uint2float_rn(r.s) / 4294967296.0f;
}
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t combine(uint32_t a, uint32_t b) {
  return mix32(a ^ mix32(b + 0x9e3779b9u));
}
__device__ __forceinline__ uint32_t sampleKey(uint32_t seed, uint32_t frame, uint32_t pixel,
                                              uint32_t sample) {
  return combine(combine(combine(seed, frame), pixel), sample);
}
__device__ __forceinline__ uint32_t childKey(uint32_t key, uint32_t i) { return combine(key, i + 1u); }
__device__ __forceinline__ uint32_t wavelengthKey(uint32_t key) { return combine(key, 0u); }
// The Russian-roulette decision of a child (an option beyond the reference):
// one number from this stream.
__device__ __forceinline__ uint32_t rouletteKey(uint32_t child_key) {
  return combine(child_key, 0xfffffffeu);
}

// ---- CIE (physics/cie.wesl) ----------------------------------------------------------
constexpr float SQRT_HALF_PI = 1.2533141373155001f;
constexpr float INV_SQRT_TWO = 0.7071067811865475f;
__device__ __forceinline__ float splitGaussian(float w, float c, float lw, float rw) {
  float width = (w < c) ? lw : rw;
  float scaled = (w - c) / width;
  return expf(-0.5f * scaled * scaled);
}
__device__ __forceinline__ float erfApprox(float x) {
  float sign = (x >= 0.0f) ? 1.0f : -1.0f;
  float ax = fabsf(x);
  float t = 1.0f / (1.0f + 0.3275911f * ax);
  float poly = (((((1.061405429f * t - 1.453152027f) * t) + 1.421413741f) * t - 0.284496736f) * t +
                0.254829592f) * t;
  return sign * (1.0f - poly * expf(-ax * ax));
}
__device__ __forceinline__ float sgAnti(float w, float c, float lw, float rw) {
  if (w < c) return SQRT_HALF_PI * lw * (1.0f + erfApprox((w - c) * INV_SQRT_TWO / lw));
  return SQRT_HALF_PI * lw + SQRT_HALF_PI * rw * erfApprox((w - c) * INV_SQRT_TWO / rw);
}
__device__ __forceinline__ float sgInt(float lo, float hi, float c, float lw, float rw) {
  return sgAnti(hi, c, lw, rw) - sgAnti(lo, c, lw, rw);
}
__device__ __forceinline__ V3 xyzMatch(float w) {
  float x = 0.362f * splitGaussian(w, 442.0f, 1.0f / 0.0624f, 1.0f / 0.0374f) +
            1.056f * splitGaussian(w, 599.8f, 1.0f / 0.0264f, 1.0f / 0.0323f) -
            0.065f * splitGaussian(w, 501.1f, 1.0f / 0.0490f, 1.0f / 0.0382f);
  float y = 0.821f * splitGaussian(w, 568.8f, 1.0f / 0.0213f, 1.0f / 0.0247f) +
            0.286f * splitGaussian(w, 530.9f, 1.0f / 0.0613f, 1.0f / 0.0322f);
  float z = 1.217f * splitGaussian(w, 437.0f, 1.0f / 0.0845f, 1.0f / 0.0278f) +
            0.681f * splitGaussian(w, 459.0f, 1.0f / 0.0385f, 1.0f / 0.0725f);
  return {x, y, z};
}
__device__ __forceinline__ float xyzMatchSumIntegral(float lo, float hi) {
  float x = 0.362f * sgInt(lo, hi, 442.0f, 1.0f / 0.0624f, 1.0f / 0.0374f) +
            1.056f * sgInt(lo, hi, 599.8f, 1.0f / 0.0264f, 1.0f / 0.0323f) -
            0.065f * sgInt(lo, hi, 501.1f, 1.0f / 0.0490f, 1.0f / 0.0382f);
  float y = 0.821f * sgInt(lo, hi, 568.8f, 1.0f / 0.0213f, 1.0f / 0.0247f) +
            0.286f * sgInt(lo, hi, 530.9f, 1.0f / 0.0613f, 1.0f / 0.0322f);
  float z = 1.217f * sgInt(lo, hi, 437.0f, 1.0f / 0.0845f, 1.0f / 0.0278f) +
            0.681f * sgInt(lo, hi, 459.0f, 1.0f / 0.0385f, 1.0f / 0.0725f);
  return x + y + z;
}

// The 16-step bisection of sampleWavelengthCdf (physics/wavelength.wesl:24-45)
// visits one of 65535 midpoints per step.  `tree` holds cdf(mid) for every
// midpoint in heap order (node k: children 2k+1 = "cdf >= target" half,
// 2k+2 = "cdf < target" half), computed once by k_wavelength_tree with the
// same float arithmetic, so the walk below takes the branches the direct
// bisection would.
__device__ __forceinline__ float sampleWavelengthTree(const float* __restrict__ tree, float u) {
  float target = wclamp(u, 0.0f, 0.999999f);
  float low = 380.0f, high = 720.0f;
  uint32_t k = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float mid = 0.5f * (low + high);
    float cdf = __ldg(tree + k);
    if (cdf < target) {
      low = mid;
      k = 2u * k + 2u;
    } else {
      high = mid;
      k = 2u * k + 1u;
    }
  }
  return 0.5f * (low + high);
}

// ---- Smits RGB -> spectrum (shading/smits.wesl, material.wesl:264-297) ---------------
// In global memory and read through the read-only data cache: lanes look up
// different bins (their wavelengths differ), which constant memory would
// serialise one address at a time; L1 serves a warp's lanes from the same
// lines in one pass.
__device__ const float kBins[10] = {380.0f, 417.7778f, 455.5556f, 493.3333f, 531.1111f,
                                    568.8889f, 606.6667f, 644.4444f, 682.2222f, 720.0f};
__device__ const float kSmits[7][10] = {
    {1.0f, 1.0f, 0.9999f, 0.9993f, 0.9992f, 0.9998f, 1.0f, 1.0f, 1.0f, 1.0f},                 // white
    {0.1012f, 0.0515f, 0.0f, 0.0f, 0.0f, 0.0f, 0.8325f, 1.0149f, 1.0149f, 1.0149f},           // red
    {0.0f, 0.0f, 0.0273f, 0.7937f, 1.0f, 0.9418f, 0.1719f, 0.0f, 0.0f, 0.0025f},              // green
    {1.0f, 1.0f, 0.8916f, 0.3323f, 0.0f, 0.0f, 0.0003f, 0.0369f, 0.0483f, 0.0496f},           // blue
    {1.0f, 1.0f, 0.9685f, 0.2229f, 0.0f, 0.0458f, 0.8369f, 1.0f, 1.0f, 0.9959f},              // magenta
    {0.971f, 0.9426f, 1.0007f, 1.0007f, 1.0007f, 1.0007f, 0.1564f, 0.0f, 0.0f, 0.0f},         // cyan
    {0.0001f, 0.0f, 0.1088f, 0.6651f, 1.0f, 1.0f, 0.9996f, 0.9586f, 0.9685f, 0.984f}};        // yellow
enum { SM_WHITE = 0, SM_RED, SM_GREEN, SM_BLUE, SM_MAGENTA, SM_CYAN, SM_YELLOW };

// Built with CG_SMITS_SHARED, the shading kernels copy the bins and curves
// into shared memory at their start (stageSmitsTables) and read them there;
// otherwise they read the global copies above through the read-only cache.
#ifdef CG_SMITS_SHARED
__shared__ float s_smits_tables[80];  // 10 bins, then the 7 curves
__device__ __forceinline__ void stageSmitsTables() {
  for (int i = threadIdx.x; i < 80; i += blockDim.x)
    s_smits_tables[i] = i < 10 ? kBins[i] : kSmits[(i - 10) / 10][(i - 10) % 10];
  __syncthreads();
}
__device__ __forceinline__ float smitsBin(uint32_t i) { return s_smits_tables[i]; }
__device__ __forceinline__ float smitsCurve(int curve, uint32_t i) {
  return s_smits_tables[10 + curve * 10 + i];
}
#else
__device__ __forceinline__ void stageSmitsTables() {}
__device__ __forceinline__ float smitsBin(uint32_t i) { return __ldg(&kBins[i]); }
__device__ __forceinline__ float smitsCurve(int curve, uint32_t i) { return __ldg(&kSmits[curve][i]); }
#endif

// Per-wavelength lookup position shared by all seven curves.
struct SmitsPos {
  int mode;  // 0: below 380, 1: above 720, 2: interpolate
  uint32_t b0, b1;
  float mixv;
};
__device__ __forceinline__ SmitsPos smitsPos(float w) {
  SmitsPos p{2, 0u, 0u, 0.0f};
  if (w <= 380.0f) {
    p.mode = 0;
    return p;
  }
  if (w >= 720.0f) {
    p.mode = 1;
    return p;
  }
  uint32_t bin = static_cast<uint32_t>(10.0f * (w - 380.0f) / 340.0f);
  p.b0 = bin > 9u ? 9u : bin;
  p.b1 = (bin + 1u) > 9u ? 9u : bin + 1u;  // WGSL robust access clamps index 10 to 9
  const float lo = smitsBin(p.b0), hi = smitsBin(p.b1);
  p.mixv = (w - lo) / (hi - lo);
  return p;
}
__device__ __forceinline__ float smits(const SmitsPos& p, int curve) {
  if (p.mode == 0) return smitsCurve(curve, 0);
  if (p.mode == 1) return smitsCurve(curve, 9);
  return (1.0f - p.mixv) * smitsCurve(curve, p.b0) + p.mixv * smitsCurve(curve, p.b1);
}
__device__ __forceinline__ float rgbToSpectrum(V3 rgb, const SmitsPos& sp) {
  float s = 0.0f;
  float r = rgb.x, g = rgb.y, b = rgb.z;
  if (r <= g && g <= b) {
    s += r * smits(sp, SM_WHITE);
    s += (g - r) * smits(sp, SM_CYAN);
    s += (b - g) * smits(sp, SM_BLUE);
  } else if (g <= r && g <= b) {
    s += g * smits(sp, SM_WHITE);
    if (r <= b) {
      s += (r - g) * smits(sp, SM_MAGENTA);
      s += (b - r) * smits(sp, SM_BLUE);
    } else {
      s += (b - g) * smits(sp, SM_MAGENTA);
      s += (r - b) * smits(sp, SM_RED);
    }
  } else {
    s += b * smits(sp, SM_WHITE);
    if (r <= g) {
      s += (r - b) * smits(sp, SM_YELLOW);
      s += (g - r) * smits(sp, SM_GREEN);
    } else {
      s += (g - b) * smits(sp, SM_YELLOW);
      s += (r - g) * smits(sp, SM_RED);
    }
  }
  return s;
}
__device__ __forceinline__ float rgbToReflectance(V3 rgb, const SmitsPos& sp) {
  return wclamp(0.94f * rgbToSpectrum(rgb, sp), 0.0f, 1.0f);
}
__device__ __forceinline__ float rgbToRadiance(V3 rgb, const SmitsPos& sp) {
  return fmaxf(rgbToSpectrum(rgb, sp), 0.0f);
}

// ---- sRGB resolve (physics/srgb.wesl:5-27) -------------------------------------------
__device__ __forceinline__ float encodeChannel(float linear) {
  float value = fmaxf(linear, 0.0f);
  float encoded = (value <= 0.0031308f) ? 12.92f * value : 1.055f * powf(value, 1.0f / 2.4f) - 0.055f;
  return wclamp(encoded, 0.0f, 1.0f);
}
__device__ __forceinline__ V3 xyzToLinearSrgb(V3 l) {
  M3 m{v3(2.36461385f, -0.51516621f, 0.0052037f), v3(-0.89654057f, 1.4264081f, -0.01440816f),
       v3(-0.46807328f, 0.0887581f, 1.00920446f)};
  return mul(m, l);
}

// ---- materials (shading/material.wesl:19-110) ------------------------------------------
struct IOR {
  float re, im;
};
struct Mat {
  float diffuse_reflectance, microfacet_roughness;
  IOR ior;
  float transmission;
  bool volume;
  float emission;
};
// decode (material.wesl:19-53) from the material values after any texture
// lookups: base color rgb, metallic, roughness, transmission (clamped) and
// the emission max(factor * strength, 0).
__device__ __forceinline__ Mat decodeValues(const DevMaterial& m, V3 base, float metallic,
                                            float roughness, float transmission, V3 emission,
                                            float w, const SmitsPos& sp) {
  float reflectance = rgbToReflectance(base, sp);
  float real_ior = m.ior;
  if (metallic == 0.0f && transmission > 0.0f && !(m.dispersion <= 0.0f)) {
    float inv_abbe = m.dispersion / 20.0f;
    real_ior = fmaxf(m.ior + (m.ior - 1.0f) * inv_abbe * (523655.0f / (w * w) - 1.5168f), 1.0f);
  }
  const float ip1 = real_ior + 1.0f;  // pow(real_ior + 1, 2) as a product
  float im = sqrtf(wclamp((4.0f * real_ior) / (1.0f - reflectance) - ip1 * ip1, 0.0f, 10.0f));
  Mat e;
  e.diffuse_reflectance = (1.0f - metallic) * (1.0f - transmission) * reflectance;
  e.microfacet_roughness = roughness * roughness;
  e.ior = IOR{real_ior, metallic * im};
  e.transmission = transmission;
  e.volume = (m.volume & 1u) != 0u;
  e.emission = rgbToReflectance(emission, sp);
  return e;
}

__device__ __forceinline__ Mat decode(const DevMaterial& m, float w, const SmitsPos& sp) {
  return decodeValues(m, V3{m.base[0], m.base[1], m.base[2]}, m.metallic, m.roughness,
                      m.transmission, V3{m.emission[0], m.emission[1], m.emission[2]}, w, sp);
}

// textureSampleLevel(material_textures, sampler, uv, layer, 0) with the
// reference's sampler (linear filtering, clamp to edge; src/wgpu/resource.cpp:
// 133-142) on the RGBA8Unorm array: texel centres at (i + 0.5) / size,
// bilinear weights in float, rounded per operation as the CPU restatement.
// x and y are clamped to [-1, size] first (beyond that every tap is the edge
// texel), which keeps the integer conversion in range.
__device__ __forceinline__ float4 sampleMaterialTexture(const SceneView& sc, int layer, float u,
                                                        float v) {
  const float W = static_cast<float>(sc.tex_w), H = static_cast<float>(sc.tex_h);
  const float x = fminf(fmaxf(__fsub_rn(__fmul_rn(u, W), 0.5f), -1.0f), W);
  const float y = fminf(fmaxf(__fsub_rn(__fmul_rn(v, H), 0.5f), -1.0f), H);
  const float fx = floorf(x), fy = floorf(y);
  const float ax = __fsub_rn(x, fx), ay = __fsub_rn(y, fy);
  const int wmax = static_cast<int>(sc.tex_w) - 1, hmax = static_cast<int>(sc.tex_h) - 1;
  const int x0 = min(max(static_cast<int>(fx), 0), wmax), x1 = min(max(static_cast<int>(fx) + 1, 0), wmax);
  const int y0 = min(max(static_cast<int>(fy), 0), hmax), y1 = min(max(static_cast<int>(fy) + 1, 0), hmax);
  const uchar4* L = sc.tex + static_cast<size_t>(layer) * sc.tex_w * sc.tex_h;
  const uchar4 t00 = __ldg(L + y0 * sc.tex_w + x0), t10 = __ldg(L + y0 * sc.tex_w + x1);
  const uchar4 t01 = __ldg(L + y1 * sc.tex_w + x0), t11 = __ldg(L + y1 * sc.tex_w + x1);
  const float bx = __fsub_rn(1.0f, ax), by = __fsub_rn(1.0f, ay);
  auto ch = [&](unsigned char a, unsigned char b, unsigned char c, unsigned char d) {
    const float fa = __fdiv_rn(static_cast<float>(a), 255.0f), fb = __fdiv_rn(static_cast<float>(b), 255.0f);
    const float fc = __fdiv_rn(static_cast<float>(c), 255.0f), fd = __fdiv_rn(static_cast<float>(d), 255.0f);
    const float top = __fadd_rn(__fmul_rn(fa, bx), __fmul_rn(fb, ax));
    const float bot = __fadd_rn(__fmul_rn(fc, bx), __fmul_rn(fd, ax));
    return __fadd_rn(__fmul_rn(top, by), __fmul_rn(bot, ay));
  };
  return make_float4(ch(t00.x, t10.x, t01.x, t11.x), ch(t00.y, t10.y, t01.y, t11.y),
                     ch(t00.z, t10.z, t01.z, t11.z), ch(t00.w, t10.w, t01.w, t11.w));
}

// decode for a material with textures: each texel multiplies its factor
// before the clamp (baseColor, roughness, metallic, transmission, emission;
// material.wesl:181-262).  uv: TEXCOORD_0.xy, TEXCOORD_1.xy at the hit.
__device__ __forceinline__ Mat decodeTextured(const SceneView& sc, const DevMaterial& m,
                                              const DevMatTex& t, float4 uv, float w,
                                              const SmitsPos& sp) {
  auto texel = [&](int k) {
    const bool set1 = (t.uv1_bits >> k) & 1u;
    return sampleMaterialTexture(sc, t.layer[k], set1 ? uv.z : uv.x, set1 ? uv.w : uv.y);
  };
  V3 base{m.base[0], m.base[1], m.base[2]};
  if (t.layer[0] >= 0) {
    const float4 c = texel(0);
    base = V3{base.x * c.x, base.y * c.y, base.z * c.z};
  }
  float metallic = m.metallic, roughness = m.roughness, transmission = m.transmission;
  if (t.layer[1] >= 0) {
    const float4 c = texel(1);
    roughness = wclamp(t.roughness * c.y, 0.0f, 1.0f);
    metallic = wclamp(t.metallic * c.z, 0.0f, 1.0f);
  }
  if (t.layer[3] >= 0) transmission = wclamp(t.transmission * texel(3).x, 0.0f, 1.0f);
  V3 emission{m.emission[0], m.emission[1], m.emission[2]};
  if (t.layer[2] >= 0) {
    const float4 c = texel(2);
    const V3 f{t.emissive[0] * c.x, t.emissive[1] * c.y, t.emissive[2] * c.z};
    emission = V3{fmaxf(f.x * t.emissive_strength, 0.0f), fmaxf(f.y * t.emissive_strength, 0.0f),
                  fmaxf(f.z * t.emissive_strength, 0.0f)};
  }
  return decodeValues(m, base, metallic, roughness, transmission, emission, w, sp);
}

// ---- shading utilities (shading/util.wesl) ------------------------------------------
__device__ __forceinline__ V3 orientedNormal(V3 curr, V3 n) { return dot(curr, n) > 0.0f ? -n : n; }
__device__ __forceinline__ IOR invIor(IOR i) {
  float ns = i.re * i.re + i.im * i.im;
  return IOR{i.re / ns, -i.im / ns};
}
__device__ __forceinline__ IOR relIor(V3 sn, V3 curr, const Mat& m) {
  return dot(sn, curr) < 0.0f ? invIor(m.ior) : m.ior;
}
__device__ __forceinline__ float complexFresnel(float c, IOR mi) {
  float re = mi.re, im = mi.im;
  float ns = re * re + im * im, cs = c * c;
  float trc = 2.0f * re * c;
  float perp = (ns - trc + cs) / fmaxf(ns + trc + cs, 1e-6f);
  float par = (ns * cs - trc + 1.0f) / fmaxf(ns * cs + trc + 1.0f, 1e-6f);
  return wclamp(0.5f * (perp + par), 0.0f, 1.0f);
}
__device__ __forceinline__ float fresnel(V3 curr, V3 normal, IOR rel) {
  float ic = wclamp(dot(-curr, normal), 0.0f, 1.0f);
  if (fabsf(rel.im) > 1e-6f) return complexFresnel(ic, rel);
  float r = rel.re;
  float tss = r * r * fmaxf(0.0f, 1.0f - ic * ic);
  if (tss >= 1.0f) return 1.0f;
  float tc = sqrtf(fmaxf(0.0f, 1.0f - tss));
  float perp = (r * ic - tc) / (r * ic + tc);
  float par = (ic - r * tc) / (ic + r * tc);
  return wclamp(0.5f * (perp * perp + par * par), 0.0f, 1.0f);
}

struct Surf {
  V3 pos, sn, gn;
};

// ---- GGX (pdf/rough_*.wesl, dist/rough_*.wesl) -------------------------------------------
constexpr float VNDF_EPS = 1e-6f;
__device__ __forceinline__ float ggxD(V3 micro, V3 macro, float alpha) {
  float nc = wclamp(dot(micro, macro), 0.0f, 1.0f);
  float nts = fmaxf(0.0f, 1.0f - nc * nc) / fmaxf(nc * nc, VNDF_EPS);
  // pow(nc, 4) and pow(alpha + nts, 2) as products (the same values up to
  // rounding; powf's log / exp sequence costs some forty instructions)
  const float nc2 = nc * nc, an = alpha + nts;
  float denom = PI * (nc2 * nc2) * (an * an);
  return alpha / fmaxf(denom, VNDF_EPS);
}
// The masking terms take the cosine c of the angle whose tangent they need:
// the reference forms tan(acos(c)), here sqrt(1 - c^2) / c, the same value
// without the two transcendental calls.  Like acos, it is NaN for c > 1 (a
// dot product of unit vectors a rounding step above 1), which keeps the
// reference's unclamped-acos NaN samples; c >= 1e-6 at every call.
__device__ __forceinline__ float tanOfAcos(float c) { return sqrtf(fmaf(-c, c, 1.0f)) / c; }
__device__ __forceinline__ float ggxLambdaTerm(float cos_angle, float alpha) {
  float t = tanOfAcos(cos_angle);
  return (sqrtf(1.0f + alpha * t * t) - 1.0f) / 2.0f;
}
__device__ __forceinline__ float ggxG1(float cos_angle, float alpha) {
  return 1.0f / (1.0f + ggxLambdaTerm(cos_angle, alpha));
}
__device__ __forceinline__ float ggxG2(float c1, float c2, float alpha) {
  return 1.0f / (1.0f + ggxLambdaTerm(c1, alpha) + ggxLambdaTerm(c2, alpha));
}
__device__ __forceinline__ V3 sampleNorm(V3 curr, const Surf& s, float alpha, Rng& rng) {
  V3 macro = orientedNormal(curr, s.sn);
  M3 ts = makeTangentSpace(macro);
  V3 lc = normalize(mulT(ts, -curr));
  V3 st = normalize(V3{alpha * lc.x, alpha * lc.y, fmaxf(lc.z, VNDF_EPS)});
  float tl2 = st.x * st.x + st.y * st.y;
  V3 tx = tl2 > VNDF_EPS ? V3{-st.y, st.x, 0.0f} / sqrtf(fmaxf(tl2, VNDF_EPS)) : V3{1.0f, 0.0f, 0.0f};
  V3 ty = cross(st, tx);
  float radius = sqrtf(randFloat(rng));
  float angle = 2.0f * PI * randFloat(rng);
  float sa, ca;
  sincosf(angle, &sa, &ca);
  float px = radius * ca;
  float py = radius * sa;
  float vis = 0.5f * (1.0f + st.z);
  py = wmix(sqrtf(fmaxf(0.0f, 1.0f - px * px)), py, vis);
  V3 lsm = px * tx + py * ty + sqrtf(fmaxf(0.0f, 1.0f - px * px - py * py)) * st;
  V3 lm = normalize(V3{alpha * lsm.x, alpha * lsm.y, fmaxf(lsm.z, VNDF_EPS)});
  return normalize(mul(ts, lm));
}
__device__ __forceinline__ float reflectPdf(V3 curr, V3 micro, V3 macro, float alpha) {
  float cmp = fmaxf(dot(-curr, macro), VNDF_EPS);
  float cmi = fmaxf(dot(-curr, micro), VNDF_EPS);
  float vnp = ggxD(micro, macro, alpha) * ggxG1(cmp, alpha) * cmi / cmp;
  return vnp / (4.0f * cmi);
}
__device__ __forceinline__ float relIorT(IOR i) { return fmaxf(i.re, VNDF_EPS); }
__device__ __forceinline__ float transmitPdf(V3 curr, V3 micro, V3 macro, V3 next, float tior,
                                             float alpha) {
  float cmp = fmaxf(dot(-curr, macro), VNDF_EPS);
  float cmi = fmaxf(dot(-curr, micro), VNDF_EPS);
  float vnp = ggxD(micro, macro, alpha) * ggxG1(cmp, alpha) * cmi / cmp;
  float nmi = dot(next, micro);
  float denom = nmi + cmi / tior;
  return vnp * cmi / fmaxf(denom * denom, VNDF_EPS);
}

// ---- lobe pdfs (shading/pdf/*.wesl) ------------------------------------------------------
__device__ __forceinline__ float diffusePdf(V3 curr, V3 next, const Surf& s) {
  return fmaxf(dot(next, orientedNormal(curr, s.sn)), 0.0f) / PI;
}
__device__ __forceinline__ V3 specularDir(V3 curr, const Surf& s) {
  return reflect(curr, orientedNormal(curr, s.sn));
}
__device__ __forceinline__ float specularReflectPdf(V3 curr, V3 next, const Surf& s) {
  V3 e = specularDir(curr, s);
  V3 d = next - e;
  return dot(d, d) <= 1e-6f ? 1.0f : 0.0f;
}
__device__ __forceinline__ float roughReflectPdf(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 macro = orientedNormal(curr, s.sn);
  if (dot(next, macro) <= 0.0f) return 0.0f;
  V3 mu = next - curr;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 micro = orientedNormal(curr, normalize(mu));
  return reflectPdf(curr, micro, macro, m.microfacet_roughness);
}
__device__ __forceinline__ V3 specularTransmissionDir(V3 curr, const Surf& s, const Mat& m) {
  if (m.volume) {
    IOR rel = relIor(s.sn, curr, m);
    return refract(curr, orientedNormal(curr, s.sn), rel.re);
  }
  return curr;
}
__device__ __forceinline__ float specularTransmitPdf(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 e = specularTransmissionDir(curr, s, m);
  V3 d = next - e;
  return (dot(e, e) > 1e-6f && dot(d, d) <= 1e-6f) ? 1.0f : 0.0f;
}
__device__ __forceinline__ float roughTransmitPdf(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 macro = orientedNormal(curr, s.sn);
  if (dot(next, macro) >= 0.0f) return 0.0f;
  float mriv = relIorT(relIor(macro, curr, m));
  V3 mu = mriv * curr - next;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 micro = orientedNormal(curr, normalize(mu));
  IOR rel = relIor(micro, curr, m);
  return transmitPdf(curr, micro, macro, next, 1.0f / relIorT(rel), m.microfacet_roughness);
}

// ---- BSDF values (shading/dist/*.wesl) ------------------------------------------------------
__device__ __forceinline__ float diffuseDist(V3 curr, V3 next, const Surf& s, const Mat& m) {
  float np = fmaxf(dot(next, orientedNormal(curr, s.sn)), 0.0f);
  return m.diffuse_reflectance * np / PI;
}
__device__ __forceinline__ float specularReflectDist(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 macro = orientedNormal(curr, s.sn);
  V3 e = reflect(curr, macro);
  V3 d = next - e;
  float dd = dot(d, d) <= 1e-6f ? 1.0f : 0.0f;
  return fresnel(curr, macro, relIor(s.sn, curr, m)) * dd;
}
__device__ __forceinline__ float roughReflectDist(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 macro = orientedNormal(curr, s.sn);
  float np = fmaxf(dot(next, macro), 0.0f);
  if (np <= 0.0f) return 0.0f;
  V3 mu = next - curr;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 raw = normalize(mu);
  V3 micro = orientedNormal(curr, raw);
  IOR rel = relIor(raw, curr, m);
  float alpha = m.microfacet_roughness;
  float cmp = fmaxf(dot(-curr, macro), VNDF_EPS);
  float nmp = fmaxf(dot(next, macro), VNDF_EPS);
  float rd = ggxD(micro, macro, alpha) * ggxG2(cmp, nmp, alpha) / (4.0f * cmp * nmp);
  return fresnel(curr, micro, rel) * rd * np;
}
__device__ __forceinline__ float specularTransmitDist(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 macro = orientedNormal(curr, s.sn);
  V3 e = specularTransmissionDir(curr, s, m);
  V3 d = next - e;
  float dd = dot(d, d) <= 1e-6f ? 1.0f : 0.0f;
  return m.transmission * (1.0f - fresnel(curr, macro, relIor(s.sn, curr, m))) * dd;
}
__device__ __forceinline__ float roughTransmitDist(V3 curr, V3 next, const Surf& s, const Mat& m) {
  V3 macro = orientedNormal(curr, s.sn);
  if (dot(next, macro) >= 0.0f) return 0.0f;
  float np = fmaxf(dot(-next, macro), 0.0f);
  float mriv = relIorT(relIor(macro, curr, m));
  V3 mu = mriv * curr - next;
  if (dot(mu, mu) <= VNDF_EPS) return 0.0f;
  V3 raw = normalize(mu);
  V3 micro = orientedNormal(curr, raw);
  IOR rel = relIor(raw, curr, m);
  float tior = 1.0f / relIorT(rel);
  float alpha = m.microfacet_roughness;
  float cmp = fmaxf(dot(-curr, macro), VNDF_EPS);
  float nmp = fmaxf(dot(-next, macro), VNDF_EPS);
  float cmi = fmaxf(dot(-curr, micro), VNDF_EPS);
  float nmi = dot(next, micro);
  float denom = nmi + cmi / tior;
  float td = m.transmission * ggxD(micro, macro, alpha) * ggxG2(cmp, nmp, alpha) *
             fabsf(cmi * nmi) / fmaxf(cmp * nmp * denom * denom, VNDF_EPS);
  return (1.0f - fresnel(curr, micro, rel)) * td * np;
}

// ---- sample counts (shading/sample.wesl:151-299, lod.wesl) ------------------------------
struct SampleCaps {
  uint32_t trace_depth, transport_cap, emission_cap, diffuse_cap, rough_cap;
};
struct Counts {
  uint32_t diffuse, specular_reflect, rough_reflect, specular_transmit, rough_transmit, light;
};
__device__ __forceinline__ uint32_t u32f(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967295.0f) return 0xffffffffu;
  return static_cast<uint32_t>(x);
}
__device__ __forceinline__ uint32_t scaledCount(float h, float scale, uint32_t maxc) {
  if (h <= 1e-6f) return 0u;
  return min(max(1u, u32f(h * scale)), maxc);
}
__device__ __forceinline__ Counts counts(const Mat& m, bool can_sample_light, int depth,
                                         const SampleCaps& c) {
  float lo = m.ior.re - 1.0f, hi = m.ior.re + 1.0f, im2 = m.ior.im * m.ior.im;
  float refl_h = wclamp((lo * lo + im2) / fmaxf(hi * hi + im2, 1e-6f), 0.0f, 1.0f);
  float diffuse_h = m.diffuse_reflectance;
  float trans_h = m.transmission;
  float sr = m.microfacet_roughness == 0.0f ? refl_h : 0.0f;
  float rr = m.microfacet_roughness > 0.0f ? refl_h : 0.0f;
  float st = (trans_h > 1e-6f && m.microfacet_roughness == 0.0f) ? trans_h : 0.0f;
  float rt = (trans_h > 1e-6f && m.microfacet_roughness > 0.0f) ? trans_h : 0.0f;
  int32_t maxd = static_cast<int32_t>(c.trace_depth);
  float heur = static_cast<float>(maxd - depth) / static_cast<float>(maxd);
  uint32_t ta = u32f(heur * static_cast<float>(min(c.transport_cap, 4u)));
  uint32_t ea = u32f(heur * static_cast<float>(min(c.emission_cap, 1u)));
  Counts out{0u, 0u, 0u, 0u, 0u, 0u};
  float hsum = diffuse_h + sr + rr + st + rt;
  if (!(ta == 0u || hsum <= 1e-6f)) {
    float scale = static_cast<float>(ta) / hsum;
    uint32_t rem = ta;
    out.diffuse = min(scaledCount(diffuse_h, scale, min(c.diffuse_cap, 1u)), rem);
    rem -= out.diffuse;
    out.specular_reflect = min(scaledCount(sr, scale, 1u), rem);
    rem -= out.specular_reflect;
    out.rough_reflect = min(scaledCount(rr, scale, min(c.rough_cap, 1u)), rem);
    rem -= out.rough_reflect;
    out.specular_transmit = min(scaledCount(st, scale, 1u), rem);
    rem -= out.specular_transmit;
    out.rough_transmit = min(scaledCount(rt, scale, min(c.rough_cap, 1u)), rem);
  }
  out.light = (can_sample_light && ea > 0u) ? max(1u, ea) : 0u;
  return out;
}

__device__ __forceinline__ bool sameCounts(const Counts& a, const Counts& b) {
  return a.diffuse == b.diffuse && a.specular_reflect == b.specular_reflect &&
         a.rough_reflect == b.rough_reflect && a.specular_transmit == b.specular_transmit &&
         a.rough_transmit == b.rough_transmit && a.light == b.light;
}

// ---- hero-wavelength sampling (an option beside the reference's sampler) -------------
// Four wavelengths per sample (Wilkie et al. 2014): the hero at offset x0 in
// [0, 400] nm above 380 (x0 = 400 u from the sample's wavelength stream), the
// others rotated by 100 nm each, wrapped into the range; each is uniform on
// [380, 780].  The offset is what the sample slot keeps; every kernel derives
// the four wavelengths from it with these same rounded operations.
constexpr int kHeroCount = 4;
__device__ __forceinline__ float heroOffset(float u) { return __fmul_rn(400.0f, u); }
__device__ __forceinline__ float heroWavelength(float x0, int j) {
  float x = __fadd_rn(x0, 100.0f * static_cast<float>(j));
  if (x >= 400.0f) x = __fsub_rn(x, 400.0f);
  return __fadd_rn(380.0f, x);
}

}  // namespace dev
}  // namespace cg

#endif
