/*
 * cg_oracle_spectral.h — spectral modules of the reference restated for the
 * oracle (TEST INFRASTRUCTURE ONLY): CIE fits (physics/cie.wesl), wavelength
 * sampling (physics/wavelength.wesl), XYZ weighting (physics/luminance.wesl),
 * sRGB resolve (physics/srgb.wesl), Smits RGB->spectrum
 * (shading/smits.wesl, shading/material.wesl:264-297,
 * shading/pdf/emission.wesl:84-118).
 */
#ifndef CG_ORACLE_SPECTRAL_H_
#define CG_ORACLE_SPECTRAL_H_

#include <cmath>
#include <cstdint>

#include "cg_oracle_math.h"

namespace oracle {

// ---- physics/cie.wesl:1-140 ---------------------------------------------
constexpr float SQRT_HALF_PI = 1.2533141373155001f;
constexpr float INV_SQRT_TWO = 0.7071067811865475f;

inline float splitGaussian(float w, float c, float lw, float rw) {
  float width = (w < c) ? lw : rw;
  float scaled = (w - c) / width;
  return std::exp(-0.5f * scaled * scaled);
}
inline float erfApprox(float x) {
  float sign = (x >= 0.0f) ? 1.0f : -1.0f;
  float ax = std::fabs(x);
  float t = 1.0f / (1.0f + 0.3275911f * ax);
  float poly = (((((1.061405429f * t - 1.453152027f) * t) + 1.421413741f) * t -
                 0.284496736f) * t + 0.254829592f) * t;
  return sign * (1.0f - poly * std::exp(-ax * ax));
}
inline float splitGaussianAntiderivative(float w, float c, float lw, float rw) {
  if (w < c) {
    return SQRT_HALF_PI * lw * (1.0f + erfApprox((w - c) * INV_SQRT_TWO / lw));
  }
  return SQRT_HALF_PI * lw + SQRT_HALF_PI * rw * erfApprox((w - c) * INV_SQRT_TWO / rw);
}
inline float splitGaussianIntegral(float lo, float hi, float c, float lw, float rw) {
  return splitGaussianAntiderivative(hi, c, lw, rw) - splitGaussianAntiderivative(lo, c, lw, rw);
}

inline float xMatch(float w) {
  return 0.362f * splitGaussian(w, 442.0f, 1.0f / 0.0624f, 1.0f / 0.0374f) +
         1.056f * splitGaussian(w, 599.8f, 1.0f / 0.0264f, 1.0f / 0.0323f) -
         0.065f * splitGaussian(w, 501.1f, 1.0f / 0.0490f, 1.0f / 0.0382f);
}
inline float yMatch(float w) {
  return 0.821f * splitGaussian(w, 568.8f, 1.0f / 0.0213f, 1.0f / 0.0247f) +
         0.286f * splitGaussian(w, 530.9f, 1.0f / 0.0613f, 1.0f / 0.0322f);
}
inline float zMatch(float w) {
  return 1.217f * splitGaussian(w, 437.0f, 1.0f / 0.0845f, 1.0f / 0.0278f) +
         0.681f * splitGaussian(w, 459.0f, 1.0f / 0.0385f, 1.0f / 0.0725f);
}
inline V3 xyzMatch(float w) { return {xMatch(w), yMatch(w), zMatch(w)}; }
inline float xyzMatchSum(float w) {
  V3 m = xyzMatch(w);
  return m.x + m.y + m.z;
}
inline float xIntegral(float lo, float hi) {
  return 0.362f * splitGaussianIntegral(lo, hi, 442.0f, 1.0f / 0.0624f, 1.0f / 0.0374f) +
         1.056f * splitGaussianIntegral(lo, hi, 599.8f, 1.0f / 0.0264f, 1.0f / 0.0323f) -
         0.065f * splitGaussianIntegral(lo, hi, 501.1f, 1.0f / 0.0490f, 1.0f / 0.0382f);
}
inline float yIntegral(float lo, float hi) {
  return 0.821f * splitGaussianIntegral(lo, hi, 568.8f, 1.0f / 0.0213f, 1.0f / 0.0247f) +
         0.286f * splitGaussianIntegral(lo, hi, 530.9f, 1.0f / 0.0613f, 1.0f / 0.0322f);
}
inline float zIntegral(float lo, float hi) {
  return 1.217f * splitGaussianIntegral(lo, hi, 437.0f, 1.0f / 0.0845f, 1.0f / 0.0278f) +
         0.681f * splitGaussianIntegral(lo, hi, 459.0f, 1.0f / 0.0385f, 1.0f / 0.0725f);
}
inline float xyzMatchSumIntegral(float lo, float hi) {
  return xIntegral(lo, hi) + yIntegral(lo, hi) + zIntegral(lo, hi);
}

// ---- physics/wavelength.wesl:14-45 -----------------------------------------
constexpr float VISIBLE_MIN = 380.0f;
constexpr float VISIBLE_MAX = 720.0f;

struct WavelengthSample {
  float wavelength, prob;
};
inline WavelengthSample sampleWavelengthCdf(float cdf_sample) {
  float total_match = xyzMatchSumIntegral(VISIBLE_MIN, VISIBLE_MAX);
  float target_cdf = wclamp(cdf_sample, 0.0f, 0.999999f);
  float low = VISIBLE_MIN, high = VISIBLE_MAX;
  for (uint32_t i = 0; i < 16u; ++i) {
    float mid = 0.5f * (low + high);
    float cdf = xyzMatchSumIntegral(VISIBLE_MIN, mid) / total_match;
    if (cdf < target_cdf)
      low = mid;
    else
      high = mid;
  }
  float wavelength = 0.5f * (low + high);
  return {wavelength, wmax(xyzMatchSum(wavelength) / total_match, 1e-6f)};
}

// ---- hero-wavelength sampling (an option beside the reference's sampler) -----
// Four wavelengths per sample: the hero uniform on [380, 780] nm from one
// random number, the others rotated by a quarter of the range each (Wilkie et
// al. 2014, "Hero Wavelength Spectral Sampling").  Each is uniform on the
// range, so a sample's estimate is (1/4) sum_j illuminate(w_j, L_j) / (1/400).
constexpr int HERO_COUNT = 4;
constexpr float HERO_MIN = 380.0f;
constexpr float HERO_SPAN = 400.0f;
inline void heroWavelengths(float u, float (&w)[HERO_COUNT]) {
  const float x0 = HERO_SPAN * u;  // offset of the hero in the range
  for (int j = 0; j < HERO_COUNT; ++j) {
    float x = x0 + (HERO_SPAN / HERO_COUNT) * static_cast<float>(j);
    if (x >= HERO_SPAN) x = x - HERO_SPAN;
    w[j] = HERO_MIN + x;
  }
}

// ---- physics/luminance.wesl:13-16 ------------------------------------------
inline V3 illuminate(float wavelength, float radiance) {
  float average_integral = xyzMatchSumIntegral(380.0f, 720.0f) / 3.0f;
  return xyzMatch(wavelength) * radiance / average_integral;
}

// ---- physics/srgb.wesl:5-27 --------------------------------------------------
inline float encodeChannel(float linear) {
  float value = wmax(linear, 0.0f);
  float encoded = (value <= 0.0031308f) ? 12.92f * value
                                        : 1.055f * std::pow(value, 1.0f / 2.4f) - 0.055f;
  return wclamp(encoded, 0.0f, 1.0f);
}
inline V3 xyzToLinearSrgb(V3 l) {
  M3 m{{v3(2.36461385f, -0.51516621f, 0.0052037f), v3(-0.89654057f, 1.4264081f, -0.01440816f),
        v3(-0.46807328f, 0.0887581f, 1.00920446f)}};
  return mul(m, l);
}
inline V3 luminanceToSrgb(V3 l) {
  V3 lin = xyzToLinearSrgb(l);
  return {encodeChannel(lin.x), encodeChannel(lin.y), encodeChannel(lin.z)};
}

// ---- shading/smits.wesl:3-124 -----------------------------------------------
// BINS are spaced 340/9 nm but bin = u32(10 * (w - 380) / 340).  For
// w in [686, 720) bin + 1 == 10 is out of range; the documented semantics is
// WGSL-robustness index clamping (10 -> 9), which makes the mix 0/0-like
// (-inf) and the curve NaN; callers' IEEE max/clamp then drop it.
constexpr float BINS[10] = {380.0f,   417.7778f, 455.5556f, 493.3333f, 531.1111f,
                            568.8889f, 606.6667f, 644.4444f, 682.2222f, 720.0f};
constexpr float WHITE[10] = {1.0f, 1.0f, 0.9999f, 0.9993f, 0.9992f, 0.9998f, 1.0f, 1.0f, 1.0f, 1.0f};
constexpr float RED[10] = {0.1012f, 0.0515f, 0.0f, 0.0f, 0.0f, 0.0f, 0.8325f, 1.0149f, 1.0149f, 1.0149f};
constexpr float GREEN[10] = {0.0f, 0.0f, 0.0273f, 0.7937f, 1.0f, 0.9418f, 0.1719f, 0.0f, 0.0f, 0.0025f};
constexpr float BLUE[10] = {1.0f, 1.0f, 0.8916f, 0.3323f, 0.0f, 0.0f, 0.0003f, 0.0369f, 0.0483f, 0.0496f};
constexpr float MAGENTA[10] = {1.0f, 1.0f, 0.9685f, 0.2229f, 0.0f, 0.0458f, 0.8369f, 1.0f, 1.0f, 0.9959f};
constexpr float CYAN[10] = {0.971f, 0.9426f, 1.0007f, 1.0007f, 1.0007f, 1.0007f, 0.1564f, 0.0f, 0.0f, 0.0f};
constexpr float YELLOW[10] = {0.0001f, 0.0f, 0.1088f, 0.6651f, 1.0f, 1.0f, 0.9996f, 0.9586f, 0.9685f, 0.984f};

inline float smitsCurve(const float* X, float w) {
  if (w <= 380.0f) return X[0];
  if (w >= 720.0f) return X[9];
  uint32_t bin = static_cast<uint32_t>(10.0f * (w - 380.0f) / 340.0f);
  uint32_t b0 = bin > 9u ? 9u : bin;
  uint32_t b1 = (bin + 1u) > 9u ? 9u : bin + 1u;
  float mixv = (w - BINS[b0]) / (BINS[b1] - BINS[b0]);
  return (1.0f - mixv) * X[b0] + mixv * X[b1];
}

// Shared body of rgbToWavelengthReflectance (material.wesl:264-297) and
// rgbToWavelengthRadiance (pdf/emission.wesl:84-118, environment.wesl:27-61).
inline float rgbToSpectrum(V3 rgb, float w) {
  float s = 0.0f;
  float r = rgb.x, g = rgb.y, b = rgb.z;
  if (r <= g && g <= b) {
    s += r * smitsCurve(WHITE, w);
    if (g <= b) {
      s += (g - r) * smitsCurve(CYAN, w);
      s += (b - g) * smitsCurve(BLUE, w);
    } else {
      s += (b - r) * smitsCurve(CYAN, w);
      s += (g - b) * smitsCurve(GREEN, w);
    }
  } else if (g <= r && g <= b) {
    s += g * smitsCurve(WHITE, w);
    if (r <= b) {
      s += (r - g) * smitsCurve(MAGENTA, w);
      s += (b - r) * smitsCurve(BLUE, w);
    } else {
      s += (b - g) * smitsCurve(MAGENTA, w);
      s += (r - b) * smitsCurve(RED, w);
    }
  } else {
    s += b * smitsCurve(WHITE, w);
    if (r <= g) {
      s += (r - b) * smitsCurve(YELLOW, w);
      s += (g - r) * smitsCurve(GREEN, w);
    } else {
      s += (g - b) * smitsCurve(YELLOW, w);
      s += (r - g) * smitsCurve(RED, w);
    }
  }
  return s;
}
inline float rgbToWavelengthReflectance(V3 rgb, float w) {
  return wclamp(0.94f * rgbToSpectrum(rgb, w), 0.0f, 1.0f);
}
inline float rgbToWavelengthRadiance(V3 rgb, float w) { return wmax(rgbToSpectrum(rgb, w), 0.0f); }

}  // namespace oracle

#endif
