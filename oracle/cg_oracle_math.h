/*
 * cg_oracle_math.h — WGSL built-ins and the reference's math modules,
 * restated in scalar C++ for the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled with -ffp-contract=off so every a*b+c rounds twice, as the
 * bit-exact traversal checks require.  Expression order follows the WGSL
 * source text (left to right).  min/max/clamp drop NaN operands (IEEE
 * fmin/fmax): the documented semantics for the NaN the reference's Smits
 * lookup produces (shading/smits.wesl:3-28).
 */
#ifndef CG_ORACLE_MATH_H_
#define CG_ORACLE_MATH_H_

#include <cmath>
#include <cstdint>

namespace oracle {

struct V3 {
  float x, y, z;
};
struct V2 {
  float x, y;
};

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }

// WGSL dot: ((x + y) + z).
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// WGSL cross (spec): (a1 b2 - b1 a2, a2 b0 - b2 a0, a0 b1 - b0 a1).
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
// WGSL normalize(e) = e / length(e).
inline V3 normalize(V3 a) { return a / length(a); }
inline float distance(V3 a, V3 b) { return length(a - b); }

inline float wmin(float a, float b) { return std::fmin(a, b); }
inline float wmax(float a, float b) { return std::fmax(a, b); }
inline float wclamp(float x, float lo, float hi) {
  return std::fmin(std::fmax(x, lo), hi);
}
inline V3 vmin(V3 a, V3 b) {
  return {wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z)};
}
inline V3 vmax(V3 a, V3 b) {
  return {wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z)};
}
// WGSL mix(e1, e2, e3) = e1 * (1 - e3) + e2 * e3.
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
// WGSL reflect(e1, e2) = e1 - 2 * dot(e2, e1) * e2.
inline V3 reflect(V3 e1, V3 e2) { return e1 - (2.0f * dot(e2, e1)) * e2; }
// WGSL refract(e1, e2, e3).
inline V3 refract(V3 e1, V3 e2, float e3) {
  float d = dot(e2, e1);
  float k = 1.0f - e3 * e3 * (1.0f - d * d);
  if (k < 0.0f) return {0.0f, 0.0f, 0.0f};
  return e3 * e1 - (e3 * d + std::sqrt(k)) * e2;
}

// Column-major 3x3 (WGSL mat3x3f): c[0..2] are columns.
struct M3 {
  V3 c[3];
};
// m * v = c0*x + c1*y + c2*z.
inline V3 mul(const M3& m, V3 v) { return (m.c[0] * v.x + m.c[1] * v.y) + m.c[2] * v.z; }
// transpose(m) * v.
inline V3 mulT(const M3& m, V3 v) {
  return {dot(m.c[0], v), dot(m.c[1], v), dot(m.c[2], v)};
}

constexpr float PI = 3.1415926535f;       // math/constant.wesl:1
constexpr float MAXD = 1e6f;              // math/constant.wesl:2

// math/geometric.wesl:28-33
inline M3 makeTangentSpace(V3 n) {
  V3 helper = (std::fabs(n.x) > 0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
  V3 tangent = normalize(cross(helper, n));
  V3 bitangent = cross(n, tangent);
  return M3{{tangent, bitangent, n}};
}

// ---- rng (math/rng.wesl:1-22) --------------------------------------------
struct Rng {
  uint32_t s;
};
inline void stepRng(Rng& r) {
  r.s = r.s * 747796405u + 2891336453u;
  uint32_t word = ((r.s >> ((r.s >> 28u) + 4u)) ^ r.s) * 277803737u;
  r.s = (word >> 22u) ^ word;
}
inline void seedRng(Rng& r, uint32_t seed) {
  r.s = seed;
  stepRng(r);
}
inline float randFloat(Rng& r) {
  stepRng(r);
  return static_cast<float>(r.s) / 4294967296.0f;
}
inline uint32_t randUInt(Rng& r) {
  stepRng(r);
  return r.s;
}

// ---- keyed streams (this backend's sample keys; the CUDA kernels use the
// same definitions) ---------------------------------------------------------
inline uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
inline uint32_t combine(uint32_t a, uint32_t b) { return mix32(a ^ mix32(b + 0x9e3779b9u)); }
inline uint32_t sampleKey(uint32_t seed, uint32_t frame, uint32_t pixel, uint32_t sample) {
  return combine(combine(combine(seed, frame), pixel), sample);
}
// Child i (0-based transport sample index) of a node.
inline uint32_t childKey(uint32_t node_key, uint32_t i) { return combine(node_key, i + 1u); }
// The Russian-roulette decision of a child (an option beyond the reference):
// one number from this stream.
inline uint32_t rouletteKey(uint32_t child_key) { return combine(child_key, 0xfffffffeu); }
// The wavelength stream of a sample.
inline uint32_t wavelengthKey(uint32_t sample_key) { return combine(sample_key, 0u); }

}  // namespace oracle

#endif
