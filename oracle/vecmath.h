/* ORACLE — test infrastructure only.  CPU restatement of the reference's arithmetic; never linked
 * into the product.  Only tests/, the smoke check and bench.py's CPU-baseline leg may load it.
 *
 * glm-semantics vector math.  The reference does all of its vector arithmetic through glm
 * (an un-vendored submodule, vendor/glm, pin unrecoverable).  Every operation below reproduces
 * glm's evaluation order in single precision so that the oracle rounds exactly like the reference:
 *   dot(vec3)  = (x*x' + y*y') + z*z'                  (glm compute_dot<vec3>)
 *   dot(vec4)  = (x*x' + y*y') + (z*z' + w*w')         (glm compute_dot<vec4>)
 *   normalize  = v * (1 / sqrt(dot(v, v)))            (glm normalize / inversesqrt)
 *   cross      = (y*z' - y'*z, z*x' - z'*x, x*y' - x'*y)
 *   reflect    = I - N * dot(N, I) * 2
 *   mat4*vec4  = (c0*v.x + c1*v.y) + (c2*v.z + c3*v.w) (glm operator*(mat4, vec4))
 *   mat3*vec3  = c0*v.x + c1*v.y + c2*v.z, row by row left to right
 * The build uses -ffp-contract=off so no multiply-add is fused (the reference's default x86-64
 * build has no FMA either).
 */
#pragma once
#include <cmath>
#include <cstdint>

namespace orc {

struct V2 {
  float x, y;
};

struct V3 {
  float x, y, z;
  float &operator[](int i) { return (&x)[i]; }
  float operator[](int i) const { return (&x)[i]; }
};

struct V4 {
  float x, y, z, w;
};

inline V3 v3(float a) { return {a, a, a}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator+(V3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }
inline V3 operator-(V3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }
inline V3 operator-(float s, V3 a) { return {s - a.x, s - a.y, s - a.z}; }
inline V3 operator/(float s, V3 a) { return {s / a.x, s / a.y, s / a.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }

inline V4 operator+(V4 a, V4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline V4 operator*(V4 a, V4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
inline V4 operator*(V4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline V4 operator*(float s, V4 a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
inline V4 operator/(V4 a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }

inline float dot(V3 a, V3 b) {
  V3 t = a * b;
  return t.x + t.y + t.z;
}
inline float dot(V4 a, V4 b) {
  V4 t = a * b;
  return (t.x + t.y) + (t.z + t.w);
}
inline float length2(V3 a) { return dot(a, a); }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 v) { return v * (1.f / std::sqrt(dot(v, v))); }
inline V4 normalize(V4 v) { return v * (1.f / std::sqrt(dot(v, v))); }
inline V3 cross(V3 x, V3 y) {
  return {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}
inline V3 reflect(V3 I, V3 N) { return I - N * dot(N, I) * 2.f; }
inline float fsign(float x) { return (0.f < x) ? 1.f : ((x < 0.f) ? -1.f : 0.f); }  // glm::sign
inline V3 vmin(V3 a, V3 b) {  // glm::min: (b < a) ? b : a per component
  return {b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y, b.z < a.z ? b.z : a.z};
}
inline V3 vmax(V3 a, V3 b) {  // glm::max: (a < b) ? b : a per component
  return {a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y, a.z < b.z ? b.z : a.z};
}

/* Column-major matrices, glm layout. */
struct M3 {
  V3 c[3];
};
struct M4 {
  V4 c[4];
};

inline V3 mul(const M3 &m, V3 v) {
  return {m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z,
          m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z,
          m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z};
}
/* transpose(m) * v: row i of the transpose is column i of m. */
inline V3 mul_t(const M3 &m, V3 v) {
  return {m.c[0].x * v.x + m.c[0].y * v.y + m.c[0].z * v.z,
          m.c[1].x * v.x + m.c[1].y * v.y + m.c[1].z * v.z,
          m.c[2].x * v.x + m.c[2].y * v.y + m.c[2].z * v.z};
}
inline V4 mul(const M4 &m, V4 v) {
  V4 add0 = m.c[0] * v.x + m.c[1] * v.y;
  V4 add1 = m.c[2] * v.z + m.c[3] * v.w;
  return add0 + add1;
}
inline M4 m4_from(const float *f) {
  M4 m;
  for (int c = 0; c < 4; c++) m.c[c] = {f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]};
  return m;
}
inline M3 m3_from(const float *f) {
  M3 m;
  for (int c = 0; c < 3; c++) m.c[c] = {f[3 * c], f[3 * c + 1], f[3 * c + 2]};
  return m;
}
inline M3 m3_of(const M4 &m) {  // glm::mat3(mat4): upper-left 3x3
  M3 r;
  for (int c = 0; c < 3; c++) r.c[c] = {m.c[c].x, m.c[c].y, m.c[c].z};
  return r;
}
inline V3 xyz(V4 v) { return {v.x, v.y, v.z}; }

/* The reference calls the float overloads of std::cos / std::sin / std::asin / std::pow, whose last
 * bit depends on the C library it links (glibc's cosf and powf, for instance, are not correctly
 * rounded: they differ from the correctly rounded value by one ulp on roughly one argument in a
 * hundred).  This restatement and the device both use the correctly rounded value: evaluated in
 * double and rounded once. */
inline float cos_rn(float x) { return (float)std::cos((double)x); }
inline float sin_rn(float x) { return (float)std::sin((double)x); }
inline float asin_rn(float x) { return (float)std::asin((double)x); }
inline float pow5_rn(float x) {
  const double d = (double)x, d2 = d * d;
  return (float)(d2 * d2 * d);
}

/* reference math::sqrt (math_utils.h:86): sqrtf(fmax(v, 0)). */
inline float msqrt(float v) { return std::sqrt(std::fmax(v, 0.f)); }
inline float sqr(float v) { return v * v; }

/* Spectrum = three floats with the reference's BaseSpectrum operators (spectrum/BaseSpectrum.h). */
using Spec = V3;
inline bool spec_nonzero(Spec s) { return s.x != 0.f || s.y != 0.f || s.z != 0.f; }

}  // namespace orc
