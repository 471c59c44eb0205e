/* Device vector math with the reference's glm evaluation order.
 *
 * The reference performs all vector arithmetic through glm in single precision.  To reproduce its
 * rounding on the device, every operation below evaluates in glm's order and the library is
 * compiled with -fmad=false (no multiply-add contraction; explicit __fmaf_rn is used only where a
 * result does not have to match, e.g. conservative box tests):
 *   dot(vec3) = (x*x' + y*y') + z*z'         dot(vec4) = (x*x' + y*y') + (z*z' + w*w')
 *   normalize(v) = v * (1 / sqrt(dot(v, v)))  cross(a, b) = (a.y b.z - b.y a.z, ...)
 *   reflect(I, N) = I - N * dot(N, I) * 2     mat4 * vec4 = (c0 x + c1 y) + (c2 z + c3 w)
 *   mat3 * vec3 = c0 x + c1 y + c2 z row by row, left to right.
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define NB_HD __host__ __device__ __forceinline__
#define NB_D __device__ __forceinline__

namespace nb {

struct V3 {
  float x, y, z;
};
struct V4 {
  float x, y, z, w;
};

NB_HD V3 v3(float a) { return {a, a, a}; }
NB_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
NB_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
NB_HD V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
NB_HD V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
NB_HD V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
NB_HD V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
NB_HD V3 operator/(float s, V3 a) { return {s / a.x, s / a.y, s / a.z}; }
NB_HD V3 operator-(V3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }
NB_HD V3 operator+(V3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }
NB_HD V3 operator-(float s, V3 a) { return {s - a.x, s - a.y, s - a.z}; }
NB_HD V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }

NB_HD V4 operator+(V4 a, V4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
NB_HD V4 operator*(V4 a, V4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
NB_HD V4 operator*(V4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
NB_HD V4 operator*(float s, V4 a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
NB_HD V4 operator/(V4 a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }

NB_HD float dot(V3 a, V3 b) {
  V3 t = a * b;
  return t.x + t.y + t.z;
}
NB_HD float dot(V4 a, V4 b) {
  V4 t = a * b;
  return (t.x + t.y) + (t.z + t.w);
}
NB_HD float length2(V3 a) { return dot(a, a); }
NB_HD float length(V3 a) { return sqrtf(dot(a, a)); }
NB_HD V3 normalize(V3 v) { return v * (1.f / sqrtf(dot(v, v))); }
NB_HD V4 normalize(V4 v) { return v * (1.f / sqrtf(dot(v, v))); }
NB_HD V3 cross(V3 x, V3 y) { return {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y}; }
NB_HD V3 reflect(V3 I, V3 N) { return I - N * dot(N, I) * 2.f; }
NB_HD float fsign(float x) { return (0.f < x) ? 1.f : ((x < 0.f) ? -1.f : 0.f); }
NB_HD float sqr(float v) { return v * v; }
NB_HD float msqrt(float v) { return sqrtf(fmaxf(v, 0.f)); } /* reference math::sqrt: sqrtf(fmax(v, 0)) */
NB_HD float fclampf(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); } /* std::clamp */
NB_HD float fmax_std(float a, float b) { return (a < b) ? b : a; } /* std::max */
NB_HD float fmin_std(float a, float b) { return (b < a) ? b : a; } /* std::min */
NB_HD bool any_nonzero(V3 s) { return s.x != 0.f || s.y != 0.f || s.z != 0.f; }
NB_HD bool all_nonzero(V3 s) { return s.x != 0.f && s.y != 0.f && s.z != 0.f; }

/* Column-major matrices (glm layout). */
struct M3 {
  V3 c[3];
};
struct M4 {
  V4 c[4];
};
NB_HD V3 mul(const M3 &m, V3 v) {
  return {m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z, m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z,
          m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z};
}
NB_HD V3 mul_t(const M3 &m, V3 v) { /* transpose(m) * v */
  return {m.c[0].x * v.x + m.c[0].y * v.y + m.c[0].z * v.z, m.c[1].x * v.x + m.c[1].y * v.y + m.c[1].z * v.z,
          m.c[2].x * v.x + m.c[2].y * v.y + m.c[2].z * v.z};
}
NB_HD V4 mul(const M4 &m, V4 v) {
  V4 a0 = m.c[0] * v.x + m.c[1] * v.y;
  V4 a1 = m.c[2] * v.z + m.c[3] * v.w;
  return a0 + a1;
}
/* xyz of m * (p, 1) and m * (d, 0) for a 4x4 given as 16 column-major floats. */
NB_HD V3 xform_point(const float *m, V3 p) {
  V4 a0 = V4{m[0], m[1], m[2], m[3]} * p.x + V4{m[4], m[5], m[6], m[7]} * p.y;
  V4 a1 = V4{m[8], m[9], m[10], m[11]} * p.z + V4{m[12], m[13], m[14], m[15]} * 1.f;
  V4 r = a0 + a1;
  return {r.x, r.y, r.z};
}
NB_HD V3 xform_dir(const float *m, V3 d) {
  V4 a0 = V4{m[0], m[1], m[2], m[3]} * d.x + V4{m[4], m[5], m[6], m[7]} * d.y;
  V4 a1 = V4{m[8], m[9], m[10], m[11]} * d.z + V4{m[12], m[13], m[14], m[15]} * 0.f;
  V4 r = a0 + a1;
  return {r.x, r.y, r.z};
}
NB_HD M3 m3_load(const float *f) { return {{{f[0], f[1], f[2]}, {f[3], f[4], f[5]}, {f[6], f[7], f[8]}}}; }
NB_HD M3 m3_of4(const float *f) { return {{{f[0], f[1], f[2]}, {f[4], f[5], f[6]}, {f[8], f[9], f[10]}}}; }
NB_HD M4 m4_load(const float *f) {
  return {{{f[0], f[1], f[2], f[3]}, {f[4], f[5], f[6], f[7]}, {f[8], f[9], f[10], f[11]}, {f[12], f[13], f[14], f[15]}}};
}

NB_HD bool finite3(V3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

/* Transcendentals evaluated in double and rounded once, so they agree with a correctly rounded
 * single-precision libm in all but double-rounding corner cases. */
NB_D float pow5f(float x) {
  double d = (double)x;
  double d2 = d * d;
  return (float)(d2 * d2 * d);
}
NB_D float cos_rn(float x) { return (float)cos((double)x); }
NB_D float sin_rn(float x) { return (float)sin((double)x); }
/* sin and cos of one argument, one shared double-precision evaluation, each rounded once */
NB_D void sincos_rn(float x, float &s, float &c) {
  double sd, cd;
  sincos((double)x, &sd, &cd);
  s = (float)sd;
  c = (float)cd;
}

}  // namespace nb
