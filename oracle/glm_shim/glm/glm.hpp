/* ORACLE PIN — test infrastructure only; never linked into the product.
 *
 * A minimal stand-in for glm (github.com/g-truc/glm, MIT licence; an empty, un-pinned submodule in
 * the reference's tree), written here so that the reference's own headers on the Nova path
 * (shape/Triangle.h, material/BxDF_math.h, material/BxDF.h, material/BSDF.h, ray/IntersectFrame.h,
 * ray/Ray.h) compile unchanged where they lie.  It holds only the types and functions those headers
 * and their includes name, and it follows glm's published definitions and evaluation order in
 * single precision:
 *   dot(vec3)    = (x*x' + y*y') + z*z'            dot(vec4) = (x*x' + y*y') + (z*z' + w*w')
 *   normalize(v) = v * (1 / sqrt(dot(v, v)))        length(v) = sqrt(dot(v, v))
 *   cross(a, b)  = (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
 *   reflect(I,N) = I - N * dot(N, I) * 2
 *   min(a, b)    = (b < a) ? b : a   max(a, b) = (a < b) ? b : a   clamp = min(max(x, lo), hi)
 *   sign(x)      = T(0 < x) - T(x < 0)
 *   mat4 * vec4  = (c0*v.x + c1*v.y) + (c2*v.z + c3*v.w)
 *   mat3 * vec3  = per row, c0*v.x + c1*v.y + c2*v.z left to right
 *   mat * mat    = per column j, A*B[j] (columns of A scaled by B[j]'s entries, summed left to right)
 *   inverse(mat3): adjugate / determinant (cofactor expansion along the first column)
 * Matrices are column-major, m[c][r].  Default-constructed vectors are zero and matrices identity.
 * Swizzles are not provided (the reference's path does not use them).
 */
#ifndef AXOMAE_ORACLE_GLM_SHIM_HPP
#define AXOMAE_ORACLE_GLM_SHIM_HPP
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <climits>
#include <cfloat>
#include <limits>

namespace glm {

template<typename T> struct tvec4;

template<typename T> struct tvec2 {
  union { T x, r, s; };
  union { T y, g, t; };
  constexpr tvec2() : x(0), y(0) {}
  constexpr explicit tvec2(T v) : x(v), y(v) {}
  template<typename A, typename B> constexpr tvec2(A a, B b) : x(T(a)), y(T(b)) {}
  template<typename U> constexpr tvec2(const tvec2<U> &o) : x(T(o.x)), y(T(o.y)) {}
  static constexpr int length() { return 2; }
  T &operator[](int i) { return i == 0 ? x : y; }
  const T &operator[](int i) const { return i == 0 ? x : y; }
};

template<typename T> struct tvec3 {
  union { T x, r, s; };
  union { T y, g, t; };
  union { T z, b, p; };
  constexpr tvec3() : x(0), y(0), z(0) {}
  constexpr explicit tvec3(T v) : x(v), y(v), z(v) {}
  template<typename A, typename B, typename C> constexpr tvec3(A a, B b_, C c) : x(T(a)), y(T(b_)), z(T(c)) {}
  template<typename C> constexpr tvec3(const tvec2<T> &v, C c) : x(v.x), y(v.y), z(T(c)) {}
  template<typename U> constexpr tvec3(const tvec3<U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
  template<typename U> constexpr tvec3(const tvec4<U> &o);
  static constexpr int length() { return 3; }
  T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  tvec3 &operator+=(const tvec3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
  tvec3 &operator-=(const tvec3 &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  tvec3 &operator*=(const tvec3 &o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
  tvec3 &operator/=(const tvec3 &o) { x /= o.x; y /= o.y; z /= o.z; return *this; }
  tvec3 &operator*=(T v) { x *= v; y *= v; z *= v; return *this; }
  tvec3 &operator/=(T v) { x /= v; y /= v; z /= v; return *this; }
  tvec3 &operator+=(T v) { x += v; y += v; z += v; return *this; }
  tvec3 &operator-=(T v) { x -= v; y -= v; z -= v; return *this; }
};

template<typename T> struct tvec4 {
  union { T x, r, s; };
  union { T y, g, t; };
  union { T z, b, p; };
  union { T w, a, q; };
  constexpr tvec4() : x(0), y(0), z(0), w(0) {}
  constexpr explicit tvec4(T v) : x(v), y(v), z(v), w(v) {}
  template<typename A, typename B, typename C, typename D>
  constexpr tvec4(A a_, B b_, C c, D d) : x(T(a_)), y(T(b_)), z(T(c)), w(T(d)) {}
  template<typename D> constexpr tvec4(const tvec3<T> &v, D d) : x(v.x), y(v.y), z(v.z), w(T(d)) {}
  template<typename U> constexpr tvec4(const tvec4<U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
  static constexpr int length() { return 4; }
  T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  tvec4 &operator+=(const tvec4 &o) { x += o.x; y += o.y; z += o.z; w += o.w; return *this; }
  tvec4 &operator*=(T v) { x *= v; y *= v; z *= v; w *= v; return *this; }
};

template<typename T> template<typename U> constexpr tvec3<T>::tvec3(const tvec4<U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}

#define AXO_GLM_BINOPS(V, N, EXPAND)                                                                               \
  template<typename T> constexpr V<T> operator+(const V<T> &a, const V<T> &b) { return V<T>(EXPAND(a, +, b)); }   \
  template<typename T> constexpr V<T> operator-(const V<T> &a, const V<T> &b) { return V<T>(EXPAND(a, -, b)); }   \
  template<typename T> constexpr V<T> operator*(const V<T> &a, const V<T> &b) { return V<T>(EXPAND(a, *, b)); }   \
  template<typename T> constexpr V<T> operator/(const V<T> &a, const V<T> &b) { return V<T>(EXPAND(a, /, b)); }

#define AXO_E2(a, op, b) a.x op b.x, a.y op b.y
#define AXO_E3(a, op, b) a.x op b.x, a.y op b.y, a.z op b.z
#define AXO_E4(a, op, b) a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w
AXO_GLM_BINOPS(tvec2, 2, AXO_E2)
AXO_GLM_BINOPS(tvec3, 3, AXO_E3)
AXO_GLM_BINOPS(tvec4, 4, AXO_E4)

/* vector (op) scalar and scalar (op) vector, component by component */
template<typename T> constexpr tvec2<T> operator*(const tvec2<T> &a, T s) { return {a.x * s, a.y * s}; }
template<typename T> constexpr tvec2<T> operator*(T s, const tvec2<T> &a) { return {s * a.x, s * a.y}; }
template<typename T> constexpr tvec2<T> operator/(const tvec2<T> &a, T s) { return {a.x / s, a.y / s}; }
template<typename T> constexpr tvec2<T> operator+(const tvec2<T> &a, T s) { return {a.x + s, a.y + s}; }
template<typename T> constexpr tvec2<T> operator-(const tvec2<T> &a, T s) { return {a.x - s, a.y - s}; }
template<typename T> constexpr tvec2<T> operator-(const tvec2<T> &a) { return {-a.x, -a.y}; }

template<typename T> constexpr tvec3<T> operator*(const tvec3<T> &a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template<typename T> constexpr tvec3<T> operator*(T s, const tvec3<T> &a) { return {s * a.x, s * a.y, s * a.z}; }
template<typename T> constexpr tvec3<T> operator/(const tvec3<T> &a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template<typename T> constexpr tvec3<T> operator/(T s, const tvec3<T> &a) { return {s / a.x, s / a.y, s / a.z}; }
template<typename T> constexpr tvec3<T> operator+(const tvec3<T> &a, T s) { return {a.x + s, a.y + s, a.z + s}; }
template<typename T> constexpr tvec3<T> operator+(T s, const tvec3<T> &a) { return {s + a.x, s + a.y, s + a.z}; }
template<typename T> constexpr tvec3<T> operator-(const tvec3<T> &a, T s) { return {a.x - s, a.y - s, a.z - s}; }
template<typename T> constexpr tvec3<T> operator-(T s, const tvec3<T> &a) { return {s - a.x, s - a.y, s - a.z}; }
template<typename T> constexpr tvec3<T> operator-(const tvec3<T> &a) { return {-a.x, -a.y, -a.z}; }

template<typename T> constexpr tvec4<T> operator*(const tvec4<T> &a, T s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template<typename T> constexpr tvec4<T> operator*(T s, const tvec4<T> &a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template<typename T> constexpr tvec4<T> operator/(const tvec4<T> &a, T s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
template<typename T> constexpr tvec4<T> operator-(const tvec4<T> &a) { return {-a.x, -a.y, -a.z, -a.w}; }

template<typename T> constexpr bool operator==(const tvec2<T> &a, const tvec2<T> &b) { return a.x == b.x && a.y == b.y; }
template<typename T> constexpr bool operator==(const tvec3<T> &a, const tvec3<T> &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
template<typename T> constexpr bool operator==(const tvec4<T> &a, const tvec4<T> &b) {
  return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}
template<typename T> constexpr bool operator!=(const tvec2<T> &a, const tvec2<T> &b) { return !(a == b); }
template<typename T> constexpr bool operator!=(const tvec3<T> &a, const tvec3<T> &b) { return !(a == b); }
template<typename T> constexpr bool operator!=(const tvec4<T> &a, const tvec4<T> &b) { return !(a == b); }

using vec2 = tvec2<float>;
using vec3 = tvec3<float>;
using vec4 = tvec4<float>;
using dvec2 = tvec2<double>;
using dvec3 = tvec3<double>;
using dvec4 = tvec4<double>;
using ivec2 = tvec2<int>;
using ivec3 = tvec3<int>;
using uvec2 = tvec2<unsigned>;
using uvec3 = tvec3<unsigned>;

/* ---- geometric functions ---- */
template<typename T> inline T dot(const tvec2<T> &a, const tvec2<T> &b) {
  const tvec2<T> m = a * b;
  return m.x + m.y;
}
template<typename T> inline T dot(const tvec3<T> &a, const tvec3<T> &b) {
  const tvec3<T> m = a * b;
  return m.x + m.y + m.z;
}
template<typename T> inline T dot(const tvec4<T> &a, const tvec4<T> &b) {
  const tvec4<T> m = a * b;
  return (m.x + m.y) + (m.z + m.w);
}
inline float dot(float a, float b) { return a * b; }
template<typename V> inline auto length2(const V &v) { return dot(v, v); }
template<typename V> inline auto length(const V &v) {
  using std::sqrt;
  return sqrt(dot(v, v));
}
template<typename T> inline T inversesqrt(T x) {
  using std::sqrt;
  return T(1) / sqrt(x);
}
template<typename V> inline V normalize(const V &v) { return v * inversesqrt(dot(v, v)); }
template<typename T> inline tvec3<T> cross(const tvec3<T> &a, const tvec3<T> &b) {
  return tvec3<T>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template<typename V> inline V reflect(const V &I, const V &N) { return I - N * dot(N, I) * decltype(dot(N, I))(2); }
template<typename V> inline auto distance(const V &a, const V &b) { return length(b - a); }

/* ---- common functions, scalar and per component ---- */
template<typename T> inline T min(T a, T b) { return (b < a) ? b : a; }
template<typename T> inline T max(T a, T b) { return (a < b) ? b : a; }
template<typename T> inline T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
template<typename T> inline T sign(T x) { return T(T(0) < x) - T(x < T(0)); }
template<typename T> inline T abs(T x) { return x >= T(0) ? x : -x; }
template<typename T> inline T mix(T a, T b, T t) { return a + t * (b - a); }

#define AXO_GLM_PER_COMPONENT(F)                                                                                   \
  template<typename T> inline tvec2<T> F(const tvec2<T> &a, const tvec2<T> &b) { return {F(a.x, b.x), F(a.y, b.y)}; } \
  template<typename T> inline tvec3<T> F(const tvec3<T> &a, const tvec3<T> &b) {                                     \
    return {F(a.x, b.x), F(a.y, b.y), F(a.z, b.z)};                                                                  \
  }                                                                                                                  \
  template<typename T> inline tvec4<T> F(const tvec4<T> &a, const tvec4<T> &b) {                                     \
    return {F(a.x, b.x), F(a.y, b.y), F(a.z, b.z), F(a.w, b.w)};                                                     \
  }
AXO_GLM_PER_COMPONENT(min)
AXO_GLM_PER_COMPONENT(max)
#undef AXO_GLM_PER_COMPONENT
template<typename T> inline tvec3<T> min(const tvec3<T> &a, T b) { return min(a, tvec3<T>(b)); }
template<typename T> inline tvec3<T> max(const tvec3<T> &a, T b) { return max(a, tvec3<T>(b)); }
template<typename T> inline tvec3<T> clamp(const tvec3<T> &x, T lo, T hi) { return min(max(x, tvec3<T>(lo)), tvec3<T>(hi)); }
template<typename T> inline tvec3<T> clamp(const tvec3<T> &x, const tvec3<T> &lo, const tvec3<T> &hi) { return min(max(x, lo), hi); }
template<typename T> inline tvec3<T> abs(const tvec3<T> &v) { return {abs(v.x), abs(v.y), abs(v.z)}; }
template<typename T> inline tvec3<T> sign(const tvec3<T> &v) { return {sign(v.x), sign(v.y), sign(v.z)}; }
template<typename T> inline tvec3<T> mix(const tvec3<T> &a, const tvec3<T> &b, T t) { return a + t * (b - a); }

/* ---- matrices: column-major, m[c] is column c ---- */
template<typename T> struct tmat4;

template<typename T> struct tmat3 {
  tvec3<T> c[3];
  constexpr tmat3() : c{tvec3<T>(1, 0, 0), tvec3<T>(0, 1, 0), tvec3<T>(0, 0, 1)} {}
  constexpr explicit tmat3(T d) : c{tvec3<T>(d, 0, 0), tvec3<T>(0, d, 0), tvec3<T>(0, 0, d)} {}
  constexpr tmat3(const tvec3<T> &a, const tvec3<T> &b, const tvec3<T> &d) : c{a, b, d} {}
  constexpr tmat3(T x0, T y0, T z0, T x1, T y1, T z1, T x2, T y2, T z2)
      : c{tvec3<T>(x0, y0, z0), tvec3<T>(x1, y1, z1), tvec3<T>(x2, y2, z2)} {}
  constexpr tmat3(const tmat4<T> &m4);
  tvec3<T> &operator[](int i) { return c[i]; }
  const tvec3<T> &operator[](int i) const { return c[i]; }
};

template<typename T> struct tmat4 {
  tvec4<T> c[4];
  constexpr tmat4()
      : c{tvec4<T>(1, 0, 0, 0), tvec4<T>(0, 1, 0, 0), tvec4<T>(0, 0, 1, 0), tvec4<T>(0, 0, 0, 1)} {}
  constexpr explicit tmat4(T d)
      : c{tvec4<T>(d, 0, 0, 0), tvec4<T>(0, d, 0, 0), tvec4<T>(0, 0, d, 0), tvec4<T>(0, 0, 0, d)} {}
  constexpr tmat4(const tvec4<T> &a, const tvec4<T> &b, const tvec4<T> &d, const tvec4<T> &e) : c{a, b, d, e} {}
  constexpr explicit tmat4(const tmat3<T> &m)
      : c{tvec4<T>(m[0], 0), tvec4<T>(m[1], 0), tvec4<T>(m[2], 0), tvec4<T>(0, 0, 0, 1)} {}
  tvec4<T> &operator[](int i) { return c[i]; }
  const tvec4<T> &operator[](int i) const { return c[i]; }
};

template<typename T> constexpr tmat3<T>::tmat3(const tmat4<T> &m4) : c{tvec3<T>(m4[0]), tvec3<T>(m4[1]), tvec3<T>(m4[2])} {}

template<typename T> constexpr bool operator==(const tmat3<T> &a, const tmat3<T> &b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }
template<typename T> constexpr bool operator==(const tmat4<T> &a, const tmat4<T> &b) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3];
}
template<typename T> constexpr bool operator!=(const tmat3<T> &a, const tmat3<T> &b) { return !(a == b); }
template<typename T> constexpr bool operator!=(const tmat4<T> &a, const tmat4<T> &b) { return !(a == b); }

using mat3 = tmat3<float>;
using mat4 = tmat4<float>;
using dmat3 = tmat3<double>;
using dmat4 = tmat4<double>;

template<typename T> inline tvec3<T> operator*(const tmat3<T> &m, const tvec3<T> &v) {
  return tvec3<T>(m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                  m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z);
}
template<typename T> inline tvec4<T> operator*(const tmat4<T> &m, const tvec4<T> &v) {
  const tvec4<T> add0 = m[0] * v.x + m[1] * v.y;
  const tvec4<T> add1 = m[2] * v.z + m[3] * v.w;
  return add0 + add1;
}
template<typename T> inline tmat3<T> operator*(const tmat3<T> &a, const tmat3<T> &b) {
  tmat3<T> r;
  for (int j = 0; j < 3; j++) r[j] = a[0] * b[j][0] + a[1] * b[j][1] + a[2] * b[j][2];
  return r;
}
template<typename T> inline tmat4<T> operator*(const tmat4<T> &a, const tmat4<T> &b) {
  tmat4<T> r;
  for (int j = 0; j < 4; j++) r[j] = a[0] * b[j][0] + a[1] * b[j][1] + a[2] * b[j][2] + a[3] * b[j][3];
  return r;
}
template<typename T> inline tmat3<T> operator*(const tmat3<T> &a, T s) { return tmat3<T>(a[0] * s, a[1] * s, a[2] * s); }

template<typename T> inline tmat3<T> transpose(const tmat3<T> &m) {
  return tmat3<T>(m[0][0], m[1][0], m[2][0], m[0][1], m[1][1], m[2][1], m[0][2], m[1][2], m[2][2]);
}
template<typename T> inline tmat4<T> transpose(const tmat4<T> &m) {
  tmat4<T> r;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) r[i][j] = m[j][i];
  return r;
}
template<typename T> inline T determinant(const tmat3<T> &m) {
  return +m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
         m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}
template<typename T> inline tmat3<T> inverse(const tmat3<T> &m) {
  const T k = T(1) / determinant(m);
  tmat3<T> r;
  r[0][0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * k;
  r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * k;
  r[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * k;
  r[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * k;
  r[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * k;
  r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * k;
  r[0][2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * k;
  r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * k;
  r[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * k;
  return r;
}
/* 4x4 inverse by cofactors in double, rounded once: the camera and transform set-up use it, the
 * pinned intersection and BSDF functions do not. */
template<typename T> inline tmat4<T> inverse(const tmat4<T> &m) {
  double a[16], inv[16];
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) a[4 * c + r] = (double)m[c][r];
  inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] + a[13] * a[6] * a[11] -
           a[13] * a[7] * a[10];
  inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] - a[12] * a[6] * a[11] +
           a[12] * a[7] * a[10];
  inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] + a[12] * a[5] * a[11] -
           a[12] * a[7] * a[9];
  inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] - a[12] * a[5] * a[10] +
            a[12] * a[6] * a[9];
  inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] - a[13] * a[2] * a[11] +
           a[13] * a[3] * a[10];
  inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] + a[12] * a[2] * a[11] -
           a[12] * a[3] * a[10];
  inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] - a[12] * a[1] * a[11] +
           a[12] * a[3] * a[9];
  inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] + a[12] * a[1] * a[10] -
            a[12] * a[2] * a[9];
  inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] + a[13] * a[2] * a[7] -
           a[13] * a[3] * a[6];
  inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] - a[12] * a[2] * a[7] +
           a[12] * a[3] * a[6];
  inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] + a[12] * a[1] * a[7] -
            a[12] * a[3] * a[5];
  inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] - a[12] * a[1] * a[6] +
            a[12] * a[2] * a[5];
  inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] - a[9] * a[2] * a[7] +
           a[9] * a[3] * a[6];
  inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] + a[8] * a[2] * a[7] -
           a[8] * a[3] * a[6];
  inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] - a[8] * a[1] * a[7] +
            a[8] * a[3] * a[5];
  inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] + a[8] * a[1] * a[6] -
            a[8] * a[2] * a[5];
  const double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
  tmat4<T> r;
  for (int c = 0; c < 4; c++)
    for (int rr = 0; rr < 4; rr++) r[c][rr] = (T)(inv[4 * c + rr] / det);
  return r;
}

/* ---- gtc/type_ptr ---- */
template<typename T> inline T *value_ptr(tvec2<T> &v) { return &v.x; }
template<typename T> inline T *value_ptr(tvec3<T> &v) { return &v.x; }
template<typename T> inline T *value_ptr(tvec4<T> &v) { return &v.x; }
template<typename T> inline const T *value_ptr(const tvec3<T> &v) { return &v.x; }
template<typename T> inline const T *value_ptr(const tvec4<T> &v) { return &v.x; }
template<typename T> inline T *value_ptr(tmat3<T> &m) { return &m[0].x; }
template<typename T> inline T *value_ptr(tmat4<T> &m) { return &m[0].x; }
template<typename T> inline const T *value_ptr(const tmat3<T> &m) { return &m[0].x; }
template<typename T> inline const T *value_ptr(const tmat4<T> &m) { return &m[0].x; }

}  // namespace glm

#endif
