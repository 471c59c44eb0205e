/* ORACLE — test infrastructure only (see oracle.h).
 *
 * Diffuse irradiance bake, CPU path of the reference:
 *   TextureOperations<float>::computeDiffuseIrradiance   sources/processing/TextureProcessing.cpp:10-64
 *   launchAsyncDiffuseIrradianceCompute / computeIrradianceImportanceSampling /
 *   computeIrradianceSingleTexel / uvSample / bilinearInterpolate / wrapAround*
 *                                                       sources/processing/TextureProcessing.h:174-303
 *   pgc3d                                                corelib/internal/common/math/math_importance_sampling.h:7-22
 * The spherical mapping uses the reference's fast approximations (atan2 polynomial, acos table).
 *
 * The reference's CUDA bake (the --gpu path), orc_bake_irradiance_texunit:
 *   gpgpu_device_compute_diffuse_irradiance             sources/processing/cuda/CubemapProcessing.cu:129-175
 *   spherical_math::*, gpu_pgc3d, dot / cross / normalize :12-105
 *   texture descriptor (wrap, linear, normalised)        :216-230
 * Its tex2D<float4> fetch is restated from the texture unit's published bilinear filter (CUDA C++
 * Programming Guide, "Texture Fetching", linear filtering): x_B = x * W - 0.5, i = floor(x_B),
 * alpha = frac(x_B) held in 9-bit fixed point with 8 fractional bits (rounded to nearest here; the
 * guide does not state the rounding), wrap addressing on the texel indices, and
 * T = (1-a)(1-b) T[i,j] + a(1-b) T[i+1,j] + (1-a) b T[i,j+1] + a b T[i+1,j+1].  The float
 * trigonometry is correctly rounded here where the device uses its own functions (within a few ulp),
 * so the two agree to a tolerance, not bit for bit.
 */
#include "oracle_internal.h"
#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace orc {
namespace {

constexpr double PI_D = M_PI;

/* uvToPixel(coord, dim) = static_cast<unsigned>(coord * dim).  A negative coordinate is converted
 * the way x86-64 GCC code does it (truncate to a 64-bit integer, keep the low 32 bits). */
inline unsigned to_pixel(float coord, unsigned dim) { return (unsigned)(int64_t)(coord * (float)dim); }

inline void pgc3d(unsigned x, unsigned y, unsigned z, float out[3]) {
  x = x * 1664525u + 1013904223u;
  y = y * 1664525u + 1013904223u;
  z = z * 1664525u + 1013904223u;
  x += y * z;
  y += z * x;
  z += x * y;
  x ^= x >> 16u;
  y ^= y >> 16u;
  z ^= z >> 16u;
  x += y * z;
  y += z * x;
  z += x * y;
  const float k = 1.f / float(0xFFFFFFFFu);
  out[0] = (float)x * k;
  out[1] = (float)y * k;
  out[2] = (float)z * k;
}

inline float horner(float x) {
  float x_sq = x * x;
  return x * (0.99997726f + x_sq * (-0.33262347f + x_sq * (0.19354346f + x_sq * (-0.11643287f +
                                                                          x_sq * (0.05265332f + x_sq * -0.01172120f)))));
}
inline float atan2_approx(float y, float x) {
  bool swap = std::fabs(x) < std::fabs(y);
  float in = (swap ? x : y) / (swap ? y : x);
  float res = horner(in);
  res = swap ? (in >= 0.0f ? (float)M_PI_2 : -(float)M_PI_2) - res : res;
  if (x >= 0.0f && y >= 0.0f) {
  } else if (x < 0.0f && y >= 0.0f) {
    res = (float)M_PI + res;
  } else if (x < 0.0f && y < 0.0f) {
    res = -(float)M_PI + res;
  }
  return res;
}
inline float acos_lt(float a) {
  int scaled = std::clamp((int)((a + 1.f) * kAcosPrecision * 0.5f), 0, kAcosPrecision - 1);
  return acos_lut()[scaled];
}
inline void to_uv(float x, float y, float z, float &u, float &v) { /* sphericalToUv(cartesianToSpherical()) */
  float phi = atan2_approx(y, x);
  float theta = acos_lt(z);
  u = (float)(phi * (1.f / (2.f * PI_D)));
  v = (float)(theta * (1.f / PI_D));
}

struct Src {
  const float *data;
  int w, h, ch;
  V3 texel(int x, int y) const { /* discreteSample + wrapAroundPixelCoords */
    int xc, yc;
    if (x >= w)
      xc = x % w;
    else if (x < 0)
      xc = w + (x % w);
    else
      xc = x;
    if (y >= h)
      yc = y % h;
    else if (y < 0)
      yc = h + (y % h);
    else
      yc = y;
    size_t i = ((size_t)yc * w + xc) * ch;
    return {data[i], data[i + 1], data[i + 2]};
  }
  V3 uv_sample(float u, float v) const { /* uvSample + wrapAroundTexCoords + bilinearInterpolate */
    float ui = std::floor(u), vi = std::floor(v);
    float uw = (u > 1. || u < 0.) ? u - ui : u;
    float vw = (v > 1. || v < 0.) ? v - vi : v;
    float px = (float)(double)to_pixel(uw, (unsigned)w);
    float py = (float)(double)to_pixel(vw, (unsigned)h);
    float tlx = std::floor(px), tly = std::floor(py);
    float trx = std::floor(px) + 1, blY = std::floor(py) + 1;
    const float fu = (px - tlx) / (trx - tlx);
    const float fv = (py - tly) / (blY - tly);
    const float hd = (1 - fu);
    V3 tl = texel((int)tlx, (int)tly), tr = texel((int)trx, (int)tly);
    V3 bl = texel((int)tlx, (int)blY), br = texel((int)trx, (int)blY);
    V3 top = hd * tl + fu * tr;
    V3 bot = hd * bl + fu * br;
    return (1 - fv) * top + fv * bot;
  }
};

V3 texel_irradiance(const Src &src, float x, float y, float z, unsigned W, unsigned H, unsigned total) {
  V3 irr{0, 0, 0};
  V3 normal{x, y, z};
  V3 right{1.f, 0.f, 0.f};
  float u, v;
  to_uv(x, y, z, u, v);
  const unsigned px = to_pixel(u, W), py = to_pixel(v, H);
  float dd = dot(right, normal);
  V3 tangent{0.f, 1.f, 0.f};
  if (1.0 - std::fabs(dd) > 1e-6) tangent = normalize(cross(right, normal));
  V3 bitangent = cross(normal, tangent);
  for (unsigned s = 0; s < total; s++) {
    float r[3];
    pgc3d(px, py, s, r);
    float phi = (float)(2 * PI_D * r[0]);
    float theta = asin_rn(std::sqrt(r[1]));
    V3 c{sin_rn(theta) * cos_rn(phi), sin_rn(theta) * sin_rn(phi), cos_rn(theta)};
    c = c.x * tangent + c.y * bitangent + c.z * normal;
    float su, sv;
    to_uv(c.x, c.y, c.z, su, sv);
    irr = irr + src.uv_sample(su, sv);
  }
  return irr / (float)total;
}

}  // namespace
}  // namespace orc

using namespace orc;

/* ---- the reference's CUDA kernel ---- */
namespace orc {
namespace {

struct F3 {
  float x, y, z;
};
inline F3 sph_to_cart(float phi, float theta) {
  return F3{sin_rn(theta) * cos_rn(phi), sin_rn(theta) * sin_rn(phi), cos_rn(theta)};
}
inline F3 cross3(F3 a, F3 b) { return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

/* tex2D<float4> with linear filtering, wrap addressing and normalised coordinates. */
struct TexUnit {
  const float *rgba;
  int w, h;
  static int wrap(int i, int n) { return ((i % n) + n) % n; }
  static float weight(float f) { return std::nearbyint(f * 256.f) / 256.f; }
  V4 fetch(float u, float v) const {
    u = u - std::floor(u), v = v - std::floor(v);
    const float xb = u * (float)w - 0.5f, yb = v * (float)h - 0.5f;
    const float fx = std::floor(xb), fy = std::floor(yb);
    const float a = weight(xb - fx), b = weight(yb - fy);
    const int i0 = wrap((int)fx, w), i1 = wrap((int)fx + 1, w), j0 = wrap((int)fy, h), j1 = wrap((int)fy + 1, h);
    auto T = [&](int i, int j) {
      const float *p = rgba + ((size_t)j * w + i) * 4;
      return V4{p[0], p[1], p[2], p[3]};
    };
    const V4 t00 = T(i0, j0), t10 = T(i1, j0), t01 = T(i0, j1), t11 = T(i1, j1);
    const float w00 = (1 - a) * (1 - b), w10 = a * (1 - b), w01 = (1 - a) * b, w11 = a * b;
    return V4{w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x, w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
              w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z, w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w};
  }
};

}  // namespace
}  // namespace orc

using namespace orc;

/* The reference's CUDA bake (CubemapProcessing.cu:129-175) on an RGBA source: out = out_w * out_h
 * * 4 floats, alpha 1.  Returns 1 for non-power-of-two sizes or no samples. */
extern "C" int32_t orc_bake_irradiance_texunit(const float *rgba, int32_t src_w, int32_t src_h, int32_t out_w,
                                               int32_t out_h, int32_t samples, int32_t threads, float *out) {
  auto pow2 = [](int32_t v) { return v > 0 && (v & (v - 1)) == 0; };
  if (!pow2(out_w) || !pow2(out_h) || samples <= 0) return 1;
  const TexUnit tex{rgba, src_w, src_h};
  const unsigned W = (unsigned)out_w, H = (unsigned)out_h, nt = threads > 0 ? (unsigned)threads : 8u;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; t++)
    pool.emplace_back([=, &tex] {
      for (unsigned j = t; j < H; j += nt)
        for (unsigned i = 0; i < W; i++) {
          const float u = (float)i / (float)W, v = (float)j / (float)H;
          const F3 normal = sph_to_cart((float)(2 * PI_D * u), (float)(PI_D * v));
          const F3 some{1.f, 0.f, 0.f};
          const float dd = some.x * normal.x + some.y * normal.y + some.z * normal.z;
          F3 tangent{0.f, 1.f, 0.f};
          if (1.0 - std::fabs(dd) > 1e-6) {
            const F3 c = cross3(some, normal);
            const float d = std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
            tangent = F3{c.x / d, c.y / d, c.z / d};
          }
          const F3 bit = cross3(normal, tangent);
          float irr[3] = {0.f, 0.f, 0.f};
          for (unsigned s = 0; s < (unsigned)samples; s++) {
            float r[3];
            pgc3d(i, j, s, r);
            const float phi = (float)(2 * PI_D * r[0]);
            const float theta = asin_rn(std::sqrt(r[1]));
            const F3 c = sph_to_cart(phi, theta);
            const F3 w{c.x * tangent.x + c.y * bit.x + c.z * normal.x, c.x * tangent.y + c.y * bit.y + c.z * normal.y,
                       c.x * tangent.z + c.y * bit.z + c.z * normal.z};
            const float th = (float)std::acos((double)w.z), ph = (float)std::atan2((double)w.y, (double)w.x);
            const V4 px = tex.fetch((float)(ph / (2 * PI_D)), (float)(th / PI_D));
            irr[0] += px.x, irr[1] += px.y, irr[2] += px.z;
          }
          float *o = out + ((size_t)j * W + i) * 4;
          o[0] = irr[0] / (float)samples;
          o[1] = irr[1] / (float)samples;
          o[2] = irr[2] / (float)samples;
          o[3] = 1.f;
        }
    });
  for (auto &t : pool) t.join();
  return 0;
}

extern "C" int32_t orc_bake_irradiance(const float *src, int32_t src_w, int32_t src_h, int32_t channels, int32_t out_w,
                                       int32_t out_h, int32_t samples, int32_t threads, float *out) {
  auto pow2 = [](int32_t v) { return v > 0 && (v & (v - 1)) == 0; };
  if (!pow2(out_w) || !pow2(out_h) || channels < 3 || samples <= 0) return 1;
  (void)acos_lut();
  Src s{src, src_w, src_h, channels};
  const unsigned W = (unsigned)out_w, H = (unsigned)out_h;
  const unsigned MAX_THREADS = threads > 0 ? (unsigned)threads : 8u; /* TextureProcessing.h:45 */
  std::vector<std::thread> pool;
  for (unsigned i = 1; i <= MAX_THREADS; i++) {
    unsigned wmax = (W / MAX_THREADS) * i, wmin = wmax - (W / MAX_THREADS);
    if (i == MAX_THREADS) wmax += W % MAX_THREADS - 1;
    pool.emplace_back([=, &s] {
      for (unsigned x = wmin; x <= wmax && x < W; x++)
        for (unsigned y = 0; y < H; y++) {
          float u = (float)((double)x / (double)W), v = (float)((double)y / (double)H);
          float phi = (float)(2 * PI_D * u), theta = (float)(PI_D * v);
          float cz = cos_rn(theta), cx = sin_rn(theta) * cos_rn(phi), cy = sin_rn(theta) * sin_rn(phi);
          V3 irr = texel_irradiance(s, cx, cy, cz, W, H, (unsigned)samples);
          size_t idx = ((size_t)y * W + x) * channels;
          out[idx] = irr.x;
          out[idx + 1] = irr.y;
          out[idx + 2] = irr.z;
        }
    });
  }
  for (auto &t : pool) t.join();
  return 0;
}
