/* Diffuse irradiance bake of an equirectangular float environment map on the device.
 *
 * Follows the reference's CPU path (sources/processing/TextureProcessing.cpp:10-64,
 * TextureProcessing.h:174-303) so results match it texel for texel: one thread per output texel
 * (x, y) -> direction from (x / W, y / H) -> tangent frame with right = (1, 0, 0) -> `samples`
 * cosine-weighted directions from the pgc3d hash (math_importance_sampling.h:7-22) seeded with the
 * texel's own approximate spherical pixel -> approximate spherical uv (atan2 polynomial, acos
 * table) -> bilinear source lookup with wrap-around -> mean.  The output keeps the source's
 * channel stride; channel 3 is left untouched (the reference never writes it).
 *
 * The reference's CUDA kernel (sources/processing/cuda/CubemapProcessing.cu:129-175) differs from
 * its CPU path (hash seeded with the output texel, exact acos/atan2, hardware filtering); this
 * kernel reproduces the CPU path, which is the one the oracle restates.
 */
#include "context.cuh"
#include "shading.cuh"

namespace {

using namespace nb;

/* float -> unsigned as compiled x86-64 code does it (64-bit truncation, low 32 bits kept), so
 * negative coordinates seed the hash the same way. */
__device__ __forceinline__ unsigned to_pixel(float coord, unsigned dim) {
  return (unsigned)(long long)(coord * (float)dim);
}

__device__ __forceinline__ void pgc3d(unsigned x, unsigned y, unsigned z, float out[3]) {
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
  out[0] = __uint2float_rn(x) * kOneOverUintMax;
  out[1] = __uint2float_rn(y) * kOneOverUintMax;
  out[2] = __uint2float_rn(z) * kOneOverUintMax;
}

struct Src {
  const float *data;
  int w, h, ch;
  bool vec4; /* 4 channels on a 16-byte aligned base: one 16-byte load per texel instead of three */
  __device__ V3 texel(int x, int y) const {
    int xc = x >= w ? x % w : (x < 0 ? w + (x % w) : x);
    int yc = y >= h ? y % h : (y < 0 ? h + (y % h) : y);
    const size_t i = (size_t)yc * w + xc;
    if (vec4) { /* the lookups scatter (each texel hashes its own directions): fewer L1 wavefronts */
      const float4 q = __ldg(reinterpret_cast<const float4 *>(data) + i);
      return {q.x, q.y, q.z};
    }
    const float *p = data + i * ch;
    return {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
  }
  __device__ V3 uv_sample(float u, float v) const {
    float ui = floorf(u), vi = floorf(v);
    float uw = (u > 1.f || u < 0.f) ? u - ui : u;
    float vw = (v > 1.f || v < 0.f) ? v - vi : v;
    float px = (float)(double)to_pixel(uw, (unsigned)w);
    float py = (float)(double)to_pixel(vw, (unsigned)h);
    float tlx = floorf(px), tly = floorf(py), trx = floorf(px) + 1, bly = floorf(py) + 1;
    const float fu = (px - tlx) / (trx - tlx);
    const float fv = (py - tly) / (bly - tly);
    const float hd = 1 - fu;
    V3 tl = texel((int)tlx, (int)tly), tr = texel((int)trx, (int)tly);
    V3 bl = texel((int)tlx, (int)bly), br = texel((int)trx, (int)bly);
    V3 top = hd * tl + fu * tr;
    V3 bot = hd * bl + fu * br;
    return (1 - fv) * top + fv * bot;
  }
};

__device__ __forceinline__ void to_uv(const float *lut, float x, float y, float z, float &u, float &v) {
  float phi = atan2_approx(y, x);
  float theta = acos_lt(lut, z);
  u = (float)((double)phi * kInv2PiD);
  v = (float)((double)theta * kInvPiD);
}

__global__ void k_bake(Src src, const float *lut, int W, int H, int samples, float *out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const float u0 = (float)((double)x / (double)W), v0 = (float)((double)y / (double)H);
  const float phi0 = (float)(2.0 * kPiD * (double)u0), theta0 = (float)(kPiD * (double)v0);
  const float st = sin_rn(theta0);
  const V3 normal{st * cos_rn(phi0), st * sin_rn(phi0), cos_rn(theta0)};
  float tu, tv;
  to_uv(lut, normal.x, normal.y, normal.z, tu, tv);
  const unsigned px = to_pixel(tu, (unsigned)W), py = to_pixel(tv, (unsigned)H);
  const V3 right{1.f, 0.f, 0.f};
  const float dd = dot(right, normal);
  V3 tangent{0.f, 1.f, 0.f};
  if (1.0 - (double)fabsf(dd) > 1e-6) tangent = normalize(cross(right, normal));
  const V3 bitangent = cross(normal, tangent);
  V3 irr{0.f, 0.f, 0.f};
  for (int s = 0; s < samples; s++) {
    float r[3];
    pgc3d(px, py, (unsigned)s, r);
    const float phi = (float)(2.0 * kPiD * (double)r[0]);
    const float theta = (float)asin((double)sqrtf(r[1]));
    const float sth = sin_rn(theta);
    V3 cdir{sth * cos_rn(phi), sth * sin_rn(phi), cos_rn(theta)};
    cdir = cdir.x * tangent + cdir.y * bitangent + cdir.z * normal;
    float su, sv;
    to_uv(lut, cdir.x, cdir.y, cdir.z, su, sv);
    irr = irr + src.uv_sample(su, sv);
  }
  irr = irr / (float)samples;
  float *o = out + ((size_t)y * W + x) * src.ch;
  o[0] = irr.x;
  o[1] = irr.y;
  o[2] = irr.z;
}

}  // namespace

nova_b200_status nb_bake(nova_b200_ctx *c, const float *src, int32_t sw, int32_t sh, int32_t ch, int32_t ow,
                         int32_t oh, int32_t samples, float *out) {
  using namespace nbctx;
  auto pow2 = [](int32_t v) { return v > 0 && (v & (v - 1)) == 0; };
  if (!src || !out) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  if (!pow2(ow) || !pow2(oh))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "irradiance size must be a power of two (TextureProcessing.cpp:11)%s");
  if (sw < 1 || sh < 1 || ch < 3 || ch > 4 || samples <= 0)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid source map or sample count%s");
  cudaSetDevice(c->device);
  /* 64-thread blocks: a 512 x 256 bake is 2048 blocks, which spread over 148 SMs within 2%, where
   * 256-thread blocks (512) leave some SMs a quarter more work than others */
  dim3 block(16, 4), grid((ow + 15) / 16, (oh + 3) / 4);
  const bool vec4 = ch == 4 && (reinterpret_cast<uintptr_t>(src) & 15u) == 0;
  k_bake<<<grid, block, 0, c->stream>>>(Src{src, sw, sh, ch, vec4}, c->d_acos, ow, oh, samples, out);
  NB_CUDA(c, cudaGetLastError(), "k_bake");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "bake");
  return NOVA_B200_SUCCESS;
}
