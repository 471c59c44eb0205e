/* Shading on the device: hit record, textures, environment lookup and the principled BSDF.
 *
 * Every function restates a reference routine (HamilcarR/Axomae, corelib/) in the reference's
 * evaluation order so the device and the reference round alike:
 *   hit record       aggregate/api/embree/embree.cpp:287-412 (geometric normal from the winding,
 *                    dpdu/dpdv from the uv determinant, interpolated TBN, Gram-Schmidt frame)
 *   u8 textures      texturing/NovaTextureInterface.h:57-145 + TextureContext.h:129-161 (the CPU
 *                    bilinear path; the reference's GPU path uses nearest tex2D instead)
 *   environment map  NovaTextureInterface.h:152-168, math_spherical.h:44-52, math_utils_approx.h:13-40,
 *                    math_acos_lt.cpp:37-40 (atan2 polynomial and the 500000-entry acos table),
 *                    TextureContext.h:196-223 (nearest texel through uv2index)
 *   material         material/NovaMaterials.h:56-137 (PrincipledMaterial::scatter, sampleBSDF)
 *   BSDF             material/BSDF.h:22-162 (lobe weights, lobe choice, local frame)
 *   lobes            material/BxDF.h:252-608 (DisneyDiffuse, Specular GGX, Dielectric)
 *   microfacet math  material/BxDF_math.h:26-343 (VNDF sampling, Fresnel, refraction)
 */
#pragma once
#include "device_scene.cuh"
#include "sampler.cuh"

namespace nb {

constexpr double kPiD = 3.14159265358979323846;
constexpr double kInvPiD = 1.0 / kPiD;          /* INV_PI  (math_spherical.h:9) */
constexpr double kInv2PiD = 1.0 / (2.0 * kPiD); /* INV_2PI (math_spherical.h:10) */
constexpr float kPiF = 3.14159265358979323846f;
constexpr float kPi2F = 1.57079632679489661923f;
constexpr float kPi4F = 0.78539816339744830962f;
constexpr float kInvPiF = 0.31830988618379067154f; /* M_1_PIf */

/* ---------------------------------------------------------------- textures */

NB_D float tex_wrap(float uv) { /* wrap, NovaTextureInterface.h:13-23 */
  if (uv < 0.f) {
    float fp = ceilf(uv) - uv;
    return 1.f - fp;
  }
  if (uv > 1.f) return uv - floorf(uv);
  return uv;
}

NB_D unsigned uv2index(float t, int dim) { /* TextureContext.h:52-58 */
  float a = fabsf(t);
  float rem = a - floorf(a);
  rem = rem == 0 ? a : rem;
  return (unsigned)(rem * (float)(unsigned)dim);
}

NB_D V4 pixel_from_format(uint32_t px, int is_rgba, int channels) {
  float b0 = (float)(px & 0xffu), b1 = (float)((px >> 8) & 0xffu), b2 = (float)((px >> 16) & 0xffu),
        b3 = (float)(px >> 24);
  float r = is_rgba ? b0 : b2, g = b1, b = is_rgba ? b2 : b0, a = b3;
  switch (channels) {
    case 1: return {r, 0.f, 0.f, 1.f};
    case 2: return {r, g, 0.f, 1.f};
    case 3: return {r, g, b, 1.f};
    default: return {r, g, b, a};
  }
}

NB_D V4 sample_u8(const DevTexture &tx, float u, float v) {
  u = tex_wrap(u);
  v = tex_wrap(v);
  u = tx.invert_u ? 1 - u : u;
  v = tx.invert_v ? 1 - v : v;
  const int width = tx.w, height = tx.h;
  float pi = fabsf(u * (float)(width - 1.f));
  float pj = fabsf(v * (float)(height - 1.f));
  unsigned i = (unsigned)floorf(pi), j = (unsigned)floorf(pj);
  if (i + 1 >= (unsigned)width) i = (unsigned)width - 2;
  if (i > (unsigned)width) i = 0;
  if (j + 1 >= (unsigned)height) j = (unsigned)height - 2;
  if (j > (unsigned)height) j = 0;
  float ftx = (pi - (float)i) / 1.f;
  float fty = (pj - (float)j) / 1.f;
  const uint32_t *p = tx.u8;
  uint32_t p0 = __ldg(p + j * width + i), p1 = __ldg(p + j * width + i + 1);
  uint32_t p2 = __ldg(p + (j + 1) * width + i), p3 = __ldg(p + (j + 1) * width + i + 1);
  V4 v0 = pixel_from_format(p0, tx.is_rgba, tx.ch), v1 = pixel_from_format(p1, tx.is_rgba, tx.ch);
  V4 v2 = pixel_from_format(p2, tx.is_rgba, tx.ch), v3 = pixel_from_format(p3, tx.is_rgba, tx.ch);
  float hd = 1 - ftx;
  V4 top = hd * v0 + ftx * v1;
  V4 bot = hd * v2 + ftx * v3;
  return (1 - fty) * top + fty * bot;
}

NB_D V4 f32pixel(const DevTexture &tx, float u, float v) {
  u = tx.invert_u ? 1 - u : u;
  v = tx.invert_v ? 1 - v : v;
  unsigned i = uv2index(u, tx.w - 1);
  unsigned j = uv2index(v, tx.h - 1);
  const float *p = tx.f32 + ((size_t)j * tx.w + i) * tx.ch;
  if (tx.ch == 4) {
    if ((((uintptr_t)p) & 15u) == 0) {
      float4 q = __ldg(reinterpret_cast<const float4 *>(p));
      return {q.x, q.y, q.z, q.w};
    }
    return {__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)};
  }
  V4 r{0.f, 0.f, 0.f, 0.f};
  if (tx.ch > 0) r.x = __ldg(p);
  if (tx.ch > 1) r.y = __ldg(p + 1);
  if (tx.ch > 2) r.z = __ldg(p + 2);
  return r;
}

NB_D float atan2_approx(float y, float x) { /* math_utils_approx.h:13-40 */
  bool swap = fabsf(x) < fabsf(y);
  float in = (swap ? x : y) / (swap ? y : x);
  float xs = in * in;
  float res = in * (0.99997726f + xs * (-0.33262347f + xs * (0.19354346f + xs * (-0.11643287f +
                                                                  xs * (0.05265332f + xs * -0.01172120f)))));
  res = swap ? (in >= 0.0f ? kPi2F : -kPi2F) - res : res;
  if (x >= 0.0f && y >= 0.0f) {
  } else if (x < 0.0f && y >= 0.0f) {
    res = kPiF + res;
  } else if (x < 0.0f && y < 0.0f) {
    res = -kPiF + res;
  }
  return res;
}

NB_D float acos_lt(const float *lut, float a) { /* math_acos_lt.cpp:37-40 */
  int scaled = (int)((a + 1.f) * (float)kAcosPrecision * 0.5f);
  scaled = scaled < 0 ? 0 : (scaled > kAcosPrecision - 1 ? kAcosPrecision - 1 : scaled);
  return __ldg(lut + scaled);
}

NB_D V4 env_sample(const DevScene &sc, V3 dir) {
  V3 n = normalize(dir);
  float phi = atan2_approx(n.y, n.x);
  float theta = acos_lt(sc.acos_lut, n.z);
  float u = (float)((double)phi * kInv2PiD);
  float v = (float)((double)theta * kInvPiD);
  return f32pixel(sc.textures[sc.envmap], tex_wrap(u), tex_wrap(v));
}

/* ---------------------------------------------------------------- hit record */

struct HitRecord {
  V3 dpdu, dpdv, ng, position;
  float u, v;
  M3 frame;
};

NB_D M3 gram_schmidt(V3 normal, V3 tangent, V3 bitangent) { /* utils_3D.h:63-70 */
  V3 N = normalize(normal);
  V3 T = normalize(tangent - N * dot(tangent, N));
  V3 B = cross(N, T);
  if (dot(B, bitangent) < 0.0f) B = -B;
  return {{T, B, N}};
}

NB_D void make_onb(V3 n, V3 &b1, V3 &b2) { /* utils_3D.h:74-81 */
  n = normalize(n);
  float sign = copysignf(1.f, n.z);
  float a = -1.f / (sign + n.z);
  float b = n.x * n.y * a;
  b1 = {1.f + sign * n.x * n.x * a, sign * b, -sign * n.x};
  b2 = {b, sign + n.y * n.y * a, -n.y};
}

NB_D V3 blerp(V3 p0, V3 p1, V3 p2, float w, float u, float v) { return p0 * w + p1 * u + p2 * v; }

struct VertexAttr {
  V3 p, n, t, b;
  float u, v;
};
NB_D VertexAttr load_vertex(const float4 *attr, uint32_t i) {
  const float4 *a = attr + 4 * (size_t)i;
  const float4 a0 = __ldg(a), a1 = __ldg(a + 1), a2 = __ldg(a + 2), a3 = __ldg(a + 3);
  return {{a0.x, a0.y, a0.z}, {a0.w, a1.x, a1.y}, {a1.z, a1.w, a2.x}, {a2.y, a2.z, a2.w}, a3.x, a3.y};
}

NB_D HitRecord make_record(const DevScene &sc, V3 ro, V3 rd, const DevInstance &I, uint32_t tri, float t, float bu,
                           float bv) {
  const uint32_t *idx = I.idx;
  const uint32_t i0 = __ldg(idx + 3 * tri), i1 = __ldg(idx + 3 * tri + 1), i2 = __ldg(idx + 3 * tri + 2);
  const VertexAttr A = load_vertex(I.attr, i0), B = load_vertex(I.attr, i1), C = load_vertex(I.attr, i2);
  HitRecord r;
  const float w = 1 - (bu + bv);
  r.u = A.u * w + B.u * bu + C.u * bv;
  r.v = A.v * w + B.v * bu + C.v * bv;
  const M3 l = m3_of4(I.m);
  const float duv02x = A.u - C.u, duv02y = A.v - C.v;
  const float duv12x = B.u - C.u, duv12y = B.v - C.v;
  const V3 dp02 = mul(l, V3{A.p.x - C.p.x, A.p.y - C.p.y, A.p.z - C.p.z});
  const V3 dp12 = mul(l, V3{B.p.x - C.p.x, B.p.y - C.p.y, B.p.z - C.p.z});
  const float det = duv02x * duv12y - duv02y * duv12x;
  const bool degen_uv = fabsf(det) < 1e-9f;
  const float invdet = 1.f / det;
  V3 dpdu = (duv12y * dp02 - duv02y * dp12) * invdet;
  V3 dpdv = (duv02x * dp12 - duv12x * dp02) * invdet;
  V3 n;
  if (degen_uv || length(cross(dpdu, dpdv)) == 0) {
    n = normalize(cross(dp12, dp02));
    make_onb(n, dpdu, dpdv);
  } else {
    n = cross(dp02, dp12);
  }
  r.ng = normalize(n);
  r.position = ro + t * rd;
  r.dpdu = dpdu;
  r.dpdv = dpdv;
  const V3 nn = blerp(A.n, B.n, C.n, w, bu, bv);
  const V3 tt = blerp(A.t, B.t, C.t, w, bu, bv);
  const V3 bb = blerp(A.b, B.b, C.b, w, bu, bv);
  const V3 tn = normalize(mul(m3_load(I.n), nn));
  const V3 tt2 = normalize(mul(l, tt));
  const V3 tb = normalize(mul(l, bb));
  r.frame = gram_schmidt(tn, tt2, tb);
  return r;
}

/* ---------------------------------------------------------------- microfacet math */

NB_D float absdot(V3 a, V3 b) { return fabsf(dot(a, b)); }
NB_D bool same_hemi(V3 a, V3 b) { return a.z * b.z > 0; }
NB_D float cos2theta(V3 v) { return sqr(v.z); }
NB_D float sin2theta(V3 v) { return fmax_std(0.f, 1.f - cos2theta(v)); }
NB_D float sin2theta_c(float c) { return fmax_std(0.f, 1.f - sqr(c)); }
NB_D float sintheta(V3 v) { return msqrt(sin2theta(v)); }
NB_D float tan2theta(V3 v) { return sin2theta(v) / cos2theta(v); }
NB_D float cosphi(V3 v) {
  float s = sintheta(v);
  if (s == 0.f) return 1.f;
  return fclampf(v.x / s, -1.f, 1.f);
}
NB_D float sinphi(V3 v) {
  float s = sintheta(v);
  if (s == 0.f) return 0.f;
  return fclampf(v.y / s, -1.f, 1.f);
}

NB_D float refract(V3 wo, V3 n, float eta, bool &valid, V3 &wt) { /* BxDF_math.h:105-124 */
  valid = true;
  float ci = dot(wo, n);
  if (ci < 0) {
    n = -n;
    eta = 1.f / eta;
    ci = -ci;
  }
  float s2t = sin2theta_c(ci) / sqr(eta);
  if (s2t >= 1.f) {
    valid = false;
    return 0.f;
  }
  float ct = msqrt(1.f - s2t);
  wt = -wo / eta + (ci / eta - ct) * n;
  return eta;
}

NB_D V3 hemisphere_cosine_sample(float u0, float u1) { /* shirley_chiu, BxDF_math.h:129-152 */
  float sx = 2 * u0 - 1, sy = 2 * u1 - 1;
  float px = 0.f, py = 0.f;
  if (!(sx == 0 && sy == 0)) {
    float r, theta;
    if (fabsf(sx) > fabsf(sy)) {
      r = sx;
      theta = kPi4F * (sy / sx);
    } else {
      r = sy;
      theta = kPi2F - kPi4F * (sx / sy);
    }
    float st, ct;
    sincos_rn(theta, st, ct);
    px = r * ct;
    py = r * st;
  }
  float z = sqrtf(fmax_std(0.f, 1 - px * px - py * py));
  return {px, py, z};
}

NB_D float schlick(float c, float F0) { return F0 + (1.f - F0) * pow5f(1.f - c); }
NB_D V3 schlick(float c, V3 F0) { return F0 + (1.f - F0) * pow5f(1.f - c); }

NB_D float fresnel_real(float etar, float ci) { /* Fresnel::real, BxDF_math.h:186-204 */
  float eta = etar;
  ci = fclampf(ci, -1.f, 1.f);
  if (ci < 0) {
    eta = 1.f / eta;
    ci = -ci;
  }
  float s2t = sin2theta_c(ci) / sqr(eta);
  if (s2t >= 1) return 1.f;
  float ct = msqrt(1.f - s2t);
  float rpar = (eta * ci - ct) / (eta * ci + ct);
  float rperp = (ci - eta * ct) / (ci + eta * ct);
  return (sqr(rpar) + sqr(rperp)) / 2.f;
}

struct VNDF { /* BxDF_math.h:226-343 */
  float ax, ay, ax_inv, ay_inv;
  NB_D void init(float anisotropy, float roughness) {
    anisotropy = fclampf(anisotropy, -1.f, 1.f);
    float aspect = msqrt(1.f - 0.9f * anisotropy);
    float a = roughness != 0 ? roughness * roughness : 1e-6f;
    ax = a / aspect;
    ay = a * aspect;
    ax_inv = 1.f / ax;
    ay_inv = 1.f / ay;
  }
  NB_D float D(V3 wm) const {
    if (wm.z < 1e-6f) return 0.f;
    float c2 = sqr(cosphi(wm)) * sqr(ax_inv);
    float s2 = sqr(sinphi(wm)) * sqr(ay_inv);
    double denom = kPiD * (double)ax * (double)ay * (double)sqr(cos2theta(wm)) *
                   (double)sqr(1.f + tan2theta(wm) * (c2 + s2));
    return 1.f / (float)denom;
  }
  NB_D float lambda(V3 v) const {
    float t2 = tan2theta(v);
    if (isinf(t2) || isnan(t2)) return 0;
    float a2 = sqr(ax) * sqr(cosphi(v)) + sqr(ay) * sqr(sinphi(v));
    return (msqrt(1 + a2 * t2) - 1) * 0.5f;
  }
  NB_D float G1(V3 v) const {
    v.z = fmax_std(v.z, 1e-6f);
    return 1.f / (1.f + lambda(v));
  }
  NB_D float G(V3 wo, V3 wi) const { return 1.f / (1.f + lambda(wo) + lambda(wi)); }
  NB_D float pdf(V3 wo, V3 wm) const { return D(wm) * absdot(wo, wm) * G1(wo) / fabsf(wo.z); }
  NB_D V3 sample(V3 wo, float u0, float u1) const {
    V3 wh = normalize(V3{wo.x * ax, wo.y * ay, wo.z});
    if (wh.z < 0) wh = -wh;
    V3 t = wh.z < 1.f ? normalize(cross(V3{0.f, 0.f, 1.f}, wh)) : V3{1.f, 0.f, 0.f};
    V3 b = cross(wh, t);
    float r = msqrt(u0);
    float th = (float)(2.0 * kPiD * (double)u1);
    float sth, cth;
    sincos_rn(th, sth, cth);
    float px = r * cth, py = r * sth;
    float s = 0.5f * (1.f + wh.z);
    py = msqrt(1.f - sqr(px)) * (1.f - s) + s * py;
    V3 nh = px * t + py * b + msqrt(fmaxf(0.f, 1.f - sqr(px) - sqr(py))) * wh;
    return normalize(V3{ax * nh.x, ay * nh.y, fmax_std(1e-6f, nh.z)});
  }
  NB_D bool full_specular() const { return fmax_std(ax, ay) < 1e-5f; }

  /* Derivatives with respect to the base width a (ax = a / aspect, ay = a * aspect, both
   * proportional to a).  D = 1 / (pi ax ay cos^4 (1 + E)^2) with E proportional to a^-2. */
  NB_D float dlnD_da(V3 wm, float a) const {
    if (wm.z < 1e-6f) return 0.f;
    const float E = tan2theta(wm) * (sqr(cosphi(wm)) * sqr(ax_inv) + sqr(sinphi(wm)) * sqr(ay_inv));
    return -2.f / a + 4.f * E / (a * (1.f + E));
  }
  /* lambda = (sqrt(1 + a2 t) - 1) / 2 with a2 proportional to a^2 */
  NB_D float dlambda_da(V3 v, float a) const {
    const float t2 = tan2theta(v);
    if (isinf(t2) || isnan(t2)) return 0.f;
    const float a2 = sqr(ax) * sqr(cosphi(v)) + sqr(ay) * sqr(sinphi(v));
    return a2 * t2 / (2.f * a * msqrt(1 + a2 * t2));
  }
  NB_D float dlnG_da(V3 wo, V3 wi, float a) const {
    return -(dlambda_da(wo, a) + dlambda_da(wi, a)) / (1.f + lambda(wo) + lambda(wi));
  }
};

/* d ln f / d theta of the sampled lobe at the sampled directions (the sampling density held fixed):
 * albedo per colour channel and the material's roughness.  Zero where f does not depend on it. */
struct Scores {
  V3 albedo;
  float roughness;
};

NB_D V3 inv_or_zero(V3 a) {
  return {a.x != 0.f ? 1.f / a.x : 0.f, a.y != 0.f ? 1.f / a.y : 0.f, a.z != 0.f ? 1.f / a.z : 0.f};
}

enum : unsigned { F_REFL = 1, F_TRANS = 2, F_DIFFUSE = 4, F_GLOSSY = 8, F_SPECULAR = 16, F_ALL = 31 };
enum Lobe : int { L_NONE = 0, L_DIFFUSE = 1, L_SPECULAR = 2, L_DIELECTRIC = 3 };

struct BsdfParams { /* bsdf_params_s, BxDF.h:22-39 (sheen/clearcoat are 0, specular 1, subsurface 1) */
  V3 ns, ng, dpdu, dpdv;
  float wo_dot_ng, metal, roughness, transmission, anisotropy;
  V3 eta, albedo;
};

struct BsdfSample {
  V3 f, wi;
  float pdf, costheta;
};

struct PrincipledBSDF {
  BsdfParams p;
  M3 frame;
  float w_diffuse, w_specular, w_transmission, p_diffuse, p_specular, p_transmission;
  int lobe;
  float lobe_w, lobe_p;
  VNDF ggx;

  NB_D void weights() { /* BSDF.h:43-67 */
    float ac = fabsf(p.wo_dot_ng);
    w_diffuse = (1 - p.transmission) * (1 - p.metal);
    w_specular = 1.f;
    w_transmission = (1.f - p.metal) * p.transmission;
    float F = schlick(ac, 1.f * 0.04f);
    float pd = w_diffuse * (1.f - F);
    float ps = w_specular * F;
    float W = pd + ps + 0.f + 0.f + w_transmission;
    if (W == 0) W = 1.f;
    p_diffuse = pd / W;
    p_specular = ps / W;
    p_transmission = w_transmission / W;
  }
  NB_D void configure(const BsdfParams &in) { /* BSDF.h:87-97 */
    p = in;
    frame = gram_schmidt(p.ns, p.dpdu, p.dpdv);
    if (p.wo_dot_ng < 0) {
      frame.c[0] = -frame.c[0];
      frame.c[1] = -frame.c[1];
      frame.c[2] = -frame.c[2];
      if (all_nonzero(p.eta)) p.eta = 1.f / p.eta;
    }
    weights();
  }
  NB_D void choose(float uc) { /* constructBXDF, BSDF.h:69-79 */
    float idx = 0.f;
    lobe = L_NONE;
    if (uc < (idx += p_diffuse)) {
      lobe = L_DIFFUSE, lobe_w = w_diffuse, lobe_p = p_diffuse;
    } else if (uc < (idx += p_specular)) {
      lobe = L_SPECULAR, lobe_w = w_specular, lobe_p = p_specular;
      ggx.init(p.anisotropy, p.roughness);
    } else if (uc < (idx += p_transmission)) {
      lobe = L_DIELECTRIC, lobe_w = w_transmission, lobe_p = p_transmission;
      ggx.init(p.anisotropy, p.roughness);
    }
  }
  NB_D unsigned flags() const {
    if (lobe == L_DIFFUSE) return F_DIFFUSE | F_REFL;
    if (lobe == L_SPECULAR) return (ggx.full_specular() ? F_SPECULAR : F_GLOSSY) | F_REFL;
    if (lobe == L_DIELECTRIC)
      return (p.eta.x == 1.f ? F_TRANS : (F_REFL | F_TRANS)) | (ggx.full_specular() ? F_SPECULAR : F_GLOSSY);
    return 0u;
  }

  NB_D bool diffuse_sample(V3 wo, float u0, float u1, BsdfSample &s, Scores *sc) const { /* BxDF.h:285-324 */
    V3 wi = normalize(hemisphere_cosine_sample(u0, u1));
    V3 h = normalize(wi + wo);
    float ci = wi.z, co = wo.z;
    if (!same_hemi(wo, wi) || ci <= 0.f || co <= 0.f) return false;
    float rough = sqr(p.roughness);
    /* fd = albedo/pi F(fd90)F(fd90) is weighted by (1 - subsurface) = 0 and is finite, so it adds 0 */
    float fss90 = rough * sqr(absdot(h, wi));
    float fwi = 1.f + (fss90 - 1) * pow5f(1.f - fabsf(wi.z));
    float fwo = 1.f + (fss90 - 1) * pow5f(1.f - fabsf(wo.z));
    V3 fss = 1.25f * p.albedo * kInvPiF * (0.5f + fwi * fwo * (-0.5f + 1 / (co + ci)));
    V3 fd = p.albedo * kInvPiF;
    V3 f = lobe_w * ((1 - 1.f) * fd + 1.f * fss);
    s.f = f;
    s.costheta = ci;
    s.pdf = lobe_p * (ci * kInvPiF);
    s.wi = wi;
    if (sc) {
      /* f = K albedo (0.5 + fwi fwo A), fss90 = r^2 cos^2(theta_d) */
      const float A = -0.5f + 1 / (co + ci);
      const float Pi = pow5f(1.f - fabsf(wi.z)), Po = pow5f(1.f - fabsf(wo.z));
      const float dfss90 = 2.f * p.roughness * sqr(absdot(h, wi));
      sc->albedo = inv_or_zero(p.albedo);
      const float den = 0.5f + fwi * fwo * A;
      sc->roughness = den != 0.f ? A * (Pi * fwo + fwi * Po) * dfss90 / den : 0.f;
    }
    return true;
  }

  /* d ln(D G) / d roughness at fixed directions (alpha = r^2; the 1e-6 floor at r = 0 is constant) */
  NB_D float dlnDG_dr(V3 wo, V3 wi, V3 wm) const {
    if (p.roughness == 0.f) return 0.f;
    const float a = p.roughness * p.roughness;
    return (ggx.dlnD_da(wm, a) + ggx.dlnG_da(wo, wi, a)) * 2.f * p.roughness;
  }

  NB_D bool specular_sample(V3 wo, float u0, float u1, BsdfSample &s, Scores *sc) const { /* BxDF.h:367-397 */
    V3 wm = ggx.sample(wo, u0, u1);
    V3 wi = reflect(-wo, wm);
    float co = wo.z, ci = wi.z;
    if (co <= 0 || ci <= 0) return false;
    float wmwo = absdot(wm, wo);
    V3 a = v3(p.metal);
    V3 F0 = v3(0.04f) * (v3(1.f) - a) + a * p.albedo;
    V3 Fr = schlick(wmwo, F0);
    V3 f = Fr * ggx.D(wm) * ggx.G(wo, wi) / (4 * co * ci);
    float pdf = ggx.pdf(wo, wm) / (4 * wmwo);
    s.f = lobe_w * f;
    s.pdf = lobe_p * pdf;
    s.wi = wi;
    s.costheta = ci;
    if (sc) {
      /* Fr = F0 + (1 - F0) P with F0 = 0.04 (1 - metal) + metal albedo */
      const float P = pow5f(1.f - wmwo);
      const float dF = p.metal * (1.f - P);
      sc->albedo = V3{Fr.x != 0.f ? dF / Fr.x : 0.f, Fr.y != 0.f ? dF / Fr.y : 0.f, Fr.z != 0.f ? dF / Fr.z : 0.f};
      sc->roughness = dlnDG_dr(wo, wi, wm);
    }
    return true;
  }

  NB_D bool dielectric_sample(V3 wo, float uc, float u0, float u1, BsdfSample &s, Scores *sc) const {
    /* BxDF.h:547-594; f is proportional to the albedo in every branch */
    if (sc) {
      sc->albedo = inv_or_zero(p.albedo);
      sc->roughness = 0.f;
    }
    const float ior = p.eta.x;
    if (ggx.full_specular() || p.eta.x == 1.f) {
      float R = fresnel_real(ior, wo.z), T = 1 - R;
      float pr = R, pt = T;
      if (pr == 0.f && pt == 0.f) return false;
      if (uc < (pr / (pr + pt))) {
        V3 wi = reflect(-wo, V3{0.f, 0.f, 1.f});
        float ci = fabsf(wi.z);
        s.costheta = ci;
        s.f = lobe_w * p.albedo * R / ci;
        s.pdf = lobe_p * pr / (pr + pt);
        s.wi = wi;
        return true;
      }
      bool ok = true;
      V3 wi{0.f, 0.f, 0.f};
      refract(wo, V3{0.f, 0.f, 1.f}, ior, ok, wi);
      if (!ok) return false;
      float ci = fabsf(wi.z);
      V3 f = T * p.albedo / ci;
      f = f / sqr(ior);
      s.f = lobe_w * f;
      s.costheta = ci;
      s.pdf = lobe_p * pt / (pr + pt);
      s.wi = wi;
      return true;
    }
    V3 wm = ggx.sample(wo, u0, u1);
    float R = fresnel_real(ior, dot(wo, wm)), T = 1 - R;
    float pr = R, pt = T;
    if (pr == 0.f && pt == 0.f) return false;
    if (uc < (pr / (pr + pt))) {
      V3 wi = reflect(-wo, wm);
      if (!same_hemi(wo, wi)) return false;
      V3 f = p.albedo * ggx.D(wm) * ggx.G(wo, wi) * R / (4 * wi.z * wo.z);
      float pdf = ggx.pdf(wo, wm) / (4 * absdot(wo, wm)) * pr / (pr + pt);
      s.f = lobe_w * f;
      s.pdf = lobe_p * pdf;
      s.wi = wi;
      s.costheta = fabsf(wi.z);
      if (sc) sc->roughness = dlnDG_dr(wo, wi, wm);
      return true;
    }
    V3 wi{0.f, 0.f, 0.f};
    bool no_tir = true;
    float eta = refract(wo, wm, ior, no_tir, wi);
    wi = normalize(wi);
    if (same_hemi(wi, wo) || wi.z == 0.f || !no_tir) return false;
    float ci = wi.z, co = wo.z;
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / eta);
    float jac = absdot(wi, wm) / denom;
    float pdf = ggx.pdf(wo, wm) * jac * pt / (pt + pr);
    V3 f = p.albedo * T * ggx.D(wm) * ggx.G(wo, wi) * fabsf(dot(wi, wm) * dot(wo, wm) / (ci * co * denom));
    f = f / sqr(eta);
    s.f = lobe_w * f;
    s.costheta = fabsf(wi.z);
    s.pdf = lobe_p * pdf;
    s.wi = wi;
    if (sc) sc->roughness = dlnDG_dr(wo, wi, wm);
    return true;
  }

  NB_D bool sample_f(V3 wo, float uc, float u0, float u1, BsdfSample &s, Scores *sc) const { /* BSDF.h:107-130 */
    if (lobe == L_NONE) return false;
    V3 lwo = normalize(mul_t(frame, wo));
    if (!(flags() & F_ALL) || lwo.z == 0.f) return false;
    bool ok;
    if (lobe == L_DIFFUSE)
      ok = diffuse_sample(lwo, u0, u1, s, sc);
    else if (lobe == L_SPECULAR)
      ok = specular_sample(lwo, u0, u1, s, sc);
    else
      ok = dielectric_sample(lwo, uc, u0, u1, s, sc);
    if (!ok) return false;
    if (!any_nonzero(s.f) || s.pdf == 0.f || s.wi.z == 0.f) return false;
    s.wi = normalize(mul(frame, s.wi));
    return true;
  }
};

NB_D V3 correct_specular_shading_normal(V3 ng, V3 wo, V3 ns) { /* BxDF_math.h:26-53 */
  V3 R = reflect(-wo, ns);
  const float woz = dot(wo, ng);
  const float threshold = fminf(0.9f * woz, 0.01f);
  if (dot(ng, R) >= threshold) return ns;
  V3 X = normalize(ns - dot(ns, ng) * ng);
  if (length2(X) == 0.f) X = ns;
  const float wox = dot(wo, X);
  const float a = sqr(wox) + sqr(woz);
  const float b = 2.0f * (a + woz * threshold);
  const float c = sqr(threshold + woz);
  const float Nz2 = (wox < 0) ? 0.25f * (b + msqrt(sqr(b) - 4.0f * a * c)) / a
                              : 0.25f * (b - msqrt(sqr(b) - 4.0f * a * c)) / a;
  if (Nz2 > 1.f || Nz2 < 0.f) return ng;
  float Nx = msqrt(1.0f - Nz2);
  float Nz = msqrt(Nz2);
  return Nx * X + Nz * ng;
}

NB_D float u8f(float v) { return v * (1.f / 255.f); } /* rgb_uint2float, math_texturing.h:8-12 */

struct ScatterResult {
  V3 weight;   /* f * |cos| / pdf: the integrator's per-level factor (Integrator.cpp:84-87) */
  V3 emissive;
  V3 wi;
  bool valid;
};

/* PrincipledMaterial::scatter + sampleBSDF (NovaMaterials.h:56-137).  Consumes four Sobol
 * dimensions starting at `dim`: uc (lobe choice), u0[2] (direction), uc (sample_f).  `prim` and
 * `mat_id` select the differentiable parameters when the scene has them (per-triangle albedo and
 * per-material roughness replace the albedo texture and the metallic texture's roughness channel);
 * `scores`, when given, receives d ln f / d(albedo, roughness) of the sampled lobe. */
/* The normal-mapped shading normal (NovaMaterials.h:103-104 with compute_local_normal): a missing
 * normal map reads as (0, 0, 1), i.e. the local normal (-1, -1, 1). */
NB_D V3 shading_normal(const DevScene &sc, const HitRecord &hr, const DevMaterial &mat) {
  V3 nmap{0.f, 0.f, 1.f};
  if (mat.normalmap >= 0) {
    V4 t = sample_u8(sc.textures[mat.normalmap], hr.u, hr.v);
    nmap = {u8f(t.x), u8f(t.y), u8f(t.z)};
  }
  return normalize(mul(hr.frame, nmap * 2.f - 1.f));
}

NB_D ScatterResult scatter(const DevScene &sc, V3 rd, const HitRecord &hr, const DevMaterial &mat, uint32_t index,
                           unsigned dim, uint32_t seed, uint32_t prim, uint32_t mat_id, Scores *scores = nullptr) {
  const float u = hr.u, v = hr.v;
  const V3 ns = shading_normal(sc, hr, mat);
  BsdfParams bp;
  bp.dpdu = hr.dpdu;
  bp.dpdv = hr.dpdv;
  bp.ns = ns;
  bp.ng = hr.ng;
  const V3 wo = normalize(-rd);
  bp.wo_dot_ng = dot(wo, hr.ng);
  V3 albedo{1.f, 1.f, 1.f};
  if (mat.albedo >= 0) {
    V4 t = sample_u8(sc.textures[mat.albedo], u, v);
    albedo = {u8f(t.x), u8f(t.y), u8f(t.z)};
  }
  if (sc.diff_albedo) albedo = {sc.diff_albedo[3 * prim], sc.diff_albedo[3 * prim + 1], sc.diff_albedo[3 * prim + 2]};
  bp.albedo = albedo;
  float rough = 0.f, metal = 0.f;
  if (mat.metallic >= 0) {
    V4 t = sample_u8(sc.textures[mat.metallic], u, v);
    rough = u8f(t.y);
    metal = u8f(t.z);
  }
  if (sc.diff_rough) rough = sc.diff_rough[mat_id];
  bp.roughness = rough;
  bp.metal = metal;
  const V3 eta{mat.eta[0], mat.eta[1], mat.eta[2]}, k{mat.k[0], mat.k[1], mat.k[2]};
  bp.transmission = (any_nonzero(eta) && !any_nonzero(k)) ? 1.f : 0.f;
  bp.anisotropy = mat.anisotropy;
  bp.eta = eta;

  float uc = sobol_sample(sc.sobol_dv, index, dim, seed);
  const float u0 = sobol_sample(sc.sobol_dv, index, dim + 1, seed);
  const float u1 = sobol_sample(sc.sobol_dv, index, dim + 2, seed);
  PrincipledBSDF bsdf;
  bsdf.configure(bp);
  bsdf.choose(uc);
  if ((bsdf.flags() & (F_GLOSSY | F_REFL)) && bp.wo_dot_ng >= 0) {
    V3 cns = normalize(correct_specular_shading_normal(bp.ng, wo, bp.ns));
    bp.ns = cns;
    bsdf.configure(bp); /* the chosen lobe keeps its weight and probability (captured at construction) */
  }
  uc = sobol_sample(sc.sobol_dv, index, dim + 3, seed);
  BsdfSample s;
  s.f = v3(0.f);
  s.pdf = 0.f;
  s.costheta = 0.f;
  ScatterResult out;
  if (scores) *scores = Scores{v3(0.f), 0.f};
  out.valid = bsdf.sample_f(wo, uc, u0, u1, s, scores);
  out.weight = s.f * s.costheta / s.pdf;
  out.wi = s.wi;
  out.emissive = v3(0.f);
  if (mat.emissive >= 0) {
    V4 t = sample_u8(sc.textures[mat.emissive], u, v);
    out.emissive = {u8f(t.x), u8f(t.y), u8f(t.z)};
  }
  return out;
}

}  // namespace nb
