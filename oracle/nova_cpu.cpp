/* ORACLE — test infrastructure only (see oracle.h).
 *
 * CPU restatement of the reference's Nova path (corelib/nova): camera rays, Embree-semantics hit
 * record, textures, the principled material / BSDF / BxDF stack, the environment map lookup, the
 * recursive PathIntegrator::Li and the tiled progressive render with its running-mean film.
 * Each function cites the reference source it follows.
 */
#include "oracle_internal.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>

namespace orc {

/* ------------------------------------------------------------------------------------------------
 * Spectrum helpers (spectrum/BaseSpectrum.h).  Spectrum != 0.f is true only when every sample
 * differs from 0 (BaseSpectrum.h operator!=); "if (eta && !k)" uses operator bool (any sample != 0). */
static inline bool spec_all_nonzero(Spec s) { return s.x != 0.f && s.y != 0.f && s.z != 0.f; }

/* ------------------------------------------------------------------------------------------------
 * Textures (texturing/NovaTextureInterface.h, texturing/TextureContext.h). */

/* wrap(), NovaTextureInterface.h:13-23 */
static inline float wrap(float uv) {
  if (uv < 0.f) {
    float fp = std::ceil(uv) - uv;
    return 1.f - fp;
  }
  if (uv > 1.f) return uv - std::floor(uv);
  return uv;
}

/* uvToPixel, math_texturing.h:19-21: unsigned(coord * dim), the product in float. */
static inline unsigned uv_to_pixel(float coord, unsigned dim) { return (unsigned)(coord * (float)dim); }

/* uv2index, TextureContext.h:52-58 */
static inline unsigned uv2index(float t, int dim) {
  float a = std::fabs(t);
  float rem = a - std::floor(a);
  rem = rem == 0 ? a : rem;
  return uv_to_pixel(rem, (unsigned)dim);
}

/* getPixelFromFormat, NovaTextureInterface.h:60-99 (little-endian byte order r,g,b,a). */
static inline V4 pixel_from_format(uint32_t px, bool is_rgba, int channels) {
  float b0 = (float)(px & 0xffu), b1 = (float)((px >> 8) & 0xffu), b2 = (float)((px >> 16) & 0xffu),
        b3 = (float)((px >> 24) & 0xffu);
  float r, g, b, a;
  if (is_rgba) {
    r = b0, g = b1, b = b2, a = b3;
  } else {
    r = b2, g = b1, b = b0, a = b3;
  }
  switch (channels) {
    case 1: return {r, 0, 0, 1.f};
    case 2: return {r, g, 0, 1.f};
    case 3: return {r, g, b, 1.f};
    default: return {r, g, b, a};
  }
}

/* ImageTexture<uint32_t>::sample on the CPU: wrap, TextureCtx::u32pixel bilinear taps
 * (TextureContext.h:129-161), bilinearInterpolate (NovaTextureInterface.h:101-116). */
static V4 sample_u8(const Texture &tx, float u, float v) {
  u = wrap(u);
  v = wrap(v);
  u = tx.invert_u ? 1 - u : u;
  v = tx.invert_v ? 1 - v : v;
  const int width = tx.w, height = tx.h;
  float pi = std::fabs(u * (float)(width - 1.f));
  float pj = std::fabs(v * (float)(height - 1.f));
  unsigned i = (unsigned)std::floor(pi);
  unsigned j = (unsigned)std::floor(pj);
  auto ensure_bound = [](unsigned index, unsigned limit) -> unsigned {
    unsigned val = index;
    if (val + 1 >= limit) val = limit - 2;
    if (val > limit) val = 0;
    return val;
  };
  i = ensure_bound(i, (unsigned)width);
  j = ensure_bound(j, (unsigned)height);
  float ftx = float(pi - (float)i) / float((i + 1) - i);
  float fty = float(pj - (float)j) / float((j + 1) - j);
  uint32_t p0 = tx.u8[j * width + i], p1 = tx.u8[j * width + i + 1];
  uint32_t p2 = tx.u8[(j + 1) * width + i], p3 = tx.u8[(j + 1) * width + i + 1];
  V4 v0 = pixel_from_format(p0, tx.is_rgba, tx.channels), v1 = pixel_from_format(p1, tx.is_rgba, tx.channels);
  V4 v2 = pixel_from_format(p2, tx.is_rgba, tx.channels), v3 = pixel_from_format(p3, tx.is_rgba, tx.channels);
  float hd = 1 - ftx;
  V4 top = hd * v0 + ftx * v1;
  V4 bot = hd * v2 + ftx * v3;
  return (1 - fty) * top + fty * bot;
}

/* TextureCtx::f32pixel on the CPU: nearest texel through uv2index(dim - 1) (TextureContext.h:196-223). */
static V4 f32pixel(const Texture &tx, float u, float v) {
  u = tx.invert_u ? 1 - u : u;
  v = tx.invert_v ? 1 - v : v;
  unsigned i = uv2index(u, tx.w - 1);
  unsigned j = uv2index(v, tx.h - 1);
  const int ch = tx.channels;
  size_t idx = ((size_t)j * tx.w + i) * ch;
  V4 rgba{0, 0, 0, 0};
  float *p = &rgba.x;
  for (int c = 0; c < ch && c < 4; c++) p[c] = tx.f32[idx + c];
  return rgba;
}

/* atan2_approx, corelib/internal/common/math/math_utils_approx.h:13-40 */
static inline float horner_approx(float x) {
  float a1 = 0.99997726f, a3 = -0.33262347f, a5 = 0.19354346f, a7 = -0.11643287f, a9 = 0.05265332f,
        a11 = -0.01172120f;
  float x_sq = x * x;
  return x * (a1 + x_sq * (a3 + x_sq * (a5 + x_sq * (a7 + x_sq * (a9 + x_sq * a11)))));
}
static inline float atan2_approx(float y, float x) {
  const float PI_F = (float)M_PI;
  const float PI_2 = (float)M_PI_2;
  bool swap = std::fabs(x) < std::fabs(y);
  float atan_input = (swap ? x : y) / (swap ? y : x);
  float res = horner_approx(atan_input);
  res = swap ? (atan_input >= 0.0f ? PI_2 : -PI_2) - res : res;
  if (x >= 0.0f && y >= 0.0f) {
  } else if (x < 0.0f && y >= 0.0f) {
    res = PI_F + res;
  } else if (x < 0.0f && y < 0.0f) {
    res = -PI_F + res;
  }
  return res;
}
/* acos_lt, math_acos_lt.cpp:37-40 */
static inline float acos_lt(float a) {
  int scaled = std::clamp((int)((a + 1.f) * kAcosPrecision * 0.5f), 0, kAcosPrecision - 1);
  return acos_lut()[scaled];
}

/* EnvmapTexture::sample (NovaTextureInterface.h:152-168): normalize, cartesianToSpherical with the
 * fast approximations (math_spherical.h:44-52), sphericalToUv in double (INV_2PI, INV_PI are
 * doubles, math_spherical.h:9-10), wrap, f32pixel. */
static V4 env_sample(const Scene &s, V3 dir) {
  V3 nrm = normalize(dir);
  float phi = atan2_approx(nrm.y, nrm.x);
  float theta = acos_lt(nrm.z);
  const double PI_D = M_PI;
  const double INV_PI_D = 1.f / PI_D;
  const double INV_2PI_D = 1.f / (2.f * PI_D);
  float u = (float)(phi * INV_2PI_D);
  float v = (float)(theta * INV_PI_D);
  u = wrap(u);
  v = wrap(v);
  return f32pixel(s.textures[s.envmap], u, v);
}

/* ------------------------------------------------------------------------------------------------
 * Hit record with Embree semantics (aggregate/api/embree/embree.cpp:287-412) from the native
 * Moller-Trumbore hit (t, u, v). */
struct HitRecord {
  V3 dpdu, dpdv, ng, position;
  float u, v, t;
  M3 frame; /* T, B, N columns */
};

/* math::gram_shmidt(normal, tangent, bitangent), utils_3D.h:63-70 */
static M3 gram_shmidt(V3 normal, V3 tangent, V3 bitangent) {
  V3 N = normalize(normal);
  V3 T = normalize(tangent - N * dot(tangent, N));
  V3 B = cross(N, T);
  if (dot(B, bitangent) < 0.0f) B = -B;
  return {{T, B, N}};
}
/* math::make_onb, utils_3D.h:74-81 */
static void make_onb(V3 n, V3 &b1, V3 &b2) {
  n = normalize(n);
  float sign = std::copysign(1.f, n.z);
  float a = -1.f / (sign + n.z);
  float b = n.x * n.y * a;
  b1 = {1.f + sign * n.x * n.x * a, sign * b, -sign * n.x};
  b2 = {b, sign + n.y * n.y * a, -n.y};
}

template <int K>
static inline V3 attr3(const std::vector<float> &a, const uint32_t *id, int k) {
  return {a[3 * id[k]], a[3 * id[k] + 1], a[3 * id[k] + 2]};
}
/* barycentric_lerp(p0, p1, p2, w, u, v) = p0*w + p1*u + p2*v (utils_3D.h:16-19) */
static inline V3 blerp(V3 p0, V3 p1, V3 p2, float w, float u, float v) { return p0 * w + p1 * u + p2 * v; }

static HitRecord make_record(const Scene &s, const Ray &ray, const Hit &h) {
  const Prim &p = s.prims[h.prim];
  const Mesh &m = s.meshes[s.inst_mesh[p.inst]];
  const Xform &x = s.xf[p.inst];
  const uint32_t *id = &m.idx[3 * p.tri];
  HitRecord r;
  const float w = 1 - (h.u + h.v);
  /* uv through rtcInterpolate0 (embree.cpp:349) */
  float uv0x = m.uv[2 * id[0]], uv0y = m.uv[2 * id[0] + 1];
  float uv1x = m.uv[2 * id[1]], uv1y = m.uv[2 * id[1] + 1];
  float uv2x = m.uv[2 * id[2]], uv2y = m.uv[2 * id[2] + 1];
  float iu = uv0x * w + uv1x * h.u + uv2x * h.v;
  float iv = uv0y * w + uv1y * h.u + uv2y * h.v;
  /* computeDerivativesTriangle, embree.cpp:287-340 */
  M3 l = m3_of(x.m);
  float duv02x = uv0x - uv2x, duv02y = uv0y - uv2y;
  float duv12x = uv1x - uv2x, duv12y = uv1y - uv2y;
  V3 v0 = attr3<0>(m.v, id, 0), v1 = attr3<0>(m.v, id, 1), v2 = attr3<0>(m.v, id, 2);
  V3 dp02 = mul(l, V3{v0.x - v2.x, v0.y - v2.y, v0.z - v2.z});
  V3 dp12 = mul(l, V3{v1.x - v2.x, v1.y - v2.y, v1.z - v2.z});
  float determinant = duv02x * duv12y - duv02y * duv12x;
  bool degen_uv = std::fabs(determinant) < 1e-9f;
  float invdet = 1.f / determinant;
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
  r.position = ray.o + h.t * ray.d;
  r.dpdu = dpdu;
  r.dpdv = dpdv;
  r.u = iu;
  r.v = iv;
  r.t = h.t;
  /* fillShadingStructure + constructTbnFrame, embree.cpp:360-390 */
  V3 nn = blerp(attr3<0>(m.n, id, 0), attr3<0>(m.n, id, 1), attr3<0>(m.n, id, 2), w, h.u, h.v);
  V3 tt = blerp(attr3<0>(m.t, id, 0), attr3<0>(m.t, id, 1), attr3<0>(m.t, id, 2), w, h.u, h.v);
  V3 bb = blerp(attr3<0>(m.b, id, 0), attr3<0>(m.b, id, 1), attr3<0>(m.b, id, 2), w, h.u, h.v);
  V3 tn = normalize(mul(x.n, nn));
  V3 tt2 = normalize(mul(l, tt));
  V3 tb = normalize(mul(l, bb));
  r.frame = gram_shmidt(tn, tt2, tb);
  return r;
}

/* ------------------------------------------------------------------------------------------------
 * BxDF math (material/BxDF_math.h). Local shading space: z is the normal. */
namespace bx {
static inline float absdot(V3 a, V3 b) { return std::fabs(dot(a, b)); }
static inline bool same_hemi(V3 a, V3 b) { return a.z * b.z > 0; }
static inline bool same_hemi3(V3 wi, V3 wo, V3 wm) { return dot(wi, wm) > 0 && dot(wo, wm) > 0; }
static inline float costheta(V3 v) { return v.z; }
static inline float abscostheta(V3 v) { return std::fabs(v.z); }
static inline float cos2theta(V3 v) { return sqr(v.z); }
static inline float sin2theta(V3 v) { return std::max(0.f, 1.f - cos2theta(v)); }
static inline float sin2theta_c(float c) { return std::max(0.f, 1.f - sqr(c)); }
static inline float sintheta(V3 v) { return msqrt(sin2theta(v)); }
static inline float tan2theta(V3 v) { return sin2theta(v) / cos2theta(v); }
static inline float cosphi(V3 v) {
  if (sintheta(v) == 0.f) return 1.f;
  return std::clamp(v.x / sintheta(v), -1.f, 1.f);
}
static inline float sinphi(V3 v) {
  if (sintheta(v) == 0.f) return 0.f;
  return std::clamp(v.y / sintheta(v), -1.f, 1.f);
}
static inline float cos2phi(V3 v) { return sqr(cosphi(v)); }
static inline float sin2phi(V3 v) { return sqr(sinphi(v)); }

/* refract, BxDF_math.h:105-124 */
static inline float refract(V3 wo, V3 n, float eta, bool &valid, V3 &wt) {
  valid = true;
  float ci = dot(wo, n);
  if (ci < 0) {
    n = -n;
    eta = 1.f / eta;
    ci = -ci;
  }
  float s2i = sin2theta_c(ci);
  float s2t = s2i / sqr(eta);
  if (s2t >= 1.f) {
    valid = false;
    return 0.f;
  }
  float ct = msqrt(1.f - s2t);
  wt = -wo / eta + (ci / eta - ct) * n;
  return eta;
}

/* shirley_chiu + hemisphere_cosine_sample, BxDF_math.h:129-152 */
static inline V3 hemisphere_cosine_sample(const float u[2]) {
  float sx = 2 * u[0] - 1;
  float sy = 2 * u[1] - 1;
  float px = 0.f, py = 0.f;
  if (!(sx == 0 && sy == 0)) {
    float r, theta;
    if (std::fabs(sx) > std::fabs(sy)) {
      r = sx;
      theta = (float)M_PI_4 * (sy / sx);
    } else {
      r = sy;
      theta = (float)M_PI_2 - (float)M_PI_4 * (sx / sy);
    }
    px = r * cos_rn(theta);
    py = r * sin_rn(theta);
  }
  float z = std::sqrt(std::max(0.f, 1 - px * px - py * py));
  return {px, py, z};
}
}  // namespace bx

/* Fresnel (BxDF_math.h:170-224) */
static inline float pow5(float x) { return pow5_rn(x); } /* std::pow(x, 5.f), correctly rounded */
static inline float schlick(float c, float F0) { return F0 + (1.f - F0) * pow5(1.f - c); }
static inline Spec schlick(float c, Spec F0) { return F0 + (1.f - F0) * pow5(1.f - c); }
static inline float fresnel_real(float etar, float ci, float &new_eta) {
  float eta = etar;
  ci = std::clamp(ci, -1.f, 1.f);
  if (ci < 0) {
    eta = 1.f / eta;
    ci = -ci;
  }
  new_eta = eta;
  float s2i = bx::sin2theta_c(ci);
  float s2t = s2i / sqr(eta);
  if (s2t >= 1) return 1.f;
  float ct = msqrt(1.f - s2t);
  float rpar = (eta * ci - ct) / (eta * ci + ct);
  float rperp = (ci - eta * ct) / (ci + eta * ct);
  return (sqr(rpar) + sqr(rperp)) / 2.f;
}

/* VNDF (BxDF_math.h:226-343) */
struct VNDF {
  float ax = 0, ax_inv = 0, ay = 0, ay_inv = 0;
  static float r2a(float r) { return r != 0 ? r * r : 1e-6f; }
  VNDF() = default;
  VNDF(float anisotropy, float roughness) {
    anisotropy = std::clamp(anisotropy, -1.f, 1.f);
    float aspect = msqrt(1.f - 0.9f * anisotropy);
    ax = r2a(roughness) / aspect;
    ay = r2a(roughness) * aspect;
    ax_inv = 1.f / ax;
    ay_inv = 1.f / ay;
  }
  float D(V3 wm) const {
    if (bx::costheta(wm) < 1e-6f) return 0.f;
    float c2 = bx::cos2phi(wm) * sqr(ax_inv);
    float s2 = bx::sin2phi(wm) * sqr(ay_inv);
    float denom = M_PI * ax * ay * sqr(bx::cos2theta(wm)) * sqr(1.f + bx::tan2theta(wm) * (c2 + s2));
    return 1.f / denom;
  }
  float lambda(V3 v) const {
    float t2 = bx::tan2theta(v);
    if (std::isinf(t2) || std::isnan(t2)) return 0;
    float axt = sqr(ax) * bx::cos2phi(v);
    float ayt = sqr(ay) * bx::sin2phi(v);
    float a2 = axt + ayt;
    return (msqrt(1 + a2 * t2) - 1) * 0.5f;
  }
  float G1(V3 v) const {
    v.z = std::max(v.z, 1e-6f);
    return 1.f / (1.f + lambda(v));
  }
  float G(V3 wo, V3 wi) const { return 1.f / (1.f + lambda(wo) + lambda(wi)); }
  float Dv(V3 wo, V3 wm) const { return D(wm) * bx::absdot(wo, wm) * G1(wo) / bx::abscostheta(wo); }
  float pdf(V3 wo, V3 wm) const { return Dv(wo, wm); }
  V3 sample(V3 wo, const float uc[2]) const {
    V3 wh = normalize(V3{wo.x * ax, wo.y * ay, wo.z});
    if (wh.z < 0) wh = -wh;
    V3 t, b;
    if (wh.z < 1.f)
      t = normalize(cross(V3{0, 0, 1}, wh));
    else
      t = {1, 0, 0};
    b = cross(wh, t);
    /* sample_uniform_disk_polar, BxDF_math.h:160-164 */
    float r = msqrt(uc[0]);
    float th = 2.f * M_PI * uc[1];
    float px = r * cos_rn(th), py = r * sin_rn(th);
    float s = 0.5f * (1.f + wh.z);
    py = msqrt(1.f - sqr(px)) * (1.f - s) + s * py; /* math::lerp(x, y, a) = x*(1-a) + a*y */
    V3 nh = px * t + py * b + msqrt(std::fmax(0.f, 1.f - sqr(px) - sqr(py))) * wh;
    return normalize(V3{ax * nh.x, ay * nh.y, std::max(1e-6f, nh.z)});
  }
  bool full_specular() const { return std::max(ax, ay) < 1e-5f; }
};

enum Flags : unsigned {
  F_NONE = 0,
  F_REFL = 1,
  F_TRANS = 2,
  F_DIFFUSE = 4,
  F_GLOSSY = 8,
  F_SPECULAR = 16,
  F_ALL = 31,
};

struct BsdfParams { /* bsdf_params_s, BxDF.h:22-39 */
  V3 ns, ng, dpdu, dpdv;
  float wo_dot_ng = 0, wo_dot_ns = 0, roughness = 0, metal = 0;
  float transmission = 0, anisotropy = 0, subsurface = 1.f, sheen = 0, clearcoat = 0, specular = 1.f;
  bool thin = false;
  Spec eta{0, 0, 0}, k{0, 0, 0}, albedo{0, 0, 0};
};

struct Sample { /* BSDFSample, BxDF_flags.h:26-35 */
  Spec f{0, 0, 0};
  V3 wi{0, 0, 0};
  float pdf = 0, costheta = 0;
  unsigned flags = 0;
  bool pdf_cosine_weighted = false;
};

enum Lobe { L_NONE, L_DIFFUSE, L_SPECULAR, L_DIELECTRIC };

/* PrincipledBSDF (material/BSDF.h:22-162) with the three reachable lobes (BxDF.h:252-608).  The
 * lobe objects keep a pointer to the BSDF's params, so a later configureBSDFParams is visible to
 * them; the lobe weight and probability are captured at construction. */
struct PrincipledBSDF {
  BsdfParams params;
  M3 frame;
  float w_diffuse = 0, w_specular = 0, w_transmission = 0, p_diffuse = 0, p_specular = 0, p_transmission = 0;
  Lobe lobe = L_NONE;
  float lobe_w = 1.f, lobe_p = 1.f;
  VNDF ggx;
  const V3 *force_wm = nullptr; /* evaluate at this microfacet normal instead of sampling one */
  mutable V3 wm_used{0, 0, 1};

  void weights() {
    float ac = std::fabs(params.wo_dot_ng);
    w_diffuse = (1 - params.transmission) * (1 - params.metal);
    float w_sheen = (1 - params.metal) * params.sheen * (1.f - params.transmission);
    float w_clearcoat = 0.25f * params.clearcoat;
    w_specular = params.specular;
    w_transmission = (1.f - params.metal) * params.transmission;
    float F = schlick(ac, params.specular * 0.04f);
    float pd = w_diffuse * (1.f - F);
    float ps = w_specular * F;
    float W = pd + ps + w_sheen + w_clearcoat + w_transmission;
    if (W == 0) {
      W = 1.f;
    }
    p_diffuse = pd / W;
    p_specular = ps / W;
    p_transmission = w_transmission / W;
  }
  void configure(const BsdfParams &p) {
    params = p;
    frame = gram_shmidt(params.ns, params.dpdu, params.dpdv); /* IntersectFrame(dpdu, dpdv, ns, true) */
    if (params.wo_dot_ng < 0) {
      frame.c[0] = -frame.c[0];
      frame.c[1] = -frame.c[1];
      frame.c[2] = -frame.c[2];
      if (!params.thin && spec_all_nonzero(params.eta)) params.eta = 1.f / params.eta;
    }
    params.ng = normalize(mul_t(frame, params.ng));
    weights();
  }
  PrincipledBSDF() = default;
  PrincipledBSDF(const BsdfParams &p, float uc) {
    configure(p);
    float idx = 0.f;
    if (uc < (idx += p_diffuse)) {
      lobe = L_DIFFUSE, lobe_w = w_diffuse, lobe_p = p_diffuse;
    } else if (uc < (idx += p_specular)) {
      lobe = L_SPECULAR, lobe_w = w_specular, lobe_p = p_specular;
      ggx = VNDF(params.anisotropy, params.roughness);
    } else if (uc < (idx += p_transmission)) {
      lobe = L_DIELECTRIC, lobe_w = w_transmission, lobe_p = p_transmission;
      ggx = VNDF(params.anisotropy, params.roughness);
    }
  }
  unsigned flags() const {
    switch (lobe) {
      case L_DIFFUSE: return F_DIFFUSE | F_REFL;
      case L_SPECULAR: return ggx.full_specular() ? (F_SPECULAR | F_REFL) : (F_GLOSSY | F_REFL);
      case L_DIELECTRIC: {
        unsigned f = params.eta.x == 1.f ? F_TRANS : (F_REFL | F_TRANS);
        return f | (ggx.full_specular() ? F_SPECULAR : F_GLOSSY);
      }
      default: return F_NONE;
    }
  }

  /* DisneyDiffuseBxDF::sample_f, BxDF.h:285-324 */
  bool diffuse_sample(V3 wo, const float u[2], Sample &s) const {
    auto fres = [](V3 w, float value) { return 1.f + (value - 1) * pow5(1.f - bx::abscostheta(w)); };
    V3 wi = normalize(bx::hemisphere_cosine_sample(u));
    V3 h = normalize(wi + wo);
    float ci = bx::costheta(wi), co = bx::costheta(wo);
    if (!bx::same_hemi(wo, wi) || ci <= 0.f || co <= 0.f) return false;
    float rough = sqr(params.roughness);
    float fd90 = 0.5f + 2 * rough * sqr(bx::absdot(wi, h));
    Spec fd = params.albedo * (float)M_1_PI * fres(wi, fd90) * fres(wo, fd90);
    float fss90 = rough * sqr(bx::absdot(h, wi));
    Spec fss = 1.25f * params.albedo * (float)M_1_PI *
               (0.5f + fres(wi, fss90) * fres(wo, fss90) * (-0.5f + 1 / (co + ci)));
    Spec f = lobe_w * ((1 - params.subsurface) * fd + params.subsurface * fss);
    s.pdf_cosine_weighted = false;
    s.costheta = ci;
    s.f = f;
    s.pdf = lobe_p * (ci * (float)M_1_PI);
    s.wi = wi;
    s.flags = F_DIFFUSE | F_REFL;
    return true;
  }

  /* SpecularBxDF::sample_f, BxDF.h:367-397 */
  bool specular_sample(V3 wo, const float u[2], Sample &s) const {
    V3 wm = force_wm ? *force_wm : ggx.sample(wo, u);
    wm_used = wm;
    V3 wi = reflect(-wo, wm);
    float co = bx::costheta(wo), ci = bx::costheta(wi);
    if (co <= 0 || ci <= 0) return false;
    float wm_dot_wo = bx::absdot(wm, wo);
    Spec F0base = v3(0.04f);
    Spec a = v3(params.metal);
    Spec F0 = F0base * (v3(1.f) - a) + a * params.albedo; /* math::lerp on Spectrum */
    Spec Fr = schlick(wm_dot_wo, F0);
    Spec f = Fr * ggx.D(wm) * ggx.G(wo, wi) / (4 * co * ci);
    float pdf = ggx.pdf(wo, wm) / (4 * wm_dot_wo);
    s.f = lobe_w * f;
    s.pdf = lobe_p * pdf;
    s.wi = wi;
    s.costheta = ci;
    s.flags = F_GLOSSY | F_REFL;
    s.pdf_cosine_weighted = false;
    return true;
  }

  /* DielectricBxDF::sample_f and helpers, BxDF.h:403-594 (radiance transport, all flags). */
  bool dielectric_sample(V3 wo, float uc, const float u[2], Sample &s) const {
    float eta_computed = 0.f;
    float ior = params.eta.x;
    if (ggx.full_specular() || params.eta.x == 1.f) {
      float R = fresnel_real(ior, bx::costheta(wo), eta_computed), T = 1 - R;
      float pr = R, pt = T;
      if (pr == 0.f && pt == 0.f) return false;
      if (uc < (pr / (pr + pt))) {
        V3 wi = reflect(-wo, V3{0, 0, 1.f});
        float ci = bx::abscostheta(wi);
        s.costheta = ci;
        s.f = lobe_w * params.albedo * R / ci;
        s.pdf = lobe_p * pr / (pr + pt);
        s.flags = F_SPECULAR | F_REFL;
        s.pdf_cosine_weighted = false;
        s.wi = wi;
        return true;
      }
      bool ok = true;
      V3 wi{0, 0, 0};
      bx::refract(wo, V3{0, 0, 1.f}, ior, ok, wi);
      if (!ok) return false;
      float ci = bx::abscostheta(wi);
      Spec f = T * params.albedo / ci;
      f = f / sqr(ior);
      s.f = lobe_w * f;
      s.costheta = ci;
      s.pdf = lobe_p * pt / (pr + pt);
      s.flags = F_SPECULAR | F_TRANS;
      s.pdf_cosine_weighted = false;
      s.wi = wi;
      return true;
    }
    V3 wm = force_wm ? *force_wm : ggx.sample(wo, u);
    wm_used = wm;
    float wo_dot_wm = dot(wo, wm);
    float R = fresnel_real(ior, wo_dot_wm, eta_computed), T = 1 - R;
    float pr = R, pt = T;
    if (pr == 0.f && pt == 0.f) return false;
    if (uc < (pr / (pr + pt))) { /* glossyReflection */
      V3 wi = reflect(-wo, wm);
      if (!bx::same_hemi(wo, wi)) return false;
      Spec f = params.albedo * ggx.D(wm) * ggx.G(wo, wi) * R / (4 * bx::costheta(wi) * bx::costheta(wo));
      float pdf = ggx.pdf(wo, wm) / (4 * bx::absdot(wo, wm)) * pr / (pr + pt);
      s.f = lobe_w * f;
      s.pdf = lobe_p * pdf;
      s.wi = wi;
      s.costheta = bx::abscostheta(wi);
      s.pdf_cosine_weighted = false;
      s.flags = F_GLOSSY | F_REFL;
      return true;
    }
    /* glossyTransmission */
    V3 wi{0, 0, 0};
    bool no_tir = true;
    float eta = bx::refract(wo, wm, ior, no_tir, wi);
    wi = normalize(wi);
    if (bx::same_hemi(wi, wo) || wi.z == 0.f || !no_tir) return false;
    float ci = bx::costheta(wi), co = bx::costheta(wo);
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / eta);
    float jac = bx::absdot(wi, wm) / denom;
    float pdf = ggx.pdf(wo, wm) * jac * pt / (pt + pr);
    Spec f = params.albedo * T * ggx.D(wm) * ggx.G(wo, wi) *
             std::fabs(dot(wi, wm) * dot(wo, wm) / (ci * co * denom));
    f = f / sqr(eta);
    s.f = lobe_w * f;
    s.costheta = bx::abscostheta(wi);
    s.pdf = lobe_p * pdf;
    s.wi = wi;
    s.pdf_cosine_weighted = false;
    s.flags = F_GLOSSY | F_TRANS;
    return true;
  }

  /* PrincipledBSDF::sample_f, BSDF.h:107-130 */
  bool sample_f(V3 wo, float uc, const float u[2], Sample &s) const {
    if (lobe == L_NONE) return false;
    V3 lwo = normalize(mul_t(frame, wo));
    if (!(flags() & F_ALL) || lwo.z == 0.f) return false;
    bool ok = false;
    switch (lobe) {
      case L_DIFFUSE: ok = diffuse_sample(lwo, u, s); break;
      case L_SPECULAR: ok = specular_sample(lwo, u, s); break;
      case L_DIELECTRIC: ok = dielectric_sample(lwo, uc, u, s); break;
      default: break;
    }
    if (!ok) return false;
    if (!spec_nonzero(s.f) || s.pdf == 0.f || s.wi.z == 0.f) return false;
    s.wi = normalize(mul(frame, s.wi));
    return true;
  }
};

/* DielectricBxDF::f (BxDF.h:497-524), radiance transport: the evaluator the reference's unit tests
 * hold the sampler to; the path itself only samples. */
static Spec dielectric_f(const PrincipledBSDF &b, V3 wo, V3 wi) {
  if (b.ggx.full_specular() || b.params.eta.x == 1.f) return v3(0.f);
  const float eta = b.params.eta.x, ci = bx::costheta(wi), co = bx::costheta(wo);
  float new_eta = 0.f;
  Spec f;
  if (bx::same_hemi(wi, wo)) {
    V3 wm = normalize(wi + wo);
    float R = fresnel_real(eta, bx::absdot(wo, wm), new_eta);
    f = b.params.albedo * b.ggx.D(wm) * b.ggx.G(wo, wi) * R / (4 * ci * co);
  } else {
    V3 wm = normalize(wi * eta + wo);
    if (dot(wo, wm) < 0) wm = -wm;
    float T = 1.f - fresnel_real(eta, bx::absdot(wo, wm), new_eta);
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / eta);
    f = b.params.albedo * T * b.ggx.D(wm) * b.ggx.G(wo, wi) * std::fabs(dot(wi, wm) * dot(wo, wm) / (ci * co * denom));
    f = f / sqr(eta);
  }
  return b.lobe_w * f;
}

/* DielectricBxDF::pdf (BxDF.h:526-557), all flags. */
static float dielectric_pdf(const PrincipledBSDF &b, V3 wo, V3 wi) {
  if (b.params.eta.x == 1.f || b.ggx.full_specular()) return 0.f;
  const float eta = b.params.eta.x;
  float new_eta = 0.f;
  if (bx::same_hemi(wi, wo)) {
    V3 wm = normalize(wi + wo);
    float wo_dot_wm = bx::absdot(wo, wm);
    float R = fresnel_real(eta, wo_dot_wm, new_eta), T = 1.f - R;
    return b.lobe_p * (b.ggx.pdf(wo, wm) / (4 * wo_dot_wm) * R / (R + T));
  }
  V3 wm = normalize(wi * eta + wo);
  if (dot(wo, wm) < 0) wm = -wm;
  float R = fresnel_real(eta, bx::absdot(wo, wm), new_eta), T = 1.f - R;
  float denom = sqr(dot(wi, wm) + dot(wo, wm) / eta);
  float jac = bx::absdot(wi, wm) / denom;
  return b.lobe_p * (b.ggx.pdf(wo, wm) * jac * T / (T + R));
}

/* bsdf::correct_specular_shading_normal, BxDF_math.h:26-53 */
static V3 correct_specular_shading_normal(V3 ng, V3 wo, V3 ns) {
  V3 R = reflect(-wo, ns);
  const float woz = dot(wo, ng);
  const float threshold = std::fmin(0.9f * woz, 0.01f);
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

struct Scatter {
  Spec attenuation{0, 0, 0}, emissive{0, 0, 0};
  Sample lobe;
};

static inline float u8f(float v) { return v * (1.f / 255.f); } /* rgb_uint2float, math_texturing.h:8-12 */

/* PrincipledMaterial::scatter + sampleBSDF (NovaMaterials.h:56-137).  Consumes four sampler
 * dimensions: uc, u0[2] (lobe choice and direction), then uc again for sample_f. */
/* Optional inputs of scatter beyond the reference's: parameter values that replace the base
 * albedo / roughness, a microfacet normal to evaluate at instead of sampling, and where to report
 * the microfacet normal used. */
struct ScatterOpts {
  const Spec *albedo = nullptr;
  const float *roughness = nullptr;
  const V3 *force_wm = nullptr;
  V3 *wm_out = nullptr;
};

static bool scatter(const Scene &s, const Ray &in, const HitRecord &hr, const Material &mat, uint32_t index,
                    unsigned &dim, uint32_t seed, Scatter &out, int32_t prim, uint32_t mat_id,
                    const ScatterOpts &so = ScatterOpts{}) {
  float u = hr.u, v = hr.v;
  V3 nmap{0.f, 0.f, 1.f};
  if (mat.normalmap >= 0) {
    V4 t = sample_u8(s.textures[mat.normalmap], u, v);
    nmap = {u8f(t.x), u8f(t.y), u8f(t.z)};
  }
  V3 local_n = nmap * 2.f - 1.f;
  V3 ns = normalize(mul(hr.frame, local_n));
  V3 ng = hr.ng;
  BsdfParams bp;
  bp.dpdu = hr.dpdu;
  bp.dpdv = hr.dpdv;
  bp.ns = ns;
  bp.ng = ng;
  V3 wo = normalize(-in.d);
  bp.wo_dot_ng = dot(wo, ng);
  bp.wo_dot_ns = dot(wo, ns);
  V4 alb{1.f, 1.f, 1.f, 1.f};
  if (mat.albedo >= 0) {
    V4 t = sample_u8(s.textures[mat.albedo], u, v);
    alb = {u8f(t.x), u8f(t.y), u8f(t.z), u8f(t.w)};
  }
  bp.albedo = {alb.x, alb.y, alb.z};
  if (!s.diff_albedo.empty())
    bp.albedo = {s.diff_albedo[3 * prim], s.diff_albedo[3 * prim + 1], s.diff_albedo[3 * prim + 2]};
  if (so.albedo) bp.albedo = *so.albedo;
  V3 met{0.f, 0.f, 0.f};
  if (mat.metallic >= 0) {
    V4 t = sample_u8(s.textures[mat.metallic], u, v);
    met = {u8f(t.x), u8f(t.y), u8f(t.z)};
  }
  bp.roughness = met.y;
  if (!s.diff_rough.empty()) bp.roughness = s.diff_rough[mat_id];
  if (so.roughness) bp.roughness = *so.roughness;
  bp.metal = met.z;
  bp.transmission = (spec_nonzero(mat.eta) && !spec_nonzero(mat.k)) ? 1.f : 0.f;
  bp.anisotropy = mat.anisotropy;
  bp.thin = false;
  bp.eta = mat.eta;
  bp.k = mat.k;

  float uc = sobol_sample(index, dim++, seed);
  float u0[2];
  u0[0] = sobol_sample(index, dim++, seed);
  u0[1] = sobol_sample(index, dim++, seed);
  PrincipledBSDF bsdf(bp, uc);
  bsdf.force_wm = so.force_wm;
  if (bsdf.flags() & (F_GLOSSY | F_REFL)) {
    if (bp.wo_dot_ng >= 0) {
      V3 cns = normalize(correct_specular_shading_normal(bp.ng, wo, bp.ns));
      bp.ns = cns;
      bp.wo_dot_ns = dot(wo, cns);
      bsdf.configure(bp);
    }
  }
  uc = sobol_sample(index, dim++, seed);
  Sample lobe;
  bool valid = bsdf.sample_f(wo, uc, u0, lobe);
  if (so.wm_out) *so.wm_out = bsdf.wm_used;
  out = Scatter{};
  out.attenuation = lobe.f;
  if (mat.emissive >= 0) {
    V4 t = sample_u8(s.textures[mat.emissive], u, v);
    out.emissive = {u8f(t.x), u8f(t.y), u8f(t.z)};
  }
  out.lobe = lobe;
  return valid;
}

/* Ray::spawn, Ray.h:22-27 */
static inline Ray spawn(V3 wi, V3 n, V3 position) {
  const float eps = 1e-3f;
  Ray r;
  r.d = normalize(wi);
  r.o = position + n * (eps + eps * fsign(dot(n, wi)));
  return r;
}

static inline bool finite4(V4 v) {
  return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z) && std::isfinite(v.w);
}

struct PathCtx {
  const Scene *s;
  uint32_t index;
  unsigned dim;
  uint32_t seed;
  int rr_start;
  uint64_t segments, traced;
  TraceCounters tc;
};

/* Russian roulette (an extension; the reference has none): after scattering at bounce b >= rr_start
 * the path survives with q = clamp(max(throughput), 0.05, 1), decided by Sobol dimension 200 + b. */
constexpr unsigned kRRDimBase = 200;

/* PathIntegrator::Li, integrator/Integrator.cpp:60-99 (recursive; DENAN per level; miss or
 * depth < 0 returns the environment without an occlusion test; failed scatter returns black). */
/* The albedo / roughness a vertex shades with (differentiable parameters or textures). */
static Spec vertex_albedo(const Scene &s, const Material &mat, const HitRecord &hr, int32_t prim) {
  if (!s.diff_albedo.empty()) return {s.diff_albedo[3 * prim], s.diff_albedo[3 * prim + 1], s.diff_albedo[3 * prim + 2]};
  if (mat.albedo < 0) return {1.f, 1.f, 1.f};
  V4 t = sample_u8(s.textures[mat.albedo], hr.u, hr.v);
  return {u8f(t.x), u8f(t.y), u8f(t.z)};
}
static float vertex_roughness(const Scene &s, const Material &mat, const HitRecord &hr, uint32_t mat_id) {
  if (!s.diff_rough.empty()) return s.diff_rough[mat_id];
  if (mat.metallic < 0) return 0.f;
  return u8f(sample_u8(s.textures[mat.metallic], hr.u, hr.v).y);
}

/* f of the lobe that `dim0` selects, at the directions of the unperturbed sample (microfacet
 * normal wm), with the given albedo / roughness. */
static Spec perturbed_f(const Scene &s, const Ray &ray, const HitRecord &hr, const Material &mat, uint32_t index,
                        unsigned dim0, uint32_t seed, int32_t prim, uint32_t mat_id, V3 wm, const Spec *albedo,
                        const float *roughness) {
  ScatterOpts so;
  so.albedo = albedo;
  so.roughness = roughness;
  so.force_wm = &wm;
  Scatter sc;
  unsigned dim = dim0;
  if (!scatter(s, ray, hr, mat, index, dim, seed, sc, prim, mat_id, so)) return {0.f, 0.f, 0.f};
  return sc.attenuation;
}

/* Optional per-thread segment log (orc_sample_path): origin, direction, hit prim, t, u, v. */
thread_local std::vector<float> *g_segment_log = nullptr;

static V4 Li(PathCtx &c, const Ray &ray, int depth, int bounce, Spec beta) {
  const Scene &s = *c.s;
  c.segments++;
  c.traced++;
  Hit hit = trace(s, ray, &c.tc);
  if (g_segment_log) {
    int32_t p = hit.is_hit ? hit.prim : -1;
    float pf;
    std::memcpy(&pf, &p, 4);
    const float rec[10] = {ray.o.x, ray.o.y, ray.o.z, ray.d.x, ray.d.y, ray.d.z, pf, hit.t, hit.u, hit.v};
    g_segment_log->insert(g_segment_log->end(), rec, rec + 10);
  }
  if (hit.is_hit && depth >= 0) {
    HitRecord hr = make_record(s, ray, hit);
    const uint32_t mat_id = s.inst_mat[s.prims[hit.prim].inst];
    const Material &mat = s.materials[mat_id];
    Scatter sc;
    const unsigned dim0 = c.dim;
    V3 wm{0, 0, 1};
    ScatterOpts so;
    so.wm_out = &wm;
    if (!scatter(s, ray, hr, mat, c.index, c.dim, c.seed, sc, hit.prim, mat_id, so)) return {0, 0, 0, 0};
    if ((s.pert_kind == 1 && s.pert_index == (uint32_t)hit.prim) || (s.pert_kind == 2 && s.pert_index == mat_id)) {
      Spec a = vertex_albedo(s, mat, hr, hit.prim);
      float r = vertex_roughness(s, mat, hr, mat_id);
      if (s.pert_kind == 1)
        (s.pert_channel == 0 ? a.x : s.pert_channel == 1 ? a.y : a.z) += s.pert_delta;
      else
        r += s.pert_delta;
      sc.attenuation = perturbed_f(s, ray, hr, mat, c.index, dim0, c.seed, hit.prim, mat_id, wm, &a, &r);
    }
    Ray out = spawn(sc.lobe.wi, hr.ng, hr.position);
    Spec color = sc.attenuation * sc.lobe.costheta / sc.lobe.pdf;
    if (c.rr_start >= 0 && bounce >= c.rr_start) {
      Spec nb = beta * color;
      float q = std::min(1.f, std::max(0.05f, std::max(nb.x, std::max(nb.y, nb.z))));
      float urr = sobol_sample(c.index, kRRDimBase + (unsigned)bounce, c.seed);
      if (!(urr < q)) {
        V4 e{sc.emissive.x, sc.emissive.y, sc.emissive.z, 1.f};
        return finite4(e) ? e : V4{0, 0, 0, 0};
      }
      color = color / q;
    }
    V4 next = Li(c, out, depth - 1, bounce + 1, beta * color);
    V4 e{sc.emissive.x, sc.emissive.y, sc.emissive.z, 1.f};
    V4 cc{color.x, color.y, color.z, 1.f};
    V4 fin = e + cc * next;
    return finite4(fin) ? fin : V4{0, 0, 0, 0};
  }
  return env_sample(s, ray.d);
}

/* screen2ndc + ray_inv_mat, math_camera.h:28-58 */
static Ray camera_ray(const Scene &s, int x, int y_screen, int W, int H, float dx, float dy) {
  const float ndc_x = (float)(2 * x - W) / (float)W;
  const float ndc_y = (float)(H - 2 * y_screen) / (float)H;
  float nx = ndc_x + dx, ny = ndc_y + dy;
  V4 o = mul(s.inv_P, V4{nx, ny, -1.f, 1.f});
  o = o / o.w;
  o = mul(s.inv_V, V4{o.x, o.y, o.z, 1.f});
  V4 d = mul(s.inv_P, V4{nx, ny, -1.f, 0.f});
  d = normalize(mul(s.inv_V, V4{d.x, d.y, -1.f, 0.f}));
  Ray r;
  r.o = {o.x, o.y, o.z};
  r.d = {d.x, d.y, d.z};
  return r;
}

static inline uint32_t sample_index(const orc_options &opt, int x, int y, int s) {
  if (opt.index_mode == 1) { /* Integrator.h:80: idx * frame_index + renderer_max_samples (0) */
    int row = opt.vertical_invert ? (opt.height - 1 - y) : y; /* generateImageOffset, Integrator.h:38-42 */
    unsigned idx = (unsigned)((row * opt.width + x) * 4);
    return idx * (unsigned)s;
  }
  return ((uint32_t)x * (uint32_t)opt.height + (uint32_t)y) * (uint32_t)opt.spp + (uint32_t)s;
}

/* One sample of pixel (x, y): AbstractIntegrator::render body (Integrator.h:66-92). */
static V4 render_sample(PathCtx &c, const orc_options &opt, int x, int y, int s) {
  constexpr float RAND_DX = 0.0005f, RAND_DY = 0.0005f;
  c.index = sample_index(opt, x, y, s);
  c.dim = 0;
  float r0 = sobol_sample(c.index, c.dim++, c.seed);
  float r1 = sobol_sample(c.index, c.dim++, c.seed);
  const float dx = r0 * RAND_DX, dy = r1 * RAND_DY;
  Ray r = camera_ray(*c.s, x, opt.height - y, opt.width, opt.height, dx, dy);
  return Li(c, r, opt.max_depth, 0, v3(1.f));
}

}  // namespace orc

using namespace orc;

static orc::Texture texture_from(const orc_texture &t) {
  orc::Texture d;
  d.w = t.width, d.h = t.height, d.channels = t.channels;
  d.is_rgba = t.is_rgba != 0, d.invert_u = t.invert_u != 0, d.invert_v = t.invert_v != 0;
  size_t n = (size_t)t.width * t.height;
  if (t.u8_pixels) d.u8.assign(t.u8_pixels, t.u8_pixels + n);
  if (t.f32_pixels) d.f32.assign(t.f32_pixels, t.f32_pixels + n * t.channels);
  return d;
}

extern "C" void *orc_build(const orc_scene *in) {
  if (!in || in->n_instances == 0 || in->envmap < 0 || (uint32_t)in->envmap >= in->n_textures) return nullptr;
  Scene *s = new Scene();
  s->meshes.resize(in->n_meshes);
  for (uint32_t i = 0; i < in->n_meshes; i++) {
    const orc_mesh &m = in->meshes[i];
    Mesh &d = s->meshes[i];
    if (!m.vertices || !m.normals || !m.tangents || !m.bitangents || !m.uv || !m.indices) {
      delete s;
      return nullptr;
    }
    d.v.assign(m.vertices, m.vertices + 3 * (size_t)m.n_verts);
    d.n.assign(m.normals, m.normals + 3 * (size_t)m.n_verts);
    d.t.assign(m.tangents, m.tangents + 3 * (size_t)m.n_verts);
    d.b.assign(m.bitangents, m.bitangents + 3 * (size_t)m.n_verts);
    d.uv.assign(m.uv, m.uv + 2 * (size_t)m.n_verts);
    d.idx.assign(m.indices, m.indices + 3 * (size_t)m.n_tris);
    d.n_tris = m.n_tris;
  }
  for (uint32_t i = 0; i < in->n_instances; i++) {
    const orc_instance &x = in->instances[i];
    s->inst_mesh.push_back(x.mesh);
    s->inst_mat.push_back(x.material);
    s->xf.push_back(Xform{m4_from(x.m), m4_from(x.inv), m3_from(x.n)});
    for (uint32_t t = 0; t < s->meshes[x.mesh].n_tris; t++) s->prims.push_back(Prim{i, t});
  }
  for (uint32_t i = 0; i < in->n_materials; i++) {
    const orc_material &m = in->materials[i];
    Material d;
    d.albedo = m.albedo, d.metallic = m.metallic, d.normalmap = m.normalmap, d.emissive = m.emissive;
    d.eta = {m.eta[0], m.eta[1], m.eta[2]};
    d.k = {m.k[0], m.k[1], m.k[2]};
    d.anisotropy = m.anisotropy;
    s->materials.push_back(d);
  }
  for (uint32_t i = 0; i < in->n_textures; i++) {
    s->textures.push_back(texture_from(in->textures[i]));
  }
  s->envmap = in->envmap;
  s->inv_P = m4_from(in->inv_P);
  s->inv_V = m4_from(in->inv_V);
  (void)sobol_table();
  (void)acos_lut();
  build_bvh(*s);
  return s;
}

extern "C" void orc_free(void *h) { delete static_cast<Scene *>(h); }

extern "C" void orc_bvh_info(void *h, int64_t *nodes, int64_t *leaves, int64_t *max_leaf) {
  Scene *s = static_cast<Scene *>(h);
  *nodes = s->nodes_used;
  int64_t l = 0, m = 0;
  for (int32_t i = 0; i < s->nodes_used; i++)
    if (s->nodes[i].count > 0) {
      l++;
      m = std::max<int64_t>(m, s->nodes[i].count);
    }
  *leaves = l;
  *max_leaf = m;
}

extern "C" void orc_trace(void *h, uint64_t n, const float *orig, const float *dir, int32_t *prim, float *t, float *u,
                          float *v, orc_stats *stats) {
  const Scene &s = *static_cast<Scene *>(h);
  TraceCounters tc;
  for (uint64_t i = 0; i < n; i++) {
    Ray r;
    r.o = {orig[3 * i], orig[3 * i + 1], orig[3 * i + 2]};
    r.d = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
    Hit hh = trace(s, r, &tc);
    prim[i] = hh.is_hit ? hh.prim : -1;
    t[i] = hh.t;
    u[i] = hh.u;
    v[i] = hh.v;
  }
  if (stats) {
    stats->traced += n;
    stats->node_visits += tc.nodes;
    stats->tri_tests += tc.tris;
  }
}

extern "C" void orc_camera_rays(void *h, const orc_options *opt, uint64_t n, const int32_t *px, const int32_t *py,
                                const int32_t *ps, float *orig, float *dir) {
  const Scene &s = *static_cast<Scene *>(h);
  for (uint64_t i = 0; i < n; i++) {
    uint32_t index = sample_index(*opt, px[i], py[i], ps[i]);
    float r0 = sobol_sample(index, 0, opt->seed);
    float r1 = sobol_sample(index, 1, opt->seed);
    Ray r = camera_ray(s, px[i], opt->height - py[i], opt->width, opt->height, r0 * 0.0005f, r1 * 0.0005f);
    orig[3 * i] = r.o.x, orig[3 * i + 1] = r.o.y, orig[3 * i + 2] = r.o.z;
    dir[3 * i] = r.d.x, dir[3 * i + 1] = r.d.y, dir[3 * i + 2] = r.d.z;
  }
}

/* The segments of one path (sample s of pixel (x, y)): 10 floats each (origin, direction, hit
 * primitive as int32 bits or -1, t, u, v); returns the number of segments written (<= max_segments). */
extern "C" int32_t orc_sample_path(void *h, const orc_options *opt, int32_t x, int32_t y, int32_t s, float *out,
                                   int32_t max_segments, float *radiance) {
  const Scene &sc = *static_cast<Scene *>(h);
  PathCtx c{&sc, 0, 0, opt->seed, opt->rr_start, 0, 0, {}};
  std::vector<float> log;
  g_segment_log = &log;
  V4 L = render_sample(c, *opt, x, y, s);
  g_segment_log = nullptr;
  if (radiance) radiance[0] = L.x, radiance[1] = L.y, radiance[2] = L.z;
  const int32_t n = std::min<int32_t>(max_segments, (int32_t)(log.size() / 10));
  std::copy(log.begin(), log.begin() + 10 * (size_t)n, out);
  return n;
}

/* One shading event per given hit (the body of Li for one level): make_record + scatter with
 * dimensions 2 + 4 * bounce .. + spawn.  valid: 1 scattered, 0 scatter failed, -1 bad input. */
extern "C" void orc_scatter(void *h, uint64_t n, const float *o, const float *d, const int32_t *prim, const float *t,
                            const float *u, const float *v, const uint32_t *index, const int32_t *bounce,
                            uint32_t seed, float *out_o, float *out_d, float *weight, float *emissive,
                            int32_t *valid) {
  const Scene &s = *static_cast<Scene *>(h);
  for (uint64_t i = 0; i < n; i++) {
    if (prim[i] < 0 || (size_t)prim[i] >= s.prims.size() || bounce[i] < 0) {
      valid[i] = -1;
      continue;
    }
    Ray ray;
    ray.o = {o[3 * i], o[3 * i + 1], o[3 * i + 2]};
    ray.d = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
    Hit hit;
    hit.is_hit = true;
    hit.prim = prim[i];
    hit.t = t[i];
    hit.u = u[i];
    hit.v = v[i];
    HitRecord hr = make_record(s, ray, hit);
    const uint32_t mat_id = s.inst_mat[s.prims[hit.prim].inst];
    const Material &mat = s.materials[mat_id];
    unsigned dim = 2u + 4u * (unsigned)bounce[i];
    Scatter sc;
    const bool ok = scatter(s, ray, hr, mat, index[i], dim, seed, sc, hit.prim, mat_id);
    Ray nx = spawn(sc.lobe.wi, hr.ng, hr.position);
    Spec w = sc.attenuation * sc.lobe.costheta / sc.lobe.pdf;
    const float oo[3] = {nx.o.x, nx.o.y, nx.o.z}, dd[3] = {nx.d.x, nx.d.y, nx.d.z}, ww[3] = {w.x, w.y, w.z},
                ee[3] = {sc.emissive.x, sc.emissive.y, sc.emissive.z};
    for (int k = 0; k < 3; k++) {
      out_o[3 * i + k] = oo[k];
      out_d[3 * i + k] = dd[k];
      weight[3 * i + k] = ww[k];
      emissive[3 * i + k] = ee[k];
    }
    valid[i] = ok ? 1 : 0;
  }
}

/* The hit record scatter() starts from, for the pin of PrincipledMaterial::scatter (tests only). */
extern "C" void orc_hit_record(void *h, uint64_t n, const float *o, const float *d, const int32_t *prim, const float *t,
                               const float *u, const float *v, float *out) {
  const Scene &s = *static_cast<Scene *>(h);
  for (uint64_t i = 0; i < n; i++) {
    float *r = out + 23 * i;
    std::fill(r, r + 23, 0.f);
    if (prim[i] < 0 || (size_t)prim[i] >= s.prims.size()) continue;
    Ray ray;
    ray.o = {o[3 * i], o[3 * i + 1], o[3 * i + 2]};
    ray.d = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
    Hit hit;
    hit.is_hit = true, hit.prim = prim[i], hit.t = t[i], hit.u = u[i], hit.v = v[i];
    const HitRecord hr = make_record(s, ray, hit);
    const V3 vs[4] = {hr.ng, hr.dpdu, hr.dpdv, hr.position};
    for (int k = 0; k < 4; k++) r[3 * k] = vs[k].x, r[3 * k + 1] = vs[k].y, r[3 * k + 2] = vs[k].z;
    r[12] = hr.u, r[13] = hr.v;
    for (int c = 0; c < 3; c++) r[14 + 3 * c] = hr.frame.c[c].x, r[15 + 3 * c] = hr.frame.c[c].y, r[16 + 3 * c] = hr.frame.c[c].z;
  }
}

extern "C" int32_t orc_set_diff_params(void *h, const float *albedo, const float *roughness) {
  Scene &s = *static_cast<Scene *>(h);
  if (albedo)
    s.diff_albedo.assign(albedo, albedo + 3 * s.prims.size());
  else
    s.diff_albedo.clear();
  if (roughness)
    s.diff_rough.assign(roughness, roughness + s.materials.size());
  else
    s.diff_rough.clear();
  return 0;
}

extern "C" int32_t orc_set_perturbation(void *h, int32_t kind, uint32_t index, int32_t channel, float delta) {
  Scene &s = *static_cast<Scene *>(h);
  if (kind < 0 || kind > 2 || channel < 0 || channel > 2) return 1;
  s.pert_kind = kind;
  s.pert_index = index;
  s.pert_channel = channel;
  s.pert_delta = delta;
  return 0;
}

/* Replay adjoint on the CPU, the checker of nova_b200_backward: for every sample, the path's
 * radiance I (primal), then the same path again from its Sobol index; at each vertex the score
 * d ln f / d theta of the sampled lobe comes from central differences of f at the sampled
 * directions (h = 1e-3, the sampling density held fixed), and
 *   grad[theta] += sum_c dI_c R_c score_c,  R = I - emission gathered up to the vertex,
 * dI = d_image / spp.  Gradients are summed in double per thread and added to the outputs. */
extern "C" int32_t orc_backward(void *h, const orc_options *opt, const float *d_image, float *grad_albedo,
                                float *grad_roughness, int32_t threads) {
  return orc_backward_range(h, opt, 0, opt->spp, d_image, grad_albedo, grad_roughness, threads);
}

/* The same over samples [sample_begin, sample_begin + sample_count) of an opt->spp-sample frame:
 * the gradient of the mean over that range (dI = d_image / sample_count), as one rank of a
 * sample-range partition computes it. */
extern "C" int32_t orc_backward_range(void *h, const orc_options *opt, int32_t sample_begin, int32_t sample_count,
                                      const float *d_image, float *grad_albedo, float *grad_roughness,
                                      int32_t threads) {
  const Scene &s = *static_cast<Scene *>(h);
  if (opt->width <= 0 || opt->height <= 0 || opt->spp <= 0 || opt->max_depth < 0 || !d_image) return 1;
  if (sample_begin < 0 || sample_count <= 0 || sample_begin + sample_count > opt->spp) return 1;
  const int W = opt->width, H = opt->height;
  const unsigned nt = threads > 0 ? (unsigned)threads : std::max(1u, std::thread::hardware_concurrency());
  const size_t na = 3 * s.prims.size(), nm = s.materials.size();
  std::vector<std::vector<double>> ga(nt, std::vector<double>(grad_albedo ? na : 0, 0.0));
  std::vector<std::vector<double>> gr(nt, std::vector<double>(grad_roughness ? nm : 0, 0.0));
  std::atomic<int> next_row{0};
  auto work = [&](unsigned wid) {
    PathCtx c{&s, 0, 0, opt->seed, opt->rr_start, 0, 0, {}};
    const float hd = 1e-3f;
    for (int y; (y = next_row.fetch_add(1)) < H;) {
      for (int x = 0; x < W; x++) {
        const size_t row = opt->vertical_invert ? (size_t)(H - 1 - y) : (size_t)y;
        const float *dp = d_image + (row * W + x) * 4;
        const Spec dl{dp[0] / (float)sample_count, dp[1] / (float)sample_count, dp[2] / (float)sample_count};
        for (int smp = sample_begin; smp < sample_begin + sample_count; smp++) {
          const V4 I = render_sample(c, *opt, x, y, smp);
          /* replay */
          constexpr float RAND_DX = 0.0005f, RAND_DY = 0.0005f;
          c.index = sample_index(*opt, x, y, smp);
          c.dim = 0;
          const float r0 = sobol_sample(c.index, c.dim++, c.seed);
          const float r1 = sobol_sample(c.index, c.dim++, c.seed);
          Ray ray = camera_ray(s, x, opt->height - y, W, H, r0 * RAND_DX, r1 * RAND_DY);
          Spec beta = v3(1.f), rem{I.x, I.y, I.z};
          for (int depth = opt->max_depth, bounce = 0;; depth--, bounce++) {
            const Hit hit = trace(s, ray, nullptr);
            if (!hit.is_hit || depth < 0) break;
            const HitRecord hr = make_record(s, ray, hit);
            const uint32_t mat_id = s.inst_mat[s.prims[hit.prim].inst];
            const Material &mat = s.materials[mat_id];
            const unsigned dim0 = c.dim;
            V3 wm{0, 0, 1};
            ScatterOpts so;
            so.wm_out = &wm;
            Scatter sc;
            const bool valid = scatter(s, ray, hr, mat, c.index, c.dim, c.seed, sc, hit.prim, mat_id, so);
            rem = rem - beta * sc.emissive;
            if (!valid) break;
            const Spec f = sc.attenuation;
            const float fv[3] = {f.x, f.y, f.z}, dv[3] = {dl.x * rem.x, dl.y * rem.y, dl.z * rem.z};
            const Spec a0 = vertex_albedo(s, mat, hr, hit.prim);
            const float r0v = vertex_roughness(s, mat, hr, mat_id);
            if (grad_albedo) {
              for (int ch = 0; ch < 3; ch++) {
                if (fv[ch] == 0.f || dv[ch] == 0.f) continue;
                Spec ap = a0, am = a0;
                (ch == 0 ? ap.x : ch == 1 ? ap.y : ap.z) += hd;
                (ch == 0 ? am.x : ch == 1 ? am.y : am.z) -= hd;
                const Spec fp = perturbed_f(s, ray, hr, mat, c.index, dim0, c.seed, hit.prim, mat_id, wm, &ap, &r0v);
                const Spec fm = perturbed_f(s, ray, hr, mat, c.index, dim0, c.seed, hit.prim, mat_id, wm, &am, &r0v);
                const float fpc = ch == 0 ? fp.x : ch == 1 ? fp.y : fp.z, fmc = ch == 0 ? fm.x : ch == 1 ? fm.y : fm.z;
                ga[wid][3 * (size_t)hit.prim + ch] += (double)dv[ch] * ((double)fpc - fmc) / (2.0 * hd * fv[ch]);
              }
            }
            if (grad_roughness && r0v > hd) {
              const float rp = r0v + hd, rm = r0v - hd;
              const Spec fp = perturbed_f(s, ray, hr, mat, c.index, dim0, c.seed, hit.prim, mat_id, wm, &a0, &rp);
              const Spec fm = perturbed_f(s, ray, hr, mat, c.index, dim0, c.seed, hit.prim, mat_id, wm, &a0, &rm);
              const float pv[3] = {fp.x, fp.y, fp.z}, mv[3] = {fm.x, fm.y, fm.z};
              double g = 0.0;
              for (int ch = 0; ch < 3; ch++)
                if (fv[ch] != 0.f) g += (double)dv[ch] * ((double)pv[ch] - mv[ch]) / (2.0 * hd * fv[ch]);
              gr[wid][mat_id] += g;
            }
            Ray out = spawn(sc.lobe.wi, hr.ng, hr.position);
            Spec color = sc.attenuation * sc.lobe.costheta / sc.lobe.pdf;
            if (c.rr_start >= 0 && bounce >= c.rr_start) {
              Spec nb = beta * color;
              float q = std::min(1.f, std::max(0.05f, std::max(nb.x, std::max(nb.y, nb.z))));
              float urr = sobol_sample(c.index, kRRDimBase + (unsigned)bounce, c.seed);
              if (!(urr < q)) break;
              color = color / q;
            }
            beta = beta * color;
            ray = out;
          }
        }
      }
    }
  };
  std::vector<std::thread> pool;
  for (unsigned i = 0; i < nt; i++) pool.emplace_back(work, i);
  for (auto &t : pool) t.join();
  for (unsigned w = 0; w < nt; w++) {
    if (grad_albedo)
      for (size_t k = 0; k < na; k++) grad_albedo[k] += (float)ga[w][k];
    if (grad_roughness)
      for (size_t k = 0; k < nm; k++) grad_roughness[k] += (float)gr[w][k];
  }
  return 0;
}

/* The BxDF math the reference's BxDFTest.cpp exercises (:27-125): Fresnel::real, VNDF::sample
 * (sampleGGXVNDF) and VNDF::G1 of the restatement above, and correct_specular_shading_normal. */
extern "C" float orc_fresnel_real(float ior, float cos_i, float *new_eta) {
  float e = 0.f;
  const float r = fresnel_real(ior, cos_i, e);
  if (new_eta) *new_eta = e;
  return r;
}
extern "C" void orc_vndf_sample(float anisotropy, float roughness, const float wo[3], const float uc[2], float wm[3]) {
  const VNDF g(anisotropy, roughness);
  const V3 m = g.sample(V3{wo[0], wo[1], wo[2]}, uc);
  wm[0] = m.x, wm[1] = m.y, wm[2] = m.z;
}
extern "C" float orc_vndf_g1(float anisotropy, float roughness, const float v[3]) {
  return VNDF(anisotropy, roughness).G1(V3{v[0], v[1], v[2]});
}
extern "C" void orc_correct_specular_normal(const float ng[3], const float wo[3], const float ns[3], float out[3]) {
  const V3 r = correct_specular_shading_normal(V3{ng[0], ng[1], ng[2]}, V3{wo[0], wo[1], wo[2]}, V3{ns[0], ns[1], ns[2]});
  out[0] = r.x, out[1] = r.y, out[2] = r.z;
}

/* EnvmapTexture::sample (env_sample above) of a float texture for n directions: the function the
 * reference's envmap tests exercise (NovaTextureInterfaceTest.cpp:56-133).  out: 4 floats each. */
extern "C" void orc_env_sample(const float *pixels, int32_t w, int32_t h, int32_t channels, uint64_t n,
                               const float *dirs, float *out) {
  Scene s;
  Texture t;
  t.f32.assign(pixels, pixels + (size_t)w * h * channels);
  t.w = w, t.h = h, t.channels = channels;
  s.textures.push_back(std::move(t));
  s.envmap = 0;
  for (uint64_t i = 0; i < n; i++) {
    const V4 r = env_sample(s, V3{dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]});
    out[4 * i] = r.x, out[4 * i + 1] = r.y, out[4 * i + 2] = r.z, out[4 * i + 3] = r.w;
  }
}

/* DielectricBxDF on its own (weight and probability 1, radiance transport, all flags), as the
 * reference's unit tests build it (BxDFTest.cpp:216-270): sample_f at (wo, uc, u), then f and pdf
 * evaluated at the normalised sampled direction.  out = f[3], pdf, wi[3], costheta, f_eval[3],
 * pdf_eval.  Returns 1 when a direction was sampled. */
extern "C" int32_t orc_dielectric_lobe(const float albedo[3], float eta, float roughness, float anisotropy,
                                       const float wo[3], float uc, const float u[2], float out[12]) {
  PrincipledBSDF b;
  b.params.albedo = {albedo[0], albedo[1], albedo[2]};
  b.params.eta = v3(eta);
  b.params.roughness = roughness;
  b.params.anisotropy = anisotropy;
  b.lobe = L_DIELECTRIC;
  b.ggx = VNDF(anisotropy, roughness);
  Sample smp;
  const V3 w{wo[0], wo[1], wo[2]};
  const bool ok = b.dielectric_sample(w, uc, u, smp);
  const V3 wi = ok ? normalize(smp.wi) : smp.wi;
  const Spec fe = ok ? dielectric_f(b, w, wi) : v3(0.f);
  const float vals[12] = {smp.f.x, smp.f.y, smp.f.z, smp.pdf, smp.wi.x, smp.wi.y, smp.wi.z, smp.costheta,
                          fe.x, fe.y, fe.z, ok ? dielectric_pdf(b, w, wi) : 0.f};
  std::copy(vals, vals + 12, out);
  return ok ? 1 : 0;
}

/* ---- pin entry points: the oracle's BSDF, triangle and spawn arithmetic on given inputs, held bit
 * for bit to the reference's own headers compiled in oracle/_ref (tests only). ---- */
static BsdfParams bsdf_params_of(const orc_bsdf_case &c) {
  BsdfParams p;
  p.ns = {c.ns[0], c.ns[1], c.ns[2]};
  p.ng = {c.ng[0], c.ng[1], c.ng[2]};
  p.dpdu = {c.dpdu[0], c.dpdu[1], c.dpdu[2]};
  p.dpdv = {c.dpdv[0], c.dpdv[1], c.dpdv[2]};
  p.wo_dot_ng = c.wo_dot_ng;
  p.roughness = c.roughness;
  p.metal = c.metal;
  p.transmission = c.transmission;
  p.anisotropy = c.anisotropy;
  p.thin = c.thin != 0;
  p.eta = v3(c.eta);
  p.albedo = {c.albedo[0], c.albedo[1], c.albedo[2]};
  return p;
}

static void store_sample(bool ok, const Sample &smp, orc_bsdf_result &r) {
  r.f[0] = smp.f.x, r.f[1] = smp.f.y, r.f[2] = smp.f.z;
  r.wi[0] = smp.wi.x, r.wi[1] = smp.wi.y, r.wi[2] = smp.wi.z;
  r.pdf = smp.pdf, r.costheta = smp.costheta, r.flags = smp.flags, r.valid = ok ? 1 : 0;
}

extern "C" void orc_principled_sample(uint64_t n, const orc_bsdf_case *cases, orc_bsdf_result *out) {
  for (uint64_t i = 0; i < n; i++) {
    const orc_bsdf_case &c = cases[i];
    const PrincipledBSDF b(bsdf_params_of(c), c.uc);
    Sample smp;
    const bool ok = b.sample_f(V3{c.wo[0], c.wo[1], c.wo[2]}, c.uc, c.u, smp);
    store_sample(ok, smp, out[i]);
  }
}

extern "C" void orc_lobe_sample(int32_t lobe, uint64_t n, const orc_bsdf_case *cases, orc_bsdf_result *out) {
  for (uint64_t i = 0; i < n; i++) {
    const orc_bsdf_case &c = cases[i];
    PrincipledBSDF b;
    b.params = bsdf_params_of(c);
    b.lobe_w = c.weight, b.lobe_p = c.probability;
    b.ggx = VNDF(c.anisotropy, c.roughness);
    Sample smp;
    const V3 wo{c.wo[0], c.wo[1], c.wo[2]};
    bool ok = false;
    if (lobe == 1) b.lobe = L_DIFFUSE, ok = b.diffuse_sample(wo, c.u, smp);
    if (lobe == 2) b.lobe = L_SPECULAR, ok = b.specular_sample(wo, c.u, smp);
    if (lobe == 3) b.lobe = L_DIELECTRIC, ok = b.dielectric_sample(wo, c.uc, c.u, smp);
    store_sample(ok, smp, out[i]);
  }
}

extern "C" void orc_dielectric_eval(uint64_t n, const orc_bsdf_case *cases, const float *wi, float *f, float *pdf) {
  for (uint64_t i = 0; i < n; i++) {
    const orc_bsdf_case &c = cases[i];
    PrincipledBSDF b;
    b.params = bsdf_params_of(c);
    b.lobe = L_DIELECTRIC, b.lobe_w = c.weight, b.lobe_p = c.probability;
    b.ggx = VNDF(c.anisotropy, c.roughness);
    const V3 wo{c.wo[0], c.wo[1], c.wo[2]}, w{wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
    const Spec fe = dielectric_f(b, wo, w);
    f[3 * i] = fe.x, f[3 * i + 1] = fe.y, f[3 * i + 2] = fe.z;
    pdf[i] = dielectric_pdf(b, wo, w);
  }
}

extern "C" void orc_triangle_hits(uint64_t n, const float *tri, const float *inv, const float *o, const float *d,
                                  float tmin, float tmax, int32_t *hit, float *t, float *u, float *v) {
  for (uint64_t i = 0; i < n; i++) {
    const float *q = tri + 9 * i;
    const M4 m = m4_from(inv + 16 * i);
    Ray r;
    r.o = {o[3 * i], o[3 * i + 1], o[3 * i + 2]};
    r.d = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
    float tt = 0.f, uu = 0.f, vv = 0.f;
    hit[i] = moller_trumbore(m, V3{q[0], q[1], q[2]}, V3{q[3], q[4], q[5]}, V3{q[6], q[7], q[8]}, r, tmin, tmax, tt, uu,
                             vv)
                 ? 1
                 : 0;
    t[i] = tt, u[i] = uu, v[i] = vv;
  }
}

extern "C" void orc_spawn(uint64_t n, const float *wi, const float *nrm, const float *pos, float *out_o, float *out_d) {
  for (uint64_t i = 0; i < n; i++) {
    const Ray r = spawn(V3{wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]}, V3{nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]},
                        V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]});
    out_o[3 * i] = r.o.x, out_o[3 * i + 1] = r.o.y, out_o[3 * i + 2] = r.o.z;
    out_d[3 * i] = r.d.x, out_d[3 * i + 1] = r.d.y, out_d[3 * i + 2] = r.d.z;
  }
}

extern "C" void orc_gram_shmidt(uint64_t n, const float *nrm, const float *tan, const float *bit, float *out) {
  for (uint64_t i = 0; i < n; i++) {
    const M3 m = gram_shmidt(V3{nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]}, V3{tan[3 * i], tan[3 * i + 1], tan[3 * i + 2]},
                             V3{bit[3 * i], bit[3 * i + 1], bit[3 * i + 2]});
    for (int c = 0; c < 3; c++)
      for (int k = 0; k < 3; k++) out[9 * i + 3 * c + k] = m.c[c][k];
  }
}

extern "C" void orc_make_onb(uint64_t n, const float *nrm, float *out) {
  for (uint64_t i = 0; i < n; i++) {
    V3 b1, b2;
    make_onb(V3{nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]}, b1, b2);
    const float vals[6] = {b1.x, b1.y, b1.z, b2.x, b2.y, b2.z};
    std::copy(vals, vals + 6, out + 6 * i);
  }
}

/* One texture lookup (property tests): an 8-bit texture through the bilinear sample, a float one
 * through the nearest-texel read; out = RGBA (8-bit channels in 0..255). */
extern "C" void orc_texture_lookup(const orc_texture *t, float u, float v, float out[4]) {
  const Texture tx = texture_from(*t);
  const V4 p = t->u8_pixels ? sample_u8(tx, u, v) : f32pixel(tx, u, v);
  out[0] = p.x, out[1] = p.y, out[2] = p.z, out[3] = p.w;
}

/* The oracle's restatements of the reference's header-only arithmetic on the texture and
 * environment path, for the pin against those headers compiled as they are (oracle/_ref):
 * atan2_approx (math_utils_approx.h:13-40), rgb_uint2float on the bilinear sample's float channels
 * (math_texturing.h:8-12), uvToPixel (math_texturing.h:19-21). */
extern "C" void orc_atan2_approx(uint64_t n, const float *y, const float *x, float *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = atan2_approx(y[i], x[i]);
}
extern "C" void orc_rgb_to_unit(uint64_t n, const float *v, float *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = u8f(v[i]);
}
extern "C" void orc_uv_to_pixel(uint64_t n, const float *t, const uint32_t *dim, uint32_t *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = uv_to_pixel(t[i], dim[i]);
}

/* Triangle::computeAABB / centroid of every primitive (prim_bounds in bvh.cpp): 6 floats of box
 * (min, max) and 3 of centroid per primitive, world space. */
extern "C" void orc_prim_bounds(void *h, float *boxes, float *centroids) {
  const Scene &s = *static_cast<Scene *>(h);
  for (size_t k = 0; k < s.prims.size(); k++) {
    Box b;
    V3 c;
    prim_bounds(s, s.prims[k], b, c);
    float *o = boxes + 6 * k;
    o[0] = b.mn.x, o[1] = b.mn.y, o[2] = b.mn.z, o[3] = b.mx.x, o[4] = b.mx.y, o[5] = b.mx.z;
    centroids[3 * k] = c.x, centroids[3 * k + 1] = c.y, centroids[3 * k + 2] = c.z;
  }
}

/* cartesianToSpherical with the fast approximations (math_spherical.h:44-52): (phi, theta) per
 * direction, the mapping the reference's TextureProcessingTest.cpp:102-110 bounds by 5e-3. */
extern "C" void orc_cartesian_to_spherical(uint64_t n, const float *xyz, float *phi_theta) {
  for (uint64_t i = 0; i < n; i++) {
    phi_theta[2 * i] = atan2_approx(xyz[3 * i + 1], xyz[3 * i]);
    phi_theta[2 * i + 1] = acos_lt(xyz[3 * i + 2]);
  }
}

/* AOV integrators (NormalIntegrator.cpp, DepthIntegrator.cpp, EmissiveIntegrator.cpp): one
 * unjittered camera ray per pixel; out = W*H*4 floats in film layout. */
extern "C" int32_t orc_render_aov(void *h, const orc_options *opt, int32_t kind, float near_plane, float far_plane,
                                  float *out) {
  const Scene &s = *static_cast<Scene *>(h);
  if (opt->width <= 0 || opt->height <= 0 || (kind != 1 && kind != 2 && kind != 4)) return 1;
  const int W = opt->width, H = opt->height;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      const Ray ray = camera_ray(s, x, H - y, W, H, 0.f, 0.f); /* screen2ndc(x, H - y), no jitter */
      const Hit hit = trace(s, ray, nullptr);
      const size_t row = opt->vertical_invert ? (size_t)(H - 1 - y) : (size_t)y;
      float *o = out + (row * W + x) * 4;
      V4 res{0.f, 0.f, 0.f, 0.f};
      if (kind == 2) {
        if (!hit.is_hit) {
          res = {far_plane, far_plane, far_plane, far_plane};
        } else {
          float depth = 1 - (hit.t - near_plane) / (far_plane - near_plane);
          depth = (2.0f * near_plane * far_plane) / (far_plane + near_plane - depth * (far_plane - near_plane)) * 2.f -
                  1.f; /* normalize_depth, DepthIntegrator.cpp:6 */
          const float v = depth / far_plane;
          res = {v, v, v, v};
        }
      } else if (hit.is_hit) {
        const HitRecord hr = make_record(s, ray, hit);
        const uint32_t mat_id = s.inst_mat[s.prims[hit.prim].inst];
        const Material &mat = s.materials[mat_id];
        if (kind == 1) { /* mat_rec.normal = ns, NovaMaterials.h:103-104,135 */
          V3 nmap{0.f, 0.f, 1.f};
          if (mat.normalmap >= 0) {
            V4 t = sample_u8(s.textures[mat.normalmap], hr.u, hr.v);
            nmap = {u8f(t.x), u8f(t.y), u8f(t.z)};
          }
          const V3 ns = normalize(mul(hr.frame, nmap * 2.f - 1.f));
          res = {ns.x, ns.y, ns.z, 1.f};
        } else { /* sampler.reset(generateImageOffset(...)), dimensions from 0 */
          const uint32_t index = (uint32_t)((row * W + x) * 4);
          unsigned dim = 0;
          Scatter sc;
          if (scatter(s, ray, hr, mat, index, dim, opt->seed, sc, hit.prim, mat_id))
            res = {sc.emissive.x, sc.emissive.y, sc.emissive.z, 1.f};
        }
      }
      o[0] = res.x, o[1] = res.y, o[2] = res.z, o[3] = res.w;
    }
  return 0;
}

extern "C" void orc_sample_radiance(void *h, const orc_options *opt, uint64_t n, const int32_t *px, const int32_t *py,
                                    const int32_t *ps, float *out) {
  PathCtx c{static_cast<Scene *>(h), 0, 0, opt->seed, opt->rr_start, 0, 0, {}};
  for (uint64_t i = 0; i < n; i++) {
    V4 L = render_sample(c, *opt, px[i], py[i], ps[i]);
    out[3 * i] = L.x, out[3 * i + 1] = L.y, out[3 * i + 2] = L.z;
  }
}

static int32_t tile_split(int W, int H, int ntw, int nth, int32_t *rects) {
  const int tw = W / ntw, th = H / nth;
  const int twr = tw + (W % tw), thr = th + (H % th);
  int32_t n = 0;
  for (int j = 0; j < nth; j++)
    for (int i = 0; i < ntw; i++, n++) {
      int32_t *r = rects + 4 * n;
      r[0] = i * tw;
      r[1] = r[0] + ((i == ntw - 1) ? twr : tw);
      r[2] = j * th;
      r[3] = r[2] + ((j == nth - 1) ? thr : th);
    }
  return n;
}

/* divideByTiles (utils/nova_utils.h:34-53): ntw x nth tiles of W / ntw x H / nth pixels, the last
 * column and row taking the remainder; rects gets (x0, x1, y0, y1) per tile, row by row. */
extern "C" int32_t orc_tile_split(int32_t W, int32_t H, int32_t ntw, int32_t nth, int32_t *rects) {
  if (W <= 0 || H <= 0 || ntw <= 0 || nth <= 0 || ntw > W || nth > H) return 0;
  return tile_split(W, H, ntw, nth, rects);
}

/* Progressive render (api/engine.cpp:498-525, utils/DrawEngine.cpp:57-89): each frame renders 1 spp
 * of every tile on a worker pool, the orchestrating thread waits on the frame fence, then folds the
 * partial buffer into the running mean (writeFramebuffer, engine.cpp:351-363). */
extern "C" int32_t orc_render(void *h, const orc_options *opt, float *out_rgba, const int32_t *pixel_ids,
                              int64_t n_pixels, orc_stats *stats) {
  const Scene &s = *static_cast<Scene *>(h);
  if (opt->width <= 0 || opt->height <= 0 || opt->spp <= 0 || opt->max_depth < 0) return 1;
  const int W = opt->width, H = opt->height;
  const int tile = opt->tile > 0 ? opt->tile : 20;
  unsigned nthreads = opt->threads > 0 ? (unsigned)opt->threads : std::max(1u, std::thread::hardware_concurrency());

  /* Work items: tiles of the full frame (the reference's 20 x 20 tiles, DrawEngine.cpp:57-89), or, for
   * a pixel subset, chunks of at most tile*tile pixels, small enough that every worker gets about four
   * per frame: a sparse subset of a small frame must not leave cores idle that a full frame of the
   * reference would keep busy. */
  struct Task {
    int x0, y0, x1, y1;
    int64_t p0, p1;
  };
  std::vector<Task> tasks;
  if (!pixel_ids) {
    const int ntw = std::max(1, W / tile), nth = std::max(1, H / tile);
    std::vector<int32_t> rects((size_t)ntw * nth * 4);
    tile_split(W, H, ntw, nth, rects.data());
    for (size_t k = 0; k < rects.size(); k += 4) {
      Task t{};
      t.x0 = rects[k], t.x1 = rects[k + 1], t.y0 = rects[k + 2], t.y1 = rects[k + 3];
      t.p0 = t.p1 = -1;
      tasks.push_back(t);
    }
  } else {
    const int64_t per_worker = (n_pixels + 4 * (int64_t)nthreads - 1) / (4 * (int64_t)nthreads);
    const int64_t chunk = std::min<int64_t>((int64_t)tile * tile, std::max<int64_t>(16, per_worker));
    for (int64_t p = 0; p < n_pixels; p += chunk) tasks.push_back(Task{0, 0, 0, 0, p, std::min(n_pixels, p + chunk)});
  }

  const size_t npx = (size_t)W * H * 4;
  std::vector<float> partial(npx, 0.f), accum(npx, 0.f);
  std::vector<float> &back = accum;
  (void)back;
  std::vector<uint64_t> seg(nthreads, 0), trc(nthreads, 0), nod(nthreads, 0), tri(nthreads, 0);

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  int frame = -1;
  std::atomic<size_t> next{0};
  size_t done = 0;
  bool quit = false;

  auto write_px = [&](PathCtx &c, int x, int y, int fr) {
    V4 L = render_sample(c, *opt, x, y, fr);
    size_t off = opt->vertical_invert ? ((size_t)(H - 1 - y) * W + x) * 4 : ((size_t)y * W + x) * 4;
    partial[off] = L.x, partial[off + 1] = L.y, partial[off + 2] = L.z, partial[off + 3] = L.w;
  };

  auto worker = [&](unsigned wid) {
    int seen = -1;
    PathCtx c{&s, 0, 0, opt->seed, opt->rr_start, 0, 0, {}};
    for (;;) {
      int fr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return quit || frame != seen; });
        if (quit) break;
        fr = frame;
        seen = fr;
      }
      for (;;) {
        size_t ti = next.fetch_add(1);
        if (ti >= tasks.size()) break;
        const Task &t = tasks[ti];
        if (t.p0 < 0) {
          for (int y = t.y1 - 1; y >= t.y0; y--) /* Integrator.h:66-67 */
            for (int x = t.x0; x < t.x1; x++) write_px(c, x, y, fr);
        } else {
          for (int64_t p = t.p0; p < t.p1; p++) write_px(c, pixel_ids[p] % W, pixel_ids[p] / W, fr);
        }
      }
      {
        /* frame fence: the orchestrating thread resumes once every worker has left the task loop */
        std::lock_guard<std::mutex> lk(mu);
        if (++done == nthreads) cv_done.notify_one();
      }
    }
    seg[wid] = c.segments;
    trc[wid] = c.traced;
    nod[wid] = c.tc.nodes;
    tri[wid] = c.tc.tris;
  };

  std::vector<std::thread> pool;
  for (unsigned i = 0; i < nthreads; i++) pool.emplace_back(worker, i);
  auto t0 = std::chrono::steady_clock::now();
  for (int fr = 0; fr < opt->spp; fr++) {
    {
      std::lock_guard<std::mutex> lk(mu);
      next = 0;
      done = 0;
      frame = fr;
    }
    cv_work.notify_all();
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_done.wait(lk, [&] { return done == nthreads; });
    }
    const float denom = float(fr + 1);
    if (!pixel_ids) {
      for (size_t i = 0; i < npx; i++) {
        accum[i] += partial[i];
        out_rgba[i] = accum[i] / denom;
      }
    } else {
      for (int64_t p = 0; p < n_pixels; p++) {
        int x = pixel_ids[p] % W, y = pixel_ids[p] / W;
        size_t off = opt->vertical_invert ? ((size_t)(H - 1 - y) * W + x) * 4 : ((size_t)y * W + x) * 4;
        for (int k = 0; k < 4; k++) {
          accum[off + k] += partial[off + k];
          out_rgba[off + k] = accum[off + k] / denom;
        }
      }
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(mu);
    quit = true;
  }
  cv_work.notify_all();
  for (auto &t : pool) t.join();
  if (stats) {
    for (unsigned i = 0; i < nthreads; i++) {
      stats->segments += seg[i];
      stats->traced += trc[i];
      stats->node_visits += nod[i];
      stats->tri_tests += tri[i];
    }
    stats->seconds += std::chrono::duration<double>(t1 - t0).count();
  }
  return 0;
}
