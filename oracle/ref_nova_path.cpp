/* ORACLE PIN — test infrastructure only; never linked into the product.
 *
 * The reference's own code on the Nova path past the sampler, compiled unchanged where it lies:
 *   nova/material/BSDF.h        PrincipledBSDF (lobe weights, lobe choice, frame, sample_f)
 *   nova/material/BxDF.h        DisneyDiffuseBxDF, SpecularBxDF, DielectricBxDF
 *   nova/material/BxDF_math.h   VNDF, Fresnel, correct_specular_shading_normal
 *   nova/shape/Triangle.h       Triangle::hit (Moller-Trumbore in object space)
 *   nova/ray/Ray.h              Ray::spawn
 *   internal/common/math/utils_3D.h   gram_shmidt, make_onb
 *   internal/geometry/BoundingBox.cpp BoundingBox::intersect (the traversal's slab test)
 *   internal/common/math/math_random.h SobolGenerator (gray code, Owen scramble, direction vectors
 *                               from the header the reference's own generator script writes)
 *   nova/texturing/NovaTextureInterface.h + TextureContext.h  EnvmapTexture::sample (spherical map,
 *                               acos table of math_acos_lt.cpp, nearest texel) and ImageTexture<u32>
 *   nova/material/NovaMaterials.h  PrincipledMaterial::scatter (texture pack, normal map, channel
 *                               mapping, specular-normal correction, sampler dimensions), with
 *                               nova/sampler/Sampler.h's SobolSampler
 * Those headers need glm, an empty submodule in the reference tree; oracle/glm_shim stands in for
 * it with glm's evaluation order.  The float transcendentals they call come from ref_libm.cpp
 * (correctly rounded, the oracle's and the device's convention).  The entry points below take the
 * same inputs as the oracle's orc_* pin functions, and tests/test_oracle_ref_pin_path.py compares the two
 * bit for bit.  No reference code is copied: it is compiled where it lies. */
#include <cstdint>
#include <cstring>
#include <vector>

#include <internal/common/math/utils_3D.h>
#include <internal/geometry/BoundingBox.h>
#include <internal/geometry/Object3D.h>
#include <internal/common/math/math_random.h>
#include <material/BSDF.h>
#include <material/BxDF.h>
#include <material/BxDF_math.h>
#include <material/NovaMaterials.h>
#include <sampler/Sampler.h>
#include <texturing/NovaTextureInterface.h>
#include <texturing/TextureContext.h>
#include <ray/Ray.h>
#include <shape/MeshContext.h>
#include <shape/Triangle.h>

#include "oracle.h"

namespace {

glm::vec3 v3(const float *p) { return glm::vec3(p[0], p[1], p[2]); }

void put3(float *out, const glm::vec3 &v) { out[0] = v.x, out[1] = v.y, out[2] = v.z; }

nova::bsdf_params_s params_of(const orc_bsdf_case &c) {
  nova::bsdf_params_s p{};
  p.ns = v3(c.ns);
  p.ng = v3(c.ng);
  p.dpdu = v3(c.dpdu);
  p.dpdv = v3(c.dpdv);
  p.wo_dot_ng = c.wo_dot_ng;
  p.roughness = c.roughness;
  p.metal = c.metal;
  p.transmission = c.transmission;
  p.anisotropy_ratio = c.anisotropy;
  p.thin_surface = c.thin != 0;
  p.eta = nova::Spectrum(c.eta);
  p.k = nova::Spectrum(0.f);
  p.albedo = nova::Spectrum(c.albedo);
  return p;
}

void store(bool ok, const nova::BSDFSample &s, orc_bsdf_result &r) {
  for (int k = 0; k < 3; k++) r.f[k] = s.f[k];
  put3(r.wi, s.wi);
  r.pdf = s.pdf, r.costheta = s.costheta, r.flags = (uint32_t)s.flags, r.valid = ok ? 1 : 0;
}

}  // namespace

/* PrincipledBSDF(params, uc, allocator).sample_f(wo, uc, u, &sample), BSDF.h:87-130. */
extern "C" void ref_principled_sample(uint64_t n, const orc_bsdf_case *cases, orc_bsdf_result *out) {
  StackAllocator allocator;
  for (uint64_t i = 0; i < n; i++) {
    const orc_bsdf_case &c = cases[i];
    allocator.reset();
    const nova::PrincipledBSDF bsdf(params_of(c), c.uc, allocator);
    nova::BSDFSample s{};
    const bool ok = bsdf.sample_f(v3(c.wo), c.uc, c.u, &s);
    store(ok, s, out[i]);
  }
}

/* One lobe's sample_f in the local frame (lobe 1 Disney diffuse, 2 GGX specular, 3 dielectric). */
extern "C" void ref_lobe_sample(int32_t lobe, uint64_t n, const orc_bsdf_case *cases, orc_bsdf_result *out) {
  for (uint64_t i = 0; i < n; i++) {
    const orc_bsdf_case &c = cases[i];
    const nova::bsdf_params_s p = params_of(c);
    nova::BSDFSample s{};
    bool ok = false;
    if (lobe == 1) ok = nova::DisneyDiffuseBxDF(p, c.weight, c.probability).sample_f(v3(c.wo), c.uc, c.u, &s);
    if (lobe == 2) ok = nova::SpecularBxDF(p, c.weight, c.probability).sample_f(v3(c.wo), c.uc, c.u, &s);
    if (lobe == 3) ok = nova::DielectricBxDF(p, c.weight, c.probability).sample_f(v3(c.wo), c.uc, c.u, &s);
    store(ok, s, out[i]);
  }
}

/* DielectricBxDF::f and ::pdf at wi (radiance transport, all flags), BxDF.h:497-545. */
extern "C" void ref_dielectric_eval(uint64_t n, const orc_bsdf_case *cases, const float *wi, float *f, float *pdf) {
  for (uint64_t i = 0; i < n; i++) {
    const orc_bsdf_case &c = cases[i];
    const nova::bsdf_params_s p = params_of(c);
    const nova::DielectricBxDF lobe(p, c.weight, c.probability);
    const nova::Spectrum fe = lobe.f(v3(c.wo), v3(wi + 3 * i));
    for (int k = 0; k < 3; k++) f[3 * i + k] = fe[k];
    pdf[i] = lobe.pdf(v3(c.wo), v3(wi + 3 * i));
  }
}

/* Triangle::hit (Triangle.h:146-213) on a one-triangle mesh with its own transform record
 * (shape_datastructures.h:41-62: m, inv, t, n; only inv and m are read by hit); uvs (0,0), (1,0),
 * (0,1) so the interpolated uv the hit stores equals its barycentrics. */
extern "C" void ref_triangle_hits(uint64_t n, const float *tri, const float *inv, const float *o, const float *d,
                                  float tmin, float tmax, int32_t *hit, float *t, float *u, float *v) {
  std::vector<float> verts(9), normals = {0, 0, 1, 0, 0, 1, 0, 0, 1}, tangents = {1, 0, 0, 1, 0, 0, 1, 0, 0},
                               bitangents = {0, 1, 0, 0, 1, 0, 0, 1, 0}, uvs = {0, 0, 1, 0, 0, 1};
  std::vector<unsigned> indices = {0, 1, 2};
  Object3D mesh;
  mesh.vertices = axstd::span<float>(verts.data(), verts.size());
  mesh.normals = axstd::span<float>(normals.data(), normals.size());
  mesh.tangents = axstd::span<float>(tangents.data(), tangents.size());
  mesh.bitangents = axstd::span<float>(bitangents.data(), bitangents.size());
  mesh.uv = axstd::span<float>(uvs.data(), uvs.size());
  mesh.indices = axstd::span<unsigned>(indices.data(), indices.size());
  std::vector<Object3D> meshes = {mesh};
  std::vector<float> record(transform4x4_t::padding(), 0.f);
  std::vector<uint64_t> offsets = {0};
  nova::shape::transform::mesh_transform_views_t tv;
  tv.matrix_components_view = axstd::span<const float>(record.data(), record.size());
  tv.mesh_offsets_to_matrix = axstd::span<const uint64_t>(offsets.data(), offsets.size());
  nova::shape::triangle::mesh_vertex_attrib_views_t gv;
  gv.host_geometry_view = axstd::span<const Object3D>(meshes.data(), meshes.size());
  const nova::shape::MeshCtx ctx{nova::shape::MeshBundleViews(tv, gv)};
  const nova::shape::Triangle triangle(0, 0);
  for (uint64_t i = 0; i < n; i++) {
    std::memcpy(verts.data(), tri + 9 * i, 9 * sizeof(float));
    for (int k = 0; k < 16; k++) {
      record[16 + k] = inv[16 * i + k];
      record[k] = (k % 5 == 0) ? 1.f : 0.f; /* m: identity (position only) */
    }
    for (int k = 0; k < 9; k++) record[48 + k] = (k % 4 == 0) ? 1.f : 0.f;
    nova::intersection_record_s data{};
    const nova::Ray ray(v3(o + 3 * i), v3(d + 3 * i));
    hit[i] = triangle.hit(ray, tmin, tmax, data, ctx) ? 1 : 0;
    t[i] = hit[i] ? data.geometry.t : 0.f;
    u[i] = hit[i] ? data.geometry.u : 0.f;
    v[i] = hit[i] ? data.geometry.v : 0.f;
  }
}

/* BoundingBox::intersect(dir, origin, dist_min), BoundingBox.cpp:150-160. */
extern "C" void ref_box_intersect(uint64_t n, const float *mn, const float *mx, const float *o, const float *d,
                                  const float *dist_min, float *out) {
  for (uint64_t i = 0; i < n; i++) {
    const geometry::BoundingBox box(v3(mn + 3 * i), v3(mx + 3 * i));
    out[i] = box.intersect(v3(d + 3 * i), v3(o + 3 * i), dist_min[i]);
  }
}

/* Ray::spawn(wi, n, position), Ray.h:22-27. */
extern "C" void ref_spawn(uint64_t n, const float *wi, const float *nrm, const float *pos, float *out_o, float *out_d) {
  for (uint64_t i = 0; i < n; i++) {
    const nova::Ray r = nova::Ray::spawn(v3(wi + 3 * i), v3(nrm + 3 * i), v3(pos + 3 * i));
    put3(out_o + 3 * i, r.origin);
    put3(out_d + 3 * i, r.direction);
  }
}

/* math::gram_shmidt(normal, tangent, bitangent) -> (T, B, N) columns, utils_3D.h:63-70. */
extern "C" void ref_gram_shmidt(uint64_t n, const float *nrm, const float *tan, const float *bit, float *out) {
  for (uint64_t i = 0; i < n; i++) {
    const glm::mat3 m = math::gram_shmidt(v3(nrm + 3 * i), v3(tan + 3 * i), v3(bit + 3 * i));
    for (int c = 0; c < 3; c++) put3(out + 9 * i + 3 * c, m[c]);
  }
}

/* math::make_onb(n, b1, b2), utils_3D.h:74-81. */
extern "C" void ref_make_onb(uint64_t n, const float *nrm, float *out) {
  for (uint64_t i = 0; i < n; i++) {
    glm::vec3 b1, b2;
    math::make_onb(v3(nrm + 3 * i), b1, b2);
    put3(out + 6 * i, b1);
    put3(out + 6 * i + 3, b2);
  }
}

/* Fresnel(eta).real(cos, new_eta), BxDF_math.h:191-207. */
extern "C" float ref_fresnel_real(float ior, float cos_i, float *new_eta) {
  float e = 0.f;
  const float r = Fresnel(ior).real(cos_i, e);
  if (new_eta) *new_eta = e;
  return r;
}

/* VNDF(anisotropy, roughness): sampleGGXVNDF, G1, D, pdf (BxDF_math.h:226-343). out per case:
 * wm[3], G1(v), D(wm), pdf(wo, wm). */
extern "C" void ref_vndf(uint64_t n, const float *aniso, const float *rough, const float *wo, const float *uc,
                         const float *v, float *out) {
  for (uint64_t i = 0; i < n; i++) {
    const VNDF g(aniso[i], rough[i]);
    const glm::vec3 wm = g.sampleGGXVNDF(v3(wo + 3 * i), uc + 2 * i);
    put3(out + 6 * i, wm);
    out[6 * i + 3] = g.G1(v3(v + 3 * i));
    out[6 * i + 4] = g.D(wm);
    out[6 * i + 5] = g.pdf(v3(wo + 3 * i), wm);
  }
}

/* bsdf::correct_specular_shading_normal(ng, wo, ns), BxDF_math.h:26-53. */
extern "C" void ref_correct_specular_normal(uint64_t n, const float *ng, const float *wo, const float *ns, float *out) {
  for (uint64_t i = 0; i < n; i++)
    put3(out + 3 * i, bsdf::correct_specular_shading_normal(v3(ng + 3 * i), v3(wo + 3 * i), v3(ns + 3 * i)));
}

/* SobolGenerator(seed).generate(index, dim), math_random.h:73-98. */
extern "C" void ref_sobol(uint64_t n, const uint32_t *index, const uint32_t *dim, uint32_t seed, float *out) {
  const math::random::SobolGenerator gen(seed);
  for (uint64_t i = 0; i < n; i++) out[i] = gen.generate(index[i], dim[i]);
}

namespace {

/* The scene's textures as the reference's texture context sees them: one 8-bit and one float slot per
 * texture index (the unused one left empty), the CPU fetch path (no interop). */
struct TextureSet {
  std::vector<U32Texture> u32;
  std::vector<F32Texture> f32;
  nova::texturing::TextureCtx ctx;
  explicit TextureSet(const orc_texture *tex, uint32_t n) : u32(n), f32(n), ctx(make(tex, n)) {}

  nova::texturing::TextureBundleViews make(const orc_texture *tex, uint32_t n) {
    for (uint32_t k = 0; k < n; k++) {
      const orc_texture &t = tex[k];
      const size_t texels = (size_t)t.width * t.height;
      U32Texture &a = u32[k];
      F32Texture &b = f32[k];
      a.width = b.width = (uint32_t)t.width;
      a.height = b.height = (uint32_t)t.height;
      a.channels = b.channels = (uint32_t)t.channels;
      a.is_rgba = b.is_rgba = t.is_rgba != 0;
      a.invert_u = b.invert_u = t.invert_u != 0;
      a.invert_v = b.invert_v = t.invert_v != 0;
      if (t.u8_pixels) a.raw_data = axstd::span<const uint32_t>(t.u8_pixels, texels);
      if (t.f32_pixels) b.raw_data = axstd::span<const float>(t.f32_pixels, texels * t.channels);
    }
    nova::texturing::u32tex_shared_views_s uv{};
    uv.managed_tex_view = CstU32ImgTexView(u32.data(), u32.size());
    nova::texturing::f32tex_shared_views_s fv{};
    fv.managed_tex_view = CstF32ImgTexView(f32.data(), f32.size());
    return nova::texturing::TextureBundleViews(uv, fv);
  }
};

}  // namespace

/* EnvmapTexture(envmap).sample for n directions (NovaTextureInterface.h:152-174): 4 floats each. */
extern "C" void ref_env_sample(const orc_texture *tex, uint32_t n_tex, int32_t envmap, uint64_t n, const float *dirs,
                               float *out) {
  const TextureSet set(tex, n_tex);
  const nova::texturing::EnvmapTexture env((std::size_t)envmap);
  nova::texturing::texture_data_aggregate_s data{};
  data.texture_ctx = &set.ctx;
  for (uint64_t i = 0; i < n; i++) {
    data.geometric_data.sampling_vector = v3(dirs + 3 * i);
    const glm::vec4 p = env.sample(0.f, 0.f, data);
    for (int k = 0; k < 4; k++) out[4 * i + k] = p[k];
  }
}

/* PrincipledMaterial::scatter (NovaMaterials.h:89-137) from a hit record (23 floats, as
 * orc_hit_record writes it) and the incoming direction, with a SobolSampler at (index, 2 + 4 * bounce)
 * (the integrator's dimension schedule), then Ray::spawn and the integrator's path weight
 * f * costheta / pdf (Integrator.cpp:80-87).  Outputs as orc_scatter. */
extern "C" void ref_material_scatter(uint64_t n, const float *records, const float *dirs, const uint32_t *material,
                                     const orc_material *mats, uint32_t n_mats, const orc_texture *tex, uint32_t n_tex,
                                     const uint32_t *index, const int32_t *bounce, uint32_t seed, float *out_o,
                                     float *out_d, float *weight, float *emissive, int32_t *valid) {
  const TextureSet set(tex, n_tex);
  std::vector<nova::texturing::ImageTexture<uint32_t>> images(n_tex);
  for (uint32_t k = 0; k < n_tex; k++) images[k] = nova::texturing::ImageTexture<uint32_t>(k);
  auto handle = [&](int32_t k) {
    return k >= 0 ? nova::texturing::NovaTextureInterface(&images[k]) : nova::texturing::NovaTextureInterface();
  };
  std::vector<nova::material::PrincipledMaterial> materials;
  for (uint32_t m = 0; m < n_mats; m++) {
    nova::material::texture_pack pack{};
    pack.albedo = handle(mats[m].albedo);
    pack.metallic = handle(mats[m].metallic);
    pack.normalmap = handle(mats[m].normalmap);
    pack.emissive = handle(mats[m].emissive);
    float eta[3] = {mats[m].eta[0], mats[m].eta[1], mats[m].eta[2]}, k[3] = {mats[m].k[0], mats[m].k[1], mats[m].k[2]};
    materials.emplace_back(pack, eta, k, mats[m].anisotropy);
  }
  nova::texturing::texture_data_aggregate_s aggregate{};
  aggregate.texture_ctx = &set.ctx;
  nova::material::shading_data_s shading{};
  shading.texture_aggregate = &aggregate;
  StackAllocator allocator;
  for (uint64_t i = 0; i < n; i++) {
    const float *r = records + 23 * i;
    nova::intersection_record_s hit{};
    hit.geometry.ng = v3(r);
    hit.geometry.dpdu = v3(r + 3);
    hit.geometry.dpdv = v3(r + 6);
    hit.geometry.position = v3(r + 9);
    hit.geometry.u = r[12], hit.geometry.v = r[13];
    hit.shading.frame = IntersectFrame(glm::mat3(v3(r + 14), v3(r + 17), v3(r + 20)));
    nova::sampler::SobolSampler<math::random::SobolGenerator> sobol{math::random::SobolGenerator(seed)};
    nova::sampler::SamplerInterface sampler(&sobol);
    sampler.reset(index[i]);
    for (int k = 0; k < 2 + 4 * bounce[i]; k++) sampler.next1D();
    const nova::Ray in(glm::vec3(0.f), v3(dirs + 3 * i));
    material_record_s rec{};
    allocator.reset();
    const bool ok = materials[material[i]].scatter(in, hit, rec, sampler, allocator, shading);
    const nova::Ray next = nova::Ray::spawn(rec.lobe.wi, hit.geometry.ng, hit.geometry.position);
    const nova::Spectrum w = rec.lobe.pdf_cosine_weighted ? rec.attenuation / rec.lobe.pdf
                                                          : rec.attenuation * rec.lobe.costheta / rec.lobe.pdf;
    put3(out_o + 3 * i, next.origin);
    put3(out_d + 3 * i, next.direction);
    for (int k = 0; k < 3; k++) weight[3 * i + k] = w[k], emissive[3 * i + k] = rec.emissive[k];
    valid[i] = ok ? 1 : 0;
  }
}
