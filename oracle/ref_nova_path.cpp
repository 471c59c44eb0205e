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
 * Those headers need glm, an empty submodule in the reference tree; oracle/glm_shim stands in for
 * it with glm's evaluation order.  The float transcendentals they call come from ref_libm.cpp
 * (correctly rounded, the oracle's and the device's convention).  The entry points below take the
 * same inputs as the oracle's orc_* pin functions, and tests/test_oracle_ref_pin.py compares the two
 * bit for bit.  No reference code is copied: it is compiled where it lies. */
#include <cstdint>
#include <cstring>
#include <vector>

#include <internal/common/math/utils_3D.h>
#include <internal/geometry/BoundingBox.h>
#include <internal/geometry/Object3D.h>
#include <material/BSDF.h>
#include <material/BxDF.h>
#include <material/BxDF_math.h>
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
