/* ORACLE — test infrastructure only.  A CPU restatement of the reference's Nova path-tracing hot
 * path (HamilcarR/Axomae, corelib/nova), used as the parity checker for the CUDA path and as the
 * timed CPU baseline.  Nothing in the product links or loads this library; only tests/, the smoke
 * check and bench.py's CPU-baseline leg do.
 *
 * Parity status: the Sobol direction vectors, the Sobol/Owen sample values and the acos lookup
 * table are pinned against fixtures produced by the reference's own generator scripts
 * (tests/golden/).  The few header-only reference functions that compile without glm (the fast
 * atan2, the texel conversions, the tile split) are compiled from the reference tree by
 * ref_pieces.cpp and the restatements below equal them bit for bit.  Everything else downstream
 * (camera, BVH, triangle test, hit record, BSDFs, envmap, integrator) is a restatement of the
 * reference sources cited per function; the reference itself cannot be built here (glm/boost/Embree
 * are empty submodules), so those parts are pinned only by the reference's own property tests and
 * are otherwise "parity unpinned".
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One triangle mesh in object space (reference Object3D spans, corelib/internal/geometry/Object3D.h:384-394).
 * All attribute arrays are required: positions/normals/tangents/bitangents 3 floats per vertex, uv 2. */
typedef struct {
  const float *vertices;
  const float *normals;
  const float *tangents;
  const float *bitangents;
  const float *uv;
  const uint32_t *indices; /* 3 per triangle */
  uint32_t n_verts;
  uint32_t n_tris;
} orc_mesh;

/* One placed mesh: the reference's per-mesh transform record transform4x4_t {m, inv, t, n}
 * (corelib/internal/common/math/utils_3D.h:84-96), column-major, and its material. */
typedef struct {
  uint32_t mesh;
  uint32_t material;
  float m[16];
  float inv[16];
  float n[9];
} orc_instance;

/* PrincipledMaterial inputs (corelib/nova/material/NovaMaterials.h:45-137, api/material.cpp:212-226):
 * u8 texture indices (-1 = absent) and the refractive indices eta, k. */
typedef struct {
  int32_t albedo;
  int32_t metallic; /* roughness = .g, metal = .b (NovaMaterials.h:116-117) */
  int32_t normalmap;
  int32_t emissive;
  float eta[3];
  float k[3];
  float anisotropy;
} orc_material;

/* A texture: exactly one of u8_pixels (packed 8-bit RGBA or BGRA words) / f32_pixels is set. */
typedef struct {
  const uint32_t *u8_pixels;
  const float *f32_pixels;
  int32_t width, height, channels;
  int32_t is_rgba, invert_u, invert_v;
} orc_texture;

typedef struct {
  const orc_mesh *meshes;
  uint32_t n_meshes;
  const orc_instance *instances;
  uint32_t n_instances;
  const orc_material *materials;
  uint32_t n_materials;
  const orc_texture *textures;
  uint32_t n_textures;
  int32_t envmap; /* index of a 4-channel f32 texture */
  float inv_P[16];
  float inv_V[16];
} orc_scene;

typedef struct {
  int32_t width, height, spp, max_depth;
  uint32_t seed;       /* Sobol/Owen seed */
  int32_t index_mode;  /* 0: (x*H+y)*spp+s (integrator_optix.cu:43); 1: 4*pixel*frame (Integrator.h:80) */
  int32_t rr_start;    /* Russian roulette from this bounce; -1 = off (the reference has none) */
  int32_t threads;     /* tile workers; 0 = hardware concurrency */
  int32_t tile;        /* tile edge in pixels (editor default 20, NovaRenderer_draw.cpp:14) */
  int32_t vertical_invert;
} orc_options;

typedef struct {
  uint64_t segments;   /* Li evaluations (one ray segment each) */
  uint64_t traced;     /* BVH queries issued */
  uint64_t node_visits;
  uint64_t tri_tests;
  double seconds;      /* wall time of the frame loop */
} orc_stats;

/* Sampler (math_random.h:29-120). */
void orc_sobol_table(uint32_t out[256 * 32]);
void orc_sobol_samples(const uint32_t *index, const uint32_t *dim, uint64_t n, uint32_t seed, float *out);
void orc_acos_lut(float *out, int32_t precision);

/* Scene + native SAH BVH (aggregate/native/BvhBuilder.cpp). Returns NULL on bad input. */
void *orc_build(const orc_scene *scene);
void orc_free(void *h);
void orc_bvh_info(void *h, int64_t *nodes, int64_t *leaves, int64_t *max_leaf);

/* Closest hit of n world-space rays (tnear 1e-6, tfar MAXFLOAT as Ray.h:14 / native.cpp:57).
 * prim = global primitive id or -1, t/u/v = Moller-Trumbore distance and barycentrics. */
void orc_trace(void *h, uint64_t n, const float *orig, const float *dir, int32_t *prim, float *t, float *u,
               float *v, orc_stats *stats);

/* Camera ray of pixel (x, y), sample s (Integrator.h:66-85 with the chosen index mapping). */
void orc_camera_rays(void *h, const orc_options *opt, uint64_t n, const int32_t *px, const int32_t *py,
                     const int32_t *s, float *orig, float *dir);

/* Full progressive render: frames of 1 spp over 20x20 tiles on a worker pool, running-mean film.
 * out_rgba = W*H*4 floats.  If pixel_ids != NULL only those pixels (y*W+x) are rendered. */
int32_t orc_render(void *h, const orc_options *opt, float *out_rgba, const int32_t *pixel_ids, int64_t n_pixels,
                   orc_stats *stats);

/* The segments of one path: 10 floats each (origin, direction, hit primitive bits, t, u, v). */
int32_t orc_sample_path(void *h, const orc_options *opt, int32_t x, int32_t y, int32_t s, float *out,
                        int32_t max_segments, float *radiance);
/* One shading event per hit: next origin / direction, weight, emission, valid. */
void orc_scatter(void *h, uint64_t n, const float *o, const float *d, const int32_t *prim, const float *t,
                 const float *u, const float *v, const uint32_t *index, const int32_t *bounce, uint32_t seed,
                 float *out_o, float *out_d, float *weight, float *emissive, int32_t *valid);
/* Differentiable parameters (3 x triangles albedo, materials roughness; NULL = textures). */
int32_t orc_set_diff_params(void *h, const float *albedo, const float *roughness);
/* Detached perturbation (kind 0 none, 1 albedo of triangle `index` channel `channel`, 2 roughness
 * of material `index`): f evaluated with the parameter moved by delta, sampling unperturbed. */
int32_t orc_set_perturbation(void *h, int32_t kind, uint32_t index, int32_t channel, float delta);
/* Replay adjoint: adds dLoss/dalbedo, dLoss/droughness for d_image = dLoss/dImage (W*H*4). */
int32_t orc_backward(void *h, const orc_options *opt, const float *d_image, float *grad_albedo,
                     float *grad_roughness, int32_t threads);
int32_t orc_backward_range(void *h, const orc_options *opt, int32_t sample_begin, int32_t sample_count,
                           const float *d_image, float *grad_albedo, float *grad_roughness, int32_t threads);
/* AOV integrators: kind 1 normal, 2 depth (camera near / far planes), 4 emissive; out = W*H*4. */
int32_t orc_render_aov(void *h, const orc_options *opt, int32_t kind, float near_plane, float far_plane, float *out);
/* Radiance of single samples (pixel x, y, sample s), RGB into out (3 per sample). */
void orc_sample_radiance(void *h, const orc_options *opt, uint64_t n, const int32_t *px, const int32_t *py,
                         const int32_t *s, float *out);

/* The reference's CUDA irradiance bake (sources/processing/cuda/CubemapProcessing.cu:129-175) with the
 * texture unit's bilinear filter restated; rgba source, out = out_w * out_h * 4 floats (alpha 1). */
int32_t orc_bake_irradiance_texunit(const float *rgba, int32_t src_w, int32_t src_h, int32_t out_w, int32_t out_h,
                                    int32_t samples, int32_t threads, float *out);
/* Diffuse irradiance bake, CPU path (sources/processing/TextureProcessing.cpp:10-64). */
int32_t orc_bake_irradiance(const float *src, int32_t src_w, int32_t src_h, int32_t channels, int32_t out_w,
                            int32_t out_h, int32_t samples, int32_t threads, float *out);

/* BxDF math of the restatement (property tests). */
float orc_fresnel_real(float ior, float cos_i, float *new_eta);
void orc_vndf_sample(float anisotropy, float roughness, const float wo[3], const float uc[2], float wm[3]);
float orc_vndf_g1(float anisotropy, float roughness, const float v[3]);
void orc_correct_specular_normal(const float ng[3], const float wo[3], const float ns[3], float out[3]);
/* Environment lookup of a float texture and the fast spherical mapping (property tests). */
void orc_env_sample(const float *pixels, int32_t w, int32_t h, int32_t channels, uint64_t n, const float *dirs,
                    float *out);
void orc_cartesian_to_spherical(uint64_t n, const float *xyz, float *phi_theta);
/* The dielectric lobe alone: sample at (wo, uc, u), then f and pdf evaluated at the sampled direction
 * (property tests); out = f[3], pdf, wi[3], costheta, f_eval[3], pdf_eval. */
int32_t orc_dielectric_lobe(const float albedo[3], float eta, float roughness, float anisotropy, const float wo[3],
                            float uc, const float u[2], float out[12]);
/* The traversal's slab test on one box: entry distance, or MAXFLOAT past dist_min (property tests). */
float orc_box_intersect(const float mn[3], const float mx[3], const float o[3], const float d[3], float dist_min);
/* One texture lookup: 8-bit bilinear sample or float nearest texel, RGBA (property tests). */
void orc_texture_lookup(const orc_texture *texture, float u, float v, float out[4]);
/* Header-only reference arithmetic as the oracle restates it (pinned against oracle/_ref). */
void orc_atan2_approx(uint64_t n, const float *y, const float *x, float *out);
void orc_rgb_to_unit(uint64_t n, const float *v, float *out);
void orc_uv_to_pixel(uint64_t n, const float *t, const uint32_t *dim, uint32_t *out);
/* Triangle bounds and centroids of every primitive, instance by instance (property tests). */
void orc_prim_bounds(void *scene, float *boxes, float *centroids);
/* The frame's tile split: (x0, x1, y0, y1) per tile; returns the tile count, 0 for bad sizes. */
int32_t orc_tile_split(int32_t width, int32_t height, int32_t tiles_w, int32_t tiles_h, int32_t *rects);

/* One BSDF query for the pin against the reference's own BxDF / BSDF code (tests only): the
 * bsdf_params_s fields the path fills (BxDF.h:22-39; eta uniform over RGB), the outgoing direction,
 * the random numbers, and for a single lobe its weight and probability.  Directions are in world
 * space for orc_principled_sample and in the local shading frame for the single lobes. */
typedef struct {
  float ns[3], ng[3], dpdu[3], dpdv[3];
  float wo_dot_ng, roughness, metal, transmission, anisotropy, eta;
  float albedo[3];
  float wo[3];
  float uc, u[2];
  float weight, probability;
  int32_t thin;
} orc_bsdf_case;
/* BSDFSample fields the integrator reads (BxDF_flags.h:26-35) and whether sampling succeeded. */
typedef struct {
  float f[3], wi[3];
  float pdf, costheta;
  uint32_t flags;
  int32_t valid;
} orc_bsdf_result;
/* PrincipledBSDF(params, uc).sample_f(wo, uc, u) (BSDF.h:87-130). */
void orc_principled_sample(uint64_t n, const orc_bsdf_case *cases, orc_bsdf_result *out);
/* One lobe's sample_f in the local frame: lobe 1 DisneyDiffuseBxDF, 2 SpecularBxDF, 3 DielectricBxDF
 * (BxDF.h:252-594). */
void orc_lobe_sample(int32_t lobe, uint64_t n, const orc_bsdf_case *cases, orc_bsdf_result *out);
/* DielectricBxDF::f / ::pdf at wi (3 floats per case) in the local frame (BxDF.h:497-545). */
void orc_dielectric_eval(uint64_t n, const orc_bsdf_case *cases, const float *wi, float *f, float *pdf);
/* Triangle::hit's Moller-Trumbore on one triangle per query (Triangle.h:146-177): tri = 9 floats of
 * object-space vertices, inv = 16 floats (column-major inverse transform), ray in world space;
 * returns hit flags, t, u, v. */
void orc_triangle_hits(uint64_t n, const float *tri, const float *inv, const float *o, const float *d, float tmin,
                       float tmax, int32_t *hit, float *t, float *u, float *v);
/* Ray::spawn(wi, n, position) (Ray.h:22-27): next origin and direction. */
void orc_spawn(uint64_t n, const float *wi, const float *nrm, const float *pos, float *out_o, float *out_d);
/* math::geometry::gram_shmidt and make_onb (utils_3D.h:52-81): 9 floats (T, B, N) / 6 floats (b1, b2). */
void orc_gram_shmidt(uint64_t n, const float *nrm, const float *tan, const float *bit, float *out);
void orc_make_onb(uint64_t n, const float *nrm, float *out);

/* The Embree-semantics hit record the oracle builds for a hit (prim, t, u, v) of a ray (embree.cpp:287-412):
 * 23 floats per hit: ng[3], dpdu[3], dpdv[3], position[3], u, v, shading frame columns T[3], B[3], N[3]. */
void orc_hit_record(void *h, uint64_t n, const float *o, const float *d, const int32_t *prim, const float *t,
                    const float *u, const float *v, float *out);

/* Film outputs and the Radiance .hdr format (film_io.cpp). */
void orc_film_accumulate(const float *partial, float *accum, float *final_buf, uint64_t n, uint32_t frame_index);
void orc_display_blend(const float *partial, const float *accum, float *out, uint64_t n, uint32_t current_frame);
void orc_snapshot(const float *film, int32_t width, int32_t height, int32_t channels, float *dst, int32_t dst_width,
                  int32_t dst_height);
void orc_rgbe_encode(const float *px, uint64_t n, int32_t channels, uint8_t *out);
void orc_rgbe_decode(const uint8_t *in, uint64_t n, float *out_rgba);
int32_t orc_hdr_parse(const uint8_t *bytes, uint64_t size, int32_t *width, int32_t *height, uint8_t *rgbe);
int32_t orc_hdr_write(const char *path, const float *px, int32_t width, int32_t height, int32_t channels, int32_t flip);

#ifdef __cplusplus
}
#endif
