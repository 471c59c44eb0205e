/* ORACLE — test infrastructure only (see oracle.h).  Internal declarations shared by the oracle's
 * translation units. */
#pragma once
#include "oracle.h"
#include "vecmath.h"
#include <cstdint>
#include <vector>

namespace orc {

constexpr int kAcosPrecision = 500000; /* PRECISION_LUT with AXOMAE_LUT_MEDIUMP (the default, CMakeLists.txt:37) */
constexpr float kMaxFloat = 3.40282347e+38f; /* MAXFLOAT */

const uint32_t *sobol_table();
float sobol_sample(uint32_t index, unsigned dim, uint32_t seed);
std::vector<float> make_acos_lut(int precision);
const float *acos_lut();

/* geometry::BoundingBox (corelib/internal/geometry/BoundingBox.h:24-26): default box is
 * min = 1e32, max = -1e32; operator+ is a component-wise glm::min / glm::max. */
struct Box {
  V3 mn{1e32f, 1e32f, 1e32f};
  V3 mx{-1e32f, -1e32f, -1e32f};
  Box operator+(const Box &b) const { return {vmin(mn, b.mn), vmax(mx, b.mx)}; }
  float half_area() const { /* BoundingBox.cpp:162-165 */
    V3 l = mx - mn;
    return l.x * l.y + l.y * l.z + l.z * l.x;
  }
};

/* aggregate/native/BvhBuilder.h:10-15 */
struct Node {
  float min[3];
  float max[3];
  int32_t left;
  int32_t count;
};

struct Mesh {
  std::vector<float> v, n, t, b, uv;
  std::vector<uint32_t> idx;
  uint32_t n_tris = 0;
};

struct Xform {
  M4 m, inv;
  M3 n;
};

struct Texture {
  std::vector<uint32_t> u8;
  std::vector<float> f32;
  int w = 0, h = 0, channels = 4;
  bool is_rgba = true, invert_u = false, invert_v = false;
};

struct Material {
  int albedo = -1, metallic = -1, normalmap = -1, emissive = -1;
  Spec eta{0, 0, 0}, k{0, 0, 0};
  float anisotropy = 0.f;
};

struct Prim {
  uint32_t inst;
  uint32_t tri; /* triangle index inside the mesh (index offset = 3 * tri) */
};

struct Scene {
  std::vector<Mesh> meshes;
  std::vector<uint32_t> inst_mesh, inst_mat;
  std::vector<Xform> xf;
  std::vector<Material> materials;
  std::vector<Texture> textures;
  int envmap = -1;
  M4 inv_P, inv_V;
  std::vector<Prim> prims;
  /* differentiable parameters (extension): per-triangle RGB albedo, per-material roughness;
   * empty = textures */
  std::vector<float> diff_albedo, diff_rough;
  /* detached perturbation of one parameter (finite differences of the detached-sampling
   * estimator): f is evaluated with the parameter moved by pert_delta at the directions and
   * densities of the unperturbed parameters.  kind 0: none, 1: albedo of triangle pert_index,
   * channel pert_channel, 2: roughness of material pert_index. */
  int pert_kind = 0;
  uint32_t pert_index = 0;
  int pert_channel = 0;
  float pert_delta = 0.f;
  /* native BVH */
  std::vector<Node> nodes;
  std::vector<int32_t> prim_idx;
  int32_t nodes_used = 0;
};

struct Ray {
  V3 o, d;
  float tnear = 0.000001f;
  float tfar = 1e30f;
};

struct Hit {
  bool is_hit = false;
  int32_t prim = -1;
  float t = 0.f, u = 0.f, v = 0.f;
};

struct TraceCounters {
  uint64_t nodes = 0, tris = 0;
};

void build_bvh(Scene &s);
void prim_bounds(const Scene &s, const Prim &p, Box &box, V3 &centroid);
Hit trace(const Scene &s, const Ray &r, TraceCounters *c);
bool triangle_hit(const Scene &s, const Prim &p, const Ray &r, float tmin, float tmax, float &t, float &u, float &v);
bool moller_trumbore(const M4 &inv, V3 v0, V3 v1, V3 v2, const Ray &in, float tmin, float tmax, float &t, float &u,
                     float &v);

}  // namespace orc
