/* Device-resident scene layout.
 *
 * HBM layout (all arrays are owned by the context, see context.cu):
 *   tris       3 float4 per triangle in BVH leaf order: (v0.xyz, prim id), (e1.xyz, instance id), (e2.xyz, 0)
 *              with object-space v0 and edges e1 = v1 - v0, e2 = v2 - v0 (Triangle.h:154-156 computes the
 *              same edges), 48 B per triangle.
 *   nodes      binary BVH, 4 float4 per node (64 B): both children's boxes and references
 *                n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)   n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
 *                n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)   n3 = (ref0, ref1, count0, count1)
 *              ref >= 0: inner node index; ref < 0: leaf whose triangles start at ~ref (count in n3.z/w).
 *   prim_inst  instance index of every global primitive (primitive order of the reference:
 *              instance by instance, triangle by triangle; api/engine.cpp:159-175).
 *   meshes / instances / materials / textures: shading data; object-space vertex attributes are
 *              interleaved per vertex (DevMesh) and gathered through the index buffer at hit time.
 */
#pragma once
#include "dmath.cuh"

namespace nb {

struct DevTexture {
  const uint32_t *u8;
  const float *f32;
  int32_t w, h, ch;
  int32_t is_rgba, invert_u, invert_v;
};

struct DevMaterial {
  int32_t albedo, metallic, normalmap, emissive;
  float eta[3];
  float k[3];
  float anisotropy;
};

/* Vertex attributes interleaved, 64 B per vertex (two 32 B sectors):
 *   attr[4 i + 0] = (p.x, p.y, p.z, n.x)   attr[4 i + 1] = (n.y, n.z, t.x, t.y)
 *   attr[4 i + 2] = (t.z, b.x, b.y, b.z)   attr[4 i + 3] = (u, v, 0, 0)                          */
struct DevMesh {
  const float4 *attr;
  const uint32_t *idx;
  uint32_t n_verts, n_tris;
};

NB_D V3 vertex_position(const DevMesh &m, uint32_t i) {
  const float4 a = __ldg(m.attr + 4 * (size_t)i);
  return {a.x, a.y, a.z};
}

struct DevInstance {
  float m[16];
  float inv[16];
  float n[9];
  uint32_t mesh;
  uint32_t material;
  uint32_t prim_offset; /* global id of this instance's first triangle */
  int32_t identity;     /* m == inv == identity: the object-space ray is the world ray bit for bit */
  uint32_t lobe_class;  /* 1: the material transmits (eta set, no absorption: the dielectric lobe) */
  const float4 *attr;   /* the mesh's interleaved vertex attributes, triangle indices and triangle */
  const uint32_t *idx;  /* count (copies of its DevMesh fields, so a hit record skips the mesh-table */
  uint32_t n_tris;      /* load) */
};

struct DevScene {
  const float4 *nodes;       /* binary BVH (width 2) or compressed 8-wide BVH (width 8, bvh_wide.cuh) */
  int32_t width;
  const float4 *tris;
  const uint32_t *prim_inst;
  const DevMesh *meshes;
  const DevInstance *instances;
  const DevMaterial *materials;
  const DevTexture *textures;
  const uint32_t *sobol_dv;  /* byte-sliced direction vectors: 256 dims x 4 x 256 (sampler.cuh) */
  const float *acos_lut;     /* 500000 entries */
  int32_t envmap;
  uint32_t n_prims;
  uint32_t n_instances, n_materials; /* table sizes: the shading kernels check every index against them */
  uint32_t has_emissive;
  const float *diff_albedo;  /* differentiable parameters (NULL: textures): 3 x n_prims RGB albedo */
  const float *diff_rough;   /* and n_materials roughness values */
  const uint32_t *blas_root; /* two-level BVH (width 1): per mesh, the node index of its bottom-level root */
};

constexpr int kAcosPrecision = 500000;

}  // namespace nb
