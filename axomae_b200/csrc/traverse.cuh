/* Closest-hit traversal of the device BVH.
 *
 * Semantics follow the reference's native accelerator (aggregate/native/native.cpp:56-114): the
 * nearer child is visited first, a box is skipped when its entry distance exceeds the current
 * closest hit, and a triangle replaces the current hit when its distance is <= the current one.
 * The triangle test is the reference's Moller-Trumbore (shape/Triangle.h:146-177) evaluated in
 * the same order (no fused multiply-add), in object space: the ray is brought into the instance's
 * space with the instance's inverse transform exactly as Triangle::hit does, and identity
 * instances skip the (bit-exact no-op) transform.
 *
 * Box tests only prune: each slab distance is (plane - origin) * rcp(direction), and the exit
 * distance is widened by 2^-21 relative, so rounding never prunes a box whose triangles the
 * Moller-Trumbore test would hit.
 *
 * Node layout and leaf encoding: see device_scene.cuh.  Leaf reference = ~((first << 4) | (count - 1)).
 * Three layouts: binary (width 2), compressed 8-wide (width 8) and two-level binary (width 1: a top
 * level over instances, a bottom level per mesh).
 */
#pragma once
#include <cfloat>
#include "bvh_wide.cuh"
#include "device_scene.cuh"

namespace nb {

constexpr int kTraversalStack = 64;

/* When both children of a binary node are hit, the deferred one's node record is prefetched into L1
 * (NB_TRACE_PREFETCH=1) so the pop later finds it near. */
#ifndef NB_TRACE_PREFETCH
#define NB_TRACE_PREFETCH 0
#endif
/* Leaves are tested one triangle per loop iteration (NB_LEAF_STEP=1): on the 32-job batch this took
 * the traversal from 193 to 179 ms per step against whole leaves per iteration. */
#ifndef NB_LEAF_STEP
#define NB_LEAF_STEP 1
#endif
NB_D void prefetch_node(const float4 *nodes, int32_t ref) {
#if NB_TRACE_PREFETCH
  if (ref >= 0) asm volatile("prefetch.global.L1 [%0];" ::"l"(nodes + 4 * (size_t)ref));
#endif
}
constexpr float kRayTNear = 0.000001f; /* Ray::tnear, ray/Ray.h:14 */
constexpr float kFarScale = 1.000000477f; /* 1 + 2^-21: covers the rounding of the slab distances */

NB_HD int32_t leaf_ref(uint32_t first, uint32_t count) { return ~(int32_t)((first << 4) | (count - 1)); }
NB_HD uint32_t leaf_first(int32_t ref) { return ((uint32_t)~ref) >> 4; }
NB_HD uint32_t leaf_count(int32_t ref) { return (((uint32_t)~ref) & 15u) + 1u; }

/* Triangle::hit, Triangle.h:154-177 (inv_det before the det == 0 test, inclusive edges). */
NB_D bool mt_hit(V3 o, V3 d, V3 v0, V3 e1, V3 e2, float tmin, float tmax, float &t, float &u, float &v) {
  const V3 P = cross(d, e2);
  const float det = dot(P, e1);
  const float inv_det = 1.f / det;
  if (det == 0.f) return false;
  const V3 T = o - v0;
  const float uu = dot(P, T) * inv_det;
  if (uu < 0 || uu > 1.f) return false;
  const V3 Q = cross(T, e1);
  const float vv = dot(Q, d) * inv_det;
  if (vv < 0.f || (uu + vv) > 1.f) return false;
  const float tt = dot(Q, e2) * inv_det;
  if (tt < tmin || tt > tmax) return false;
  t = tt;
  u = uu;
  v = vv;
  return true;
}

struct TraceResult {
  int32_t prim;
  float t, u, v;
  uint32_t inst; /* the hit triangle's instance (valid when prim >= 0) */
};

NB_D float safe_rcp(float d) {
  /* reciprocal for the slab test; zero components get a huge finite value of the right sign */
  const float big = 1e30f;
  return fabsf(d) > 1e-30f ? __frcp_rn(d) : copysignf(big, d);
}

/* Closest hit of one world-space ray on the binary BVH. */
NB_D TraceResult trace_closest2(const DevScene &sc, V3 o, V3 d, uint64_t *node_visits = nullptr,
                               uint64_t *tri_tests = nullptr) {
  TraceResult r{-1, 0.f, 0.f, 0.f, 0u};
  float tmax = FLT_MAX; /* native.cpp:57 starts from MAXFLOAT */
  const float ix = safe_rcp(d.x), iy = safe_rcp(d.y), iz = safe_rcp(d.z);
  int32_t stack[kTraversalStack];
  int sp = 0;
  int32_t cur = 0; /* the root is always an inner node (a one-leaf scene gets an empty sibling) */
  int32_t cached_inst = -1;
  V3 lo_o = o, lo_d = d;
  uint64_t nv = 0, tt = 0;
#if NB_LEAF_STEP
  uint32_t lk = 0, le = 0; /* the current leaf's next and end triangle */
#endif
  for (;;) {
    if (cur >= 0) {
      nv++;
      const float4 n0 = __ldg(&sc.nodes[4 * cur + 0]);
      const float4 n1 = __ldg(&sc.nodes[4 * cur + 1]);
      const float4 n2 = __ldg(&sc.nodes[4 * cur + 2]);
      const float4 n3 = __ldg(&sc.nodes[4 * cur + 3]);
      /* slabs as (plane - origin) * rcp(dir): two roundings per distance, far end widened by 2^-21 */
      float a0 = (n0.x - o.x) * ix, b0 = (n0.y - o.x) * ix;
      float a1 = (n0.z - o.y) * iy, b1 = (n0.w - o.y) * iy;
      float a2 = (n2.x - o.z) * iz, b2 = (n2.y - o.z) * iz;
      float c0n = fmaxf(fmaxf(fminf(a0, b0), fminf(a1, b1)), fmaxf(fminf(a2, b2), 0.f));
      float c0f = fminf(fminf(fminf(fmaxf(a0, b0), fmaxf(a1, b1)), fmaxf(a2, b2)) * kFarScale, tmax);
      float d0 = (n1.x - o.x) * ix, e0 = (n1.y - o.x) * ix;
      float d1 = (n1.z - o.y) * iy, e1 = (n1.w - o.y) * iy;
      float d2 = (n2.z - o.z) * iz, e2 = (n2.w - o.z) * iz;
      float c1n = fmaxf(fmaxf(fminf(d0, e0), fminf(d1, e1)), fmaxf(fminf(d2, e2), 0.f));
      float c1f = fminf(fminf(fminf(fmaxf(d0, e0), fmaxf(d1, e1)), fmaxf(d2, e2)) * kFarScale, tmax);
      const bool h0 = c0n <= c0f, h1 = c1n <= c1f;
      const int32_t r0 = __float_as_int(n3.x), r1 = __float_as_int(n3.y);
      if (h0 && h1) {
        int32_t first = r0, second = r1;
        if (c1n < c0n) {
          first = r1;
          second = r0;
        }
        prefetch_node(sc.nodes, second);
        if (sp < kTraversalStack) stack[sp++] = second;
        cur = first;
        continue;
      } else if (h0) {
        cur = r0;
        continue;
      } else if (h1) {
        cur = r1;
        continue;
      }
    } else {
#if NB_LEAF_STEP
      /* one triangle per loop iteration: a lane in a leaf costs its warp one triangle test per
       * iteration, not the whole leaf, while the other lanes visit nodes */
      if (lk >= le) {
        lk = leaf_first(cur);
        le = lk + leaf_count(cur);
      }
      {
        const uint32_t k = lk++;
#else
      const uint32_t first = leaf_first(cur), count = leaf_count(cur);
      for (uint32_t k = first; k < first + count; k++) {
#endif
        const float4 t0 = __ldg(&sc.tris[3 * k + 0]);
        const float4 t1 = __ldg(&sc.tris[3 * k + 1]);
        const float4 t2 = __ldg(&sc.tris[3 * k + 2]);
        const int32_t inst = __float_as_int(t1.w);
        if (inst != cached_inst) {
          cached_inst = inst;
          const DevInstance &I = sc.instances[inst];
          if (I.identity) {
            lo_o = o;
            lo_d = d;
          } else {
            lo_o = xform_point(I.inv, o);
            lo_d = xform_dir(I.inv, d);
          }
        }
        tt++;
        float ht, hu, hv;
        if (mt_hit(lo_o, lo_d, V3{t0.x, t0.y, t0.z}, V3{t1.x, t1.y, t1.z}, V3{t2.x, t2.y, t2.z}, kRayTNear, tmax, ht,
                   hu, hv)) {
          tmax = ht;
          r.prim = __float_as_int(t0.w);
          r.inst = (uint32_t)inst;
          r.t = ht;
          r.u = hu;
          r.v = hv;
        }
      }
#if NB_LEAF_STEP
      if (lk < le) continue;
#endif
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
  if (node_visits) *node_visits += nv;
  if (tri_tests) *tri_tests += tt;
  return r;
}

/* Triangle tests of one leaf range with the instance-transform cache (Triangle.h:146-153). */
template <class S>
NB_D void test_triangles(const S &sc, uint32_t first, uint32_t count, V3 o, V3 d, int32_t &cached_inst, V3 &lo_o,
                         V3 &lo_d, float &tmax, TraceResult &r) {
  /* count: the caller counts triangle tests (trace_closest8's tri_tests) */
  for (uint32_t k = first; k < first + count; k++) {
    const float4 t0 = __ldg(&sc.tris[3 * k + 0]);
    const float4 t1 = __ldg(&sc.tris[3 * k + 1]);
    const float4 t2 = __ldg(&sc.tris[3 * k + 2]);
    const int32_t inst = __float_as_int(t1.w);
    if (inst != cached_inst) {
      cached_inst = inst;
      const DevInstance &I = sc.instances[inst];
      if (I.identity) {
        lo_o = o;
        lo_d = d;
      } else {
        lo_o = xform_point(I.inv, o);
        lo_d = xform_dir(I.inv, d);
      }
    }
    float ht, hu, hv;
    if (mt_hit(lo_o, lo_d, V3{t0.x, t0.y, t0.z}, V3{t1.x, t1.y, t1.z}, V3{t2.x, t2.y, t2.z}, kRayTNear, tmax, ht, hu,
               hv)) {
      tmax = ht;
      r.prim = __float_as_int(t0.w);
      r.inst = (uint32_t)inst;
      r.t = ht;
      r.u = hu;
      r.v = hv;
    }
  }
}

/* The binary-BVH walk of trace_closest2 as a resumable state: step() does one loop iteration (an
 * inner node, or a leaf and the pop after it) with the same arithmetic and order, so a walk driven
 * to the end reports exactly trace_closest2's hit.  Used where a thread interleaves several rays.
 * The traversal stack (kTraversalStack entries) is the caller's, so the scalar state can stay in
 * registers. */
/* The three tables a binary walk reads, held in registers by a thread that switches between rays
 * of different jobs. */
struct WalkScene {
  const float4 *nodes;
  const float4 *tris;
  const DevInstance *instances;
};

struct Walk2 {
  V3 o, d;
  float ix, iy, iz, tmax;
  TraceResult r;
  int32_t cur, cached_inst;
  int sp;
  V3 lo_o, lo_d;

  NB_D void init(V3 ro, V3 rd) {
    o = ro;
    d = rd;
    ix = safe_rcp(d.x), iy = safe_rcp(d.y), iz = safe_rcp(d.z);
    tmax = FLT_MAX;
    r = TraceResult{-1, 0.f, 0.f, 0.f, 0u};
    cur = 0;
    cached_inst = -1;
    sp = 0;
    lo_o = o;
    lo_d = d;
  }

  /* false once the walk is over (r holds the closest hit); S is any scene view with the nodes,
   * tris and instances tables (DevScene, WalkScene) */
  template <class S>
  NB_D bool step(const S &sc, int32_t *stack) {
    if (cur >= 0) {
      const float4 n0 = __ldg(&sc.nodes[4 * cur + 0]);
      const float4 n1 = __ldg(&sc.nodes[4 * cur + 1]);
      const float4 n2 = __ldg(&sc.nodes[4 * cur + 2]);
      const float4 n3 = __ldg(&sc.nodes[4 * cur + 3]);
      const float a0 = (n0.x - o.x) * ix, b0 = (n0.y - o.x) * ix;
      const float a1 = (n0.z - o.y) * iy, b1 = (n0.w - o.y) * iy;
      const float a2 = (n2.x - o.z) * iz, b2 = (n2.y - o.z) * iz;
      const float c0n = fmaxf(fmaxf(fminf(a0, b0), fminf(a1, b1)), fmaxf(fminf(a2, b2), 0.f));
      const float c0f = fminf(fminf(fminf(fmaxf(a0, b0), fmaxf(a1, b1)), fmaxf(a2, b2)) * kFarScale, tmax);
      const float d0 = (n1.x - o.x) * ix, e0 = (n1.y - o.x) * ix;
      const float d1 = (n1.z - o.y) * iy, e1 = (n1.w - o.y) * iy;
      const float d2 = (n2.z - o.z) * iz, e2 = (n2.w - o.z) * iz;
      const float c1n = fmaxf(fmaxf(fminf(d0, e0), fminf(d1, e1)), fmaxf(fminf(d2, e2), 0.f));
      const float c1f = fminf(fminf(fminf(fmaxf(d0, e0), fmaxf(d1, e1)), fmaxf(d2, e2)) * kFarScale, tmax);
      const bool h0 = c0n <= c0f, h1 = c1n <= c1f;
      const int32_t r0 = __float_as_int(n3.x), r1 = __float_as_int(n3.y);
      if (h0 && h1) {
        int32_t first = r0, second = r1;
        if (c1n < c0n) {
          first = r1;
          second = r0;
        }
        if (sp < kTraversalStack) stack[sp++] = second;
        cur = first;
        return true;
      } else if (h0) {
        cur = r0;
        return true;
      } else if (h1) {
        cur = r1;
        return true;
      }
    } else {
      test_triangles(sc, leaf_first(cur), leaf_count(cur), o, d, cached_inst, lo_o, lo_d, tmax, r);
    }
    if (sp == 0) return false;
    cur = stack[--sp];
    return true;
  }
};

/* Closest hit on the compressed 8-wide BVH (layout in bvh_wide.cuh).  Every visited node tests its
 * eight quantised child boxes, tests the triangles of hit leaf children in slot order, then
 * descends into the first hit inner child; the other hit inner children stay on a stack as one
 * (child_base, hit mask, inner mask) group.  Child slots are visited in increasing (slot ^ oct)
 * order, oct being the ray's direction-sign bits, which is near-to-far for the slot assignment.
 * node_visits / tri_tests (optional) add the nodes visited and the triangles tested. */
NB_D TraceResult trace_closest8(const DevScene &sc, V3 o, V3 d, uint64_t *node_visits = nullptr,
                               uint64_t *tri_tests = nullptr) {
  TraceResult r{-1, 0.f, 0.f, 0.f, 0u};
  float tmax = FLT_MAX;
  const float ix = safe_rcp(d.x), iy = safe_rcp(d.y), iz = safe_rcp(d.z);
  const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
  uint2 stack[kWideStack];
  int sp = 0;
  uint32_t node = 0;
  int32_t cached_inst = -1;
  V3 lo_o = o, lo_d = d;
  uint32_t nv = 0, tt = 0;
  for (;;) {
    nv++;
    const float4 *np = sc.nodes + 5 * (size_t)node;
    const float4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
    const uint32_t hdr = __float_as_uint(w0.w);
    const uint32_t imask = hdr >> 24;
    const float sx = __uint_as_float((hdr & 0xffu) << 23), sy = __uint_as_float(((hdr >> 8) & 0xffu) << 23),
                sz = __uint_as_float(((hdr >> 16) & 0xffu) << 23);
    /* plane distance = (p + q s - o) * idir = q (s idir) + (p - o) idir; the near plane of each
     * axis is the low plane when the direction component is positive, the high plane otherwise */
    const float ax = (w0.x - o.x) * ix, ay = (w0.y - o.y) * iy, az = (w0.z - o.z) * iz;
    const float bx = sx * ix, by = sy * iy, bz = sz * iz;
    const uint32_t child_base = __float_as_uint(w1.x), tri_base = __float_as_uint(w1.y);
    const uint32_t meta[2] = {__float_as_uint(w1.z), __float_as_uint(w1.w)};
    const bool px = ix >= 0.f, py = iy >= 0.f, pz = iz >= 0.f;
    const uint32_t nx[2] = {px ? __float_as_uint(w2.x) : __float_as_uint(w3.z), px ? __float_as_uint(w2.y) : __float_as_uint(w3.w)};
    const uint32_t fx[2] = {px ? __float_as_uint(w3.z) : __float_as_uint(w2.x), px ? __float_as_uint(w3.w) : __float_as_uint(w2.y)};
    const uint32_t ny[2] = {py ? __float_as_uint(w2.z) : __float_as_uint(w4.x), py ? __float_as_uint(w2.w) : __float_as_uint(w4.y)};
    const uint32_t fy[2] = {py ? __float_as_uint(w4.x) : __float_as_uint(w2.z), py ? __float_as_uint(w4.y) : __float_as_uint(w2.w)};
    const uint32_t nz[2] = {pz ? __float_as_uint(w3.x) : __float_as_uint(w4.z), pz ? __float_as_uint(w3.y) : __float_as_uint(w4.w)};
    const uint32_t fz[2] = {pz ? __float_as_uint(w4.z) : __float_as_uint(w3.x), pz ? __float_as_uint(w4.w) : __float_as_uint(w3.y)};
    uint32_t inner_hits = 0, leaf_hits = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int w = i >> 2;
      const uint32_t sel = 0x7540u + (uint32_t)(i & 3);
      /* byte -> exact float: 0x4B0000bb is 2^23 + bb */
      const float qnx = __uint_as_float(__byte_perm(nx[w], 0x4B000000u, sel)) - 8388608.f;
      const float qfx = __uint_as_float(__byte_perm(fx[w], 0x4B000000u, sel)) - 8388608.f;
      const float qny = __uint_as_float(__byte_perm(ny[w], 0x4B000000u, sel)) - 8388608.f;
      const float qfy = __uint_as_float(__byte_perm(fy[w], 0x4B000000u, sel)) - 8388608.f;
      const float qnz = __uint_as_float(__byte_perm(nz[w], 0x4B000000u, sel)) - 8388608.f;
      const float qfz = __uint_as_float(__byte_perm(fz[w], 0x4B000000u, sel)) - 8388608.f;
      const float nr = fmaxf(fmaxf(__fmaf_rn(qnx, bx, ax), __fmaf_rn(qny, by, ay)), fmaxf(__fmaf_rn(qnz, bz, az), 0.f));
      const float fr =
          fminf(fminf(fminf(__fmaf_rn(qfx, bx, ax), __fmaf_rn(qfy, by, ay)), __fmaf_rn(qfz, bz, az)) * kFarScale, tmax);
      /* empty slots store qlo = 255, qhi = 0 on every axis: near > far for either ray sign */
      if (nr <= fr) {
        const uint32_t bit = 1u << (i ^ oct);
        if ((imask >> i) & 1u)
          inner_hits |= bit;
        else
          leaf_hits |= bit;
      }
    }
    while (leaf_hits) {
      const uint32_t slot = (uint32_t)(__ffs(leaf_hits) - 1) ^ oct;
      leaf_hits &= leaf_hits - 1;
      const uint32_t m = (meta[slot >> 2] >> (8 * (slot & 3))) & 0xffu;
      tt += ((m >> 5) & 3u) + 1u;
      test_triangles(sc, tri_base + (m & 31u), ((m >> 5) & 3u) + 1u, o, d, cached_inst, lo_o, lo_d, tmax, r);
    }
    if (inner_hits) {
      const uint32_t slot = (uint32_t)(__ffs(inner_hits) - 1) ^ oct;
      inner_hits &= inner_hits - 1;
      if (inner_hits && sp < kWideStack) stack[sp++] = make_uint2(child_base, inner_hits | (imask << 8));
      node = child_base + __popc(imask & ((1u << slot) - 1u));
      continue;
    }
    if (sp == 0) break;
    uint2 g = stack[--sp];
    uint32_t hits = g.y & 0xffu;
    const uint32_t gmask = g.y >> 8;
    const uint32_t slot = (uint32_t)(__ffs(hits) - 1) ^ oct;
    hits &= hits - 1;
    if (hits) stack[sp++] = make_uint2(g.x, hits | (gmask << 8));
    node = g.x + __popc(gmask & ((1u << slot) - 1u));
  }
  if (node_visits) *node_visits += nv;
  if (tri_tests) *tri_tests += tt;
  return r;
}

/* Closest hit on the two-level BVH (width 1): the top level's binary nodes over instance boxes, one
 * instance per leaf; at a top leaf the ray is brought into the instance's object space (its
 * inverse transform, Triangle.h:150-153; identity instances keep the world ray bit for bit) and the
 * walk goes on in the mesh's bottom-level BVH, with a marker on the stack that restores the world
 * ray when that subtree is done.  t is the same in both spaces (the direction is not renormalised),
 * so the closest distance found so far prunes both levels.  Node tests, ordering and the triangle
 * test are trace_closest2's. */
constexpr int32_t kLeaveInstance = 0x7fffffff; /* stack marker: back to the top level */

NB_D TraceResult trace_closest_tl(const DevScene &sc, V3 o, V3 d, uint64_t *node_visits = nullptr,
                                  uint64_t *tri_tests = nullptr) {
  TraceResult r{-1, 0.f, 0.f, 0.f, 0u};
  float tmax = FLT_MAX;
  V3 ro = o, rd = d;
  float ix = safe_rcp(d.x), iy = safe_rcp(d.y), iz = safe_rcp(d.z);
  int32_t stack[kTraversalStack];
  int sp = 0;
  int32_t cur = 0;
  uint32_t prim_base = 0, inst_in = 0;
#if NB_LEAF_STEP
  uint32_t lk = 0, le = 0; /* the current bottom-level leaf's next and end triangle */
#endif
  bool inside = false;
  uint32_t nv = 0, tt = 0;
  for (;;) {
    if (cur >= 0) {
      nv++;
      const float4 n0 = __ldg(&sc.nodes[4 * cur + 0]);
      const float4 n1 = __ldg(&sc.nodes[4 * cur + 1]);
      const float4 n2 = __ldg(&sc.nodes[4 * cur + 2]);
      const float4 n3 = __ldg(&sc.nodes[4 * cur + 3]);
      float a0 = (n0.x - ro.x) * ix, b0 = (n0.y - ro.x) * ix;
      float a1 = (n0.z - ro.y) * iy, b1 = (n0.w - ro.y) * iy;
      float a2 = (n2.x - ro.z) * iz, b2 = (n2.y - ro.z) * iz;
      float c0n = fmaxf(fmaxf(fminf(a0, b0), fminf(a1, b1)), fmaxf(fminf(a2, b2), 0.f));
      float c0f = fminf(fminf(fminf(fmaxf(a0, b0), fmaxf(a1, b1)), fmaxf(a2, b2)) * kFarScale, tmax);
      float d0 = (n1.x - ro.x) * ix, e0 = (n1.y - ro.x) * ix;
      float d1 = (n1.z - ro.y) * iy, e1 = (n1.w - ro.y) * iy;
      float d2 = (n2.z - ro.z) * iz, e2 = (n2.w - ro.z) * iz;
      float c1n = fmaxf(fmaxf(fminf(d0, e0), fminf(d1, e1)), fmaxf(fminf(d2, e2), 0.f));
      float c1f = fminf(fminf(fminf(fmaxf(d0, e0), fmaxf(d1, e1)), fmaxf(d2, e2)) * kFarScale, tmax);
      const bool h0 = c0n <= c0f, h1 = c1n <= c1f;
      const int32_t r0 = __float_as_int(n3.x), r1 = __float_as_int(n3.y);
      if (h0 && h1) {
        int32_t first = r0, second = r1;
        if (c1n < c0n) {
          first = r1;
          second = r0;
        }
        if (sp < kTraversalStack) stack[sp++] = second;
        cur = first;
        continue;
      } else if (h0) {
        cur = r0;
        continue;
      } else if (h1) {
        cur = r1;
        continue;
      }
    } else if (!inside) { /* top-level leaf: enter the instance */
      const DevInstance &I = sc.instances[leaf_first(cur)];
      if (!I.identity) {
        ro = xform_point(I.inv, o);
        rd = xform_dir(I.inv, d);
        ix = safe_rcp(rd.x), iy = safe_rcp(rd.y), iz = safe_rcp(rd.z);
      }
      prim_base = I.prim_offset;
      inst_in = leaf_first(cur);
      inside = true;
      if (sp < kTraversalStack) stack[sp++] = kLeaveInstance;
      cur = (int32_t)sc.blas_root[I.mesh];
      continue;
    } else { /* bottom-level leaf: object-space triangles, mesh-local ids */
#if NB_LEAF_STEP
      if (lk >= le) {
        lk = leaf_first(cur);
        le = lk + leaf_count(cur);
      }
      {
        const uint32_t k = lk++;
#else
      const uint32_t first = leaf_first(cur), count = leaf_count(cur);
      for (uint32_t k = first; k < first + count; k++) {
#endif
        const float4 t0 = __ldg(&sc.tris[3 * k + 0]);
        const float4 t1 = __ldg(&sc.tris[3 * k + 1]);
        const float4 t2 = __ldg(&sc.tris[3 * k + 2]);
        tt++;
        float ht, hu, hv;
        if (mt_hit(ro, rd, V3{t0.x, t0.y, t0.z}, V3{t1.x, t1.y, t1.z}, V3{t2.x, t2.y, t2.z}, kRayTNear, tmax, ht, hu,
                   hv)) {
          tmax = ht;
          r.prim = (int32_t)(prim_base + (uint32_t)__float_as_int(t0.w));
          r.inst = inst_in;
          r.t = ht;
          r.u = hu;
          r.v = hv;
        }
      }
#if NB_LEAF_STEP
      if (lk < le) continue;
#endif
    }
    /* pop; the marker returns the walk to the top level and the world ray */
    for (;;) {
      if (sp == 0) {
        if (node_visits) *node_visits += nv;
        if (tri_tests) *tri_tests += tt;
        return r;
      }
      cur = stack[--sp];
      if (cur != kLeaveInstance) break;
      inside = false;
      ro = o;
      rd = d;
      ix = safe_rcp(d.x), iy = safe_rcp(d.y), iz = safe_rcp(d.z);
    }
  }
}

template <int WIDTH>
NB_D TraceResult trace_closest_w(const DevScene &sc, V3 o, V3 d, uint64_t *node_visits = nullptr,
                                 uint64_t *tri_tests = nullptr) {
  if constexpr (WIDTH == 8)
    return trace_closest8(sc, o, d, node_visits, tri_tests);
  else if constexpr (WIDTH == 1)
    return trace_closest_tl(sc, o, d, node_visits, tri_tests);
  else
    return trace_closest2(sc, o, d, node_visits, tri_tests);
}

NB_D TraceResult trace_closest(const DevScene &sc, V3 o, V3 d) {
  return sc.width == 8 ? trace_closest8(sc, o, d) : sc.width == 1 ? trace_closest_tl(sc, o, d) : trace_closest2(sc, o, d);
}

}  // namespace nb
