/* ORACLE — test infrastructure only (see oracle.h).
 *
 * The reference's native binary SAH BVH and its traversal:
 *   build      corelib/nova/aggregate/native/BvhBuilder.cpp:48-253 (PERFORMANCE = 4 candidates per axis,
 *              selected by native.cpp:25-27),
 *   traversal  corelib/nova/aggregate/native/native.cpp:56-114 with the slab test of
 *              corelib/internal/geometry/BoundingBox.cpp:150-160,
 *   triangle   corelib/nova/shape/Triangle.h:127-213 (Moller-Trumbore in object space).
 */
#include "oracle_internal.h"
#include <algorithm>
#include <climits>
#include <utility>

namespace orc {

/* Triangle::computeAABB / centroid (Triangle.h:99-114; compute_center Object3D.h:194-199). */
void prim_bounds(const Scene &s, const Prim &p, Box &box, V3 &centroid) {
  const Mesh &m = s.meshes[s.inst_mesh[p.inst]];
  const Xform &x = s.xf[p.inst];
  const uint32_t *id = &m.idx[3 * p.tri];
  V3 v[3];
  for (int k = 0; k < 3; k++) v[k] = {m.v[3 * id[k]], m.v[3 * id[k] + 1], m.v[3 * id[k] + 2]};
  V3 w[3];
  for (int k = 0; k < 3; k++) w[k] = xyz(mul(x.m, V4{v[k].x, v[k].y, v[k].z, 1.f}));
  box.mn = vmin(w[0], vmin(w[1], w[2]));
  box.mx = vmax(w[0], vmax(w[1], w[2]));
  V3 c{(v[0].x + v[1].x + v[2].x) * 0.333333f, (v[0].y + v[1].y + v[2].y) * 0.333333f,
       (v[0].z + v[1].z + v[2].z) * 0.333333f};
  centroid = xyz(mul(x.m, V4{c.x, c.y, c.z, 1.f}));
}

namespace {

struct Cache {
  std::vector<Box> aabbs;
  std::vector<V3> centroids;
};

/* update_aabb, BvhBuilder.cpp:77-99: starts from (INT_MAX, INT_MIN) and unions the prims. */
void update_aabb(const Cache &c, Scene &s, int32_t node_id) {
  Node &node = s.nodes[node_id];
  Box nb{v3((float)INT_MAX), v3((float)INT_MIN)};
  for (int32_t i = 0; i < node.count; i++) {
    nb = nb + c.aabbs[s.prim_idx[i + node.left]];
    node.min[0] = nb.mn.x, node.min[1] = nb.mn.y, node.min[2] = nb.mn.z;
    node.max[0] = nb.mx.x, node.max[1] = nb.mx.y, node.max[2] = nb.mx.z;
  }
}

/* eval_sah, BvhBuilder.cpp:114-137.  An empty side has an infinite half area; inf * 0 is NaN and
 * "cost > 0 ? cost : INT_MAX" maps it to INT_MAX, exactly as in the reference. */
float eval_sah(const Cache &c, const Scene &s, const Node &node, int axis, float pos) {
  Box l, r;
  int nl = 0, nr = 0;
  for (int32_t i = 0; i < node.count; i++) {
    int32_t p = s.prim_idx[i + node.left];
    if (c.centroids[p][axis] < pos) {
      nl++;
      l = l + c.aabbs[p];
    } else {
      nr++;
      r = r + c.aabbs[p];
    }
  }
  const float cost = l.half_area() * (float)nl + r.half_area() * (float)nr;
  return cost > 0.f ? cost : (float)INT_MAX;
}

int axis_subdiv_sah(const Cache &c, const Scene &s, int32_t node_id, float &best_cost_r, float split[3]) {
  const unsigned SEGMENT_COUNT = 4;
  int best_axis = 0;
  float best_position = 0.f;
  float best_cost = (float)INT_MAX;
  const Node &node = s.nodes[node_id];
  for (int axis = 0; axis < 3; axis++) {
    const float bmin = node.min[axis], bmax = node.max[axis];
    float dist = bmax - bmin;
    if (dist == 0) continue;
    float seg = dist / (float)SEGMENT_COUNT;
    for (unsigned i = 0; i < SEGMENT_COUNT; i++) {
      float cand = seg * (float)i + bmin;
      const float cost = eval_sah(c, s, node, axis, cand);
      if (cost < best_cost) {
        best_cost = cost;
        best_axis = axis;
        best_position = cand;
      }
    }
  }
  split[best_axis] = best_position;
  best_cost_r = best_cost;
  return best_axis;
}

/* create_nodes, BvhBuilder.cpp:186-203: in-place partition with swaps from the back. */
int32_t create_nodes(const Cache &c, std::vector<int32_t> &pidx, const Node &node, const float split[3], int axis) {
  int32_t i = node.left;
  int32_t j = i + node.count - 1;
  while (i <= j) {
    int32_t p = pidx[i];
    float cen = c.centroids[p][axis];
    if (cen < split[axis])
      i++;
    else
      std::swap(pidx[i], pidx[j--]);
  }
  return i;
}

/* subdivide, BvhBuilder.cpp:205-253, as a pre-order walk with an explicit stack (same node order
 * as the recursion: left subtree completely before right). */
void subdivide_all(const Cache &c, Scene &s) {
  std::vector<int32_t> stack{0};
  while (!stack.empty()) {
    int32_t node_id = stack.back();
    stack.pop_back();
    float split[3] = {0.f, 0.f, 0.f};
    float best_cost = 0.f;
    int axis = axis_subdiv_sah(c, s, node_id, best_cost, split);
    Node &node = s.nodes[node_id];
    Box nb{{node.min[0], node.min[1], node.min[2]}, {node.max[0], node.max[1], node.max[2]}};
    const float cost = nb.half_area() * (float)node.count;
    if (best_cost >= cost) continue;
    int32_t i = create_nodes(c, s.prim_idx, node, split, axis);
    int32_t left_count = i - node.left;
    if (left_count == 0 || left_count == node.count) continue;
    int32_t li = s.nodes_used++;
    int32_t ri = s.nodes_used++;
    s.nodes[li].left = node.left;
    s.nodes[li].count = left_count;
    s.nodes[ri].left = i;
    s.nodes[ri].count = node.count - left_count;
    s.nodes[node_id].count = 0;
    s.nodes[node_id].left = li;
    update_aabb(c, s, li);
    update_aabb(c, s, ri);
    stack.push_back(ri);
    stack.push_back(li);
  }
}

/* BoundingBox::intersect(dir, origin, dist_min), BoundingBox.cpp:150-160, with std::min/std::max. */
inline float box_intersect(const Node &n, const V3 &d, const V3 &o, float dist_min) {
  float tx1 = (n.min[0] - o.x) / d.x, tx2 = (n.max[0] - o.x) / d.x;
  float tmin = std::min(tx1, tx2), tmax = std::max(tx1, tx2);
  float ty1 = (n.min[1] - o.y) / d.y, ty2 = (n.max[1] - o.y) / d.y;
  tmin = std::max(tmin, std::min(ty1, ty2)), tmax = std::min(tmax, std::max(ty1, ty2));
  float tz1 = (n.min[2] - o.z) / d.z, tz2 = (n.max[2] - o.z) / d.z;
  tmin = std::max(tmin, std::min(tz1, tz2)), tmax = std::min(tmax, std::max(tz1, tz2));
  if (tmax >= tmin && tmax > 0 && tmin <= dist_min) return tmin;
  return kMaxFloat;
}

}  // namespace

void build_bvh(Scene &s) {
  const size_t n = s.prims.size();
  Cache c;
  c.aabbs.resize(n);
  c.centroids.resize(n);
  for (size_t i = 0; i < n; i++) prim_bounds(s, s.prims[i], c.aabbs[i], c.centroids[i]);
  s.nodes.assign(2 * n - 1, Node{{0, 0, 0}, {0, 0, 0}, 0, 0});
  s.prim_idx.resize(n);
  for (size_t i = 0; i < n; i++) s.prim_idx[i] = (int32_t)i;
  s.nodes[0].left = 0;
  s.nodes[0].count = (int32_t)n;
  update_aabb(c, s, 0);
  s.nodes_used = 1;
  subdivide_all(c, s);
}

/* Triangle::hit's intersection (Triangle.h:150-177): ray to object space through the inverse
 * transform, Moller-Trumbore with inv_det computed before the det == 0 test; edges inclusive; no
 * culling. */
bool moller_trumbore(const M4 &inv, V3 v0, V3 v1, V3 v2, const Ray &in, float tmin, float tmax, float &t_out,
                     float &u_out, float &v_out) {
  const V3 o = xyz(mul(inv, V4{in.o.x, in.o.y, in.o.z, 1.f}));
  const V3 d = xyz(mul(inv, V4{in.d.x, in.d.y, in.d.z, 0.f}));
  const V3 e1 = v1 - v0, e2 = v2 - v0;
  const V3 P = cross(d, e2);
  const float det = dot(P, e1);
  const float inv_det = 1.f / det;
  if (det == 0.f) return false;
  const V3 T = o - v0;
  const float u = dot(P, T) * inv_det;
  if (u < 0 || u > 1.f) return false;
  const V3 Q = cross(T, e1);
  const float v = dot(Q, d) * inv_det;
  if (v < 0.f || (u + v) > 1.f) return false;
  float t = dot(Q, e2) * inv_det;
  if (t < tmin || t > tmax) return false;
  t_out = t;
  u_out = u;
  v_out = v;
  return true;
}

/* Triangle::hit (Triangle.h:146-177): degenerate check (isDegenerate, :127-132), then the
 * intersection above. */
bool triangle_hit(const Scene &s, const Prim &p, const Ray &in, float tmin, float tmax, float &t_out, float &u_out,
                  float &v_out) {
  const Mesh &m = s.meshes[s.inst_mesh[p.inst]];
  const uint32_t *id = &m.idx[3 * p.tri];
  if (id[0] == id[1] || id[2] == id[1] || id[2] == id[0]) return false;
  const Xform &x = s.xf[p.inst];
  const V3 v0{m.v[3 * id[0]], m.v[3 * id[0] + 1], m.v[3 * id[0] + 2]};
  const V3 v1{m.v[3 * id[1]], m.v[3 * id[1] + 1], m.v[3 * id[1] + 2]};
  const V3 v2{m.v[3 * id[2]], m.v[3 * id[2] + 1], m.v[3 * id[2] + 2]};
  return moller_trumbore(x.inv, v0, v1, v2, in, tmin, tmax, t_out, u_out, v_out);
}

/* iter_traverse, native.cpp:56-114.  Stack of 2048 node pointers; both children slab-tested;
 * nearer pushed last; leaf prims accepted when t <= current tmax (later equal t wins). */
Hit trace(const Scene &s, const Ray &r, TraceCounters *cnt) {
  Hit h;
  constexpr int MAX_STACK = 2048;
  float tmax = kMaxFloat;
  const Node *stack[MAX_STACK];
  stack[0] = &s.nodes[0];
  int top = 0;
  uint64_t nodes = 0, tris = 0;
  while (top != -1) {
    const Node *it = stack[top--];
    if (it->count == 0) {
      nodes++;
      const Node *left = &s.nodes[it->left];
      const Node *right = &s.nodes[it->left + 1];
      float li = box_intersect(*left, r.d, r.o, tmax);
      float ri = box_intersect(*right, r.d, r.o, tmax);
      if (li > ri) {
        std::swap(li, ri);
        std::swap(left, right);
      }
      if (li == kMaxFloat) continue;
      if (ri == kMaxFloat) {
        if (top + 1 < MAX_STACK && top + 1 < MAX_STACK) stack[++top] = left;
        continue;
      }
      if (top + 1 < MAX_STACK) stack[++top] = right;
      if (top + 1 < MAX_STACK) stack[++top] = left;
    }
    if (it->count == 0) continue;
    for (int32_t i = 0; i < it->count; i++) {
      int32_t pidx = s.prim_idx[it->left + i];
      tris++;
      float t, u, v;
      if (!triangle_hit(s, s.prims[pidx], r, r.tnear, tmax, t, u, v)) continue;
      h.is_hit = true;
      if (t <= tmax) {
        h.prim = pidx;
        h.t = t;
        h.u = u;
        h.v = v;
        tmax = t;
      }
    }
  }
  if (cnt) {
    cnt->nodes += nodes;
    cnt->tris += tris;
  }
  return h;
}

}  // namespace orc

/* The traversal's slab test on one box (property tests): the entry distance of the ray (o, d) when
 * it meets [mn, mx] no farther than dist_min, else MAXFLOAT. */
extern "C" float orc_box_intersect(const float mn[3], const float mx[3], const float o[3], const float d[3],
                                   float dist_min) {
  orc::Node n{{mn[0], mn[1], mn[2]}, {mx[0], mx[1], mx[2]}, 0, 0};
  return orc::box_intersect(n, orc::V3{d[0], d[1], d[2]}, orc::V3{o[0], o[1], o[2]}, dist_min);
}
