/* Collapse of the binary SAH BVH into the compressed 8-wide layout (bvh_wide.cuh), on the device.
 *
 * Level-synchronous top-down pass, one thread per wide node: starting from the binary node's two
 * children, the inner child with the largest surface area is replaced by its own two children
 * until eight children are gathered or only leaves remain; children are assigned to slots by
 * their centroid direction (greedy, most aligned first); the node box is quantised to 8 bits per
 * plane against per-axis power-of-two scales (rounded outwards, so decoded boxes contain the
 * exact ones); inner children get consecutive node indices and leaf triangles consecutive records
 * (atomics), both in slot order.  Children are always allocated after their parent, so every
 * child index exceeds its parent's and traversal cannot cycle.
 */
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <vector>

#include "bvh_wide.cuh"
#include "traverse.cuh"

namespace nb {
namespace {

struct WTask {
  uint32_t node2, wnode, depth;
};

struct Child {
  int32_t ref;
  float lo[3], hi[3];
};

__device__ __forceinline__ float child_half_area(const Child &c) {
  float dx = c.hi[0] - c.lo[0], dy = c.hi[1] - c.lo[1], dz = c.hi[2] - c.lo[2];
  return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ void read_children(const float4 *nodes2, uint32_t node, Child out[2], int &n) {
  const float *f = reinterpret_cast<const float *>(nodes2 + 4 * (size_t)node);
  const int32_t *r = reinterpret_cast<const int32_t *>(nodes2 + 4 * (size_t)node);
  n = 0;
  for (int s = 0; s < 2; s++) {
    Child c;
    c.ref = r[12 + s];
    c.lo[0] = f[4 * s + 0], c.hi[0] = f[4 * s + 1];
    c.lo[1] = f[4 * s + 2], c.hi[1] = f[4 * s + 3];
    c.lo[2] = f[8 + 2 * s], c.hi[2] = f[9 + 2 * s];
    if (c.lo[0] <= c.hi[0] && c.lo[1] <= c.hi[1] && c.lo[2] <= c.hi[2]) out[n++] = c; /* skip empty boxes */
  }
}

/* Smallest power-of-two scale 2^k with 255 * 2^k >= hi - lo (checked in double), as a biased
 * exponent k + 127 in 1..254. */
__device__ __forceinline__ uint32_t scale_exponent(float lo, float hi) {
  const double ext = (double)hi - (double)lo;
  if (!(ext > 0.0)) return 1u;
  int k = ilogb(ext / 255.0);
  while (ldexp(255.0, k) < ext) k++;
  k = k < -126 ? -126 : (k > 127 ? 127 : k);
  return (uint32_t)(k + 127);
}

__global__ void k_collapse(const float4 *nodes2, const float4 *tris2, const WTask *tasks, uint32_t n_tasks,
                           float4 *wnodes, float4 *tris_out, unsigned *counters, WTask *next) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= n_tasks) return;
  const WTask t = tasks[tid];
  Child ch[8];
  int n = 0;
  {
    Child two[2];
    int m;
    read_children(nodes2, t.node2, two, m);
    for (int k = 0; k < m; k++) ch[n++] = two[k];
  }
  while (n < 8) {
    int best = -1;
    float best_area = -1.f;
    for (int j = 0; j < n; j++)
      if (ch[j].ref >= 0) {
        float a = child_half_area(ch[j]);
        if (a > best_area) best_area = a, best = j;
      }
    if (best < 0) break;
    Child two[2];
    int m;
    read_children(nodes2, (uint32_t)ch[best].ref, two, m);
    if (m == 0) { /* an inner node without children cannot occur in a validated tree */
      atomicAdd(counters + 3, 1u);
      return;
    }
    ch[best] = two[0];
    if (m == 2) ch[n++] = two[1];
  }
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int j = 0; j < n; j++)
    for (int k = 0; k < 3; k++) lo[k] = fminf(lo[k], ch[j].lo[k]), hi[k] = fmaxf(hi[k], ch[j].hi[k]);
  /* greedy slot assignment by centroid direction */
  int slot_child[8];
  for (int s = 0; s < 8; s++) slot_child[s] = -1;
  {
    float cx[8], cy[8], cz[8];
    const float mx = 0.5f * (lo[0] + hi[0]), my = 0.5f * (lo[1] + hi[1]), mz = 0.5f * (lo[2] + hi[2]);
    for (int j = 0; j < n; j++) {
      cx[j] = 0.5f * (ch[j].lo[0] + ch[j].hi[0]) - mx;
      cy[j] = 0.5f * (ch[j].lo[1] + ch[j].hi[1]) - my;
      cz[j] = 0.5f * (ch[j].lo[2] + ch[j].hi[2]) - mz;
    }
    unsigned child_done = 0, slot_used = 0;
    for (int it = 0; it < n; it++) {
      float best = -FLT_MAX;
      int bj = -1, bs = -1;
      for (int j = 0; j < n; j++) {
        if (child_done & (1u << j)) continue;
        for (int s = 0; s < 8; s++) {
          if (slot_used & (1u << s)) continue;
          const float v = ((s & 1) ? cx[j] : -cx[j]) + ((s & 2) ? cy[j] : -cy[j]) + ((s & 4) ? cz[j] : -cz[j]);
          if (v > best) best = v, bj = j, bs = s;
        }
      }
      child_done |= 1u << bj;
      slot_used |= 1u << bs;
      slot_child[bs] = bj;
    }
  }
  /* quantisation */
  uint32_t ebias[3];
  float scale[3];
  for (int k = 0; k < 3; k++) {
    ebias[k] = scale_exponent(lo[k], hi[k]);
    scale[k] = __uint_as_float(ebias[k] << 23);
  }
  uint32_t qlo[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qhi[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  uint32_t meta[2] = {0, 0};
  uint32_t imask = 0, n_inner = 0, n_tri = 0;
  uint32_t leaf_first_[8], leaf_cnt[8], leaf_off[8];
  for (int s = 0; s < 8; s++) {
    const int j = slot_child[s];
    const int w = s >> 2, sh = 8 * (s & 3);
    if (j < 0) {
      for (int k = 0; k < 3; k++) qlo[k][w] |= 255u << sh;
      leaf_cnt[s] = 0;
      continue;
    }
    for (int k = 0; k < 3; k++) {
      const double p = (double)lo[k], sc = (double)scale[k];
      double a = floor(((double)ch[j].lo[k] - p) / sc);
      double b = ceil(((double)ch[j].hi[k] - p) / sc);
      while (a > 0 && p + a * sc > (double)ch[j].lo[k]) a -= 1;
      while (b < 255 && p + b * sc < (double)ch[j].hi[k]) b += 1;
      a = a < 0 ? 0 : (a > 255 ? 255 : a);
      b = b < 0 ? 0 : (b > 255 ? 255 : b);
      qlo[k][w] |= (uint32_t)a << sh;
      qhi[k][w] |= (uint32_t)b << sh;
    }
    if (ch[j].ref >= 0) {
      imask |= 1u << s;
      n_inner++;
      leaf_cnt[s] = 0;
    } else {
      const uint32_t cnt = leaf_count(ch[j].ref);
      if (cnt > (uint32_t)kWideLeafMax) atomicAdd(counters + 3, 1u);
      leaf_first_[s] = leaf_first(ch[j].ref);
      leaf_cnt[s] = cnt;
      leaf_off[s] = n_tri;
      meta[w] |= ((n_tri & 31u) | ((cnt - 1u) << 5)) << sh;
      n_tri += cnt;
    }
  }
  const uint32_t child_base = n_inner ? atomicAdd(counters + 0, n_inner) : 0u;
  const uint32_t tri_base = n_tri ? atomicAdd(counters + 1, n_tri) : 0u;
  float4 *wn = wnodes + 5 * (size_t)t.wnode;
  wn[0] = make_float4(lo[0], lo[1], lo[2], __uint_as_float(ebias[0] | (ebias[1] << 8) | (ebias[2] << 16) | (imask << 24)));
  wn[1] = make_float4(__uint_as_float(child_base), __uint_as_float(tri_base), __uint_as_float(meta[0]),
                      __uint_as_float(meta[1]));
  wn[2] = make_float4(__uint_as_float(qlo[0][0]), __uint_as_float(qlo[0][1]), __uint_as_float(qlo[1][0]),
                      __uint_as_float(qlo[1][1]));
  wn[3] = make_float4(__uint_as_float(qlo[2][0]), __uint_as_float(qlo[2][1]), __uint_as_float(qhi[0][0]),
                      __uint_as_float(qhi[0][1]));
  wn[4] = make_float4(__uint_as_float(qhi[1][0]), __uint_as_float(qhi[1][1]), __uint_as_float(qhi[2][0]),
                      __uint_as_float(qhi[2][1]));
  if (n_inner) {
    const uint32_t q = atomicAdd(counters + 2, n_inner);
    uint32_t rank = 0;
    for (int s = 0; s < 8; s++)
      if (imask & (1u << s)) {
        next[q + rank] = WTask{(uint32_t)ch[slot_child[s]].ref, child_base + rank, t.depth + 1};
        rank++;
      }
  }
  for (int s = 0; s < 8; s++)
    for (uint32_t k = 0; k < leaf_cnt[s]; k++) {
      const size_t src = 3 * (size_t)(leaf_first_[s] + k), dst = 3 * (size_t)(tri_base + leaf_off[s] + k);
      tris_out[dst] = tris2[src];
      tris_out[dst + 1] = tris2[src + 1];
      tris_out[dst + 2] = tris2[src + 2];
    }
  atomicMax(reinterpret_cast<int *>(counters + 4), (int)t.depth);
}

}  // namespace

cudaError_t build_wide_bvh(const float4 *nodes2, uint32_t n_nodes2, const float4 *tris2, uint32_t n_tris,
                           float4 *wnodes, float4 *tris_out, cudaStream_t stream, WideBuildResult *res) {
  auto t0 = std::chrono::steady_clock::now();
  WTask *qa = nullptr, *qb = nullptr;
  unsigned *counters = nullptr;
  cudaError_t err = cudaSuccess;
  unsigned h[5] = {1u, 0u, 0u, 0u, 0u};
  uint32_t n_level = 1;
#define NB_TRY(x)                         \
  do {                                    \
    err = (x);                            \
    if (err != cudaSuccess) goto cleanup; \
  } while (0)
  NB_TRY(cudaMallocAsync(&qa, sizeof(WTask) * (n_nodes2 + 1), stream));
  NB_TRY(cudaMallocAsync(&qb, sizeof(WTask) * (n_nodes2 + 1), stream));
  NB_TRY(cudaMallocAsync(&counters, sizeof(unsigned) * 5, stream));
  NB_TRY(cudaMemcpyAsync(counters, h, sizeof(h), cudaMemcpyHostToDevice, stream));
  {
    const WTask root{0u, 0u, 0u};
    NB_TRY(cudaMemcpyAsync(qa, &root, sizeof(WTask), cudaMemcpyHostToDevice, stream));
  }
  while (n_level) {
    NB_TRY(cudaMemsetAsync(counters + 2, 0, sizeof(unsigned), stream));
    k_collapse<<<(n_level + 127) / 128, 128, 0, stream>>>(nodes2, tris2, qa, n_level, wnodes, tris_out, counters, qb);
    NB_TRY(cudaGetLastError());
    NB_TRY(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, stream));
    NB_TRY(cudaStreamSynchronize(stream));
    if (h[3] != 0 || h[0] > n_nodes2 + 1) {
      err = cudaErrorUnknown; /* malformed input tree: reported as a build failure */
      goto cleanup;
    }
    n_level = h[2];
    std::swap(qa, qb);
  }
  if (h[1] != n_tris) err = cudaErrorUnknown;
  if (res) {
    res->n_nodes = h[0];
    res->n_tris = h[1];
    res->depth = (int)h[4];
  }
cleanup:
  cudaFreeAsync(qa, stream);
  cudaFreeAsync(qb, stream);
  cudaFreeAsync(counters, stream);
  cudaStreamSynchronize(stream);
#undef NB_TRY
  if (res) res->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return err;
}

}  // namespace nb
