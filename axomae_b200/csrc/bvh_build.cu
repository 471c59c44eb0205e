/* On-device binned-SAH BVH build.
 *
 * The reference builds its binary SAH BVH on one CPU thread (aggregate/native/BvhBuilder.cpp:48-253,
 * four candidate planes per axis, one O(n) pass per candidate) and its OptiX path hands the
 * build to the driver (aggregate/api/optix/host.cpp:440-480).  Here the build runs on the GPU,
 * top-down and breadth-first, with centroid binning:
 *
 *   large nodes (> small_task primitives), one level per host iteration:
 *     k_init_level   reset per-node centroid bounds and bins
 *     k_cbounds      centroid bounds, one CTA per chunk of kChunk (1024) primitives, merged with atomics
 *     k_bin          centroid bins per axis in shared memory, merged into the node's global bins
 *     k_split        one CTA per node: SAH over bins*3 candidate planes, node allocation, children
 *     k_partition    primitive ids scattered to the children's ranges of the other id buffer
 *     k_make_chunks  the next level's chunk list (the host reads back only the task and chunk counts)
 *   small nodes (<= small_task): k_build_small, one CTA per node builds its whole subtree with a
 *     CTA-local task stack, shared-memory bins and a stable block-scan partition; nodes of at most
 *     32 primitives are handed to single warps (exact sweep SAH over sorted centroids, no barriers).
 *
 * Leaves list their primitives in a contiguous range of `order`; each leaf's range is finally
 * sorted by primitive index so the layout is deterministic (atomics only reorder primitives
 * inside a node's range, and SAH decisions depend on the set of primitives, not their order).
 * Child boxes are padded outwards by 2^-20 relative so transformed-instance boxes stay
 * conservative.  Below depth kMedianDepth nodes are split at their median position, which bounds
 * the depth (and the traversal stack) for any input.
 */
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <vector>

#include "bvh_build.cuh"
#include "traverse.cuh"

namespace nb {
namespace {

constexpr int kMaxBins = 32;
constexpr uint32_t kSmallTaskDefault = 256;
/* Primitives per CTA in the level kernels: the top levels of a scene have few large nodes, so
 * smaller chunks put more CTAs on the GPU.  32 batch scenes: 4096 -> 57.5 ms build_batch, 116.6 ms
 * one after another; 1024 -> 55.4 / 100.7 ms; 512 -> 54.6 / 99.1 ms; 256 -> 55.9 / 101.1 ms.  The
 * tree does not depend on it. */
#ifndef NB_BUILD_CHUNK
#define NB_BUILD_CHUNK 1024
#endif
constexpr uint32_t kChunk = NB_BUILD_CHUNK;
constexpr int kMedianDepth = 40;
constexpr int kBlock = 256;
/* Threads of a subtree CTA (a subtree of <= small_task primitives needs few per node).  128: 72
 * registers and 28.5 KB of shared memory, 7 CTAs = 28 warps per SM; 64 held 9 CTAs = 18 warps (93
 * registers, 23.8 KB).  32 batch scenes 26.3 -> 25.6 ms concurrent, heightfield 5.0 -> 4.8 ms, same
 * trees. */
constexpr int kSmallBlock = 128;
constexpr int kHardLeaf = 16;
constexpr int kSmallStack = 64;

struct Task {
  uint32_t begin, end;
  int32_t parent, slot, depth, buf;
  float lo[3], hi[3];
};

struct Bins {
  unsigned cnt[3][kMaxBins];
  float lo[3][kMaxBins][3];
  float hi[3][kMaxBins][3];
};

struct SplitInfo {
  int axis, bin, median;
  uint32_t mid;
  unsigned left_ptr, right_ptr;
  float cmin[3], scale[3];
};

struct Chunk {
  uint32_t task, begin, end;
};

struct Shared {
  const float4 *lo, *hi;
  uint32_t *ids0, *ids1;
  float4 *nodes;
  uint32_t *order;
  unsigned *node_counter;
  Task *large_next;
  unsigned *large_next_count;
  Task *small;
  unsigned *small_count;
  uint2 *leaves;
  unsigned *leaf_count;
  int *max_depth;
  int bins, max_leaf, hard_leaf;
  uint32_t small_task;
  float cost_trav;
};

__device__ __forceinline__ uint32_t *ids_of(const Shared &s, int buf) { return buf ? s.ids1 : s.ids0; }

__device__ __forceinline__ void atomic_min_f(float *a, float v) {
  if (v >= 0.f)
    atomicMin(reinterpret_cast<int *>(a), __float_as_int(v));
  else
    atomicMax(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float *a, float v) {
  if (v >= 0.f)
    atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
  else
    atomicMin(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}

/* Adds each valid lane's primitive (box bl, bh) to bin b of one axis's shared bins.  When every lane
 * of the warp falls in the same bin (neighbouring primitives of a large node often do) the warp
 * reduces first and one lane adds, instead of 32 same-address atomics that execute one after the
 * other.  Counts, minima and maxima are exact, so the bins are the same either way.  All 32 lanes
 * call it. */
__device__ __forceinline__ void bin_add(unsigned *cnt, float (*lo)[3], float (*hi)[3], int b, bool valid,
                                        const float4 &bl, const float4 &bh) {
  const unsigned same = __match_any_sync(0xffffffffu, valid ? b : -1);
  if (same == 0xffffffffu) {
    if (!valid) return; /* uniform: an invalid lane's -1 matches only other invalid lanes */
    float l0 = bl.x, l1 = bl.y, l2 = bl.z, h0 = bh.x, h1 = bh.y, h2 = bh.z;
    for (int o = 16; o > 0; o >>= 1) {
      l0 = fminf(l0, __shfl_xor_sync(0xffffffffu, l0, o)), l1 = fminf(l1, __shfl_xor_sync(0xffffffffu, l1, o));
      l2 = fminf(l2, __shfl_xor_sync(0xffffffffu, l2, o)), h0 = fmaxf(h0, __shfl_xor_sync(0xffffffffu, h0, o));
      h1 = fmaxf(h1, __shfl_xor_sync(0xffffffffu, h1, o)), h2 = fmaxf(h2, __shfl_xor_sync(0xffffffffu, h2, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&cnt[b], 32u);
      atomic_min_f(&lo[b][0], l0), atomic_min_f(&lo[b][1], l1), atomic_min_f(&lo[b][2], l2);
      atomic_max_f(&hi[b][0], h0), atomic_max_f(&hi[b][1], h1), atomic_max_f(&hi[b][2], h2);
    }
  } else if (valid) {
    atomicAdd(&cnt[b], 1u);
    atomic_min_f(&lo[b][0], bl.x), atomic_min_f(&lo[b][1], bl.y), atomic_min_f(&lo[b][2], bl.z);
    atomic_max_f(&hi[b][0], bh.x), atomic_max_f(&hi[b][1], bh.y), atomic_max_f(&hi[b][2], bh.z);
  }
}

__device__ __forceinline__ float3 centroid(const Shared &s, uint32_t i) {
  float4 a = __ldg(s.lo + i), b = __ldg(s.hi + i);
  return make_float3((a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f);
}
__device__ __forceinline__ float comp(float3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

__device__ __forceinline__ float half_area(const float lo[3], const float hi[3]) {
  float dx = fmaxf(hi[0] - lo[0], 0.f), dy = fmaxf(hi[1] - lo[1], 0.f), dz = fmaxf(hi[2] - lo[2], 0.f);
  return dx * dy + dy * dz + dz * dx;
}

/* Bin mapping shared by binning and partitioning (identical inputs give identical bins). */
__device__ __forceinline__ float bin_scale(float cmin, float cmax, int nb) {
  float ext = cmax - cmin;
  return ext > 0.f ? (float)nb * (1.f - 1e-6f) / ext : 0.f;
}
__device__ __forceinline__ int bin_of(float c, float cmin, float scale, int nb) {
  int b = (int)((c - cmin) * scale);
  return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

__device__ __forceinline__ float pad_lo(float x) { return x - (fabsf(x) * 9.5367431640625e-07f + 1e-30f); }
__device__ __forceinline__ float pad_hi(float x) { return x + (fabsf(x) * 9.5367431640625e-07f + 1e-30f); }

__device__ void write_child(float4 *nodes, int node, int slot, const float lo[3], const float hi[3]) {
  float *n = reinterpret_cast<float *>(nodes + 4 * node);
  const float lx = pad_lo(lo[0]), ly = pad_lo(lo[1]), lz = pad_lo(lo[2]);
  const float hx = pad_hi(hi[0]), hy = pad_hi(hi[1]), hz = pad_hi(hi[2]);
  if (slot == 0) {
    n[0] = lx, n[1] = hx, n[2] = ly, n[3] = hy;
    n[8] = lz, n[9] = hz;
  } else {
    n[4] = lx, n[5] = hx, n[6] = ly, n[7] = hy;
    n[10] = lz, n[11] = hz;
  }
}
__device__ void write_ref(float4 *nodes, int node, int slot, int32_t ref) {
  int32_t *n = reinterpret_cast<int32_t *>(nodes + 4 * node);
  n[12 + slot] = ref;
  n[14 + slot] = 0;
}

/* Thread 0 only: records a finished leaf (ids already copied into order[begin, end)). */
__device__ void finish_leaf(const Shared &s, const Task &t) {
  const uint32_t n = t.end - t.begin;
  const int32_t ref = leaf_ref(t.begin, n);
  if (t.parent < 0) { /* whole scene in one leaf: root with an empty second child */
    const float elo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ehi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    const int node = (int)atomicAdd(s.node_counter, 1u);
    write_child(s.nodes, node, 0, t.lo, t.hi);
    write_child(s.nodes, node, 1, elo, ehi);
    write_ref(s.nodes, node, 0, ref);
    write_ref(s.nodes, node, 1, ref);
  } else {
    write_ref(s.nodes, t.parent, t.slot, ref);
  }
  unsigned li = atomicAdd(s.leaf_count, 1u);
  s.leaves[li] = make_uint2(t.begin, n);
  atomicMax(s.max_depth, t.depth);
}

__device__ __forceinline__ void push_task(const Shared &s, const Task &t) {
  if (t.end - t.begin > s.small_task) {
    unsigned i = atomicAdd(s.large_next_count, 1u);
    s.large_next[i] = t;
  } else {
    unsigned i = atomicAdd(s.small_count, 1u);
    s.small[i] = t;
  }
}

/* ------------------------------------------------------------------ whole-scene box */

__global__ void k_scene_box(const float4 *lo, const float4 *hi, uint32_t n, float *out /* 6 */) {
  float l[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, h[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 a = lo[i], b = hi[i];
    l[0] = fminf(l[0], a.x), l[1] = fminf(l[1], a.y), l[2] = fminf(l[2], a.z);
    h[0] = fmaxf(h[0], b.x), h[1] = fmaxf(h[1], b.y), h[2] = fmaxf(h[2], b.z);
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; k++) {
      l[k] = fminf(l[k], __shfl_xor_sync(0xffffffffu, l[k], o));
      h[k] = fmaxf(h[k], __shfl_xor_sync(0xffffffffu, h[k], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) {
      atomic_min_f(out + k, l[k]);
      atomic_max_f(out + 3 + k, h[k]);
    }
}

__global__ void k_iota(uint32_t *ids, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ids[i] = i;
}

/* ------------------------------------------------------------------ large nodes */

__global__ void k_init_level(Bins *bins, float *cb, uint32_t n_tasks, int nb) {
  uint32_t t = blockIdx.x;
  if (t >= n_tasks) return;
  for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) {
    int a = i / nb, b = i % nb;
    bins[t].cnt[a][b] = 0u;
    for (int k = 0; k < 3; k++) {
      bins[t].lo[a][b][k] = FLT_MAX;
      bins[t].hi[a][b][k] = -FLT_MAX;
    }
  }
  if (threadIdx.x < 3) {
    cb[6 * t + threadIdx.x] = FLT_MAX;
    cb[6 * t + 3 + threadIdx.x] = -FLT_MAX;
  }
}

__device__ __forceinline__ void block_minmax3(float l[3], float h[3], float *sh /* 6 * 32 */) {
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; k++) {
      l[k] = fminf(l[k], __shfl_xor_sync(0xffffffffu, l[k], o));
      h[k] = fmaxf(h[k], __shfl_xor_sync(0xffffffffu, h[k], o));
    }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < 3; k++) {
      sh[k * 32 + w] = l[k];
      sh[(3 + k) * 32 + w] = h[k];
    }
  __syncthreads();
  for (int k = 0; k < 3; k++) {
    float a = FLT_MAX, b = -FLT_MAX;
    for (int j = 0; j < nw; j++) {
      a = fminf(a, sh[k * 32 + j]);
      b = fmaxf(b, sh[(3 + k) * 32 + j]);
    }
    l[k] = a;
    h[k] = b;
  }
  __syncthreads();
}

__global__ void k_cbounds(Shared s, const Task *tasks, const Chunk *chunks, float *cb) {
  __shared__ float sh[6 * 32];
  const Chunk c = chunks[blockIdx.x];
  const Task &t = tasks[c.task];
  const uint32_t *src = ids_of(s, t.buf);
  float l[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, h[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) {
    float3 p = centroid(s, src[i]);
    l[0] = fminf(l[0], p.x), l[1] = fminf(l[1], p.y), l[2] = fminf(l[2], p.z);
    h[0] = fmaxf(h[0], p.x), h[1] = fmaxf(h[1], p.y), h[2] = fmaxf(h[2], p.z);
  }
  block_minmax3(l, h, sh);
  if (threadIdx.x < 3) {
    atomic_min_f(cb + 6 * c.task + threadIdx.x, l[threadIdx.x]);
    atomic_max_f(cb + 6 * c.task + 3 + threadIdx.x, h[threadIdx.x]);
  }
}

__global__ void k_bin(Shared s, const Task *tasks, const Chunk *chunks, const float *cb, Bins *bins) {
  __shared__ unsigned scnt[3][kMaxBins];
  __shared__ float slo[3][kMaxBins][3], shi[3][kMaxBins][3];
  const int nb = s.bins;
  const Chunk c = chunks[blockIdx.x];
  const Task &t = tasks[c.task];
  const uint32_t *src = ids_of(s, t.buf);
  for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) {
    int a = i / nb, b = i % nb;
    scnt[a][b] = 0u;
    for (int k = 0; k < 3; k++) slo[a][b][k] = FLT_MAX, shi[a][b][k] = -FLT_MAX;
  }
  float cmin[3], scale[3];
  for (int a = 0; a < 3; a++) {
    cmin[a] = cb[6 * c.task + a];
    scale[a] = bin_scale(cmin[a], cb[6 * c.task + 3 + a], nb);
  }
  __syncthreads();
  for (uint32_t r0 = c.begin; r0 < c.end; r0 += blockDim.x) { /* whole warps: bin_add votes */
    const uint32_t i = r0 + threadIdx.x;
    const bool valid = i < c.end;
    float4 bl = make_float4(0.f, 0.f, 0.f, 0.f), bh = bl;
    if (valid) {
      const uint32_t id = src[i];
      bl = __ldg(s.lo + id), bh = __ldg(s.hi + id);
    }
    const float3 p = make_float3((bl.x + bh.x) * 0.5f, (bl.y + bh.y) * 0.5f, (bl.z + bh.z) * 0.5f);
    for (int a = 0; a < 3; a++)
      bin_add(scnt[a], slo[a], shi[a], bin_of(comp(p, a), cmin[a], scale[a], nb), valid, bl, bh);
  }
  __syncthreads();
  Bins &g = bins[c.task];
  for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) {
    int a = i / nb, b = i % nb;
    if (scnt[a][b] == 0u) continue;
    atomicAdd(&g.cnt[a][b], scnt[a][b]);
    for (int k = 0; k < 3; k++) {
      atomic_min_f(&g.lo[a][b][k], slo[a][b][k]);
      atomic_max_f(&g.hi[a][b][k], shi[a][b][k]);
    }
  }
}

/* SAH sweep over bins: best (cost, axis, plane) with a deterministic tie order. */
struct Best {
  float cost;
  int key; /* axis * kMaxBins + plane; planes 1..nb-1 */
};
__device__ __forceinline__ bool better(const Best &a, const Best &b) {
  return a.cost < b.cost || (a.cost == b.cost && a.key < b.key);
}

template <class CntF, class LoF, class HiF>
__device__ Best sah_best(int nb, float parent_area, float cost_trav, CntF cnt, LoF blo, HiF bhi) {
  Best best{FLT_MAX, 0x7fffffff};
  for (int cand = threadIdx.x; cand < 3 * (nb - 1); cand += blockDim.x) {
    const int a = cand / (nb - 1), plane = cand % (nb - 1) + 1;
    unsigned nl = 0, nr = 0;
    float ll[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lh[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float rl[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rh[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int b = 0; b < nb; b++) {
      unsigned c = cnt(a, b);
      if (!c) continue;
      if (b < plane) {
        nl += c;
        for (int k = 0; k < 3; k++) ll[k] = fminf(ll[k], blo(a, b, k)), lh[k] = fmaxf(lh[k], bhi(a, b, k));
      } else {
        nr += c;
        for (int k = 0; k < 3; k++) rl[k] = fminf(rl[k], blo(a, b, k)), rh[k] = fmaxf(rh[k], bhi(a, b, k));
      }
    }
    if (nl == 0 || nr == 0) continue;
    const float cost = cost_trav + (half_area(ll, lh) * (float)nl + half_area(rl, rh) * (float)nr) / parent_area;
    Best c{cost, a * kMaxBins + plane};
    if (better(c, best)) best = c;
  }
  return best;
}

__device__ Best block_best(Best b, Best *sh) {
  for (int o = 16; o > 0; o >>= 1) {
    Best q{__shfl_xor_sync(0xffffffffu, b.cost, o), __shfl_xor_sync(0xffffffffu, b.key, o)};
    if (better(q, b)) b = q;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = b;
  __syncthreads();
  Best r = sh[0];
  for (int j = 1; j < (int)(blockDim.x >> 5); j++)
    if (better(sh[j], r)) r = sh[j];
  __syncthreads();
  return r;
}

__global__ void k_split(Shared s, const Task *tasks, const float *cb, const Bins *bins, SplitInfo *splits) {
  __shared__ Best sh[kBlock / 32];
  const Task t = tasks[blockIdx.x];
  const Bins &B = bins[blockIdx.x];
  const int nb = s.bins;
  const float area = half_area(t.lo, t.hi);
  Best best{FLT_MAX, 0x7fffffff};
  if (area > 0.f && t.depth < kMedianDepth)
    best = sah_best(
        nb, area, s.cost_trav, [&](int a, int b) { return B.cnt[a][b]; },
        [&](int a, int b, int k) { return B.lo[a][b][k]; }, [&](int a, int b, int k) { return B.hi[a][b][k]; });
  best = block_best(best, sh);
  if (threadIdx.x != 0) return;
  SplitInfo sp;
  for (int a = 0; a < 3; a++) {
    sp.cmin[a] = cb[6 * blockIdx.x + a];
    sp.scale[a] = bin_scale(sp.cmin[a], cb[6 * blockIdx.x + 3 + a], nb);
  }
  float llo[3], lhi[3], rlo[3], rhi[3];
  const uint32_t n = t.end - t.begin;
  if (best.key != 0x7fffffff) {
    sp.median = 0;
    sp.axis = best.key / kMaxBins;
    sp.bin = best.key % kMaxBins - 1; /* left side: bins <= sp.bin */
    unsigned nl = 0;
    for (int k = 0; k < 3; k++) llo[k] = rlo[k] = FLT_MAX, lhi[k] = rhi[k] = -FLT_MAX;
    for (int b = 0; b < nb; b++) {
      const unsigned c = B.cnt[sp.axis][b];
      if (!c) continue;
      float *l = b <= sp.bin ? llo : rlo, *h = b <= sp.bin ? lhi : rhi;
      if (b <= sp.bin) nl += c;
      for (int k = 0; k < 3; k++) l[k] = fminf(l[k], B.lo[sp.axis][b][k]), h[k] = fmaxf(h[k], B.hi[sp.axis][b][k]);
    }
    sp.mid = t.begin + nl;
  } else {
    sp.median = 1;
    sp.axis = 0;
    sp.bin = 0;
    sp.mid = t.begin + n / 2;
    for (int k = 0; k < 3; k++) llo[k] = rlo[k] = t.lo[k], lhi[k] = rhi[k] = t.hi[k];
  }
  sp.left_ptr = t.begin;
  sp.right_ptr = sp.mid;
  splits[blockIdx.x] = sp;
  const int node = (int)atomicAdd(s.node_counter, 1u);
  if (t.parent >= 0) write_ref(s.nodes, t.parent, t.slot, node);
  write_child(s.nodes, node, 0, llo, lhi);
  write_child(s.nodes, node, 1, rlo, rhi);
  Task L{t.begin, sp.mid, node, 0, t.depth + 1, 1 - t.buf, {llo[0], llo[1], llo[2]}, {lhi[0], lhi[1], lhi[2]}};
  Task R{sp.mid, t.end, node, 1, t.depth + 1, 1 - t.buf, {rlo[0], rlo[1], rlo[2]}, {rhi[0], rhi[1], rhi[2]}};
  push_task(s, L);
  push_task(s, R);
}

__global__ void k_partition(Shared s, const Task *tasks, const Chunk *chunks, SplitInfo *splits) {
  __shared__ unsigned warp_l[kBlock / 32], warp_r[kBlock / 32];
  __shared__ unsigned base_l, base_r;
  const Chunk c = chunks[blockIdx.x];
  const Task &t = tasks[c.task];
  SplitInfo &sp = splits[c.task];
  const uint32_t *src = ids_of(s, t.buf);
  uint32_t *dst = ids_of(s, 1 - t.buf);
  const int nb = s.bins;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t r0 = c.begin; r0 < c.end; r0 += blockDim.x) {
    const uint32_t i = r0 + threadIdx.x;
    const bool valid = i < c.end;
    uint32_t id = 0;
    bool left = false;
    if (valid) {
      id = src[i];
      if (sp.median)
        left = i < sp.mid;
      else
        left = bin_of(comp(centroid(s, id), sp.axis), sp.cmin[sp.axis], sp.scale[sp.axis], nb) <= sp.bin;
    }
    const unsigned ml = __ballot_sync(0xffffffffu, valid && left), mr = __ballot_sync(0xffffffffu, valid && !left);
    if (lane == 0) warp_l[w] = __popc(ml), warp_r[w] = __popc(mr);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tl = 0, tr = 0;
      for (int j = 0; j < (int)(blockDim.x >> 5); j++) {
        unsigned a = warp_l[j], b = warp_r[j];
        warp_l[j] = tl, warp_r[j] = tr;
        tl += a, tr += b;
      }
      base_l = atomicAdd(&sp.left_ptr, tl);
      base_r = atomicAdd(&sp.right_ptr, tr);
    }
    __syncthreads();
    const unsigned below = (1u << lane) - 1u;
    if (valid) {
      /* positions stay inside [begin, mid) / [mid, end) because partition and binning share
       * bin_of(); the guard keeps a bookkeeping error from ever writing outside the node */
      const unsigned pos = left ? base_l + warp_l[w] + __popc(ml & below) : base_r + warp_r[w] + __popc(mr & below);
      if (left ? (pos < sp.mid) : (pos < t.end))
        dst[pos] = id;
      else
        atomicAdd(s.leaf_count + 1, 1u);
    }
    __syncthreads();
  }
}

/* The next level's chunk list, on the device: every task's primitives cut into kChunk pieces, in
 * task order (one block; an exclusive scan of the tasks' chunk counts, tile by tile).  The host
 * then reads only the task and chunk counts. */
__global__ void k_make_chunks(const Task *tasks, const unsigned *n_tasks, Chunk *chunks, unsigned max_chunks,
                              unsigned *n_chunks, unsigned *errors) {
  __shared__ unsigned warp_sum[32];
  __shared__ unsigned base;
  const unsigned nt = *n_tasks;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (unsigned t0 = 0; t0 < nt; t0 += blockDim.x) {
    const unsigned t = t0 + threadIdx.x;
    uint32_t b = 0, e = 0;
    unsigned c = 0;
    if (t < nt) {
      b = tasks[t].begin;
      e = tasks[t].end;
      c = (e - b + kChunk - 1) / kChunk;
    }
    unsigned x = c; /* inclusive scan within the warp, then over the warps */
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    unsigned before = 0, tile = 0;
    for (int j = 0; j < nw; j++) {
      if (j < w) before += warp_sum[j];
      tile += warp_sum[j];
    }
    const unsigned off = base + before + x - c;
    for (unsigned k = 0; k < c; k++) {
      if (off + k < max_chunks)
        chunks[off + k] = Chunk{t, b + k * kChunk, min(e, b + (k + 1) * kChunk)};
      else
        atomicAdd(errors, 1u); /* cannot happen (the capacity bounds the chunks): a build failure */
    }
    __syncthreads();
    if (threadIdx.x == 0) base += tile;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_chunks = base;
}

/* ------------------------------------------------------------------ small nodes */

/* Sum of v over the block (every thread gets it).  sh: blockDim.x / 32 entries.  Two barriers. */
__device__ __forceinline__ unsigned block_sum(unsigned v, unsigned *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = __reduce_add_sync(0xffffffffu, v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  unsigned t = 0;
  for (int j = 0; j < nw; j++) t += sh[j];
  __syncthreads();
  return t;
}

/* One round of a stable two-way partition over the block: this thread's rank among the round's
 * valid left (or right) threads in thread order, and the round's left and right totals.
 * sh: 2 * (blockDim.x / 32) entries.  Two barriers. */
__device__ __forceinline__ unsigned round_rank(bool valid, bool left, unsigned *sh, unsigned &tl, unsigned &tr) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned ml = __ballot_sync(0xffffffffu, valid && left), mr = __ballot_sync(0xffffffffu, valid && !left);
  if (lane == 0) sh[w] = __popc(ml), sh[nw + w] = __popc(mr);
  __syncthreads();
  unsigned bl = 0, br = 0;
  tl = tr = 0;
  for (int j = 0; j < nw; j++) {
    if (j < w) bl += sh[j], br += sh[nw + j];
    tl += sh[j], tr += sh[nw + j];
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  return left ? bl + __popc(ml & below) : br + __popc(mr & below);
}

/* ------------------------------------------------------------------ warp subtrees (<= 32 primitives)
 *
 * A node of at most 32 primitives is built by one warp, one primitive per lane, without block
 * barriers: per axis the lanes sort their centroids (bitonic, ties by primitive id), scan the sorted boxes
 * from both ends and evaluate the SAH of every split position (an exact sweep, where the larger
 * nodes use bins); the best (cost, axis, position) wins, the ids go to the other buffer in that
 * axis's sorted order.  Leaf rules, cost model and the median split below kMedianDepth are those of
 * the CTA path.
 *
 * The work runs on lane segments: a segment of W lanes (W = 32 is the whole warp) builds a node of
 * at most W primitives.  When both children of a split fit in W / 2 lanes the segment forks: its
 * lower half builds the left subtree while its upper half builds the right one, each as a segment of
 * W / 2 lanes, down to single lanes (one-primitive leaves); otherwise the left child continues on
 * the segment and the right one waits on the segment's stack.  A half whose subtree is done waits
 * for its sibling, and the two continue as their parent segment.  The splits do not depend on which
 * lanes compute them or in which order, so the tree is the one a single warp building node after
 * node produces. */
constexpr int kWarpPrims = 32;
constexpr int kWarpList = 256;   /* subtrees of <= kWarpPrims handed from the CTA loop to its warps */
/* Right siblings a W-lane segment keeps: it pushes only at nodes of >= W / 2 + 2 primitives (smaller
 * ones fork), nested with strictly decreasing sizes <= W, so at most W / 2 - 1 at once (none for
 * W <= 2).  Per warp: one segment of 32 lanes (15 entries), 2 of 16 (7 each), 4 of 8 (3 each) and 8
 * of 4 (1 each). */
constexpr int kWarpStack = 15 + 2 * 7 + 4 * 3 + 8 * 1;

__device__ __forceinline__ unsigned seg_mask(int W) {
  return W == 32 ? 0xffffffffu : ((1u << W) - 1u) << ((threadIdx.x & 31) & ~(W - 1));
}

/* The stack of the calling lane's W-lane segment, at level log2(32 / W) (W >= 4). */
__device__ __forceinline__ Task *seg_stack(Task *stacks, int level, int W) {
  const int base = level == 0 ? 0 : (level == 1 ? 15 : (level == 2 ? 29 : 41));
  return stacks + base + ((threadIdx.x & 31) / W) * (W / 2 - 1);
}

/* Sorts the segment's (key, tie) pairs ascending over each group of `span` lanes (a power of two,
 * 2..W) and returns, for this lane's rank, the segment lane that held it.  tie must be unique per
 * lane (the primitive id, so equal centroids sort the same way whatever order the ids arrive in;
 * empty lanes use 0xffffffff - lane).  A node of n primitives sits in segment lanes 0..n-1 with empty
 * lanes above, so the smallest power of two >= n sorts it: the bitonic stages above span only order
 * the empty lanes. */
__device__ __forceinline__ int seg_sort_idx(float key, uint32_t tie, int span, int W, unsigned mask) {
  const int lane = threadIdx.x & (W - 1);
  int idx = lane;
  for (int k = 2; k <= span; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      const float ok = __shfl_xor_sync(mask, key, j, W);
      const uint32_t ot = __shfl_xor_sync(mask, tie, j, W);
      const int oi = __shfl_xor_sync(mask, idx, j, W);
      const bool other_less = ok < key || (ok == key && ot < tie);
      const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
      if (keep_min ? other_less : !other_less) key = ok, tie = ot, idx = oi;
    }
  return idx;
}

/* Inclusive prefix (from segment lane 0) and suffix (towards the segment's last lane) bounds of the
 * boxes held by the segment's lanes.  Each lane's scan reaches `span` lanes (a power of two): with
 * the node's boxes in lanes 0..n-1, n <= span, and empty boxes above, the prefix of lane i < n and
 * the suffix of lane i (over i..n-1) are exact, the same values as a scan over the whole segment
 * (min and max are exact). */
__device__ __forceinline__ void seg_scan_boxes(const float lo[3], const float hi[3], float pl[3], float ph[3],
                                               float sl[3], float sh[3], int span, int W, unsigned mask) {
  const int lane = threadIdx.x & (W - 1);
  for (int k = 0; k < 3; k++) pl[k] = sl[k] = lo[k], ph[k] = sh[k] = hi[k];
  for (int o = 1; o < span; o <<= 1)
    for (int k = 0; k < 3; k++) {
      const float a = __shfl_up_sync(mask, pl[k], o, W), b = __shfl_up_sync(mask, ph[k], o, W);
      const float c = __shfl_down_sync(mask, sl[k], o, W), d = __shfl_down_sync(mask, sh[k], o, W);
      if (lane >= o) pl[k] = fminf(pl[k], a), ph[k] = fmaxf(ph[k], b);
      if (lane + o < W) sl[k] = fminf(sl[k], c), sh[k] = fmaxf(sh[k], d);
    }
}

__device__ __forceinline__ Best seg_best(Best b, int W, unsigned mask) {
  for (int o = W / 2; o > 0; o >>= 1) {
    Best q{__shfl_xor_sync(mask, b.cost, o, W), __shfl_xor_sync(mask, b.key, o, W)};
    if (better(q, b)) b = q;
  }
  return b;
}

/* Builds the subtree of `root` (<= 32 primitives) with the calling warp; all 32 lanes call it.
 * stacks: the warp's kWarpStack entries. */
__device__ void warp_build(const Shared &s, Task root, Task *stacks) {
  int W = 32, level = 0; /* this lane's segment: width and log2(32 / W) */
  uint32_t depth_sp = 0; /* per level (4 bits each, levels 0..3), the segment's stack depth */
  bool failed = false;
  Task t = root;
  for (int iter = 0;; iter++) {
    const int lane = threadIdx.x & (W - 1);
    unsigned mask = seg_mask(W);
    const uint32_t n = t.end - t.begin;
    const uint32_t *src = ids_of(s, t.buf);
    uint32_t *dst = ids_of(s, 1 - t.buf);
    const bool act = (uint32_t)lane < n;
    const uint32_t id = act ? src[t.begin + lane] : 0u;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX}, c[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    if (act) {
      const float4 a = __ldg(s.lo + id), b = __ldg(s.hi + id);
      lo[0] = a.x, lo[1] = a.y, lo[2] = a.z, hi[0] = b.x, hi[1] = b.y, hi[2] = b.z;
      c[0] = (a.x + b.x) * 0.5f, c[1] = (a.y + b.y) * 0.5f, c[2] = (a.z + b.z) * 0.5f;
    }
    /* a lane processes distinct nodes of a <= 32-primitive subtree, at most 63: past 2 * 63
     * iterations something is broken, and every further node becomes a leaf, so the segments still
     * drain their stacks and meet their siblings (no lane leaves while another waits for it).  The
     * vote keeps the decision uniform over the segment (lanes of a joined segment count differently) */
    if (__any_sync(mask, iter >= 2 * (2 * kWarpPrims - 1)) && !failed) {
      failed = true;
      if (lane == 0) atomicAdd(s.leaf_count + 1, 1u); /* reported as a build failure */
    }
    bool make_leaf = n <= 1 || failed;
    const float area = half_area(t.lo, t.hi);
    Best best{FLT_MAX, 0x7fffffff};
    float pl[3], ph[3], sl[3], sh[3];
    /* sorts and scans reach the smallest power of two >= n lanes (uniform over the segment) */
    const int span = n <= 2u ? 2 : 1 << (32 - __clz((int)n - 1));
    int from_a[3] = {0, 0, 0}; /* per axis, the lane holding each sorted rank */
    bool sorted = false;
    if (!make_leaf && area > 0.f && t.depth < kMedianDepth) {
      sorted = true;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const int from = seg_sort_idx(act ? c[a] : FLT_MAX, act ? id : 0xffffffffu - (uint32_t)lane, span, W, mask);
        from_a[a] = from;
        float bl[3], bh[3];
        for (int k = 0; k < 3; k++)
          bl[k] = __shfl_sync(mask, lo[k], from, W), bh[k] = __shfl_sync(mask, hi[k], from, W);
        seg_scan_boxes(bl, bh, pl, ph, sl, sh, span, W, mask);
        float rl[3], rh[3];
        for (int k = 0; k < 3; k++)
          rl[k] = __shfl_down_sync(mask, sl[k], 1, W), rh[k] = __shfl_down_sync(mask, sh[k], 1, W);
        Best mine{FLT_MAX, 0x7fffffff};
        if ((uint32_t)lane + 1 < n) { /* split after sorted position lane: left = lane + 1 primitives */
          const float cost =
              s.cost_trav + (half_area(pl, ph) * (float)(lane + 1) + half_area(rl, rh) * (float)(n - 1 - lane)) / area;
          mine = Best{cost, a * 64 + lane};
        }
        mine = seg_best(mine, W, mask);
        if (better(mine, best)) best = mine;
      }
    }
    const bool has_split = best.key != 0x7fffffff;
    if (!make_leaf) {
      if ((int)n <= s.max_leaf && (!has_split || (float)n <= best.cost)) make_leaf = true;
      if ((int)n <= s.hard_leaf && !has_split) make_leaf = true;
    }
    if (!make_leaf) {
      /* the split: best SAH position, or the median along the widest centroid extent */
      int axis, left_n;
      if (has_split) {
        axis = best.key / 64;
        left_n = best.key % 64 + 1;
      } else {
        float ext[3];
        for (int k = 0; k < 3; k++) {
          float mn = act ? c[k] : FLT_MAX, mx = act ? c[k] : -FLT_MAX;
          for (int o = W / 2; o > 0; o >>= 1)
            mn = fminf(mn, __shfl_xor_sync(mask, mn, o, W)), mx = fmaxf(mx, __shfl_xor_sync(mask, mx, o, W));
          ext[k] = mx - mn;
        }
        axis = ext[1] > ext[0] ? (ext[2] > ext[1] ? 2 : 1) : (ext[2] > ext[0] ? 2 : 0);
        left_n = (int)n / 2;
      }
      /* the SAH pass already sorted every axis: reuse its order for the chosen one */
      const int from = sorted ? (axis == 0 ? from_a[0] : (axis == 1 ? from_a[1] : from_a[2]))
                              : seg_sort_idx(act ? c[axis] : FLT_MAX, act ? id : 0xffffffffu - (uint32_t)lane, span,
                                             W, mask);
      const uint32_t sid = __shfl_sync(mask, id, from, W);
      float bl[3], bh[3];
      for (int k = 0; k < 3; k++)
        bl[k] = __shfl_sync(mask, lo[k], from, W), bh[k] = __shfl_sync(mask, hi[k], from, W);
      if (act) dst[t.begin + lane] = sid;
      seg_scan_boxes(bl, bh, pl, ph, sl, sh, span, W, mask);
      float cl[3], ch[3], dl[3], dh[3];
      for (int k = 0; k < 3; k++) {
        cl[k] = __shfl_sync(mask, pl[k], left_n - 1, W), ch[k] = __shfl_sync(mask, ph[k], left_n - 1, W);
        dl[k] = __shfl_sync(mask, sl[k], left_n, W), dh[k] = __shfl_sync(mask, sh[k], left_n, W);
      }
      const uint32_t mid = t.begin + (uint32_t)left_n;
      int node = 0;
      if (lane == 0) {
        node = (int)atomicAdd(s.node_counter, 1u);
        if (t.parent >= 0) write_ref(s.nodes, t.parent, t.slot, node);
        write_child(s.nodes, node, 0, cl, ch);
        write_child(s.nodes, node, 1, dl, dh);
      }
      node = __shfl_sync(mask, node, 0, W);
      __syncwarp(mask); /* the children read ids written by other lanes */
      const Task L{t.begin, mid, node, 0, t.depth + 1, 1 - t.buf, {cl[0], cl[1], cl[2]}, {ch[0], ch[1], ch[2]}};
      const Task R{mid, t.end, node, 1, t.depth + 1, 1 - t.buf, {dl[0], dl[1], dl[2]}, {dh[0], dh[1], dh[2]}};
      if ((uint32_t)left_n <= (uint32_t)(W / 2) && n - (uint32_t)left_n <= (uint32_t)(W / 2)) {
        /* fork: the lower half builds the left subtree, the upper half the right one */
        t = lane < W / 2 ? L : R;
        W >>= 1;
        level++;
        if (level < 4) depth_sp &= ~(15u << (4 * level));
        continue;
      }
      const int sp = (int)((depth_sp >> (4 * level)) & 15u);
      if (sp < W / 2 - 1) {
        if (lane == 0) seg_stack(stacks, level, W)[sp] = R;
        depth_sp += 1u << (4 * level);
      } else if (lane == 0) {
        atomicAdd(s.leaf_count + 1, 1u); /* cannot happen (see kWarpStack): reported as a build failure */
      }
      __syncwarp(mask);
      t = L;
      continue;
    }
    if (act) s.order[t.begin + lane] = id;
    if (lane == 0) finish_leaf(s, t);
    /* next: the segment's pending sibling; a segment with none waits for its sibling half and the
     * two continue as their parent */
    for (;;) {
      const int sp = level < 4 ? (int)((depth_sp >> (4 * level)) & 15u) : 0;
      if (sp > 0) {
        __syncwarp(mask);
        t = seg_stack(stacks, level, W)[sp - 1];
        depth_sp -= 1u << (4 * level);
        __syncwarp(mask);
        break;
      }
      if (level == 0) return;
      W <<= 1;
      level--;
      mask = seg_mask(W);
      __syncwarp(mask);
    }
  }
}

__global__ void __launch_bounds__(kSmallBlock) k_build_small(Shared s, const Task *small_tasks) {
  __shared__ Task stack[kSmallStack];
  __shared__ int sp, have;
  __shared__ unsigned scnt[3][kMaxBins];
  __shared__ float slo[3][kMaxBins][3], shi[3][kMaxBins][3];
  __shared__ float red[6 * 32];
  __shared__ unsigned scan_sh[32];
  __shared__ Best best_sh[kBlock / 32];
  __shared__ Task cur;
  __shared__ float cmin_s[3], scale_s[3];
  __shared__ Task wlist[kWarpList];
  __shared__ Task wstack[kSmallBlock / 32][kWarpStack];
  __shared__ int wl_count, wl_next;
  const int nb = s.bins;
  if (threadIdx.x == 0) {
    const Task t0 = small_tasks[blockIdx.x];
    wl_count = wl_next = 0;
    sp = 0;
    if (t0.end - t0.begin <= (uint32_t)kWarpPrims)
      wlist[wl_count++] = t0;
    else
      stack[sp++] = t0;
  }
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) {
      have = sp > 0;
      if (have) cur = stack[--sp];
    }
    __syncthreads();
    if (!have) break;
    const Task t = cur;
    const uint32_t n = t.end - t.begin;
    const uint32_t *src = ids_of(s, t.buf);
    uint32_t *dst = ids_of(s, 1 - t.buf);
    bool make_leaf = n <= 1;
    /* centroid bounds */
    float l[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, h[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += blockDim.x) {
      float3 p = centroid(s, src[i]);
      l[0] = fminf(l[0], p.x), l[1] = fminf(l[1], p.y), l[2] = fminf(l[2], p.z);
      h[0] = fmaxf(h[0], p.x), h[1] = fmaxf(h[1], p.y), h[2] = fmaxf(h[2], p.z);
    }
    block_minmax3(l, h, red);
    if (threadIdx.x < 3) {
      cmin_s[threadIdx.x] = l[threadIdx.x];
      scale_s[threadIdx.x] = bin_scale(l[threadIdx.x], h[threadIdx.x], nb);
    }
    for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) {
      int a = i / nb, b = i % nb;
      scnt[a][b] = 0u;
      for (int k = 0; k < 3; k++) slo[a][b][k] = FLT_MAX, shi[a][b][k] = -FLT_MAX;
    }
    __syncthreads();
    Best best{FLT_MAX, 0x7fffffff};
    const float area = half_area(t.lo, t.hi);
    if (!make_leaf) {
      for (uint32_t r0 = t.begin; r0 < t.end; r0 += blockDim.x) { /* whole warps: bin_add votes */
        const uint32_t i = r0 + threadIdx.x;
        const bool valid = i < t.end;
        float4 bl = make_float4(0.f, 0.f, 0.f, 0.f), bh = bl;
        if (valid) {
          const uint32_t id = src[i];
          bl = __ldg(s.lo + id), bh = __ldg(s.hi + id);
        }
        const float3 p = make_float3((bl.x + bh.x) * 0.5f, (bl.y + bh.y) * 0.5f, (bl.z + bh.z) * 0.5f);
        for (int a = 0; a < 3; a++)
          bin_add(scnt[a], slo[a], shi[a], bin_of(comp(p, a), cmin_s[a], scale_s[a], nb), valid, bl, bh);
      }
      __syncthreads();
      if (area > 0.f && t.depth < kMedianDepth)
        best = sah_best(
            nb, area, s.cost_trav, [&](int a, int b) { return scnt[a][b]; },
            [&](int a, int b, int k) { return slo[a][b][k]; }, [&](int a, int b, int k) { return shi[a][b][k]; });
    }
    best = block_best(best, best_sh);
    const bool has_split = best.key != 0x7fffffff;
    if (!make_leaf) {
      const float leaf_cost = (float)n;
      if ((int)n <= s.max_leaf && (!has_split || leaf_cost <= best.cost)) make_leaf = true;
      if ((int)n <= s.hard_leaf && !has_split) make_leaf = true;
    }
    if (make_leaf) {
      for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += blockDim.x) s.order[i] = src[i];
      if (threadIdx.x == 0) finish_leaf(s, t);
      continue;
    }
    /* partition into dst (stable), then child boxes */
    const int axis = has_split ? best.key / kMaxBins : 0;
    const int split_bin = has_split ? best.key % kMaxBins - 1 : 0;
    const uint32_t mid_med = t.begin + n / 2;
    unsigned left_total = 0;
    {
      /* count left first */
      unsigned cnt = 0;
      for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += blockDim.x) {
        bool left = has_split ? bin_of(comp(centroid(s, src[i]), axis), cmin_s[axis], scale_s[axis], nb) <= split_bin
                              : i < mid_med;
        cnt += left;
      }
      left_total = block_sum(cnt, scan_sh);
    }
    const uint32_t mid = t.begin + left_total;
    unsigned run_l = 0, run_r = 0;
    for (uint32_t r0 = t.begin; r0 < t.end; r0 += blockDim.x) {
      const uint32_t i = r0 + threadIdx.x;
      const bool valid = i < t.end;
      uint32_t id = 0;
      bool left = false;
      if (valid) {
        id = src[i];
        left = has_split ? bin_of(comp(centroid(s, id), axis), cmin_s[axis], scale_s[axis], nb) <= split_bin
                         : i < mid_med;
      }
      unsigned tl, tr;
      const unsigned rank = round_rank(valid, left, scan_sh, tl, tr);
      if (valid) {
        const uint32_t pos = left ? t.begin + run_l + rank : mid + run_r + rank;
        if (left ? (pos < mid) : (pos < t.end))
          dst[pos] = id;
        else
          atomicAdd(s.leaf_count + 1, 1u);
      }
      run_l += tl;
      run_r += tr;
    }
    __syncthreads();
    /* exact child boxes */
    float cl[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ch[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float dl[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, dh[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += blockDim.x) {
      const uint32_t id = dst[i];
      const float4 bl = __ldg(s.lo + id), bh = __ldg(s.hi + id);
      float *ol = i < mid ? cl : dl, *oh = i < mid ? ch : dh;
      ol[0] = fminf(ol[0], bl.x), ol[1] = fminf(ol[1], bl.y), ol[2] = fminf(ol[2], bl.z);
      oh[0] = fmaxf(oh[0], bh.x), oh[1] = fmaxf(oh[1], bh.y), oh[2] = fmaxf(oh[2], bh.z);
    }
    block_minmax3(cl, ch, red);
    block_minmax3(dl, dh, red);
    if (threadIdx.x == 0) {
      const int node = (int)atomicAdd(s.node_counter, 1u);
      if (t.parent >= 0) write_ref(s.nodes, t.parent, t.slot, node);
      write_child(s.nodes, node, 0, cl, ch);
      write_child(s.nodes, node, 1, dl, dh);
      Task L{t.begin, mid, node, 0, t.depth + 1, 1 - t.buf, {cl[0], cl[1], cl[2]}, {ch[0], ch[1], ch[2]}};
      Task R{mid, t.end, node, 1, t.depth + 1, 1 - t.buf, {dl[0], dl[1], dl[2]}, {dh[0], dh[1], dh[2]}};
      /* subtrees of <= kWarpPrims primitives go to the warps; larger ones stay on the CTA stack
       * (depth-first: at most one pending sibling per level) */
      for (const Task &ch : {R, L}) {
        if (ch.end - ch.begin <= (uint32_t)kWarpPrims && wl_count < kWarpList)
          wlist[wl_count++] = ch;
        else if (sp < kSmallStack)
          stack[sp++] = ch;
        else
          atomicAdd(s.leaf_count + 1, 1u); /* a lost subtree: reported as a build failure */
      }
    }
  }
  /* the warps build the small subtrees, each taking the next one from the list */
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(&wl_next, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= wl_count) break;
    warp_build(s, wlist[item], wstack[warp]);
  }
}

__global__ void k_sort_leaves(const uint2 *leaves, unsigned n, uint32_t *order) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint2 L = leaves[i];
  uint32_t *o = order + L.x;
  for (uint32_t a = 1; a < L.y; a++) {
    uint32_t v = o[a];
    int b = (int)a - 1;
    while (b >= 0 && o[b] > v) {
      o[b + 1] = o[b];
      b--;
    }
    o[b + 1] = v;
  }
}

/* ------------------------------------------------------------------ depth-first node order
 *
 * Nodes are numbered as they are created: level by level for large nodes, then by many CTAs at
 * once for the small subtrees, so a subtree's nodes end up interleaved with other subtrees'.  The
 * final pass renumbers them in depth-first preorder (left child first), so a node's descendants
 * follow it in memory.  Subtree sizes come bottom-up (the last child to finish continues to its
 * parent); a node's preorder number is its depth plus the sizes of the left siblings along its
 * path to the root. */

constexpr uint32_t kNoParent = 0xffffffffu;

__global__ void k_dfs_init(const float4 *nodes, uint32_t n, uint32_t *parent, uint8_t *side, uint32_t *need,
                           uint32_t *arrived) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 n3 = nodes[4 * i + 3];
  const int32_t r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
  uint32_t k = 0;
  for (int c = 0; c < 2; c++)
    if (r[c] >= 0 && (uint32_t)r[c] < n) {
      parent[r[c]] = i;
      side[r[c]] = (uint8_t)c;
      k++;
    }
  need[i] = k;
  arrived[i] = 0;
  if (i == 0) parent[0] = kNoParent;
}

__global__ void k_dfs_sizes(const float4 *nodes, uint32_t n, const uint32_t *parent, const uint32_t *need,
                            uint32_t *arrived, uint32_t *size) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || need[i] != 0) return;
  uint32_t v = i;
  size[v] = 1;
  for (int guard = 0; guard < 4 * kSmallStack; guard++) {
    __threadfence();
    const uint32_t p = parent[v];
    if (p == kNoParent || p >= n) return;
    if (atomicAdd(&arrived[p], 1u) + 1u < need[p]) return; /* a sibling subtree is still open */
    __threadfence();
    const float4 n3 = nodes[4 * p + 3];
    const int32_t r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
    uint32_t sz = 1;
    for (int c = 0; c < 2; c++)
      if (r[c] >= 0 && (uint32_t)r[c] < n) sz += __ldcg(size + r[c]);
    size[p] = sz;
    v = p;
  }
}

__global__ void k_dfs_number(const float4 *nodes, uint32_t n, const uint32_t *parent, const uint8_t *side,
                             const uint32_t *size, uint32_t *number) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t idx = 0, v = i;
  for (int guard = 0; guard < 4 * kSmallStack && v != 0; guard++) {
    const uint32_t p = parent[v];
    if (p >= n) break;
    idx += 1;
    if (side[v] == 1) {
      const int32_t left = __float_as_int(nodes[4 * p + 3].x);
      if (left >= 0 && (uint32_t)left < n) idx += size[left];
    }
    v = p;
  }
  number[i] = idx;
}

__global__ void k_dfs_permute(const float4 *nodes, uint32_t n, const uint32_t *number, float4 *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = number[i];
  if (j >= n) return;
  float4 n3 = nodes[4 * i + 3];
  const int32_t r0 = __float_as_int(n3.x), r1 = __float_as_int(n3.y);
  if (r0 >= 0 && (uint32_t)r0 < n) n3.x = __int_as_float((int32_t)number[r0]);
  if (r1 >= 0 && (uint32_t)r1 < n) n3.y = __int_as_float((int32_t)number[r1]);
  out[4 * j + 0] = nodes[4 * i + 0];
  out[4 * j + 1] = nodes[4 * i + 1];
  out[4 * j + 2] = nodes[4 * i + 2];
  out[4 * j + 3] = n3;
}

}  // namespace

cudaError_t reorder_depth_first(float4 *nodes, uint32_t n, cudaStream_t stream) {
  if (n <= 1) return cudaSuccess;
  uint32_t *parent = nullptr, *need = nullptr, *arrived = nullptr, *size = nullptr, *number = nullptr;
  uint8_t *side = nullptr;
  float4 *tmp = nullptr;
  cudaError_t err = cudaSuccess;
  const unsigned grid = (n + 255) / 256;
  if ((err = cudaMallocAsync(&parent, sizeof(uint32_t) * n, stream)) != cudaSuccess) goto done;
  if ((err = cudaMallocAsync(&need, sizeof(uint32_t) * n, stream)) != cudaSuccess) goto done;
  if ((err = cudaMallocAsync(&arrived, sizeof(uint32_t) * n, stream)) != cudaSuccess) goto done;
  if ((err = cudaMallocAsync(&size, sizeof(uint32_t) * n, stream)) != cudaSuccess) goto done;
  if ((err = cudaMallocAsync(&number, sizeof(uint32_t) * n, stream)) != cudaSuccess) goto done;
  if ((err = cudaMallocAsync(&side, n, stream)) != cudaSuccess) goto done;
  if ((err = cudaMallocAsync(&tmp, sizeof(float4) * 4 * (size_t)n, stream)) != cudaSuccess) goto done;
  k_dfs_init<<<grid, 256, 0, stream>>>(nodes, n, parent, side, need, arrived);
  k_dfs_sizes<<<grid, 256, 0, stream>>>(nodes, n, parent, need, arrived, size);
  k_dfs_number<<<grid, 256, 0, stream>>>(nodes, n, parent, side, size, number);
  k_dfs_permute<<<grid, 256, 0, stream>>>(nodes, n, number, tmp);
  if ((err = cudaGetLastError()) != cudaSuccess) goto done;
  err = cudaMemcpyAsync(nodes, tmp, sizeof(float4) * 4 * (size_t)n, cudaMemcpyDeviceToDevice, stream);
done:
  cudaFreeAsync(parent, stream);
  cudaFreeAsync(need, stream);
  cudaFreeAsync(arrived, stream);
  cudaFreeAsync(size, stream);
  cudaFreeAsync(number, stream);
  cudaFreeAsync(side, stream);
  cudaFreeAsync(tmp, stream);
  return err;
}

cudaError_t build_bvh(const float4 *lo, const float4 *hi, uint32_t n, const BvhBuildParams &p, float4 *nodes,
                      uint32_t *order, cudaStream_t stream, BvhBuildResult *res) {
  auto t0 = std::chrono::steady_clock::now();
  if (n == 0) return cudaErrorInvalidValue;
  const int nb = std::max(4, std::min(kMaxBins, p.bins > 0 ? p.bins : 16));
  const int hard_leaf = std::max(1, std::min(kHardLeaf, p.hard_leaf > 0 ? p.hard_leaf : kHardLeaf));
  const int max_leaf = std::max(1, std::min(hard_leaf, p.max_leaf > 0 ? p.max_leaf : 8));
  const uint32_t small_task = p.small_task >= 64 ? p.small_task : kSmallTaskDefault;
  const size_t max_large = n / small_task + 2;
  const size_t max_small = n + 1;
  /* scratch */
  uint32_t *ids0 = nullptr, *ids1 = nullptr;
  Task *large_a = nullptr, *large_b = nullptr, *small = nullptr;
  unsigned *counters = nullptr; /* node, large_next, small, leaf, partition errors, next level's chunks */
  uint2 *leaves = nullptr;
  int *maxdepth = nullptr;
  float *scene = nullptr, *cb = nullptr;
  Bins *bins = nullptr;
  SplitInfo *splits = nullptr;
  Chunk *chunks = nullptr;
  const size_t max_chunks = n / kChunk + max_large + 2;
  cudaError_t err = cudaSuccess;
#define NB_TRY(x)                        \
  do {                                   \
    err = (x);                           \
    if (err != cudaSuccess) goto cleanup; \
  } while (0)
  {
    NB_TRY(cudaMallocAsync(&ids0, sizeof(uint32_t) * n, stream));
    NB_TRY(cudaMallocAsync(&ids1, sizeof(uint32_t) * n, stream));
    NB_TRY(cudaMallocAsync(&large_a, sizeof(Task) * max_large, stream));
    NB_TRY(cudaMallocAsync(&large_b, sizeof(Task) * max_large, stream));
    NB_TRY(cudaMallocAsync(&small, sizeof(Task) * max_small, stream));
    NB_TRY(cudaMallocAsync(&counters, sizeof(unsigned) * 6, stream));
    NB_TRY(cudaMallocAsync(&leaves, sizeof(uint2) * n, stream));
    NB_TRY(cudaMallocAsync(&maxdepth, sizeof(int), stream));
    NB_TRY(cudaMallocAsync(&scene, sizeof(float) * 6, stream));
    NB_TRY(cudaMallocAsync(&cb, sizeof(float) * 6 * max_large, stream));
    NB_TRY(cudaMallocAsync(&bins, sizeof(Bins) * max_large, stream));
    NB_TRY(cudaMallocAsync(&splits, sizeof(SplitInfo) * max_large, stream));
    NB_TRY(cudaMallocAsync(&chunks, sizeof(Chunk) * max_chunks, stream));
    NB_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * 6, stream));
    NB_TRY(cudaMemsetAsync(maxdepth, 0, sizeof(int), stream));
    {
      const float init[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
      NB_TRY(cudaMemcpyAsync(scene, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    }
    k_scene_box<<<std::min<uint32_t>(1024, (n + 255) / 256), 256, 0, stream>>>(lo, hi, n, scene);
    k_iota<<<(n + 255) / 256, 256, 0, stream>>>(ids0, n);
    NB_TRY(cudaGetLastError());
    float hscene[6];
    NB_TRY(cudaMemcpyAsync(hscene, scene, sizeof(hscene), cudaMemcpyDeviceToHost, stream));
    NB_TRY(cudaStreamSynchronize(stream));

    Shared sh;
    sh.lo = lo;
    sh.hi = hi;
    sh.ids0 = ids0;
    sh.ids1 = ids1;
    sh.nodes = nodes;
    sh.order = order;
    sh.node_counter = counters + 0;
    sh.large_next_count = counters + 1;
    sh.small_count = counters + 2;
    sh.leaf_count = counters + 3;
    sh.small = small;
    sh.leaves = leaves;
    sh.max_depth = maxdepth;
    sh.bins = nb;
    sh.max_leaf = max_leaf;
    sh.hard_leaf = hard_leaf;
    sh.cost_trav = p.cost_trav > 0.f ? p.cost_trav : 1.0f;
    sh.small_task = small_task;

    Task root{0u, n, -1, 0, 0, 0, {hscene[0], hscene[1], hscene[2]}, {hscene[3], hscene[4], hscene[5]}};
    Task *cur = large_a, *next = large_b;
    uint32_t nt = 0, nc = 0; /* tasks and chunks of the current level */
    if (n > small_task) {
      std::vector<Chunk> ch;
      for (uint32_t b = 0; b < n; b += kChunk) ch.push_back(Chunk{0u, b, std::min(n, b + kChunk)});
      nt = 1;
      nc = (uint32_t)ch.size();
      NB_TRY(cudaMemcpyAsync(cur, &root, sizeof(Task), cudaMemcpyHostToDevice, stream));
      NB_TRY(cudaMemcpyAsync(chunks, ch.data(), sizeof(Chunk) * nc, cudaMemcpyHostToDevice, stream));
    } else {
      NB_TRY(cudaMemcpyAsync(small, &root, sizeof(Task), cudaMemcpyHostToDevice, stream));
      const unsigned one = 1;
      NB_TRY(cudaMemcpyAsync(counters + 2, &one, sizeof(unsigned), cudaMemcpyHostToDevice, stream));
    }
    /* one level per iteration: the level's tasks and chunks stay on the device, the host reads their
     * counts (one synchronisation per level) */
    while (nt > 0) {
      NB_TRY(cudaMemsetAsync(counters + 1, 0, sizeof(unsigned), stream));
      sh.large_next = next;
      k_init_level<<<nt, 128, 0, stream>>>(bins, cb, nt, nb);
      k_cbounds<<<nc, kBlock, 0, stream>>>(sh, cur, chunks, cb);
      k_bin<<<nc, kBlock, 0, stream>>>(sh, cur, chunks, cb, bins);
      k_split<<<nt, kBlock, 0, stream>>>(sh, cur, cb, bins, splits);
      k_partition<<<nc, kBlock, 0, stream>>>(sh, cur, chunks, splits);
      k_make_chunks<<<1, 1024, 0, stream>>>(next, counters + 1, chunks, (unsigned)max_chunks, counters + 5,
                                            counters + 4);
      NB_TRY(cudaGetLastError());
      unsigned hn[5]; /* counters 1..5: next level's tasks, small tasks, leaves, errors, next level's chunks */
      NB_TRY(cudaMemcpyAsync(hn, counters + 1, sizeof(hn), cudaMemcpyDeviceToHost, stream));
      NB_TRY(cudaStreamSynchronize(stream));
      nt = hn[0];
      nc = hn[4];
      std::swap(cur, next);
    }
    unsigned n_small = 0;
    NB_TRY(cudaMemcpyAsync(&n_small, counters + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    NB_TRY(cudaStreamSynchronize(stream));
    if (n_small) k_build_small<<<n_small, kSmallBlock, 0, stream>>>(sh, small);
    NB_TRY(cudaGetLastError());
    unsigned hc[5];
    int hdepth = 0;
    NB_TRY(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, stream));
    NB_TRY(cudaMemcpyAsync(&hdepth, maxdepth, sizeof(int), cudaMemcpyDeviceToHost, stream));
    NB_TRY(cudaStreamSynchronize(stream));
    if (hc[3]) k_sort_leaves<<<(hc[3] + 255) / 256, 256, 0, stream>>>(leaves, hc[3], order);
    NB_TRY(cudaGetLastError());
    NB_TRY(cudaStreamSynchronize(stream));
    if (hc[4] != 0) {
      err = cudaErrorUnknown; /* partition inconsistency: never expected, reported as a build failure */
      goto cleanup;
    }
    NB_TRY(reorder_depth_first(nodes, hc[0], stream));
    if (res) {
      res->n_nodes = hc[0];
      res->n_leaves = hc[3];
      res->max_depth = hdepth;
    }
  }
cleanup:
  cudaFreeAsync(ids0, stream);
  cudaFreeAsync(ids1, stream);
  cudaFreeAsync(large_a, stream);
  cudaFreeAsync(large_b, stream);
  cudaFreeAsync(small, stream);
  cudaFreeAsync(counters, stream);
  cudaFreeAsync(leaves, stream);
  cudaFreeAsync(maxdepth, stream);
  cudaFreeAsync(scene, stream);
  cudaFreeAsync(cb, stream);
  cudaFreeAsync(bins, stream);
  cudaFreeAsync(splits, stream);
  cudaFreeAsync(chunks, stream);
  cudaStreamSynchronize(stream);
#undef NB_TRY
  if (res) res->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return err;
}

}  // namespace nb
