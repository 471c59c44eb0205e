/* C-ABI entry points: context lifecycle, scene upload, BVH build, queries.
 *
 * Upload (Engine::buildScene, api/engine.cpp:201-233): mesh attribute spans, instances with their
 * transform records, materials and textures are validated on the host and copied to device
 * memory; the global primitive order is the reference's (instance by instance, triangle by
 * triangle, api/engine.cpp:159-175).  Triangles whose indices repeat are never hit by the
 * reference (Triangle::isDegenerate, shape/Triangle.h:127-132) and are left out of the BVH.
 *
 * Build (Engine::buildAcceleration, api/engine.cpp:235): world boxes of the valid triangles
 * (transform.m * vertex, Triangle::computeAABB, Triangle.h:99-109) -> device binned SAH
 * (bvh_build.cu) -> structural validation (every inner reference points to a later node, every
 * leaf range is in bounds, so traversal always terminates) -> triangle records in leaf order.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>

#include "bvh_build.cuh"
#include "sampler.cuh"
#include "bvh_wide.cuh"
#include "context.cuh"
#include "traverse.cuh"

namespace {

struct JoeKuoRow {
  int d, s, a;
  int m[12];
};
const JoeKuoRow kJoeKuo[255] = {
#include "joe_kuo_params.inc"
};

/* Direction numbers V_i = m_i << (32 - i) from the Joe & Kuo recurrence
 * m_k = (m_{k-s} << s) ^ m_{k-s} ^ XOR_{j=1..s-1} a_j (m_{k-j} << j), a_1 the most significant
 * of the s - 1 coefficient bits (the reference's scripts/generate_luts_sobol.py:51-95). */
void sobol_table(std::vector<uint32_t> &t) {
  t.assign(256 * 32, 0u);
  for (int d = 0; d < 255; d++) {
    const JoeKuoRow &r = kJoeKuo[d];
    uint64_t m[32];
    for (int k = 0; k < 32; k++) {
      if (k < r.s) {
        m[k] = (uint64_t)r.m[k];
        continue;
      }
      uint64_t v = (m[k - r.s] << r.s) ^ m[k - r.s];
      for (int j = 1; j < r.s; j++)
        if ((r.a >> (r.s - 1 - j)) & 1) v ^= m[k - j] << j;
      m[k] = v;
    }
    for (int i = 0; i < 32; i++) t[d * 32 + i] = (uint32_t)(m[i] << (31 - i));
  }
}

/* The device form of the direction vectors: for every dimension four 256-entry tables, entry b of
 * table k the XOR of the vectors of the set bits of byte value b at bit position 8k..8k+7, so the
 * XOR over the set bits of a 32-bit gray code is four lookups (sampler.cuh). */
void sobol_byte_tables(const std::vector<uint32_t> &dv, std::vector<uint32_t> &t) {
  t.assign((size_t)nb::kSobolDims * nb::kSobolByteTable, 0u);
  for (int d = 0; d < nb::kSobolDims; d++)
    for (int k = 0; k < 4; k++)
      for (int b = 0; b < 256; b++) {
        uint32_t x = 0;
        for (int j = 0; j < 8; j++)
          if ((b >> j) & 1) x ^= dv[d * 32 + 8 * k + j];
        t[(size_t)d * nb::kSobolByteTable + 256 * k + b] = x;
      }
}

/* acos table f(i) = acos(2 i / P - 1), P = 500000, rounded to float
 * (scripts/generate_luts_trigonometrics.py:11-18, looked up by math_acos_lt.cpp:37-40). */
void acos_table(std::vector<float> &t) {
  t.resize(nb::kAcosPrecision);
  for (int i = 0; i < nb::kAcosPrecision; i++)
    t[i] = (float)std::acos(((double)i / (double)nb::kAcosPrecision) * 2.0 - 1.0);
}

bool is_identity(const float *m) {
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++)
      if (m[4 * c + r] != (c == r ? 1.f : 0.f)) return false;
  return true;
}

/* Scene uploads go to one device arena per scene (one pool allocation instead of one cudaMalloc per
 * texture / mesh / table; cudaMalloc and cudaFree synchronise the device).  Pieces up to kSmallPiece
 * bytes are read by a gather kernel when the caller's memory is pinned, else gathered in a pinned
 * host buffer and copied with one transfer; larger ones are copied directly from the caller's
 * memory. */
/* 32 batch scenes (2,738 meshes, 444 MB, each array pinned on its own): with 64 KB the mesh arrays
 * above it went one cudaMemcpyAsync each and the uploads took 24.7 ms (18 GB/s); with 256 KB they
 * take 14.7 ms (30 GB/s), with 1 MB 16.6 ms. */
constexpr size_t kSmallPiece = 1 << 18;

struct Piece {
  const void *src;
  size_t bytes;
  size_t off;   /* offset in its region */
  bool temp;    /* region: temporary SoA staging (true) or the persistent arena */
};

struct UploadPlan {
  std::vector<Piece> pieces;
  size_t arena = 0, temp = 0;
  static size_t align(size_t b) { return (b + 255) & ~(size_t)255; }
  size_t add(const void *src, size_t bytes, bool temp_region = false) {
    size_t &top = temp_region ? temp : arena;
    const size_t off = top;
    top += align(bytes);
    pieces.push_back(Piece{src, bytes, off, temp_region});
    return off;
  }
};

nova_b200_status ensure_pinned_stage(nova_b200_ctx *c, size_t bytes) {
  if (c->h_stage_bytes >= bytes) return NOVA_B200_SUCCESS;
  if (c->h_stage) cudaFreeHost(c->h_stage);
  c->h_stage = nullptr;
  c->h_stage_bytes = 0;
  const size_t want = std::max<size_t>(bytes, 1 << 20);
  NB_CUDA(c, cudaMallocHost(&c->h_stage, want), "cudaMallocHost(upload staging)");
  c->h_stage_bytes = want;
  return NOVA_B200_SUCCESS;
}

/* One small piece read by the device straight from the caller's pinned host memory. */
struct GatherPiece {
  const char *src; /* device-accessible address of pinned host memory */
  char *dst;
  uint32_t bytes;
};

/* One block per piece: 16-byte words when both ends are 16-byte aligned, else bytes. */
__global__ void k_gather_pieces(const GatherPiece *pieces) {
  const GatherPiece g = pieces[blockIdx.x];
  if (!((reinterpret_cast<uintptr_t>(g.src) | reinterpret_cast<uintptr_t>(g.dst)) & 15)) {
    const uint32_t n16 = g.bytes >> 4;
    const uint4 *s4 = reinterpret_cast<const uint4 *>(g.src);
    uint4 *d4 = reinterpret_cast<uint4 *>(g.dst);
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) d4[i] = s4[i];
    for (uint32_t i = (n16 << 4) + threadIdx.x; i < g.bytes; i += blockDim.x) g.dst[i] = g.src[i];
  } else {
    for (uint32_t i = threadIdx.x; i < g.bytes; i += blockDim.x) g.dst[i] = g.src[i];
  }
}

/* Device-accessible address of pinned (page-locked, mapped) host memory, or null for anything else. */
const char *pinned_device_address(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? static_cast<const char *>(a.devicePointer) : nullptr;
}

/* Copies the plan's pieces: large ones with one transfer each; small ones from pinned caller memory
 * by one gather kernel that reads them over the bus (no host copy, one launch), the rest through
 * the context's pinned staging buffer (one transfer per run of adjacent pieces). */
nova_b200_status copy_pieces(nova_b200_ctx *c, const UploadPlan &plan, char *arena, char *temp) {
  std::vector<GatherPiece> gather;
  std::vector<char> pinned(plan.pieces.size(), 0);
  size_t small = 0;
  for (size_t k = 0; k < plan.pieces.size(); k++) {
    const Piece &p = plan.pieces[k];
    if (p.bytes > kSmallPiece || p.bytes == 0) continue;
    if (const char *src = pinned_device_address(p.src)) {
      pinned[k] = 1;
      gather.push_back(GatherPiece{src, (p.temp ? temp : arena) + p.off, (uint32_t)p.bytes});
    } else {
      small += UploadPlan::align(p.bytes);
    }
  }
  const size_t table = gather.size() * sizeof(GatherPiece);
  nova_b200_status st = ensure_pinned_stage(c, small + table + 256);
  if (st != NOVA_B200_SUCCESS) return st;
  if (!gather.empty()) {
    /* the table goes at the end of the staging buffer, read by the kernel over the bus as well */
    char *tab = static_cast<char *>(c->h_stage) + UploadPlan::align(small);
    std::memcpy(tab, gather.data(), table);
    const char *tab_dev = pinned_device_address(tab);
    if (!tab_dev) return nbctx::fail(c, NOVA_B200_RENDERER_EXCEPTION, "staging buffer is not device-accessible%s");
    k_gather_pieces<<<(unsigned)gather.size(), 256, 0, c->stream>>>(reinterpret_cast<const GatherPiece *>(tab_dev));
    NB_CUDA(c, cudaGetLastError(), "k_gather_pieces");
  }
  /* small pieces are packed per region in plan order; each region's packed pieces are contiguous
   * neither on the host nor on the device in general, so runs of adjacent pieces are merged */
  char *h = static_cast<char *>(c->h_stage);
  size_t hoff = 0;
  struct Run {
    char *dst;
    size_t hbegin, bytes;
  };
  std::vector<Run> runs;
  for (size_t k = 0; k < plan.pieces.size(); k++) {
    const Piece &p = plan.pieces[k];
    char *dst = (p.temp ? temp : arena) + p.off;
    if (p.bytes > kSmallPiece) {
      NB_CUDA(c, cudaMemcpyAsync(dst, p.src, p.bytes, cudaMemcpyHostToDevice, c->stream), "upload(scene)");
      continue;
    }
    if (pinned[k] || p.bytes == 0) continue;
    std::memcpy(h + hoff, p.src, p.bytes);
    const size_t step = UploadPlan::align(p.bytes);
    if (!runs.empty() && runs.back().dst + runs.back().bytes == dst && runs.back().hbegin + runs.back().bytes == hoff)
      runs.back().bytes += step;
    else
      runs.push_back(Run{dst, hoff, step});
    hoff += step;
  }
  for (const Run &r : runs)
    NB_CUDA(c, cudaMemcpyAsync(r.dst, h + r.hbegin, r.bytes, cudaMemcpyHostToDevice, c->stream), "upload(scene)");
  return NOVA_B200_SUCCESS;
}

void free_scene(nova_b200_ctx *c) {
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->d_arena) cudaFreeAsync(c->d_arena, c->stream);
  if (c->d_nodes) cudaFreeAsync(c->d_nodes, c->stream);
  if (c->d_tris) cudaFreeAsync(c->d_tris, c->stream);
  if (c->d_valid) cudaFreeAsync(c->d_valid, c->stream);
  if (c->d_blas_root) cudaFreeAsync(c->d_blas_root, c->stream);
  c->d_blas_root = nullptr;
  c->h_meshes.clear();
  c->d_arena = nullptr;
  c->d_nodes = nullptr;
  c->d_tris = nullptr;
  c->d_valid = nullptr;
  c->n_valid = 0;
  c->scene = nb::DevScene{};
  c->h_instances.clear();
  c->scene_ready = c->bvh_ready = false;
  c->primal_valid = false;
  c->scene_bytes = 0;
  c->n_nodes = c->n_leaves = 0;
}

/* ------------------------------------------------------------------ build kernels */

__global__ void k_prim_boxes(nb::DevScene sc, const uint32_t *valid, uint32_t n, float4 *lo, float4 *hi) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t prim = valid[i];
  const uint32_t inst = sc.prim_inst[prim];
  const nb::DevInstance &I = sc.instances[inst];
  const nb::DevMesh &m = sc.meshes[I.mesh];
  const uint32_t tri = prim - I.prim_offset;
  nb::V3 w[3];
  for (int k = 0; k < 3; k++) {
    const nb::V3 v = nb::vertex_position(m, m.idx[3 * tri + k]);
    w[k] = I.identity ? v : nb::xform_point(I.m, v);
  }
  lo[i] = make_float4(fminf(w[0].x, fminf(w[1].x, w[2].x)), fminf(w[0].y, fminf(w[1].y, w[2].y)),
                      fminf(w[0].z, fminf(w[1].z, w[2].z)), 0.f);
  hi[i] = make_float4(fmaxf(w[0].x, fmaxf(w[1].x, w[2].x)), fmaxf(w[0].y, fmaxf(w[1].y, w[2].y)),
                      fmaxf(w[0].z, fmaxf(w[1].z, w[2].z)), 0.f);
}

/* Triangle records in leaf order: (v0, prim id), (v1 - v0, instance), (v2 - v0, 0), object space. */
__global__ void k_write_tris(nb::DevScene sc, const uint32_t *valid, const uint32_t *order, uint32_t n, float4 *tris) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t prim = valid[order[k]];
  const uint32_t inst = sc.prim_inst[prim];
  const nb::DevInstance &I = sc.instances[inst];
  const nb::DevMesh &m = sc.meshes[I.mesh];
  const uint32_t tri = prim - I.prim_offset;
  const uint32_t a = m.idx[3 * tri], b = m.idx[3 * tri + 1], cc = m.idx[3 * tri + 2];
  const nb::V3 v0 = nb::vertex_position(m, a), v1 = nb::vertex_position(m, b), v2 = nb::vertex_position(m, cc);
  const nb::V3 e1 = v1 - v0, e2 = v2 - v0;
  tris[3 * k + 0] = make_float4(v0.x, v0.y, v0.z, __int_as_float((int)prim));
  tris[3 * k + 1] = make_float4(e1.x, e1.y, e1.z, __int_as_float((int)inst));
  tris[3 * k + 2] = make_float4(e2.x, e2.y, e2.z, 0.f);
}

/* Where one mesh's SoA attributes sit in the staging region and its 64 B records in the arena
 * (byte offsets), and its first vertex in the scene-wide vertex numbering. */
struct InterleaveMesh {
  uint64_t v, n, t, b, uv, attr;
  uint32_t first_vertex, n_verts;
};

/* Interleaves the SoA vertex attributes of every mesh into 64 B records (layout in
 * device_scene.cuh): one thread per vertex of the scene, the mesh found by binary search. */
__global__ void k_interleave(const InterleaveMesh *meshes, uint32_t n_meshes, uint32_t total, const char *stage,
                             char *arena) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  uint32_t lo = 0, hi = n_meshes;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (meshes[mid].first_vertex <= g)
      lo = mid;
    else
      hi = mid;
  }
  const InterleaveMesh &m = meshes[lo];
  const uint32_t i = g - m.first_vertex;
  if (i >= m.n_verts) return;
  const float *v = reinterpret_cast<const float *>(stage + m.v), *n = reinterpret_cast<const float *>(stage + m.n);
  const float *t = reinterpret_cast<const float *>(stage + m.t), *b = reinterpret_cast<const float *>(stage + m.b);
  const float *uv = reinterpret_cast<const float *>(stage + m.uv);
  float4 *attr = reinterpret_cast<float4 *>(arena + m.attr);
  attr[4 * (size_t)i + 0] = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], n[3 * i]);
  attr[4 * (size_t)i + 1] = make_float4(n[3 * i + 1], n[3 * i + 2], t[3 * i], t[3 * i + 1]);
  attr[4 * (size_t)i + 2] = make_float4(t[3 * i + 2], b[3 * i], b[3 * i + 1], b[3 * i + 2]);
  attr[4 * (size_t)i + 3] = make_float4(uv[2 * i], uv[2 * i + 1], 0.f, 0.f);
}

/* Per global primitive (instance by instance, triangle by triangle): its instance (binary search on
 * the instances' first primitive ids), a flag for "can be hit" (no repeated vertex index,
 * Triangle.h:127-132) and the check that its indices name vertices of its mesh (bad[0] |= 1). */
__global__ void k_scene_tables(const nb::DevInstance *inst, uint32_t n_inst, const nb::DevMesh *meshes, uint32_t n_prims,
                               uint32_t *prim_inst, uint32_t *can_hit, unsigned *bad) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_prims) return;
  uint32_t lo = 0, hi = n_inst;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (inst[mid].prim_offset <= p)
      lo = mid;
    else
      hi = mid;
  }
  const nb::DevMesh &m = meshes[inst[lo].mesh];
  const uint32_t t = p - inst[lo].prim_offset;
  const uint32_t a = m.idx[3 * (size_t)t], b = m.idx[3 * (size_t)t + 1], c = m.idx[3 * (size_t)t + 2];
  if (a >= m.n_verts || b >= m.n_verts || c >= m.n_verts) atomicOr(bad, 1u);
  prim_inst[p] = lo;
  can_hit[p] = (a == b || c == b || c == a) ? 0u : 1u;
}

/* Stable compaction of the primitives that can be hit: per block of kCompactItems flags a count,
 * one block scans the counts (block offsets and the total), then each block writes its ids. */
constexpr uint32_t kCompactThreads = 1024, kCompactPer = 4, kCompactItems = kCompactThreads * kCompactPer;

__device__ __forceinline__ uint32_t block_excl_scan1024(uint32_t v, uint32_t *sh /* 32 */, uint32_t *total) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = sh[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    sh[lane] = s; /* inclusive over warps */
  }
  __syncthreads();
  const uint32_t before = (w ? sh[w - 1] : 0u) + x - v;
  *total = sh[31];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kCompactThreads) k_compact_count(const uint32_t *flags, uint32_t n, uint32_t *counts) {
  __shared__ uint32_t sh[32];
  const uint32_t base = blockIdx.x * kCompactItems + threadIdx.x * kCompactPer;
  uint32_t c = 0;
  for (uint32_t k = 0; k < kCompactPer; k++)
    if (base + k < n) c += flags[base + k];
  uint32_t total;
  block_excl_scan1024(c, sh, &total);
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kCompactThreads) k_compact_offsets(uint32_t *counts, uint32_t n_blocks,
                                                                     uint32_t *total_out) {
  __shared__ uint32_t sh[32];
  const uint32_t per = (n_blocks + kCompactThreads - 1) / kCompactThreads;
  const uint32_t b = threadIdx.x * per, e = min(b + per, n_blocks);
  uint32_t sum = 0;
  for (uint32_t i = b; i < e; i++) sum += counts[i];
  uint32_t total;
  uint32_t run = block_excl_scan1024(sum, sh, &total);
  for (uint32_t i = b; i < e; i++) {
    const uint32_t cnt = counts[i];
    counts[i] = run;
    run += cnt;
  }
  if (threadIdx.x == 0) *total_out = total;
}

__global__ void __launch_bounds__(kCompactThreads) k_compact_write(const uint32_t *flags, uint32_t n,
                                                                   const uint32_t *offsets, uint32_t *out) {
  __shared__ uint32_t sh[32];
  const uint32_t base = blockIdx.x * kCompactItems + threadIdx.x * kCompactPer;
  uint32_t f[kCompactPer], c = 0;
  for (uint32_t k = 0; k < kCompactPer; k++) {
    f[k] = base + k < n ? flags[base + k] : 0u;
    c += f[k];
  }
  uint32_t total;
  uint32_t pos = offsets[blockIdx.x] + block_excl_scan1024(c, sh, &total);
  for (uint32_t k = 0; k < kCompactPer; k++)
    if (f[k]) out[pos++] = base + k;
}

__global__ void k_validate(const float4 *nodes, uint32_t n_nodes, uint32_t n_tris, unsigned *bad) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_nodes) return;
  const float4 n3 = nodes[4 * i + 3];
  const int32_t r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
  for (int s = 0; s < 2; s++) {
    if (r[s] >= 0) {
      if ((uint32_t)r[s] <= i || (uint32_t)r[s] >= n_nodes) atomicAdd(bad, 1u);
    } else {
      const uint32_t f = nb::leaf_first(r[s]), cnt = nb::leaf_count(r[s]);
      if (f + cnt > n_tris) atomicAdd(bad, 1u);
    }
  }
}

/* ------------------------------------------------------------------ two-level BVH (width 1)
 *
 * The reference's Embree accelerator keeps one sub-scene per mesh under its instances
 * (aggregate/api/embree/embree.cpp:236-254).  Here: a binary BVH per mesh over its object-space
 * triangles that can be hit (bottom level, built once however many instances use the mesh), and a
 * binary BVH over the instances' world-space boxes with one instance per leaf (top level), in one
 * node array: the top level first, then each mesh's nodes with their references relocated.  Bottom
 * triangle records hold the mesh-local triangle id; the hit's primitive id is the instance's first
 * primitive id plus it, the reference's numbering (api/engine.cpp:159-175). */

/* 1 where a mesh triangle can be hit (no repeated vertex index, Triangle.h:127-132). */
__global__ void k_mesh_flags(nb::DevMesh m, uint32_t *flags) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.n_tris) return;
  const uint32_t a = m.idx[3 * (size_t)t], b = m.idx[3 * (size_t)t + 1], c = m.idx[3 * (size_t)t + 2];
  flags[t] = (a == b || c == b || c == a) ? 0u : 1u;
}

__global__ void k_mesh_boxes(nb::DevMesh m, const uint32_t *ids, uint32_t n, float4 *lo, float4 *hi) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t t = ids[i];
  nb::V3 w[3];
  for (int k = 0; k < 3; k++) w[k] = nb::vertex_position(m, m.idx[3 * (size_t)t + k]);
  lo[i] = make_float4(fminf(w[0].x, fminf(w[1].x, w[2].x)), fminf(w[0].y, fminf(w[1].y, w[2].y)),
                      fminf(w[0].z, fminf(w[1].z, w[2].z)), 0.f);
  hi[i] = make_float4(fmaxf(w[0].x, fmaxf(w[1].x, w[2].x)), fmaxf(w[0].y, fmaxf(w[1].y, w[2].y)),
                      fmaxf(w[0].z, fmaxf(w[1].z, w[2].z)), 0.f);
}

/* Bottom-level triangle records in leaf order: (v0, mesh-local triangle id), (v1 - v0, 0), (v2 - v0, 0). */
__global__ void k_write_blas_tris(nb::DevMesh m, const uint32_t *ids, const uint32_t *order, uint32_t n, float4 *tris) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t t = ids[order[k]];
  const uint32_t a = m.idx[3 * (size_t)t], b = m.idx[3 * (size_t)t + 1], cc = m.idx[3 * (size_t)t + 2];
  const nb::V3 v0 = nb::vertex_position(m, a), v1 = nb::vertex_position(m, b), v2 = nb::vertex_position(m, cc);
  const nb::V3 e1 = v1 - v0, e2 = v2 - v0;
  tris[3 * k + 0] = make_float4(v0.x, v0.y, v0.z, __int_as_float((int)t));
  tris[3 * k + 1] = make_float4(e1.x, e1.y, e1.z, 0.f);
  tris[3 * k + 2] = make_float4(e2.x, e2.y, e2.z, 0.f);
}

/* A bottom level built at node 0 moved to node_base, its triangles to tri_base. */
__global__ void k_relocate(float4 *nodes, uint32_t n_nodes, uint32_t node_base, uint32_t tri_base) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_nodes) return;
  float4 &n3 = nodes[4 * (size_t)(node_base + i) + 3];
  int32_t r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
  for (int s = 0; s < 2; s++)
    r[s] = r[s] >= 0 ? r[s] + (int32_t)node_base : nb::leaf_ref(nb::leaf_first(r[s]) + tri_base, nb::leaf_count(r[s]));
  n3.x = __int_as_float(r[0]);
  n3.y = __int_as_float(r[1]);
}

/* World box of each instance: the eight corners of its mesh's bottom-level root box, transformed. */
__global__ void k_instance_boxes(const nb::DevInstance *inst, uint32_t n, const float4 *nodes, const uint32_t *blas_root,
                                 float4 *lo, float4 *hi) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const nb::DevInstance &I = inst[i];
  const float4 *rn = nodes + 4 * (size_t)blas_root[I.mesh];
  const float4 n0 = rn[0], n1 = rn[1], n2 = rn[2];
  /* union of the root's two child boxes (an empty child box is inverted and drops out) */
  const nb::V3 bl{fminf(n0.x, n1.x), fminf(n0.z, n1.z), fminf(n2.x, n2.z)};
  const nb::V3 bh{fmaxf(n0.y, n1.y), fmaxf(n0.w, n1.w), fmaxf(n2.y, n2.w)};
  nb::V3 wl{FLT_MAX, FLT_MAX, FLT_MAX}, wh{-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int k = 0; k < 8; k++) {
    const nb::V3 p{(k & 1) ? bh.x : bl.x, (k & 2) ? bh.y : bl.y, (k & 4) ? bh.z : bl.z};
    const nb::V3 w = I.identity ? p : nb::xform_point(I.m, p);
    wl = nb::V3{fminf(wl.x, w.x), fminf(wl.y, w.y), fminf(wl.z, w.z)};
    wh = nb::V3{fmaxf(wh.x, w.x), fmaxf(wh.y, w.y), fmaxf(wh.z, w.z)};
  }
  lo[i] = make_float4(wl.x, wl.y, wl.z, 0.f);
  hi[i] = make_float4(wh.x, wh.y, wh.z, 0.f);
}

/* Top-level leaves (one instance each) name the instance itself instead of its slot in `order`. */
__global__ void k_top_leaves(float4 *nodes, uint32_t n_nodes, const uint32_t *order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_nodes) return;
  float4 &n3 = nodes[4 * (size_t)i + 3];
  int32_t r[2] = {__float_as_int(n3.x), __float_as_int(n3.y)};
  for (int s = 0; s < 2; s++)
    if (r[s] < 0) r[s] = nb::leaf_ref(order[nb::leaf_first(r[s])], 1u);
  n3.x = __int_as_float(r[0]);
  n3.y = __int_as_float(r[1]);
}

/* Builds the two-level BVH into c->d_nodes / c->d_tris / c->d_blas_root.  res: total nodes, leaves,
 * and the deepest top + bottom path (for the traversal stack). */
nova_b200_status build_two_level(nova_b200_ctx *c, const nb::BvhBuildParams &p, nb::BvhBuildResult &res) {
  using namespace nbctx;
  const uint32_t n_inst = (uint32_t)c->h_instances.size(), n_meshes = (uint32_t)c->h_meshes.size();
  std::vector<char> used(n_meshes, 0);
  for (const nb::DevInstance &I : c->h_instances) used[I.mesh] = 1;
  /* per used mesh: the triangles that can be hit, compacted on the device */
  std::vector<uint32_t *> ids(n_meshes, nullptr);
  std::vector<uint32_t> count(n_meshes, 0);
  uint32_t *counts_h = c->h_counters; /* 16 pinned words: done in batches of 8 meshes (count, bad) */
  auto free_ids = [&] {
    for (uint32_t *q : ids)
      if (q) cudaFreeAsync(q, c->stream);
  };
  for (uint32_t m0 = 0; m0 < n_meshes; m0 += 8) {
    const uint32_t m1 = std::min(n_meshes, m0 + 8);
    for (uint32_t m = m0; m < m1; m++) {
      if (!used[m]) continue;
      const nb::DevMesh &M = c->h_meshes[m];
      const uint32_t T = M.n_tris, nb_ = (T + kCompactItems - 1) / kCompactItems;
      uint32_t *flags = nullptr, *cnts = nullptr;
      cudaError_t e = cudaMallocAsync(&ids[m], sizeof(uint32_t) * T, c->stream);
      if (e == cudaSuccess) e = cudaMallocAsync(&flags, sizeof(uint32_t) * T, c->stream);
      if (e == cudaSuccess) e = cudaMallocAsync(&cnts, sizeof(uint32_t) * (nb_ + 1), c->stream);
      if (e == cudaSuccess) {
        k_mesh_flags<<<(T + 255) / 256, 256, 0, c->stream>>>(M, flags);
        k_compact_count<<<nb_, kCompactThreads, 0, c->stream>>>(flags, T, cnts);
        k_compact_offsets<<<1, kCompactThreads, 0, c->stream>>>(cnts, nb_, c->d_counters + (m - m0));
        k_compact_write<<<nb_, kCompactThreads, 0, c->stream>>>(flags, T, cnts, ids[m]);
        e = cudaGetLastError();
      }
      if (flags) cudaFreeAsync(flags, c->stream);
      if (cnts) cudaFreeAsync(cnts, c->stream);
      if (e != cudaSuccess) {
        free_ids();
        return cuda_fail(c, e, "two-level BVH: triangle lists");
      }
    }
    NB_CUDA(c, cudaMemcpyAsync(counts_h, c->d_counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream),
            "readback");
    NB_CUDA(c, cudaStreamSynchronize(c->stream), "two-level BVH");
    for (uint32_t m = m0; m < m1; m++)
      if (used[m]) count[m] = counts_h[m - m0];
  }
  /* node and triangle offsets: top level first */
  const size_t top_nodes = std::max<size_t>(2 * (size_t)n_inst, 2);
  std::vector<uint32_t> node_off(n_meshes, 0), tri_off(n_meshes, 0);
  size_t total_nodes = top_nodes, total_tris = 0;
  size_t real_tris = 0;
  for (uint32_t m = 0; m < n_meshes; m++) {
    if (!used[m]) continue;
    node_off[m] = (uint32_t)total_nodes;
    tri_off[m] = (uint32_t)total_tris;
    /* a mesh of degenerate triangles only gets one node over one zero triangle (never hit) */
    total_nodes += std::max<size_t>(2 * (size_t)count[m], 2);
    total_tris += std::max<uint32_t>(count[m], 1u);
    real_tris += count[m];
  }
  if (real_tris == 0 || total_nodes >= (1ull << 31) || total_tris >= (1ull << 27)) {
    free_ids();
    return fail(c, NOVA_B200_INVALID_SCENE_TYPE, "two-level BVH: no triangle can be hit, or too many%s");
  }
  float4 *lo = nullptr, *hi = nullptr;
  uint32_t *order = nullptr;
  size_t scratch = n_inst;
  for (uint32_t m = 0; m < n_meshes; m++) scratch = std::max<size_t>(scratch, count[m]);
  cudaError_t e = cudaMallocAsync(&c->d_nodes, sizeof(float4) * 4 * total_nodes, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&c->d_tris, sizeof(float4) * 3 * total_tris, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&c->d_blas_root, sizeof(uint32_t) * n_meshes, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_nodes, 0, sizeof(float4) * 4 * total_nodes, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_tris, 0, sizeof(float4) * 3 * total_tris, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&lo, sizeof(float4) * scratch, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&hi, sizeof(float4) * scratch, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&order, sizeof(uint32_t) * scratch, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_counters, 0, 4, c->stream);
  auto cleanup = [&] {
    free_ids();
    if (lo) cudaFreeAsync(lo, c->stream);
    if (hi) cudaFreeAsync(hi, c->stream);
    if (order) cudaFreeAsync(order, c->stream);
  };
  if (e != cudaSuccess) {
    cleanup();
    return cuda_fail(c, e, "cudaMalloc(two-level BVH)");
  }
  /* bottom levels */
  std::vector<uint32_t> roots(n_meshes, 0);
  nb::BvhBuildResult r{};
  int bottom_depth = 0;
  res = nb::BvhBuildResult{};
  for (uint32_t m = 0; m < n_meshes; m++) {
    if (!used[m]) continue;
    if (count[m] == 0) { /* the placeholder: a point box at the origin over a zero triangle */
      float4 node[4] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f),
                        make_float4(0.f, 0.f, 0.f, 0.f)};
      const int32_t ref = nb::leaf_ref(tri_off[m], 1u);
      node[3].x = node[3].y = *reinterpret_cast<const float *>(&ref);
      e = cudaMemcpyAsync(c->d_nodes + 4 * (size_t)node_off[m], node, sizeof(node), cudaMemcpyHostToDevice, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream); /* `node` is a stack array */
      if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(c, e, "two-level BVH: placeholder");
      }
      roots[m] = node_off[m]; /* its triangle record stays zero (the array was cleared) */
      continue;
    }
    const uint32_t n = count[m];
    const nb::DevMesh &M = c->h_meshes[m];
    float4 *nodes = c->d_nodes + 4 * (size_t)node_off[m];
    float4 *tris = c->d_tris + 3 * (size_t)tri_off[m];
    k_mesh_boxes<<<(n + 255) / 256, 256, 0, c->stream>>>(M, ids[m], n, lo, hi);
    e = nb::build_bvh(lo, hi, n, p, nodes, order, c->stream, &r);
    if (e == cudaSuccess) {
      k_write_blas_tris<<<(n + 255) / 256, 256, 0, c->stream>>>(M, ids[m], order, n, tris);
      k_validate<<<(r.n_nodes + 255) / 256, 256, 0, c->stream>>>(nodes, r.n_nodes, n, c->d_counters);
      k_relocate<<<(r.n_nodes + 255) / 256, 256, 0, c->stream>>>(c->d_nodes, r.n_nodes, node_off[m], tri_off[m]);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess || r.n_nodes > std::max<uint32_t>(2 * n, 2)) {
      cleanup();
      return e != cudaSuccess ? cuda_fail(c, e, "two-level BVH: bottom level")
                              : fail(c, NOVA_B200_RENDERER_EXCEPTION, "BVH validation failed%s");
    }
    roots[m] = node_off[m];
    res.n_nodes += r.n_nodes;
    res.n_leaves += r.n_leaves;
    res.ms += r.ms;
    bottom_depth = std::max(bottom_depth, r.max_depth);
  }
  NB_CUDA(c, cudaMemcpyAsync(c->d_blas_root, roots.data(), sizeof(uint32_t) * n_meshes, cudaMemcpyHostToDevice,
                             c->stream),
          "upload(bottom-level roots)");
  /* top level: one instance per leaf */
  nb::BvhBuildParams pt = p;
  pt.max_leaf = 1;
  pt.hard_leaf = 1;
  const nb::DevInstance *d_inst = c->scene.instances;
  k_instance_boxes<<<(n_inst + 255) / 256, 256, 0, c->stream>>>(d_inst, n_inst, c->d_nodes, c->d_blas_root, lo, hi);
  e = nb::build_bvh(lo, hi, n_inst, pt, c->d_nodes, order, c->stream, &r);
  if (e == cudaSuccess) {
    k_validate<<<(r.n_nodes + 255) / 256, 256, 0, c->stream>>>(c->d_nodes, r.n_nodes, n_inst, c->d_counters);
    k_top_leaves<<<(r.n_nodes + 255) / 256, 256, 0, c->stream>>>(c->d_nodes, r.n_nodes, order);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->h_counters, c->d_counters, 4, cudaMemcpyDeviceToHost, c->stream);
  cleanup();
  if (e != cudaSuccess) return cuda_fail(c, e, "two-level BVH: top level");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "two-level BVH");
  res.n_nodes += r.n_nodes;
  res.n_leaves += r.n_leaves;
  res.ms += r.ms;
  res.max_depth = r.max_depth + bottom_depth + 1; /* + the stack entry that leaves an instance */
  if (c->h_counters[0] != 0 || r.n_nodes == 0 || r.n_nodes > top_nodes || res.max_depth >= nb::kTraversalStack)
    return fail(c, NOVA_B200_RENDERER_EXCEPTION, "BVH validation failed%s");
  return NOVA_B200_SUCCESS;
}

/* Runs op(k) for k < n on up to 16 host threads; returns the first failing status (its message is
 * copied to ctxs[0]). */
template <class Op>
nova_b200_status for_each_context(nova_b200_ctx *const *ctxs, uint32_t n, Op op) {
  if (!ctxs || n == 0 || !ctxs[0]) return NOVA_B200_INVALID_ARGUMENT;
  for (uint32_t k = 0; k < n; k++)
    if (!ctxs[k]) return nbctx::fail(ctxs[0], NOVA_B200_INVALID_ARGUMENT, "null context in batch%s");
  for (uint32_t k = 0; k < n; k++)
    for (uint32_t m = 0; m < k; m++)
      if (ctxs[k] == ctxs[m]) return nbctx::fail(ctxs[0], NOVA_B200_INVALID_ARGUMENT, "a context appears twice%s");
  std::vector<nova_b200_status> st(n, NOVA_B200_SUCCESS);
  std::atomic<uint32_t> next{0};
  const unsigned nt = std::max(1u, std::min(std::min(n, 16u), std::max(1u, std::thread::hardware_concurrency())));
  auto work = [&] {
    for (uint32_t k; (k = next.fetch_add(1)) < n;) st[k] = op(k);
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
  work();
  for (auto &t : pool) t.join();
  for (uint32_t k = 0; k < n; k++)
    if (st[k] != NOVA_B200_SUCCESS) {
      if (k != 0) ctxs[0]->error = ctxs[k]->error;
      return st[k];
    }
  return NOVA_B200_SUCCESS;
}

}  // namespace

extern "C" {

nova_b200_status nova_b200_create(nova_b200_ctx **out, int32_t device) {
  if (!out) return NOVA_B200_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return NOVA_B200_NOT_GPU_BUILD;
  if (device < 0 || device >= count) return NOVA_B200_INVALID_ARGUMENT;
  nova_b200_ctx *c = new nova_b200_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev_begin) != cudaSuccess || cudaEventCreate(&c->ev_end) != cudaSuccess ||
      cudaEventCreate(&c->ev_a) != cudaSuccess || cudaEventCreate(&c->ev_b) != cudaSuccess) {
    delete c;
    return NOVA_B200_RENDER_ENGINE_NOT_INITIALIZED;
  }
  /* keep memory freed with cudaFreeAsync (BVH build scratch, upload staging) in the device pool
   * instead of returning it to the driver at every synchronisation */
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  std::vector<uint32_t> dv, sob;
  std::vector<float> ac;
  sobol_table(dv);
  sobol_byte_tables(dv, sob);
  acos_table(ac);
  if (cudaMalloc(&c->d_sobol, sob.size() * 4) != cudaSuccess || cudaMalloc(&c->d_acos, ac.size() * 4) != cudaSuccess ||
      cudaMalloc(&c->d_counters, 64) != cudaSuccess || cudaMallocHost(&c->h_counters, 64) != cudaSuccess) {
    nova_b200_destroy(c);
    return NOVA_B200_OUT_OF_MEMORY;
  }
  cudaMemcpy(c->d_sobol, sob.data(), sob.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(c->d_acos, ac.data(), ac.size() * 4, cudaMemcpyHostToDevice);
  /* the allocation-free render's device memory (its static scratch array and its kernel's local
   * memory) is taken here, so that nova_b200_render_noalloc itself never allocates */
  const nova_b200_status st = nb_noalloc_prepare(c);
  if (st != NOVA_B200_SUCCESS) {
    nova_b200_destroy(c);
    return st;
  }
  *out = c;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_destroy(nova_b200_ctx *c) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  free_scene(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  cudaFree(c->d_adj);
  cudaFree(c->d_sobol);
  cudaFree(c->d_acos);
  cudaFree(c->d_counters);
  cudaFree(c->d_film_acc);
  cudaFree(c->d_queue);
  cudaFree(c->d_radiance);
  cudaFree(c->d_film_out);
  cudaFree(c->d_wave);
  cudaFree(c->d_persist);
  if (c->h_cancel_map) cudaFreeHost(const_cast<int *>(c->h_cancel_map));
  if (c->h_wave) cudaFreeHost(c->h_wave);
  for (cudaGraphExec_t g : c->graph_exec)
    if (g) cudaGraphExecDestroy(g);
  for (cudaEvent_t e : c->ev_done)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : c->ev_wave)
    if (e) cudaEventDestroy(e);
  if (c->h_counters) cudaFreeHost(c->h_counters);
  if (c->ev_begin) cudaEventDestroy(c->ev_begin);
  if (c->ev_end) cudaEventDestroy(c->ev_end);
  if (c->ev_a) cudaEventDestroy(c->ev_a);
  if (c->ev_b) cudaEventDestroy(c->ev_b);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream), cudaStreamDestroy(c->copy_stream);
  if (c->ev_copy) cudaEventDestroy(c->ev_copy);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_upload_scene(nova_b200_ctx *c, const nova_b200_scene_desc *d) {
  using namespace nbctx;
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (!d) return fail(c, NOVA_B200_INVALID_ARGUMENT, "scene descriptor is null%s");
  cudaSetDevice(c->device);
  free_scene(c);
  if (d->n_instances == 0 || !d->instances || !d->meshes || d->n_meshes == 0)
    return fail(c, NOVA_B200_INVALID_SCENE_TYPE, "scene has no meshes or instances%s");
  if (d->envmap < 0 || (uint32_t)d->envmap >= d->n_textures || !d->textures[d->envmap].f32_pixels ||
      d->textures[d->envmap].channels != 4)
    return fail(c, NOVA_B200_INVALID_SCENE_TYPE, "environment map must be a 4-channel float texture%s");
  UploadPlan plan;
  /* textures: the device pointers are patched in once the arena exists */
  std::vector<nb::DevTexture> tex(d->n_textures);
  std::vector<size_t> tex_off(d->n_textures);
  for (uint32_t i = 0; i < d->n_textures; i++) {
    const nova_b200_texture &t = d->textures[i];
    if ((!t.u8_pixels) == (!t.f32_pixels) || t.width < 2 || t.height < 2 || t.channels < 1 || t.channels > 4)
      return fail(c, NOVA_B200_INVALID_CHANNEL_DESCRIPTOR, "texture needs exactly one pixel buffer, >= 2x2 texels%s");
    nb::DevTexture &o = tex[i];
    o.w = t.width, o.h = t.height, o.ch = t.channels;
    o.is_rgba = t.is_rgba, o.invert_u = t.invert_u, o.invert_v = t.invert_v;
    const size_t px = (size_t)t.width * t.height;
    tex_off[i] = t.u8_pixels ? plan.add(t.u8_pixels, px * sizeof(uint32_t))
                             : plan.add(t.f32_pixels, px * t.channels * sizeof(float));
  }
  /* materials */
  std::vector<nb::DevMaterial> mats(d->n_materials);
  bool emissive = false;
  for (uint32_t i = 0; i < d->n_materials; i++) {
    const nova_b200_material &m = d->materials[i];
    const int32_t slots[4] = {m.albedo, m.metallic, m.normalmap, m.emissive};
    for (int32_t s : slots)
      if (s >= (int32_t)d->n_textures || (s >= 0 && !d->textures[s].u8_pixels))
        return fail(c, NOVA_B200_INVALID_ARGUMENT, "material texture slot must name an 8-bit texture or be -1%s");
    mats[i].albedo = m.albedo, mats[i].metallic = m.metallic, mats[i].normalmap = m.normalmap;
    mats[i].emissive = m.emissive;
    for (int k = 0; k < 3; k++) mats[i].eta[k] = m.eta[k], mats[i].k[k] = m.k[k];
    mats[i].anisotropy = m.anisotropy;
    emissive |= m.emissive >= 0;
  }
  /* meshes: indices to the arena, SoA attributes to the temporary staging region, interleaved
   * into the arena's 64 B records by k_interleave */
  std::vector<nb::DevMesh> meshes(d->n_meshes);
  struct MeshOffsets {
    size_t idx, attr, v, n, t, b, uv;
  };
  std::vector<MeshOffsets> moff(d->n_meshes);
  std::vector<InterleaveMesh> ilv(d->n_meshes);
  uint64_t total_verts = 0;
  for (uint32_t i = 0; i < d->n_meshes; i++) {
    const nova_b200_mesh &m = d->meshes[i];
    if (!m.vertices || !m.normals || !m.tangents || !m.bitangents || !m.uv || !m.indices || m.n_tris == 0)
      return fail(c, NOVA_B200_INVALID_ARGUMENT, "mesh needs vertices, normals, tangents, bitangents, uv, indices%s");
    meshes[i].n_verts = m.n_verts, meshes[i].n_tris = m.n_tris;
    const size_t nv = m.n_verts;
    MeshOffsets &o = moff[i];
    o.idx = plan.add(m.indices, 3ull * m.n_tris * sizeof(uint32_t));
    o.attr = plan.arena;
    plan.arena += UploadPlan::align(nv * 64);
    o.v = plan.add(m.vertices, 12 * nv, true);
    o.n = plan.add(m.normals, 12 * nv, true);
    o.t = plan.add(m.tangents, 12 * nv, true);
    o.b = plan.add(m.bitangents, 12 * nv, true);
    o.uv = plan.add(m.uv, 8 * nv, true);
    ilv[i] = InterleaveMesh{o.v, o.n, o.t, o.b, o.uv, o.attr, (uint32_t)total_verts, m.n_verts};
    total_verts += nv;
  }
  if (total_verts >= (1ull << 32)) return fail(c, NOVA_B200_OUT_OF_MEMORY, "more than 2^32 vertices%s");
  const size_t off_ilv = plan.add(ilv.data(), ilv.size() * sizeof(InterleaveMesh), true);
  /* instances + primitive tables */
  c->h_instances.resize(d->n_instances);
  uint64_t offset = 0;
  for (uint32_t i = 0; i < d->n_instances; i++) {
    const nova_b200_instance &x = d->instances[i];
    if (x.mesh >= d->n_meshes || x.material >= d->n_materials)
      return fail(c, NOVA_B200_INVALID_ARGUMENT, "instance references a missing mesh or material%s");
    nb::DevInstance &o = c->h_instances[i];
    std::memcpy(o.m, x.m, sizeof(o.m));
    std::memcpy(o.inv, x.inv, sizeof(o.inv));
    std::memcpy(o.n, x.n, sizeof(o.n));
    o.mesh = x.mesh;
    o.material = x.material;
    o.prim_offset = (uint32_t)offset;
    o.identity = is_identity(x.m) && is_identity(x.inv);
    {
      const nova_b200_material &mt = d->materials[x.material];
      const bool eta = mt.eta[0] != 0.f || mt.eta[1] != 0.f || mt.eta[2] != 0.f;
      const bool k = mt.k[0] != 0.f || mt.k[1] != 0.f || mt.k[2] != 0.f;
      o.lobe_class = eta && !k ? 1u : 0u; /* NovaMaterials.h:118-121 */
    }
    offset += d->meshes[x.mesh].n_tris;
  }
  if (offset >= (1ull << 27))
    return fail(c, NOVA_B200_OUT_OF_MEMORY, "more than 2^27 triangles are not supported by the leaf encoding%s");
  c->n_prims = offset;
  c->n_materials = d->n_materials;
  /* per-triangle tables (instance of each primitive, which primitives can be hit) and the index
   * check are built on the device after the copies */
  const size_t off_mats = plan.add(mats.data(), mats.size() * sizeof(nb::DevMaterial));
  const size_t off_inst = plan.add(c->h_instances.data(), c->h_instances.size() * sizeof(nb::DevInstance));
  const size_t off_pi = plan.arena;
  plan.arena += UploadPlan::align(offset * sizeof(uint32_t));
  const uint32_t n_cblocks = (uint32_t)((offset + kCompactItems - 1) / kCompactItems);
  const size_t off_flags = plan.add(nullptr, offset * sizeof(uint32_t), true);
  const size_t off_counts = plan.add(nullptr, (n_cblocks + 2) * sizeof(uint32_t), true);
  plan.pieces.pop_back();
  plan.pieces.pop_back();
  /* texture and mesh tables hold device pointers: reserve their space now, fill after allocation */
  const size_t off_tex = plan.arena;
  plan.arena += UploadPlan::align(tex.size() * sizeof(nb::DevTexture));
  const size_t off_mesh = plan.arena;
  plan.arena += UploadPlan::align(meshes.size() * sizeof(nb::DevMesh));

  char *arena = nullptr, *temp = nullptr;
  NB_CUDA(c, cudaMallocAsync(reinterpret_cast<void **>(&arena), plan.arena, c->stream), "cudaMalloc(scene)");
  c->d_arena = arena;
  c->scene_bytes = plan.arena;
  NB_CUDA(c, cudaMallocAsync(reinterpret_cast<void **>(&temp), std::max<size_t>(plan.temp, 256), c->stream),
          "cudaMalloc(staging)");
  for (uint32_t i = 0; i < d->n_textures; i++) {
    if (d->textures[i].u8_pixels)
      tex[i].u8 = reinterpret_cast<const uint32_t *>(arena + tex_off[i]), tex[i].f32 = nullptr;
    else
      tex[i].f32 = reinterpret_cast<const float *>(arena + tex_off[i]), tex[i].u8 = nullptr;
  }
  for (uint32_t i = 0; i < d->n_meshes; i++) {
    meshes[i].idx = reinterpret_cast<const uint32_t *>(arena + moff[i].idx);
    meshes[i].attr = reinterpret_cast<const float4 *>(arena + moff[i].attr);
  }
  for (nb::DevInstance &I : c->h_instances) { /* copied with the pieces below */
    I.attr = meshes[I.mesh].attr;
    I.idx = meshes[I.mesh].idx;
    I.n_tris = meshes[I.mesh].n_tris;
  }
  plan.pieces.push_back(Piece{tex.data(), tex.size() * sizeof(nb::DevTexture), off_tex, false});
  plan.pieces.push_back(Piece{meshes.data(), meshes.size() * sizeof(nb::DevMesh), off_mesh, false});
  c->h_meshes = meshes;
  nova_b200_status st = copy_pieces(c, plan, arena, temp);
  if (st != NOVA_B200_SUCCESS) {
    cudaFreeAsync(temp, c->stream);
    return st;
  }
  if (total_verts)
    k_interleave<<<(unsigned)((total_verts + 255) / 256), 256, 0, c->stream>>>(
        reinterpret_cast<const InterleaveMesh *>(temp + off_ilv), d->n_meshes, (uint32_t)total_verts, temp, arena);
  uint32_t *flags = reinterpret_cast<uint32_t *>(temp + off_flags), *counts = reinterpret_cast<uint32_t *>(temp + off_counts);
  unsigned *bad = counts + n_cblocks; /* bad, total */
  cudaError_t e_launch = cudaGetLastError();
  if (e_launch == cudaSuccess) e_launch = cudaMallocAsync(&c->d_valid, offset * sizeof(uint32_t), c->stream);
  if (e_launch == cudaSuccess) e_launch = cudaMemsetAsync(bad, 0, sizeof(unsigned), c->stream);
  if (e_launch == cudaSuccess) {
    k_scene_tables<<<(unsigned)((offset + 255) / 256), 256, 0, c->stream>>>(
        reinterpret_cast<const nb::DevInstance *>(arena + off_inst), d->n_instances,
        reinterpret_cast<const nb::DevMesh *>(arena + off_mesh), (uint32_t)offset,
        reinterpret_cast<uint32_t *>(arena + off_pi), flags, bad);
    k_compact_count<<<n_cblocks, kCompactThreads, 0, c->stream>>>(flags, (uint32_t)offset, counts);
    k_compact_offsets<<<1, kCompactThreads, 0, c->stream>>>(counts, n_cblocks, bad + 1);
    k_compact_write<<<n_cblocks, kCompactThreads, 0, c->stream>>>(flags, (uint32_t)offset, counts, c->d_valid);
    e_launch = cudaGetLastError();
  }
  if (e_launch == cudaSuccess)
    e_launch = cudaMemcpyAsync(c->h_counters, bad, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(temp, c->stream);
  if (e_launch != cudaSuccess) {
    free_scene(c);
    return cuda_fail(c, e_launch, "scene tables");
  }
  c->scene.textures = reinterpret_cast<const nb::DevTexture *>(arena + off_tex);
  c->scene.materials = reinterpret_cast<const nb::DevMaterial *>(arena + off_mats);
  c->scene.meshes = reinterpret_cast<const nb::DevMesh *>(arena + off_mesh);
  c->scene.instances = reinterpret_cast<const nb::DevInstance *>(arena + off_inst);
  c->scene.prim_inst = reinterpret_cast<const uint32_t *>(arena + off_pi);
  c->scene.sobol_dv = c->d_sobol;
  c->scene.acos_lut = c->d_acos;
  c->scene.envmap = d->envmap;
  c->scene.n_prims = (uint32_t)offset;
  c->scene.n_instances = d->n_instances;
  c->scene.n_materials = d->n_materials;
  c->scene.has_emissive = emissive ? 1u : 0u;
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "upload_scene");
  if (c->h_counters[0] != 0) {
    free_scene(c);
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "mesh index out of range%s");
  }
  c->n_valid = c->h_counters[1];
  if (c->n_valid == 0) {
    free_scene(c);
    return fail(c, NOVA_B200_INVALID_SCENE_TYPE, "scene has no non-degenerate triangle%s");
  }
  c->scene_ready = true;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_build_bvh(nova_b200_ctx *c, const nova_b200_bvh_options *opts) {
  using namespace nbctx;
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (!c->scene_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "upload a scene before building%s");
  cudaSetDevice(c->device);
  const uint32_t n = c->n_valid;
  const int width = opts && opts->width ? opts->width : 2;
  if (width != 1 && width != 2 && width != 8)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "BVH width must be 1 (two-level), 2 or 8%s");
  nb::BvhBuildParams p;
  p.max_leaf = opts && opts->max_leaf_size > 0 ? opts->max_leaf_size : (width == 8 ? nb::kWideLeafMax : 8);
  p.hard_leaf = width == 8 ? nb::kWideLeafMax : 16;
  p.bins = opts && opts->bins > 0 ? opts->bins : 16;
  p.cost_trav = 0.5f; /* node visits are cheap relative to triangle tests here: measured 2-3 % faster traversal than 1.0 */
  p.small_task = opts && opts->small_subtree > 0 ? (uint32_t)opts->small_subtree : 0u;
  if (opts && (opts->small_subtree < 0 || (opts->small_subtree > 0 && (opts->small_subtree < 64 || opts->small_subtree > 65536))))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "small_subtree must be 0 or 64..65536%s");
  if (p.max_leaf > p.hard_leaf || p.bins < 4 || p.bins > 32)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "max_leaf_size must be 1..16 (1..4 for width 8) and bins 4..32%s");
  if (c->d_nodes) cudaFreeAsync(c->d_nodes, c->stream);
  if (c->d_tris) cudaFreeAsync(c->d_tris, c->stream);
  if (c->d_blas_root) cudaFreeAsync(c->d_blas_root, c->stream);
  c->d_nodes = nullptr;
  c->d_tris = nullptr;
  c->d_blas_root = nullptr;
  c->scene.blas_root = nullptr;
  c->bvh_ready = false;
  c->primal_valid = false;
  if (width == 1) {
    nb::BvhBuildResult r{};
    const nova_b200_status st = build_two_level(c, p, r);
    if (st != NOVA_B200_SUCCESS) return st;
    c->scene.nodes = c->d_nodes;
    c->scene.tris = c->d_tris;
    c->scene.blas_root = c->d_blas_root;
    c->scene.width = 1;
    c->bvh_width = 1;
    c->n_nodes = r.n_nodes;
    c->n_leaves = r.n_leaves;
    c->bvh_depth = r.max_depth;
    c->bvh_ms = r.ms;
    c->bvh_ready = true;
    return NOVA_B200_SUCCESS;
  }
  const uint32_t *d_valid = c->d_valid;
  uint32_t *d_order = nullptr;
  float4 *d_lo = nullptr, *d_hi = nullptr;
  const size_t max_nodes = std::max<size_t>(2 * (size_t)n, 2);
  NB_CUDA(c, cudaMallocAsync(&c->d_nodes, sizeof(float4) * 4 * max_nodes, c->stream), "cudaMalloc(nodes)");
  NB_CUDA(c, cudaMallocAsync(&c->d_tris, sizeof(float4) * 3 * (size_t)n, c->stream), "cudaMalloc(tris)");
  NB_CUDA(c, cudaMemsetAsync(c->d_nodes, 0, sizeof(float4) * 4 * max_nodes, c->stream), "memset(nodes)");
  NB_CUDA(c, cudaMallocAsync(&d_order, sizeof(uint32_t) * n, c->stream), "cudaMalloc(order)");
  NB_CUDA(c, cudaMallocAsync(&d_lo, sizeof(float4) * n, c->stream), "cudaMalloc(lo)");
  NB_CUDA(c, cudaMallocAsync(&d_hi, sizeof(float4) * n, c->stream), "cudaMalloc(hi)");
  k_prim_boxes<<<(n + 255) / 256, 256, 0, c->stream>>>(c->scene, d_valid, n, d_lo, d_hi);
  NB_CUDA(c, cudaGetLastError(), "k_prim_boxes");
  nb::BvhBuildResult r{};
  cudaError_t e = nb::build_bvh(d_lo, d_hi, n, p, c->d_nodes, d_order, c->stream, &r);
  if (e != cudaSuccess) return cuda_fail(c, e, "build_bvh");
  k_write_tris<<<(n + 255) / 256, 256, 0, c->stream>>>(c->scene, d_valid, d_order, n, c->d_tris);
  NB_CUDA(c, cudaMemsetAsync(c->d_counters, 0, 4, c->stream), "memset");
  k_validate<<<(r.n_nodes + 255) / 256, 256, 0, c->stream>>>(c->d_nodes, r.n_nodes, n, c->d_counters);
  NB_CUDA(c, cudaMemcpyAsync(c->h_counters, c->d_counters, 4, cudaMemcpyDeviceToHost, c->stream), "readback");
  cudaFreeAsync(d_order, c->stream);
  cudaFreeAsync(d_lo, c->stream);
  cudaFreeAsync(d_hi, c->stream);
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "build_bvh");
  if (c->h_counters[0] != 0 || r.n_nodes == 0 || r.n_nodes > max_nodes || r.max_depth >= nb::kTraversalStack)
    return fail(c, NOVA_B200_RENDERER_EXCEPTION, "BVH validation failed%s");
  if (width == 8) {
    float4 *wnodes = nullptr, *wtris = nullptr;
    NB_CUDA(c, cudaMallocAsync(&wnodes, sizeof(float4) * 5 * ((size_t)r.n_nodes + 1), c->stream),
            "cudaMalloc(wide nodes)");
    cudaError_t we = cudaMallocAsync(&wtris, sizeof(float4) * 3 * (size_t)n, c->stream);
    if (we != cudaSuccess) {
      cudaFreeAsync(wnodes, c->stream);
      return cuda_fail(c, we, "cudaMalloc(wide triangles)");
    }
    nb::WideBuildResult wr{};
    we = nb::build_wide_bvh(c->d_nodes, r.n_nodes, c->d_tris, n, wnodes, wtris, c->stream, &wr);
    if (we != cudaSuccess || wr.depth >= nb::kWideStack) {
      cudaFreeAsync(wnodes, c->stream);
      cudaFreeAsync(wtris, c->stream);
      if (we != cudaSuccess) return cuda_fail(c, we, "build_wide_bvh");
      return fail(c, NOVA_B200_RENDERER_EXCEPTION, "wide BVH deeper than the traversal stack%s");
    }
    cudaFreeAsync(c->d_nodes, c->stream);
    cudaFreeAsync(c->d_tris, c->stream);
    c->d_nodes = wnodes;
    c->d_tris = wtris;
    r.n_nodes = wr.n_nodes;
    r.max_depth = wr.depth;
    r.ms += wr.ms;
  }
  c->scene.nodes = c->d_nodes;
  c->scene.tris = c->d_tris;
  c->scene.width = width;
  c->bvh_width = width;
  c->n_nodes = r.n_nodes;
  c->n_leaves = r.n_leaves;
  c->bvh_depth = r.max_depth;
  c->bvh_ms = r.ms;
  c->bvh_ready = true;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_upload_scene_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                              uint32_t n) {
  if (!descs) return ctxs && ctxs[0] ? nbctx::fail(ctxs[0], NOVA_B200_INVALID_ARGUMENT, "descs is null%s")
                                     : NOVA_B200_INVALID_ARGUMENT;
  return for_each_context(ctxs, n, [&](uint32_t k) { return nova_b200_upload_scene(ctxs[k], &descs[k]); });
}

nova_b200_status nova_b200_build_bvh_batch(nova_b200_ctx *const *ctxs, uint32_t n, const nova_b200_bvh_options *opts) {
  return for_each_context(ctxs, n, [&](uint32_t k) { return nova_b200_build_bvh(ctxs[k], opts); });
}

nova_b200_status nova_b200_upload_build_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                              uint32_t n, const nova_b200_bvh_options *opts) {
  if (!descs) return ctxs && n && ctxs[0] ? nbctx::fail(ctxs[0], NOVA_B200_INVALID_ARGUMENT, "descs is null%s")
                                          : NOVA_B200_INVALID_ARGUMENT;
  return for_each_context(ctxs, n, [&](uint32_t k) {
    const nova_b200_status st = nova_b200_upload_scene(ctxs[k], &descs[k]);
    return st != NOVA_B200_SUCCESS ? st : nova_b200_build_bvh(ctxs[k], opts);
  });
}

nova_b200_status nova_b200_render(nova_b200_ctx *c, const nova_b200_frame *f, float *film_host, float *film_device,
                                  nova_b200_render_stats *stats) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_render(c, f, film_host, film_device, stats);
}

nova_b200_status nova_b200_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_frame *frames, uint32_t n,
                                        float *const *films_host, float *const *films_device,
                                        nova_b200_render_stats *stats) {
  return nb_render_batch(ctxs, frames, n, films_host, films_device, stats);
}

nova_b200_status nova_b200_upload_build_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                                     const nova_b200_frame *frames, uint32_t n,
                                                     const nova_b200_bvh_options *opts, float *const *films_host,
                                                     float *const *films_device, nova_b200_render_stats *stats) {
  return nb_upload_build_render_batch(ctxs, descs, frames, n, opts, films_host, films_device, stats);
}

nova_b200_status nova_b200_trace(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, int32_t *prim, float *t,
                                 float *u, float *v) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_trace(c, n, o, d, prim, t, u, v);
}

nova_b200_status nova_b200_cancel(nova_b200_ctx *c) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  c->cancel.store(true);
  if (c->h_cancel_map) *c->h_cancel_map = 1; /* the persistent wavefront reads this one */
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_trace_host(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, int32_t *prim,
                                      float *t, float *u, float *v) {
  using namespace nbctx;
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (n == 0) return NOVA_B200_SUCCESS;
  if (!o || !d || !prim || !t || !u || !v) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  cudaSetDevice(c->device);
  char *buf = nullptr; /* origins, directions, prim, t, u, v */
  const size_t b3 = n * 3 * sizeof(float), b1 = n * sizeof(float);
  NB_CUDA(c, cudaMallocAsync(reinterpret_cast<void **>(&buf), 2 * b3 + 4 * b1, c->stream), "cudaMalloc(rays)");
  float *d_o = reinterpret_cast<float *>(buf), *d_d = reinterpret_cast<float *>(buf + b3);
  int32_t *d_p = reinterpret_cast<int32_t *>(buf + 2 * b3);
  float *d_t = reinterpret_cast<float *>(buf + 2 * b3 + b1), *d_u = d_t + n, *d_v = d_u + n;
  cudaError_t e = cudaMemcpyAsync(d_o, o, b3, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_d, d, b3, cudaMemcpyHostToDevice, c->stream);
  nova_b200_status st = e == cudaSuccess ? nb_trace(c, n, d_o, d_d, d_p, d_t, d_u, d_v) : NOVA_B200_SUCCESS;
  if (e == cudaSuccess && st == NOVA_B200_SUCCESS) {
    e = cudaMemcpyAsync(prim, d_p, b1, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t, d_t, b1, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(u, d_u, b1, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v, d_v, b1, cudaMemcpyDeviceToHost, c->stream);
  }
  cudaFreeAsync(buf, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "trace_host");
  if (st != NOVA_B200_SUCCESS) return st;
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "trace_host");
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_sobol(nova_b200_ctx *c, uint64_t n, const uint32_t *idx, const uint32_t *dim, uint32_t seed,
                                 float *out) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_sobol(c, n, idx, dim, seed, out);
}

nova_b200_status nova_b200_scatter(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, const int32_t *prim,
                                   const float *t, const float *u, const float *v, const uint32_t *index,
                                   const int32_t *bounce, uint32_t seed, float *out_o, float *out_d, float *weight,
                                   float *emissive, int32_t *valid) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_scatter(c, n, o, d, prim, t, u, v, index, bounce, seed, out_o, out_d, weight, emissive, valid);
}

nova_b200_status nova_b200_bake_irradiance(nova_b200_ctx *c, const float *src, int32_t sw, int32_t sh, int32_t ch,
                                           int32_t ow, int32_t oh, int32_t samples, float *out) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_bake(c, src, sw, sh, ch, ow, oh, samples, out);
}

nova_b200_status nova_b200_bake_irradiance_texunit(nova_b200_ctx *c, const float *src, int32_t sw, int32_t sh,
                                                   int32_t ch, int32_t ow, int32_t oh, int32_t samples, float *out) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_bake_texunit(c, src, sw, sh, ch, ow, oh, samples, out);
}

void nova_b200_get_error(nova_b200_ctx *c, char buf[1024], size_t *size) {
  if (!buf) return;
  const std::string &e = c ? c->error : std::string("null context");
  size_t n = std::min<size_t>(e.size(), 1023);
  std::memcpy(buf, e.data(), n);
  buf[n] = 0;
  if (size) *size = n;
}

nova_b200_status nova_b200_set_diff_params(nova_b200_ctx *c, const float *albedo, const float *roughness) {
  using namespace nbctx;
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (!c->scene_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "upload a scene first%s");
  c->scene.diff_albedo = albedo;
  c->scene.diff_rough = roughness;
  c->primal_valid = false;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_backward(nova_b200_ctx *c, const nova_b200_frame *f, const float *d_image,
                                    float *grad_albedo, float *grad_roughness, uint32_t flags,
                                    nova_b200_render_stats *stats) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  return nb_backward(c, f, d_image, grad_albedo, grad_roughness, flags, stats);
}

nova_b200_status nova_b200_scene_info(nova_b200_ctx *c, uint64_t *tris, uint64_t *insts, uint64_t *nodes,
                                      uint64_t *leaves, uint64_t *bytes) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (tris) *tris = c->n_prims;
  if (insts) *insts = c->h_instances.size();
  if (nodes) *nodes = c->n_nodes;
  if (leaves) *leaves = c->n_leaves;
  if (bytes)
    *bytes = c->scene_bytes + (uint64_t)c->n_nodes * (c->bvh_width == 8 ? 80 : 64) +
             (uint64_t)c->n_valid * 48 + c->queue_bytes + c->radiance_cap * 16;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_synchronize(nova_b200_ctx *c) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
  return NOVA_B200_SUCCESS;
}

}  // extern "C"
