/* Wavefront path tracer: the reference's PathIntegrator::Li (integrator/Integrator.cpp:60-99) as
 * sm_100a kernels over a path queue in HBM, for one frame or a batch of frames of different scenes.
 *
 *   k_refill   fills free queue slots with camera rays of new paths (Integrator.h:66-85 with the
 *              OptiX raygen's sample index (x * H + y) * spp + s, integrator_optix.cu:43; Sobol
 *              dimensions 0 and 1 jitter NDC)
 *   k_trace    closest hit per queued ray (traverse.cuh); a miss finishes its path with the
 *              environment lookup, hits go to a compact hit list
 *   k_shade    per hit: principled scatter (Sobol dimensions 2 + 4b .. 5 + 4b at bounce b),
 *              throughput update, spawned ray appended to the next queue with warp-aggregated
 *              atomics; after the last allowed scatter the spawned direction looks up the
 *              environment directly (the reference traces that ray but discards the hit,
 *              Integrator.cpp:94-98)
 *   k_wave_end advances the device-side wave counters
 *   k_resolve  per pixel, adds the per-path radiance of the call's samples to the running sum in
 *              sample order and writes sum / samples (writeFramebuffer, api/engine.cpp:351-363)
 *
 * Jobs: every path carries its job index (a frame of one context: scene, BVH, camera, sample
 * range) and every kernel reads the chunk's job table, so a batch of frames of different scenes
 * runs as one wavefront.  A single render is a batch of one.  The table travels in the kernel
 * parameter space (__grid_constant__, read through the constant cache): one Job for a single
 * frame, up to kParamJobs for a batch chunk.  The per-path arithmetic does not depend on the batch,
 * and each pixel's samples are added in sample order, so a frame rendered in a batch equals the
 * same frame rendered alone, bit for bit.
 *
 * Wave loop: the counters (active paths, next path, hits, survivors) live on the device and the
 * kernels read device-resident counts, so the host never waits between waves.  Waves are enqueued
 * in groups of four, two groups in flight: while the GPU runs one group the host reads the
 * previous group's counters (pinned memory, event-synchronised) and enqueues the next, so the GPU
 * does not wait for the host; a group issued after the last path finished finds empty queues and
 * returns at once.  A single-frame chunk launches its kernels directly; a batch chunk replays each
 * slot's group from a CUDA graph (captured once per job table, with event-record nodes timing
 * every trace and shade kernel).
 *
 * The recursive estimator e_0 + c_0 (e_1 + c_1 (... env)) is evaluated forward as
 * sum_k beta_k e_k + beta_K env with beta_k = c_0 ... c_{k-1}; a path whose result is not finite
 * contributes 0 (DENAN, Integrator.cpp:92).  Path state: origin + radiance slot, direction + bounce +
 * job, throughput + Sobol sample index (3 x 16 B); hits 16 B + 4 B slot; per-path radiance 16 B,
 * written once.
 */
#include <algorithm>
#include <cfloat>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "context.cuh"
#include "shading.cuh"
#include "traverse.cuh"

namespace {

using namespace nb;

constexpr uint32_t kQueueCapDefault = 1u << 23; /* rays per wave unless tuned */
constexpr size_t kRadianceCapBytes = 4ull << 30;
constexpr unsigned kRRDimBase = 200; /* Russian roulette decisions use Sobol dimension 200 + bounce */
constexpr int kMaxDepth = 48;        /* 2 + 4 (depth + 1) Sobol dimensions must stay below 200 */
constexpr int kWavesPerGraph = 4;    /* even: the queues end each graph launch where they started */

struct RenderParams {
  int32_t W, H;
  uint32_t NP;    /* pixels */
  uint32_t count; /* samples traced for this job in the current chunk */
  uint32_t begin; /* first of those samples */
  uint32_t spp_total;
  int32_t max_depth;
  uint32_t seed;
  int32_t rr_start;
  float inv_P[16], inv_V[16];
  uint32_t tile_w, tile_h; /* consecutive paths walk tile_w x tile_h pixel tiles (0: image rows) */
  int32_t vinv;            /* film rows stored top-down (vertical_invert) */
};

struct Job {
  DevScene sc;
  RenderParams rp;
  uint32_t path_begin; /* first path id of this job in the chunk (radiance slot of its first path) */
  uint32_t n_paths;
};

struct WaveCounters {
  uint32_t n_active; /* rays waiting in the input queue */
  uint32_t next;     /* next path id to start */
  uint32_t total;    /* paths in the chunk */
  uint32_t cap;      /* queue capacity */
  uint32_t hit_count, out_count;
  uint32_t hit_back; /* NB_HIT_CLASSES: hits of transmissive materials, from the end of the hit list */
  uint32_t done;
  uint32_t waves; /* waves that did work */
  uint32_t trace_next; /* next queued ray handed out by the persistent trace kernel */
  uint32_t shade_next; /* next hit handed out in the persistent wavefront */
  /* device status of the whole loop (never reset between waves): path radiance values that were not
   * finite and were written as 0 (the reference's DENAN, Integrator.cpp:92), and hits whose
   * primitive, instance or material id is out of range (the path ends black, the render fails) */
  uint32_t nonfinite, bad_index;
  unsigned long long traced;
  unsigned long long node_visits, tri_tests; /* trace_mode 2 only: the traversal's own work */
};

/* The chunk's job table as a kernel parameter. */
struct OneJob {
  Job j;
  __device__ __forceinline__ const Job &at(uint32_t) const { return j; }
  __device__ __forceinline__ uint32_t find(uint32_t) const { return 0u; }
};

constexpr uint32_t kParamJobs = 104;

struct ManyJobs {
  uint32_t n;
  Job j[kParamJobs];
  __device__ __forceinline__ const Job &at(uint32_t k) const { return j[k]; }
  /* the last job whose first path id is <= g */
  __device__ __forceinline__ uint32_t find(uint32_t g) const {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (j[mid].path_begin <= g)
        lo = mid;
      else
        hi = mid;
    }
    return lo;
  }
};
static_assert(sizeof(ManyJobs) + 256 <= 32764, "a batch job table must fit the 32 KB kernel parameter space");

struct Queue {
  float4 *o, *d, *beta;
};

__device__ __forceinline__ uint32_t wave_new(const WaveCounters &wc) {
  return min(wc.cap - wc.n_active, wc.total - wc.next);
}

constexpr uint32_t kTileW = 8, kTileH = 4; /* default pixel tile: one warp of camera rays per tile */

/* Tiles of a tuning: 0 x 0 = the default tile, 1 x 1 = image rows (tile_w = 0 below). */
void set_tiles(RenderParams &rp, const nova_b200_tuning &tu) {
  if (tu.tile_w == 0) {
    rp.tile_w = kTileW;
    rp.tile_h = kTileH;
  } else if (tu.tile_w == 1 && tu.tile_h == 1) {
    rp.tile_w = rp.tile_h = 0u;
  } else {
    rp.tile_w = tu.tile_w;
    rp.tile_h = tu.tile_h;
  }
}

/* The q-th pixel a frame's paths visit: row-major, or tile_w x tile_h tiles in row-major tile
 * order (partial tiles at the right and bottom edges), so a warp's primary rays cover a compact
 * patch of the image. */
__device__ __forceinline__ void tile_pixel(const RenderParams &rp, uint32_t q, uint32_t &x, uint32_t &y) {
  const uint32_t W = (uint32_t)rp.W, H = (uint32_t)rp.H;
  if (rp.tile_w == 0) {
    y = q / W;
    x = q - y * W;
    return;
  }
  const uint32_t tw = rp.tile_w, th = rp.tile_h;
  const uint32_t ty = q / (W * th), r = q - ty * W * th;
  const uint32_t h_r = min(th, H - ty * th);
  const uint32_t tx = r / (tw * h_r), r2 = r - tx * tw * h_r;
  const uint32_t w_c = min(tw, W - tx * tw);
  const uint32_t ly = r2 / w_c;
  x = tx * tw + (r2 - ly * w_c);
  y = ty * th + ly;
}

/* The camera ray of path g of the chunk: pixel (x, y), radiance slot and Sobol index. */
struct CameraPath {
  uint32_t job, x, y, rslot, index;
  V4 o, d;
};

template <class JS>
__device__ __forceinline__ CameraPath camera_path(const JS &js, uint32_t g) {
  CameraPath c;
  c.job = js.find(g);
  const Job &J = js.at(c.job);
  const RenderParams &rp = J.rp;
  const uint32_t p = g - J.path_begin;
  const uint32_t s_local = p / rp.NP, q_pix = p - s_local * rp.NP;
  uint32_t x, y;
  tile_pixel(rp, q_pix, x, y);
  c.x = x;
  c.y = y;
  /* the radiance slot stays keyed by the row-major pixel, whatever order paths start in */
  c.rslot = J.path_begin + s_local * rp.NP + y * (uint32_t)rp.W + x;
  const uint32_t index = ((uint32_t)x * (uint32_t)rp.H + (uint32_t)y) * rp.spp_total + (rp.begin + s_local);
  c.index = index;
  const float r0 = sobol_sample(J.sc.sobol_dv, index, 0, rp.seed);
  const float r1 = sobol_sample(J.sc.sobol_dv, index, 1, rp.seed);
  const float dx = r0 * 0.0005f, dy = r1 * 0.0005f; /* RAND_DX / RAND_DY, Integrator.h:54-55 */
  const int ys = rp.H - (int)y;                     /* screen row, Integrator.h:84 */
  const float ndc_x = (float)(2 * (int)x - rp.W) / (float)rp.W;
  const float ndc_y = (float)(rp.H - 2 * ys) / (float)rp.H;
  const float nx = ndc_x + dx, ny = ndc_y + dy;
  const M4 iP = m4_load(rp.inv_P), iV = m4_load(rp.inv_V);
  V4 o = mul(iP, V4{nx, ny, -1.f, 1.f});
  o = o / o.w;
  o = mul(iV, V4{o.x, o.y, o.z, 1.f});
  V4 d = mul(iP, V4{nx, ny, -1.f, 0.f});
  d = normalize(mul(iV, V4{d.x, d.y, -1.f, 0.f}));
  c.o = o;
  c.d = d;
  return c;
}

/* Camera ray of new path `next + i` into queue slot `n_active + i`. */
template <class JS>
__device__ __forceinline__ void refill_one(const Queue &q, uint32_t next, uint32_t n_active, float4 *L, const JS &js,
                                           uint32_t i) {
  const CameraPath c = camera_path(js, next + i);
  const uint32_t slot = n_active + i;
  q.o[slot] = make_float4(c.o.x, c.o.y, c.o.z, __uint_as_float(c.rslot));
  q.d[slot] = make_float4(c.d.x, c.d.y, c.d.z, __uint_as_float(c.job << 8));
  q.beta[slot] = make_float4(1.f, 1.f, 1.f, __uint_as_float(c.index));
  if (js.at(c.job).sc.has_emissive) L[c.rslot] = make_float4(0.f, 0.f, 0.f, 0.f);
}

template <class JS>
__global__ void __launch_bounds__(256) k_refill(Queue q, const WaveCounters *wcp, float4 *L,
                                                const __grid_constant__ JS js) {
  const WaveCounters wc = *wcp;
  const uint32_t n_new = wave_new(wc);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x)
    refill_one(q, wc.next, wc.n_active, L, js, i);
}

/* Non-finite radiance becomes 0 (DENAN), counted in *nonfinite (rare: a plain atomic). */
__device__ __forceinline__ float4 finite_or_zero(V3 L, float alpha, unsigned *nonfinite) {
  if (!finite3(L)) {
    atomicAdd(nonfinite, 1u);
    return make_float4(0.f, 0.f, 0.f, 0.f);
  }
  return make_float4(L.x, L.y, L.z, alpha);
}

/* Loads of data written earlier in the same launch by other blocks: through L2 (ld.global.cg) when P,
 * the persistent wavefront; plain loads otherwise (a kernel boundary orders them). */
template <bool P, class T>
__device__ __forceinline__ T ldq(const T *p) {
  if constexpr (P)
    return __ldcg(p);
  else
    return *p;
}

/* Writes a finished path's radiance (adds the emission gathered so far when the scene has any). */
template <bool P = false>
__device__ __forceinline__ void finish_path(const DevScene &sc, float4 *L, uint32_t g, float4 result,
                                            unsigned *nonfinite) {
  if (sc.has_emissive) {
    const float4 acc = ldq<P>(&L[g]);
    float4 r = make_float4(acc.x + result.x, acc.y + result.y, acc.z + result.z, result.w);
    if (!isfinite(r.x) || !isfinite(r.y) || !isfinite(r.z)) {
      atomicAdd(nonfinite, 1u);
      r = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    L[g] = r;
  } else {
    L[g] = result;
  }
}

/* The hit's primitive, its instance (from the hit list) and the instance's material all index their
 * tables, and the primitive is one of the instance's triangles. */
__device__ __forceinline__ bool hit_ids_valid(const DevScene &sc, int prim, uint32_t inst) {
  if (prim < 0 || (uint32_t)prim >= sc.n_prims || inst >= sc.n_instances) return false;
  const DevInstance &I = sc.instances[inst];
  return (uint32_t)prim - I.prim_offset < I.n_tris && I.material < sc.n_materials;
}

/* Warp-aggregated append: returns the slot of every lane with `flag` set. */
__device__ __forceinline__ unsigned warp_append(bool flag, unsigned *counter) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  unsigned base = 0;
  if (m) {
    if (lane == (unsigned)(__ffs(m) - 1)) base = atomicAdd(counter, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  }
  return base + __popc(m & ((1u << lane) - 1u));
}

/* Closest hit of every queued ray.  A miss finishes its path here (environment lookup,
 * Integrator.cpp:94-98); hits are appended to a compact hit list so the shading kernel only runs
 * on rays that hit.  At least 10 resident blocks of 128 (48 registers): the walk is latency-bound,
 * and 40 warps per SM beat 32 (-4% on the batched scenes); 12 blocks spill the walk state. */
/* Resident blocks of 128 threads per SM that k_trace is compiled for (the register bound is
 * 65536 / (128 * blocks)): binary layouts and the 8-wide one separately. */
#ifndef NB_TRACE_MIN_BLOCKS
#define NB_TRACE_MIN_BLOCKS 10
#endif
#ifndef NB_TRACE8_MIN_BLOCKS
#define NB_TRACE8_MIN_BLOCKS 10
#endif

/* NB_HIT_CLASSES=1: the hit list holds non-transmissive hits from its front and transmissive ones
 * from its back (k_shade reads both ranges), so shading warps mostly run one lobe family: the
 * dielectric lobe's refraction code or the reflective lobes'.  The class is the instance's (its
 * material's eta and k, NovaMaterials.h:118-121), read next to the identity flag the traversal
 * already loaded.  On the 32-job batch k_shade went from 107.3 to 80.9 ms per step (films
 * bit-identical); only the order in which hits are shaded changes.  A third list for fully metal
 * materials measured equal (shading -0.6 %, the third append +0.4 % in k_trace). */
#ifndef NB_HIT_CLASSES
#define NB_HIT_CLASSES 1
#endif

/* The closest-hit pass for one warp's lanes (ray i of n queued; the warp's lanes call together: the
 * hit append is a warp ballot). */
template <int WIDTH, class JS, bool ADJ, bool COUNT, bool P>
__device__ __forceinline__ void trace_warp(const Queue &q, WaveCounters *wcp, float4 *hits, uint2 *hit_slot,
                                           float4 *L, const JS &js, uint32_t i, uint32_t n,
                                           const uint32_t *order = nullptr) {
  {
    bool is_hit = false, back = false;
    TraceResult r{-1, 0.f, 0.f, 0.f, 0u};
    uint64_t nv = 0, tt = 0;
    if (i < n) {
      if (order) i = order[i]; /* the queue slot this lane traces (k_order_rays) */
      const float4 o = ldq<P>(&q.o[i]), d = ldq<P>(&q.d[i]);
      const DevScene &sc = js.at(__float_as_uint(d.w) >> 8).sc;
      r = trace_closest_w<WIDTH>(sc, V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, COUNT ? &nv : nullptr,
                                 COUNT ? &tt : nullptr);
      if (r.prim >= 0) {
        is_hit = true;
        if constexpr (NB_HIT_CLASSES && !COUNT && !P) back = sc.instances[r.inst].lobe_class != 0u;
      } else if (!ADJ) { /* a replayed path's radiance is already known */
        const float4 b4 = ldq<P>(&q.beta[i]);
        const V4 e = env_sample(sc, V3{d.x, d.y, d.z});
        finish_path<P>(sc, L, __float_as_uint(o.w),
                    finite_or_zero(V3{b4.x, b4.y, b4.z} * V3{e.x, e.y, e.z},
                                   (float)(__float_as_uint(d.w) & 0xffu) + e.w, &wcp->nonfinite),
                    &wcp->nonfinite);
      }
    }
    if constexpr (COUNT) { /* one atomic per warp for each counter */
      for (int off = 16; off > 0; off >>= 1) {
        nv += __shfl_down_sync(0xffffffffu, nv, off);
        tt += __shfl_down_sync(0xffffffffu, tt, off);
      }
      if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&wcp->node_visits, (unsigned long long)nv);
        atomicAdd(&wcp->tri_tests, (unsigned long long)tt);
      }
    }
    uint32_t slot;
    if constexpr (NB_HIT_CLASSES && !COUNT && !P) {
      /* transmissive hits go to the end of the list, the others to the front, so the shading warps
       * mostly take one lobe family (BSDF.h:69-79) */
      const unsigned f = warp_append(is_hit && !back, &wcp->hit_count);
      const unsigned b = warp_append(back, &wcp->hit_back);
      slot = back ? wcp->cap - 1u - b : f;
    } else {
      slot = warp_append(is_hit, &wcp->hit_count);
    }
    if (is_hit) {
      hits[slot] = make_float4(r.t, r.u, r.v, __int_as_float(r.prim));
      hit_slot[slot] = make_uint2(i, r.inst);
    }
  }
}

template <int WIDTH, class JS, bool ADJ = false, bool COUNT = false>
__global__ void __launch_bounds__(128, WIDTH == 8 ? NB_TRACE8_MIN_BLOCKS : NB_TRACE_MIN_BLOCKS) k_trace(Queue q, WaveCounters *wcp, float4 *hits, uint2 *hit_slot, float4 *L,
                                               const __grid_constant__ JS js, const uint32_t *order = nullptr) {
  const uint32_t n = wcp->n_active + wave_new(*wcp);
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if ((i & ~31u) >= n) return; /* whole warps leave together (the append below is a warp ballot) */
  trace_warp<WIDTH, JS, ADJ, COUNT, false>(q, wcp, hits, hit_slot, L, js, i, n, order);
}

/* Ray ordering before the trace (NB_RAY_ORDER = window of queue slots, 0 = off): each window of
 * consecutive slots, whose rays come from neighbouring pixel tiles, is counting-sorted by direction
 * (8 x 8 octahedral bins), and k_trace's warps take the window's rays in that order, so a warp's
 * rays start out alike.  Only the order in which rays are traced and appended changes; a path's
 * result does not depend on it. */
#ifndef NB_RAY_ORDER
#define NB_RAY_ORDER 0
#endif
constexpr int kOrderThreads = 1024;

__device__ __forceinline__ uint32_t direction_bin(float4 d) {
  const float s = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
  float x = d.x / s, y = d.y / s;
  if (d.z < 0.f) {
    const float ax = fabsf(x), ay = fabsf(y);
    x = copysignf(1.f - ay, x);
    y = copysignf(1.f - ax, y);
  }
  const int bx = min(7, max(0, (int)((x + 1.f) * 4.f))), by = min(7, max(0, (int)((y + 1.f) * 4.f)));
  return (uint32_t)(bx + 8 * by);
}

template <int WINDOW>
__global__ void __launch_bounds__(kOrderThreads) k_order_rays(Queue q, const WaveCounters *wcp, uint32_t *order) {
  constexpr int kPer = WINDOW / kOrderThreads;
  __shared__ uint32_t s_bin[64];
  const uint32_t n = wcp->n_active + wave_new(*wcp);
  const uint32_t start = blockIdx.x * (uint32_t)WINDOW;
  if (start >= n) return;
  if (threadIdx.x < 64) s_bin[threadIdx.x] = 0;
  __syncthreads();
  uint32_t key[kPer];
#pragma unroll
  for (int k = 0; k < kPer; k++) {
    const uint32_t slot = start + (uint32_t)k * kOrderThreads + threadIdx.x;
    key[k] = 64u;
    if (slot < n) {
      key[k] = direction_bin(q.d[slot]);
      atomicAdd(&s_bin[key[k]], 1u);
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) { /* exclusive scan of the 64 bins by one warp, two bins a lane */
    const uint32_t a = s_bin[2 * threadIdx.x], b = s_bin[2 * threadIdx.x + 1];
    uint32_t x = a + b;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
      if ((int)threadIdx.x >= off) x += y;
    }
    const uint32_t excl = x - a - b;
    s_bin[2 * threadIdx.x] = excl;
    s_bin[2 * threadIdx.x + 1] = excl + a;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kPer; k++) {
    const uint32_t slot = start + (uint32_t)k * kOrderThreads + threadIdx.x;
    if (key[k] < 64u) order[start + atomicAdd(&s_bin[key[k]], 1u)] = slot;
  }
}

/* Persistent variant of k_trace (binary BVH): a fixed grid of warps hands out the queued rays with
 * a warp-wide counter, and lanes whose walk has ended take new rays while the warp's other lanes
 * keep walking, so lanes do not idle behind the warp's longest walk.  Work goes in rounds: every lane
 * advances its walk by up to kDynSteps iterations of trace_closest2's loop (an inner node, or a leaf
 * and the pop after it), leaving the round early once kRefillLanes lanes are done; then finished
 * walks report (miss: environment, hit: the compact hit list, one warp append per round) and idle
 * lanes take new rays.  The walk's arithmetic and order are trace_closest2's, so the hits are the
 * same.  A lane keeps its ray's scene tables in registers (WalkScene), so a batch's job table is
 * read once per ray. */
/* Measured on the 32-job batch (trace time per step): 8 blocks per SM and 32 steps 221 ms, 16 steps
 * 222 ms, 8 steps 282 ms; 10 blocks per SM (spills) and 16 steps 245 ms; the per-ray kernel 195 ms.
 * The hits also reach the shading pass in finishing order instead of queue order, which costs
 * k_shade 11 % (121 vs 109 ms). */
#ifndef NB_DYN_STEPS
#define NB_DYN_STEPS 32
#endif
#ifndef NB_DYN_MIN_BLOCKS
#define NB_DYN_MIN_BLOCKS 8
#endif
constexpr int kDynSteps = NB_DYN_STEPS;
constexpr int kRefillLanes = 8;

template <class JS>
__global__ void __launch_bounds__(128, NB_DYN_MIN_BLOCKS) k_trace_dyn(Queue q, WaveCounters *wcp, float4 *hits,
                                                                      uint2 *hit_slot, float4 *L,
                                                                      const __grid_constant__ JS js) {
  const uint32_t n = wcp->n_active + wave_new(*wcp);
  const unsigned full = 0xffffffffu, lane = threadIdx.x & 31u;
  Walk2 w;
  WalkScene ws{nullptr, nullptr, nullptr};
  int32_t stack[kTraversalStack];
  int32_t ray = -1;
  bool exhausted = false;
  /* every round hands out rays or advances a walk; the bound only guards against a bug */
  for (uint32_t round = 0; round < (1u << 30); round++) {
    const bool idle = ray < 0 && !exhausted;
    const unsigned need = __ballot_sync(full, idle);
    if (need) {
      const int leader = __ffs(need) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(&wcp->trace_next, (unsigned)__popc(need));
      base = __shfl_sync(full, base, leader);
      if (idle) {
        const uint32_t i = base + (uint32_t)__popc(need & ((1u << lane) - 1u));
        if (i < n) {
          const float4 o = q.o[i], d = q.d[i];
          const DevScene &sc = js.at(__float_as_uint(d.w) >> 8).sc;
          ws = WalkScene{sc.nodes, sc.tris, sc.instances};
          ray = (int32_t)i;
          w.init(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z});
        } else {
          exhausted = true;
        }
      }
    }
    if (__ballot_sync(full, ray >= 0) == 0) break; /* every lane idle after a refill: all rays handed out */
    bool fin = false;
    for (int k = 0; k < kDynSteps; k++) {
      if (ray >= 0 && !fin) fin = !w.step(ws, stack);
      if (__popc(__ballot_sync(full, ray < 0 || fin)) >= kRefillLanes) break;
    }
    const bool is_hit = fin && w.r.prim >= 0;
    if (fin && !is_hit) {
      const float4 o = q.o[ray], b4 = q.beta[ray], d = q.d[ray];
      const DevScene &sc = js.at(__float_as_uint(d.w) >> 8).sc;
      const V4 e = env_sample(sc, V3{d.x, d.y, d.z});
      finish_path(sc, L, __float_as_uint(o.w),
                  finite_or_zero(V3{b4.x, b4.y, b4.z} * V3{e.x, e.y, e.z}, (float)(__float_as_uint(d.w) & 0xffu) + e.w,
                                 &wcp->nonfinite),
                  &wcp->nonfinite);
    }
    if (__ballot_sync(full, fin)) {
      const unsigned slot = warp_append(is_hit, &wcp->hit_count);
      if (is_hit) {
        hits[slot] = make_float4(w.r.t, w.r.u, w.r.v, __int_as_float(w.r.prim));
        hit_slot[slot] = make_uint2((uint32_t)ray, w.r.inst);
      }
    }
    if (fin) ray = -1;
  }
}

/* The shading pass for one warp's lanes (hit i of n; the warp's lanes call together: the continuation
 * append is a warp ballot). */
template <class JS, bool P>
__device__ __forceinline__ void shade_warp(const Queue &in, const Queue &out, WaveCounters *wcp, const float4 *hits,
                                           const uint2 *hit_slot, float4 *L, const JS &js, uint32_t i, uint32_t n) {
  {
    bool enq = false;
    float4 no{}, nd{}, nbeta{};
    if (i < n) {
      const uint2 hs = ldq<P>(&hit_slot[i]);
      const uint32_t slot_in = hs.x, inst = hs.y;
      const float4 o4 = ldq<P>(&in.o[slot_in]), d4 = ldq<P>(&in.d[slot_in]), b4 = ldq<P>(&in.beta[slot_in]),
                   h = ldq<P>(&hits[i]);
      const uint32_t g = __float_as_uint(o4.w);
      const uint32_t tag = __float_as_uint(d4.w);
      const int bounce = (int)(tag & 0xffu);
      const Job &J = js.at(tag >> 8);
      const DevScene &sc = J.sc;
      const RenderParams &rp = J.rp;
      const uint32_t index = __float_as_uint(b4.w); /* the path's Sobol index, set by k_refill */
      const V3 ro{o4.x, o4.y, o4.z}, rd{d4.x, d4.y, d4.z};
      V3 beta{b4.x, b4.y, b4.z};
      const int prim = __float_as_int(h.w);
      bool done = false;
      float4 result = make_float4(0.f, 0.f, 0.f, 0.f);
      if (!hit_ids_valid(sc, prim, inst)) {
        atomicAdd(&wcp->bad_index, 1u);
        L[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        goto append;
      }
      {
      const DevInstance &I = sc.instances[inst];
      const HitRecord hr = make_record(sc, ro, rd, I, (uint32_t)prim - I.prim_offset, h.x, h.y, h.z);
      const ScatterResult sr = scatter(sc, rd, hr, sc.materials[I.material], index, 2u + 4u * (unsigned)bounce, rp.seed,
                                       (uint32_t)prim, I.material);
      /* a failed scatter returns black, emission included (Integrator.cpp:73-79) */
      if (sr.valid && sc.has_emissive && any_nonzero(sr.emissive)) {
        const V3 em = beta * sr.emissive;
        const float4 acc = ldq<P>(&L[g]);
        L[g] = make_float4(acc.x + em.x, acc.y + em.y, acc.z + em.z, acc.w);
      }
      if (!sr.valid) {
        result = make_float4(0.f, 0.f, 0.f, (float)bounce);
        done = true;
      } else {
        V3 c = sr.weight;
        bool alive = true;
        if (rp.rr_start >= 0 && bounce >= rp.rr_start) {
          const V3 nbt = beta * c;
          const float q = fmin_std(1.f, fmax_std(0.05f, fmax_std(nbt.x, fmax_std(nbt.y, nbt.z))));
          const float urr = sobol_sample(sc.sobol_dv, index, kRRDimBase + (unsigned)bounce, rp.seed);
          if (!(urr < q)) {
            alive = false;
            result = make_float4(0.f, 0.f, 0.f, (float)bounce + 1.f);
            done = true;
          } else {
            c = c / q;
          }
        }
        if (alive) {
          beta = beta * c;
          const float eps = 1e-3f; /* Ray::spawn, ray/Ray.h:22-27 */
          const V3 nd3 = normalize(sr.wi);
          const V3 no3 = hr.position + hr.ng * (eps + eps * fsign(dot(hr.ng, sr.wi)));
          if (bounce + 1 > rp.max_depth) {
            const V4 e = env_sample(sc, nd3);
            result = finite_or_zero(beta * V3{e.x, e.y, e.z}, (float)bounce + 1.f + e.w, &wcp->nonfinite);
            done = true;
          } else {
            enq = true;
            no = make_float4(no3.x, no3.y, no3.z, o4.w);
            nd = make_float4(nd3.x, nd3.y, nd3.z, __uint_as_float(tag + 1u));
            nbeta = make_float4(beta.x, beta.y, beta.z, b4.w);
          }
        }
      }
      if (done) finish_path<P>(sc, L, g, result, &wcp->nonfinite);
      }
    }
  append:
    const unsigned slot = warp_append(enq, &wcp->out_count);
    if (enq) {
      out.o[slot] = no;
      out.d[slot] = nd;
      out.beta[slot] = nbeta;
    }
  }
}

/* Lobe class of hit i, the key k_shade groups a block's hits by (BSDF.h:69-79 picks the lobe from
 * the material's transmission and metallic inputs): 0 diffuse-only material, 1 a material with a
 * metallic/roughness texture, 2 a transmissive one (eta set, no absorption), 3 no hit / bad index. */
template <class JS>
__device__ __forceinline__ uint32_t lobe_class(const Queue &in, const float4 *hits, const uint2 *hit_slot,
                                               const JS &js, uint32_t i, uint32_t n) {
  if (i >= n) return 3u;
  const uint2 hs = hit_slot[i];
  const uint32_t tag = __float_as_uint(in.d[hs.x].w), inst = hs.y;
  const DevScene &sc = js.at(tag >> 8).sc;
  const int prim = __float_as_int(hits[i].w);
  if (!hit_ids_valid(sc, prim, inst)) return 3u;
  const DevMaterial &m = sc.materials[sc.instances[inst].material];
  const bool eta = m.eta[0] != 0.f || m.eta[1] != 0.f || m.eta[2] != 0.f;
  const bool k = m.k[0] != 0.f || m.k[1] != 0.f || m.k[2] != 0.f;
  return (eta && !k) ? 2u : (m.metallic >= 0 ? 1u : 0u);
}

#ifndef NB_SHADE_SORT
#define NB_SHADE_SORT 0
#endif
static_assert(!(NB_HIT_CLASSES && NB_SHADE_SORT), "one hit ordering at a time");

/* Resident blocks of 128 per SM that k_shade is compiled for.  With hits of one lobe family per
 * warp (NB_HIT_CLASSES), 8 blocks (64 registers) are best on the 32-job batch: 79.5 ms per step,
 * against 79.9 at 9, 80.7 at 10 (48 registers, more spills) and 81.4 at 12; before the split 10
 * blocks led (107.5 ms against 108.6 at 8), and 8 also suits the heightfield (11.7 against 12.1). */
#ifndef NB_SHADE_MIN_BLOCKS
#define NB_SHADE_MIN_BLOCKS 8
#endif

template <class JS>
__global__ void __launch_bounds__(128, NB_SHADE_MIN_BLOCKS) k_shade(Queue in, Queue out, WaveCounters *wcp, const float4 *hits,
                                               const uint2 *hit_slot, float4 *L, const __grid_constant__ JS js) {
  const uint32_t n = wcp->hit_count;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
#if NB_SHADE_SORT
  /* The block's 128 hits are permuted so that each lobe class runs contiguously (a counting sort of
   * four keys with warp ballots): warps then take one lobe's code path.  Only the order of the
   * continuation rays changes, never a path's result. */
  if (blockIdx.x * blockDim.x >= n) return; /* whole blocks leave together (barriers below) */
  __shared__ uint32_t s_cnt[4][4];
  __shared__ uint8_t s_perm[128];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t cls = lobe_class(in, hits, hit_slot, js, i, n);
  const unsigned mine = __ballot_sync(0xffffffffu, cls == 0u) * (cls == 0u) |
                        __ballot_sync(0xffffffffu, cls == 1u) * (cls == 1u) |
                        __ballot_sync(0xffffffffu, cls == 2u) * (cls == 2u) |
                        __ballot_sync(0xffffffffu, cls == 3u) * (cls == 3u);
  if (threadIdx.x < 16u) (&s_cnt[0][0])[threadIdx.x] = 0; /* blocks of fewer than 4 warps count 0 for the rest */
  __syncthreads();
  if (lane == (uint32_t)(__ffs(mine) - 1)) s_cnt[warp][cls] = (uint32_t)__popc(mine);
  __syncthreads();
  uint32_t pos = (uint32_t)__popc(mine & ((1u << lane) - 1u));
  for (uint32_t c = 0; c < cls; c++)
    pos += s_cnt[0][c] + s_cnt[1][c] + s_cnt[2][c] + s_cnt[3][c];
  for (uint32_t w = 0; w < warp; w++) pos += s_cnt[w][cls];
  s_perm[pos] = (uint8_t)threadIdx.x;
  __syncthreads();
  i = blockIdx.x * blockDim.x + s_perm[threadIdx.x];
  if (__all_sync(0xffffffffu, i >= n)) return;
#elif NB_HIT_CLASSES
  const uint32_t nf = n, nb = wcp->hit_back, cap = wcp->cap;
  if ((i & ~31u) >= nf + nb) return;
  /* hit i of the front range, or of the back range counted from the end of the list */
  const uint32_t h = i < nf ? i : (i < nf + nb ? cap - 1u - (i - nf) : 0u);
  shade_warp<JS, false>(in, out, wcp, hits, hit_slot, L, js, h, i < nf + nb ? 0xffffffffu : 0u);
  return;
#else
  if ((i & ~31u) >= n) return;
#endif
  shade_warp<JS, false>(in, out, wcp, hits, hit_slot, L, js, i, n);
}

/* ---------------------------------------------------------------- replay adjoint
 *
 * Path-replay backpropagation (detached sampling).  A path's estimate is
 *   I = sum_k beta_k e_k + beta_K env,  beta_k = w_0 ... w_{k-1},  w_k = f_k |cos| / pdf_k.
 * With the sampling densities held fixed, d w_k / d theta = w_k d ln f_k / d theta, and theta_k
 * (the albedo of the triangle hit at vertex k, the roughness of its material) scales everything
 * the path gathers after vertex k's own emission: R_k = I - sum_{m <= k} beta_m e_m.  So
 *   dLoss/dtheta_k += sum_c dLoss/dI_c R_k,c d ln f_k,c / d theta_k.
 * The replay starts with R = I (the path's radiance from the primal pass, read from the radiance
 * buffer) and subtracts emission as it walks the path again from the same Sobol index; vertices
 * add their terms to the gradients with atomics.  Extra path state: R and dLoss/dI (2 x 16 B). */

struct AdjQueue {
  float4 *rem, *dl;
};

/* Adds v[0..N) to base[key * N + 0..N) for every active lane.  Lanes of the warp with the same key
 * are summed first (pointer jumping along the lanes that share the key: after five rounds the
 * first lane of each key holds its sum), so a key costs one atomic per value per warp.  Camera
 * paths of neighbouring pixels share triangles and materials, and a large triangle can be hit by a
 * sizeable part of the image: without the warp sum, its atomics serialise.  All 32 lanes must call
 * this together. */
template <int N>
__device__ __forceinline__ void warp_add_by_key(bool active, uint32_t key, const float (&v)[N], float *base) {
  const unsigned full = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned peers = __match_any_sync(full, active ? key : 0xffffffffu);
  const unsigned above = lane == 31u ? 0u : (peers & (0xffffffffu << (lane + 1u)));
  int nxt = above ? __ffs(above) - 1 : 32;
  float sum[N];
#pragma unroll
  for (int k = 0; k < N; k++) sum[k] = active ? v[k] : 0.f;
#pragma unroll
  for (int it = 0; it < 5; it++) {
    const int src = nxt < 32 ? nxt : (int)lane;
    float t[N];
#pragma unroll
    for (int k = 0; k < N; k++) t[k] = __shfl_sync(full, sum[k], src);
    const int nn = __shfl_sync(full, nxt, src);
    if (nxt < 32) {
#pragma unroll
      for (int k = 0; k < N; k++) sum[k] += t[k];
      nxt = nn;
    }
  }
  if (active && lane == (unsigned)(__ffs(peers) - 1)) {
#pragma unroll
    for (int k = 0; k < N; k++)
      if (sum[k] != 0.f) atomicAdd(base + (size_t)key * N + k, sum[k]);
  }
}

template <class JS>
__global__ void __launch_bounds__(256) k_refill_adj(Queue q, AdjQueue a, const WaveCounters *wcp, const float4 *L,
                                                    const float4 *d_image, const __grid_constant__ JS js) {
  const WaveCounters wc = *wcp;
  const uint32_t n_new = wave_new(wc);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
    const CameraPath c = camera_path(js, wc.next + i);
    const RenderParams &rp = js.at(c.job).rp;
    const uint32_t slot = wc.n_active + i;
    q.o[slot] = make_float4(c.o.x, c.o.y, c.o.z, __uint_as_float(c.rslot));
    q.d[slot] = make_float4(c.d.x, c.d.y, c.d.z, __uint_as_float(c.job << 8));
    q.beta[slot] = make_float4(1.f, 1.f, 1.f, __uint_as_float(c.index));
    const float4 I = L[c.rslot];
    a.rem[slot] = make_float4(I.x, I.y, I.z, 0.f);
    /* the film pixel of (x, y): rows flipped when the frame asks for it (k_resolve) */
    const uint32_t row = rp.vinv ? (uint32_t)rp.H - 1u - c.y : c.y;
    const float4 g = d_image[(size_t)row * rp.W + c.x];
    const float inv = 1.f / (float)rp.count; /* the image is the mean of the frame's samples */
    a.dl[slot] = make_float4(g.x * inv, g.y * inv, g.z * inv, 0.f);
  }
}

template <class JS>
__global__ void __launch_bounds__(128, 8) k_shade_adj(Queue in, Queue out, AdjQueue ain, AdjQueue aout,
                                                      WaveCounters *wcp, const float4 *hits, const uint2 *hit_slot,
                                                      float *g_alb, float *g_rough, const __grid_constant__ JS js) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#if NB_HIT_CLASSES
  /* the front range of the hit list, then its back range counted from the end (see k_shade) */
  const uint32_t nf = wcp->hit_count, nb = wcp->hit_back, cap = wcp->cap;
  if ((t & ~31u) >= nf + nb) return;
  const bool valid = t < nf + nb;
  const uint32_t i = t < nf ? t : (valid ? cap - 1u - (t - nf) : 0u);
#else
  const uint32_t n = wcp->hit_count;
  if ((t & ~31u) >= n) return;
  const bool valid = t < n;
  const uint32_t i = t;
#endif
  bool enq = false, g_act = false;
  float4 no{}, nd{}, nbeta{}, nrem{}, ndl{};
  uint32_t g_prim = 0, g_mat = 0;
  float va[3] = {0.f, 0.f, 0.f}, vr[1] = {0.f};
  if (valid) {
    const uint2 hs = hit_slot[i];
    const uint32_t slot_in = hs.x, inst = hs.y;
    const float4 o4 = in.o[slot_in], d4 = in.d[slot_in], b4 = in.beta[slot_in], h = hits[i];
    const float4 r4 = ain.rem[slot_in], l4 = ain.dl[slot_in];
    const uint32_t tag = __float_as_uint(d4.w);
    const int bounce = (int)(tag & 0xffu);
    const Job &J = js.at(tag >> 8);
    const DevScene &sc = J.sc;
    const RenderParams &rp = J.rp;
    const uint32_t index = __float_as_uint(b4.w);
    const V3 ro{o4.x, o4.y, o4.z}, rd{d4.x, d4.y, d4.z};
    V3 beta{b4.x, b4.y, b4.z};
    V3 rem{r4.x, r4.y, r4.z};
    const V3 dl{l4.x, l4.y, l4.z};
    const int prim = __float_as_int(h.w);
    if (!hit_ids_valid(sc, prim, inst)) {
      atomicAdd(&wcp->bad_index, 1u);
      goto gather;
    }
    {
    const DevInstance &I = sc.instances[inst];
    const HitRecord hr = make_record(sc, ro, rd, I, (uint32_t)prim - I.prim_offset, h.x, h.y, h.z);
    Scores scs;
    const ScatterResult sr = scatter(sc, rd, hr, sc.materials[I.material], index, 2u + 4u * (unsigned)bounce, rp.seed,
                                     (uint32_t)prim, I.material, &scs);
    if (sr.valid && sc.has_emissive) rem = rem - beta * sr.emissive;
    if (sr.valid) {
      const V3 cw = dl * rem;
      g_act = true;
      g_prim = (uint32_t)prim;
      g_mat = I.material;
      va[0] = cw.x * scs.albedo.x;
      va[1] = cw.y * scs.albedo.y;
      va[2] = cw.z * scs.albedo.z;
      const float gr = ((cw.x + cw.y) + cw.z) * scs.roughness;
      vr[0] = isfinite(gr) ? gr : 0.f;
      V3 c = sr.weight;
      bool alive = true;
      if (rp.rr_start >= 0 && bounce >= rp.rr_start) {
        const V3 nbt = beta * c;
        const float q = fmin_std(1.f, fmax_std(0.05f, fmax_std(nbt.x, fmax_std(nbt.y, nbt.z))));
        const float urr = sobol_sample(sc.sobol_dv, index, kRRDimBase + (unsigned)bounce, rp.seed);
        if (!(urr < q))
          alive = false;
        else
          c = c / q;
      }
      if (alive && bounce + 1 <= rp.max_depth) {
        beta = beta * c;
        const float eps = 1e-3f;
        const V3 nd3 = normalize(sr.wi);
        const V3 no3 = hr.position + hr.ng * (eps + eps * fsign(dot(hr.ng, sr.wi)));
        enq = true;
        no = make_float4(no3.x, no3.y, no3.z, o4.w);
        nd = make_float4(nd3.x, nd3.y, nd3.z, __uint_as_float(tag + 1u));
        nbeta = make_float4(beta.x, beta.y, beta.z, b4.w);
        nrem = make_float4(rem.x, rem.y, rem.z, 0.f);
        ndl = l4;
      }
    }
    }
  }
gather:
  if (g_alb) warp_add_by_key<3>(g_act, g_prim, va, g_alb);
  if (g_rough) warp_add_by_key<1>(g_act, g_mat, vr, g_rough);
  const unsigned slot = warp_append(enq, &wcp->out_count);
  if (enq) {
    out.o[slot] = no;
    out.d[slot] = nd;
    out.beta[slot] = nbeta;
    aout.rem[slot] = nrem;
    aout.dl[slot] = ndl;
  }
}

__global__ void k_wave_end(WaveCounters *wc) {
  const uint32_t n_new = wave_new(*wc);
  const uint32_t n = wc->n_active + n_new;
  if (n) {
    wc->waves++;
    wc->traced += n;
  }
  wc->next += n_new;
  wc->n_active = wc->out_count;
  wc->out_count = 0;
  wc->hit_count = 0;
  wc->hit_back = 0;
  wc->trace_next = 0;
  wc->shade_next = 0;
  wc->done = (wc->n_active == 0 && wc->next == wc->total) ? 1u : 0u;
}

/* ---------------------------------------------------------------- persistent wavefront (trace_mode 3)
 *
 * One cooperative launch runs every wave of a chunk: refill -> trace -> shade -> wave end, the same
 * device functions as the per-wave kernels, separated by a grid barrier.  Warps take 32 rays (hits)
 * at a time from a counter, so the block scheduler's balancing of the per-wave kernels is kept.
 * Data one phase writes and a later phase reads on another SM is loaded through L2 (ldq<true>).
 *
 * The barrier is this file's own and its wait is bounded: block leaders arrive on a counter and
 * spin on a generation word with a time limit (globaltimer); a leader that waits past the limit sets
 * the status word to 1 and every block leaves at its next barrier, so the kernel always ends and the
 * host reports RENDERER_EXCEPTION.  A cancel (the context's mapped flag) sets status 2 the same way. */
struct PersistSync {
  unsigned arrive, gen, status, pad;
  unsigned long long trace_ns, shade_ns; /* phase times seen by block 0 */
};

__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) { return *(const volatile unsigned *)p; }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* false once any block gave up waiting (or the render was cancelled): the caller returns.  The leader's
 * reading of the status word is shared through shared memory, so a block leaves as a whole. */
__device__ bool grid_barrier(PersistSync *s, unsigned long long limit_ns) {
  __shared__ unsigned s_status;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_volatile(&s->gen);
    __threadfence();
    if (atomicAdd(&s->arrive, 1u) == gridDim.x - 1u) {
      atomicExch(&s->arrive, 0u);
      __threadfence();
      atomicAdd(&s->gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (ld_volatile(&s->gen) == gen) {
        if (ld_volatile(&s->status) != 0u) break;
        if (global_ns() - t0 > limit_ns) {
          atomicCAS(&s->status, 0u, 1u);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_status = ld_volatile(&s->status);
  }
  __syncthreads();
  return s_status == 0u;
}

/* A warp's next 32 items from a counter (lane 0 takes them, the warp shares the base). */
__device__ __forceinline__ uint32_t warp_take(unsigned *counter) {
  uint32_t base = 0;
  if ((threadIdx.x & 31u) == 0) base = atomicAdd(counter, 32u);
  return __shfl_sync(0xffffffffu, base, 0);
}

/* Resident blocks of 128 per SM that k_persist is compiled for.  It holds both the walk and the
 * shading state, so its register budget is the larger of the two phases': on the 32-job batch, 6
 * blocks (80 registers) took 379 ms per step, 5 (96) 408 ms and 4 (128, no spills) 465 ms, against
 * 316 ms for the per-wave kernels (40 resident warps for k_trace, 32 for k_shade when measured). */
#ifndef NB_PERSIST_MIN_BLOCKS
#define NB_PERSIST_MIN_BLOCKS 6
#endif

template <int WIDTH, class JS>
__global__ void __launch_bounds__(128, NB_PERSIST_MIN_BLOCKS) k_persist(Queue qa, Queue qb, WaveCounters *wcp, float4 *hits,
                                                 uint2 *hit_slot, float4 *L, PersistSync *sync,
                                                 const volatile int *cancel, unsigned long long limit_ns,
                                                 const __grid_constant__ JS js) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31u;
  const bool leader = tid == 0;
  for (uint32_t w = 0;; w++) {
    const Queue &in = (w & 1u) ? qb : qa;
    const Queue &out = (w & 1u) ? qa : qb;
    const uint32_t n_active = __ldcg(&wcp->n_active), next = __ldcg(&wcp->next);
    const uint32_t total = __ldcg(&wcp->total), cap = __ldcg(&wcp->cap);
    if (__ldcg(&wcp->done)) return;
    const uint32_t n_new = min(cap - n_active, total - next), n = n_active + n_new;
    for (uint32_t i = tid; i < n_new; i += nthreads) refill_one(in, next, n_active, L, js, i);
    if (!grid_barrier(sync, limit_ns)) return;
    const unsigned long long t0 = leader ? global_ns() : 0ull;
    for (;;) {
      const uint32_t base = warp_take(&wcp->trace_next);
      if (base >= n) break;
      trace_warp<WIDTH, JS, false, false, true>(in, wcp, hits, hit_slot, L, js, base + lane, n);
    }
    if (!grid_barrier(sync, limit_ns)) return;
    const unsigned long long t1 = leader ? global_ns() : 0ull;
    const uint32_t nh = __ldcg(&wcp->hit_count);
    for (;;) {
      const uint32_t base = warp_take(&wcp->shade_next);
      if (base >= nh) break;
      shade_warp<JS, true>(in, out, wcp, hits, hit_slot, L, js, base + lane, nh);
    }
    if (!grid_barrier(sync, limit_ns)) return;
    if (leader) { /* k_wave_end's update */
      sync->trace_ns += t1 - t0;
      sync->shade_ns += global_ns() - t1;
      WaveCounters *wc = wcp;
      if (n) {
        wc->waves++;
        wc->traced += n;
      }
      wc->next = next + n_new;
      wc->n_active = __ldcg(&wcp->out_count);
      wc->out_count = 0;
      wc->hit_count = 0;
      wc->hit_back = 0;
      wc->trace_next = 0;
      wc->shade_next = 0;
      wc->done = (wc->n_active == 0 && wc->next == total) ? 1u : 0u;
      if (*cancel) atomicCAS(&sync->status, 0u, 2u);
      __threadfence();
    }
    if (!grid_barrier(sync, limit_ns)) return;
  }
}

__global__ void k_resolve(const float4 *L, uint32_t NP, uint32_t count, float4 *acc, float denom, float *out, int W,
                          int H, int vinv) {
  const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= NP) return;
  float4 a = acc[pix];
  for (uint32_t s = 0; s < count; s++) {
    const float4 l = L[(size_t)s * NP + pix];
    a.x += l.x, a.y += l.y, a.z += l.z, a.w += l.w;
  }
  acc[pix] = a;
  const uint32_t y = pix / (uint32_t)W, x = pix - y * (uint32_t)W;
  const uint32_t row = vinv ? (uint32_t)H - 1u - y : y;
  reinterpret_cast<float4 *>(out)[(size_t)row * W + x] = make_float4(a.x / denom, a.y / denom, a.z / denom, a.w / denom);
}

__global__ void k_trace_api(DevScene sc, uint64_t n, const float *o, const float *d, int32_t *prim, float *t, float *u,
                            float *v) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TraceResult r =
      trace_closest(sc, V3{o[3 * i], o[3 * i + 1], o[3 * i + 2]}, V3{d[3 * i], d[3 * i + 1], d[3 * i + 2]});
  prim[i] = r.prim;
  t[i] = r.t;
  u[i] = r.u;
  v[i] = r.v;
}

/* One shading event per given hit: the hit record, the principled scatter with Sobol dimensions
 * 2 + 4 * bounce .. 5 + 4 * bounce, and the spawned ray (the body of k_shade for one path). */
__global__ void k_scatter_api(DevScene sc, uint64_t n, const float *o, const float *d, const int32_t *prim,
                              const float *t, const float *u, const float *v, const uint32_t *index,
                              const int32_t *bounce, uint32_t seed, float *out_o, float *out_d, float *weight,
                              float *emissive, int32_t *valid) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t p = prim[i];
  if (p < 0 || (uint64_t)p >= sc.n_prims || bounce[i] < 0 || bounce[i] > kMaxDepth) {
    valid[i] = -1;
    return;
  }
  const V3 ro{o[3 * i], o[3 * i + 1], o[3 * i + 2]}, rd{d[3 * i], d[3 * i + 1], d[3 * i + 2]};
  const DevInstance &I = sc.instances[__ldg(sc.prim_inst + p)];
  const HitRecord hr = make_record(sc, ro, rd, I, (uint32_t)p - I.prim_offset, t[i], u[i], v[i]);
  const ScatterResult sr =
      scatter(sc, rd, hr, sc.materials[I.material], index[i], 2u + 4u * (unsigned)bounce[i], seed, (uint32_t)p,
              I.material);
  const float eps = 1e-3f;
  const V3 nd3 = normalize(sr.wi);
  const V3 no3 = hr.position + hr.ng * (eps + eps * fsign(dot(hr.ng, sr.wi)));
  for (int k = 0; k < 3; k++) {
    out_o[3 * i + k] = k == 0 ? no3.x : k == 1 ? no3.y : no3.z;
    out_d[3 * i + k] = k == 0 ? nd3.x : k == 1 ? nd3.y : nd3.z;
    weight[3 * i + k] = k == 0 ? sr.weight.x : k == 1 ? sr.weight.y : sr.weight.z;
    emissive[3 * i + k] = k == 0 ? sr.emissive.x : k == 1 ? sr.emissive.y : sr.emissive.z;
  }
  valid[i] = sr.valid ? 1 : 0;
}

__global__ void k_sobol_api(const uint32_t *dv, uint64_t n, const uint32_t *idx, const uint32_t *dim, uint32_t seed,
                            float *out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t dm = dim[i];
  out[i] = dm < (uint32_t)kSobolDims ? sobol_sample(dv, idx[i], dm, seed) : __int_as_float(0x7fc00000);
}

/* ------------------------------------------------------------------ host side */

nova_b200_status ensure_film(nova_b200_ctx *c, int W, int H) {
  const size_t npx = (size_t)W * H;
  if (c->film_w != W || c->film_h != H || !c->d_film_acc) {
    cudaFree(c->d_film_acc);
    c->d_film_acc = nullptr;
    NB_CUDA(c, cudaMalloc(&c->d_film_acc, npx * sizeof(float4)), "cudaMalloc(film)");
    NB_CUDA(c, cudaMemsetAsync(c->d_film_acc, 0, npx * sizeof(float4), c->stream), "memset(film)");
    c->film_w = W;
    c->film_h = H;
    c->film_samples = 0;
  }
  if (c->film_out_cap < npx * 4) {
    cudaFree(c->d_film_out);
    c->d_film_out = nullptr;
    NB_CUDA(c, cudaMalloc(&c->d_film_out, npx * 4 * sizeof(float)), "cudaMalloc(film out)");
    c->film_out_cap = npx * 4;
  }
  return NOVA_B200_SUCCESS;
}

nova_b200_status ensure_wave_buffers(nova_b200_ctx *c, uint32_t cap, size_t radiance) {
  bool changed = false;
  if (c->queue_cap < cap) {
    cudaFree(c->d_queue);
    c->d_queue = nullptr;
    c->queue_cap = 0;
    c->queue_bytes = 0;
    const size_t bytes = (size_t)cap * (16 * 7 + 8 + (NB_RAY_ORDER ? 4 : 0));
    NB_CUDA(c, cudaMalloc(&c->d_queue, bytes), "cudaMalloc(queue)");
    c->queue_cap = cap;
    c->queue_bytes = bytes;
    changed = true;
  }
  if (c->radiance_cap < radiance) {
    cudaFree(c->d_radiance);
    c->d_radiance = nullptr;
    c->radiance_cap = 0;
    NB_CUDA(c, cudaMalloc(&c->d_radiance, radiance * sizeof(float4)), "cudaMalloc(radiance)");
    c->radiance_cap = radiance;
    changed = true;
  }
  if (!c->d_wave) {
    NB_CUDA(c, cudaMalloc(&c->d_wave, sizeof(WaveCounters)), "cudaMalloc(wave counters)");
    NB_CUDA(c, cudaMallocHost(&c->h_wave, 3 * sizeof(WaveCounters)), "cudaMallocHost(wave counters)");
    for (int k = 0; k < 2 * 3 * kWavesPerGraph; k++) NB_CUDA(c, cudaEventCreate(&c->ev_wave[k]), "cudaEventCreate");
    for (int k = 0; k < 2; k++)
      NB_CUDA(c, cudaEventCreateWithFlags(&c->ev_done[k], cudaEventDisableTiming), "cudaEventCreate");
    changed = true;
  }
  if (changed) {
    for (cudaGraphExec_t &g : c->graph_exec)
      if (g) cudaGraphExecDestroy(g), g = nullptr;
    c->graph_key.clear();
  }
  return NOVA_B200_SUCCESS;
}

/* Launch shape of one render: rays per wave and the trace / shade block sizes. */
struct LaunchShape {
  uint32_t cap;
  uint32_t trace_block, shade_block;
  uint32_t trace_mode; /* 0: one ray per thread, 1: persistent warps with ray hand-out (binary BVH),
                         2: one ray per thread, counting node visits and triangle tests,
                         3: the persistent wavefront (one cooperative launch per chunk) */
  uint32_t wait_limit_us; /* trace_mode 3: longest grid-barrier wait before the render fails */
};

struct WaveBuffers {
  Queue qa, qb;
  float4 *hits;
  uint2 *hit_slot; /* per hit: its ray's queue slot and the hit triangle's instance */
  uint32_t *order; /* k_order_rays' slot order (NB_RAY_ORDER builds only) */
  WaveCounters *wc;
};

WaveBuffers wave_buffers(nova_b200_ctx *c) {
  const uint32_t cap = c->queue_cap;
  float4 *base = static_cast<float4 *>(c->d_queue);
  WaveBuffers b;
  b.qa = Queue{base, base + cap, base + 2 * (size_t)cap};
  b.qb = Queue{base + 3 * (size_t)cap, base + 4 * (size_t)cap, base + 5 * (size_t)cap};
  b.hits = base + 6 * (size_t)cap;
  b.hit_slot = reinterpret_cast<uint2 *>(base + 7 * (size_t)cap);
  b.order = NB_RAY_ORDER ? reinterpret_cast<uint32_t *>(b.hit_slot + cap) : nullptr;
  b.wc = static_cast<WaveCounters *>(c->d_wave);
  return b;
}

/* Enqueues one group of kWavesPerGraph waves for pipeline slot `slot` (queues alternating
 * A -> B -> A ...): an event record around each trace and shade kernel (`external` while capturing,
 * so they become graph event-record nodes), the read-back of the counters into the slot's pinned
 * copy and the slot's completion event. */
/* Replay-loop arguments: the adjoint queues (A, B), the image adjoint and the gradients. */
struct AdjArgs {
  AdjQueue qa, qb;
  const float4 *d_image;
  float *g_alb, *g_rough;
};

template <class JS, int WIDTH, bool ADJ = false>
void enqueue_waves(nova_b200_ctx *c, const JS &js, const LaunchShape &ls, int slot, bool external,
                   const AdjArgs *adj = nullptr) {
  const WaveBuffers b = wave_buffers(c);
  int dev_sms = 148, occ_r = 1;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_r, k_refill<JS>, 256, 0);
  /* trace and shade: one ray per thread over the wave capacity, so the hardware block scheduler
   * balances rays of very different cost; blocks past the live count exit at once */
  const unsigned g_trace = (ls.cap + ls.trace_block - 1) / ls.trace_block;
  const unsigned g_shade = (ls.cap + ls.shade_block - 1) / ls.shade_block;
  const unsigned g_refill = (unsigned)(dev_sms * std::max(1, occ_r) * 2);
  int occ_t = 1;
  if (WIDTH == 2 && ls.trace_mode == 1)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, k_trace_dyn<JS>, 128, 0);
  const unsigned g_dyn = (unsigned)std::min<uint64_t>((uint64_t)dev_sms * std::max(1, occ_t), (ls.cap + 127) / 128);
  const unsigned flags = external ? cudaEventRecordExternal : cudaEventRecordDefault;
  cudaEvent_t *ev = c->ev_wave + 3 * kWavesPerGraph * slot;
  for (int w = 0; w < kWavesPerGraph; w++) {
    const Queue &in = (w & 1) ? b.qb : b.qa;
    const Queue &out = (w & 1) ? b.qa : b.qb;
    if constexpr (ADJ) {
      const AdjQueue &ain = (w & 1) ? adj->qb : adj->qa;
      const AdjQueue &aout = (w & 1) ? adj->qa : adj->qb;
      k_refill_adj<JS><<<g_refill, 256, 0, c->stream>>>(in, ain, b.wc, c->d_radiance, adj->d_image, js);
      cudaEventRecordWithFlags(ev[3 * w + 0], c->stream, flags);
      k_trace<WIDTH, JS, true><<<g_trace, ls.trace_block, 0, c->stream>>>(in, b.wc, b.hits, b.hit_slot, nullptr, js);
      cudaEventRecordWithFlags(ev[3 * w + 1], c->stream, flags);
      k_shade_adj<JS><<<g_shade, ls.shade_block, 0, c->stream>>>(in, out, ain, aout, b.wc, b.hits, b.hit_slot,
                                                                 adj->g_alb, adj->g_rough, js);
      cudaEventRecordWithFlags(ev[3 * w + 2], c->stream, flags);
    } else {
      k_refill<JS><<<g_refill, 256, 0, c->stream>>>(in, b.wc, c->d_radiance, js);
      const bool ordered = NB_RAY_ORDER && !(WIDTH == 2 && ls.trace_mode == 1);
#if NB_RAY_ORDER
      if (ordered)
        k_order_rays<NB_RAY_ORDER><<<(ls.cap + NB_RAY_ORDER - 1) / NB_RAY_ORDER, kOrderThreads, 0, c->stream>>>(
            in, b.wc, b.order);
#endif
      const uint32_t *order = ordered ? b.order : nullptr;
      cudaEventRecordWithFlags(ev[3 * w + 0], c->stream, flags);
      if (WIDTH == 2 && ls.trace_mode == 1)
        k_trace_dyn<JS><<<g_dyn, 128, 0, c->stream>>>(in, b.wc, b.hits, b.hit_slot, c->d_radiance, js);
      else if (ls.trace_mode == 2)
        k_trace<WIDTH, JS, false, true>
            <<<g_trace, ls.trace_block, 0, c->stream>>>(in, b.wc, b.hits, b.hit_slot, c->d_radiance, js, order);
      else
        k_trace<WIDTH, JS>
            <<<g_trace, ls.trace_block, 0, c->stream>>>(in, b.wc, b.hits, b.hit_slot, c->d_radiance, js, order);
      cudaEventRecordWithFlags(ev[3 * w + 1], c->stream, flags);
      k_shade<JS><<<g_shade, ls.shade_block, 0, c->stream>>>(in, out, b.wc, b.hits, b.hit_slot, c->d_radiance, js);
      cudaEventRecordWithFlags(ev[3 * w + 2], c->stream, flags);
    }
    k_wave_end<<<1, 1, 0, c->stream>>>(b.wc);
  }
  cudaMemcpyAsync(static_cast<WaveCounters *>(c->h_wave) + slot, b.wc, sizeof(WaveCounters), cudaMemcpyDeviceToHost,
                  c->stream);
  cudaEventRecordWithFlags(c->ev_done[slot], c->stream, flags);
}

template <class JS>
void enqueue_group(nova_b200_ctx *c, const JS &js, const LaunchShape &ls, int width, int slot, bool external) {
  if (width == 8)
    enqueue_waves<JS, 8>(c, js, ls, slot, external);
  else if (width == 1)
    enqueue_waves<JS, 1>(c, js, ls, slot, external);
  else
    enqueue_waves<JS, 2>(c, js, ls, slot, external);
}

/* Batch chunks: each slot's group is captured into a CUDA graph for the chunk's job table (the
 * table is a kernel parameter); the graphs are kept while the same table and width come back. */
nova_b200_status capture_graphs(nova_b200_ctx *c, const ManyJobs &js, const LaunchShape &ls, int width) {
  const size_t key_bytes = sizeof(ManyJobs) + sizeof(LaunchShape) + sizeof(int);
  std::vector<char> key(key_bytes);
  std::memcpy(key.data(), &js, sizeof(ManyJobs));
  std::memcpy(key.data() + sizeof(ManyJobs), &ls, sizeof(LaunchShape));
  std::memcpy(key.data() + sizeof(ManyJobs) + sizeof(LaunchShape), &width, sizeof(int));
  if (c->graph_exec[0] && c->graph_exec[1] && c->graph_key == key) return NOVA_B200_SUCCESS;
  c->graph_key.clear();
  for (int slot = 0; slot < 2; slot++) {
    if (c->graph_exec[slot]) cudaGraphExecDestroy(c->graph_exec[slot]), c->graph_exec[slot] = nullptr;
    cudaGraph_t graph = nullptr;
    NB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "capture");
    enqueue_group(c, js, ls, width, slot, true);
    const cudaError_t e_launch = cudaGetLastError();
    const cudaError_t e_end = cudaStreamEndCapture(c->stream, &graph);
    if (e_launch != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return nbctx::cuda_fail(c, e_launch, "capture kernels");
    }
    if (e_end != cudaSuccess) return nbctx::cuda_fail(c, e_end, "cudaStreamEndCapture");
    const cudaError_t e_inst = cudaGraphInstantiate(&c->graph_exec[slot], graph, 0);
    cudaGraphDestroy(graph);
    if (e_inst != cudaSuccess) {
      c->graph_exec[slot] = nullptr;
      return nbctx::cuda_fail(c, e_inst, "cudaGraphInstantiate");
    }
  }
  c->graph_key = std::move(key);
  return NOVA_B200_SUCCESS;
}

/* Counters of wave loops. */
struct LoopStats {
  float t_trace = 0.f, t_shade = 0.f;
  uint64_t kernels = 0, traced = 0;
  uint64_t nonfinite = 0, bad_index = 0, node_visits = 0, tri_tests = 0;
  uint32_t waves = 0;
  void add_to(nova_b200_render_stats &s) const {
    s.node_visits += node_visits;
    s.tri_tests += tri_tests;
    s.nonfinite += nonfinite;
    s.bad_index += bad_index;
    s.traced += traced;
    s.segments += traced;
    s.waves += waves;
    s.kernels += kernels;
    s.trace_ms += t_trace;
    s.shade_ms += t_shade;
  }
};

/* Runs the device-driven wave loop over `total` paths: uploads the counters, keeps two groups of
 * waves in flight (launch(slot) enqueues one), reads each finished group's counters and event
 * times, and stops once the device reports every path finished.  The group still in flight then
 * finds empty queues. */
template <class Launch>
nova_b200_status run_waves(nova_b200_ctx *x, uint32_t total, uint32_t cap, Launch &&launch, LoopStats &ls) {
  WaveCounters *hw = static_cast<WaveCounters *>(x->h_wave); /* [0], [1]: read-back slots, [2]: upload */
  /* a previous loop's last (empty) group may still be running: it is stream-ordered before this
   * upload, and the upload slot is only rewritten once the previous upload has completed */
  hw[2] = WaveCounters{};
  hw[2].total = total;
  hw[2].cap = cap;
  NB_CUDA(x, cudaMemcpyAsync(x->d_wave, hw + 2, sizeof(WaveCounters), cudaMemcpyHostToDevice, x->stream),
          "upload(wave counters)");
  NB_CUDA(x, launch(0), "wave group");
  NB_CUDA(x, launch(1), "wave group");
  int slot = 0;
  for (;;) {
    NB_CUDA(x, cudaEventSynchronize(x->ev_done[slot]), "waves");
    const cudaEvent_t *ev = x->ev_wave + 3 * kWavesPerGraph * slot;
    for (int w = 0; w < kWavesPerGraph; w++) {
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, ev[3 * w], ev[3 * w + 1]);
      cudaEventElapsedTime(&b, ev[3 * w + 1], ev[3 * w + 2]);
      ls.t_trace += a;
      ls.t_shade += b;
    }
    ls.kernels += 4 * kWavesPerGraph;
    const WaveCounters r = hw[slot];
    if (r.bad_index) { /* the device status word: stop after this group, as the reference aborts a tile
                        * once its exception manager holds an error (integrator/Integrator.h:74-78) */
      NB_CUDA(x, cudaEventSynchronize(x->ev_done[slot ^ 1]), "waves");
      const WaveCounters last = hw[slot ^ 1];
      ls.bad_index += std::max(r.bad_index, last.bad_index);
      ls.nonfinite += std::max(r.nonfinite, last.nonfinite);
      char msg[160];
      std::snprintf(msg, sizeof(msg), "device status: %u hits with an out-of-range primitive, instance or material id",
                    (unsigned)std::max(r.bad_index, last.bad_index));
      return nbctx::fail(x, NOVA_B200_RENDERER_EXCEPTION, "%s", msg);
    }
    if (r.done) {
      ls.waves += r.waves;
      ls.traced += r.traced;
      ls.nonfinite += r.nonfinite;
      ls.node_visits += r.node_visits;
      ls.tri_tests += r.tri_tests;
      break;
    }
    if (x->cancel.load()) { /* nova_b200_cancel: let the group in flight finish, enqueue nothing more */
      NB_CUDA(x, cudaEventSynchronize(x->ev_done[slot ^ 1]), "waves");
      return nbctx::fail(x, NOVA_B200_RENDERER_EXCEPTION, "render cancelled%s");
    }
    NB_CUDA(x, launch(slot), "wave group");
    slot ^= 1;
  }
  ls.kernels += 4 * kWavesPerGraph; /* the empty group */
  return NOVA_B200_SUCCESS;
}

/* The persistent wavefront over `total` paths: counters and barrier reset, one cooperative launch of
 * k_persist with every block resident (the occupancy calculator's count per SM), then the counters'
 * read-back.  Status 1 (a barrier wait ran out) and 2 (cancelled) fail the call; the context stays
 * usable either way (the kernel has returned). */
template <int WIDTH, class JS>
nova_b200_status run_persistent(nova_b200_ctx *x, const JS &js, const LaunchShape &ls, uint32_t total, uint32_t cap,
                                LoopStats &st) {
  using namespace nbctx;
  WaveCounters *hw = static_cast<WaveCounters *>(x->h_wave);
  if (!x->d_persist) {
    NB_CUDA(x, cudaMalloc(&x->d_persist, sizeof(PersistSync)), "cudaMalloc(persistent barrier)");
    void *flag = nullptr;
    NB_CUDA(x, cudaHostAlloc(&flag, sizeof(int), cudaHostAllocMapped), "cudaHostAlloc(cancel flag)");
    x->h_cancel_map = static_cast<volatile int *>(flag);
    *x->h_cancel_map = x->cancel.load() ? 1 : 0;
  }
  void *d_cancel_v = nullptr;
  NB_CUDA(x, cudaHostGetDevicePointer(&d_cancel_v, const_cast<int *>(x->h_cancel_map), 0), "cancel flag");
  int *d_cancel = static_cast<int *>(d_cancel_v);
  hw[2] = WaveCounters{};
  hw[2].total = total;
  hw[2].cap = cap;
  NB_CUDA(x, cudaMemcpyAsync(x->d_wave, hw + 2, sizeof(WaveCounters), cudaMemcpyHostToDevice, x->stream),
          "upload(wave counters)");
  NB_CUDA(x, cudaMemsetAsync(x->d_persist, 0, sizeof(PersistSync), x->stream), "reset(barrier)");
  int sms = 148, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device);
  NB_CUDA(x, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_persist<WIDTH, JS>, 128, 0), "occupancy");
  if (occ < 1) return fail(x, NOVA_B200_RENDERER_EXCEPTION, "persistent wavefront: no resident block fits%s");
  const WaveBuffers b = wave_buffers(x);
  PersistSync *sync = static_cast<PersistSync *>(x->d_persist);
  float4 *L = x->d_radiance;
  const volatile int *cancel = d_cancel;
  const unsigned long long limit_ns = 1000ull * ls.wait_limit_us;
  void *args[] = {const_cast<Queue *>(&b.qa), const_cast<Queue *>(&b.qb), const_cast<WaveCounters **>(&b.wc),
                  const_cast<float4 **>(&b.hits), const_cast<uint2 **>(&b.hit_slot), &L, &sync,
                  const_cast<const volatile int **>(&cancel), const_cast<unsigned long long *>(&limit_ns),
                  const_cast<JS *>(&js)};
  NB_CUDA(x, cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(k_persist<WIDTH, JS>), dim3(sms * occ),
                                         dim3(128), args, 0, x->stream),
          "persistent wavefront launch");
  PersistSync hs{};
  NB_CUDA(x, cudaMemcpyAsync(hw, x->d_wave, sizeof(WaveCounters), cudaMemcpyDeviceToHost, x->stream), "readback");
  NB_CUDA(x, cudaMemcpyAsync(&hs, x->d_persist, sizeof(PersistSync), cudaMemcpyDeviceToHost, x->stream), "readback");
  NB_CUDA(x, cudaStreamSynchronize(x->stream), "persistent wavefront");
  const WaveCounters r = hw[0];
  st.kernels += 1;
  st.t_trace += (float)(hs.trace_ns * 1e-6);
  st.t_shade += (float)(hs.shade_ns * 1e-6);
  st.waves += r.waves;
  st.traced += r.traced;
  st.nonfinite += r.nonfinite;
  st.bad_index += r.bad_index;
  if (hs.status == 2u) return fail(x, NOVA_B200_RENDERER_EXCEPTION, "render cancelled%s");
  if (hs.status != 0u) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "persistent wavefront: a grid barrier waited longer than %u us", ls.wait_limit_us);
    return fail(x, NOVA_B200_RENDERER_EXCEPTION, "%s", msg);
  }
  if (r.bad_index) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "device status: %u hits with an out-of-range primitive, instance or material id",
                  (unsigned)r.bad_index);
    return fail(x, NOVA_B200_RENDERER_EXCEPTION, "%s", msg);
  }
  if (!r.done) return fail(x, NOVA_B200_RENDERER_EXCEPTION, "persistent wavefront ended before its paths%s");
  return NOVA_B200_SUCCESS;
}

template <class JS>
nova_b200_status run_persistent_w(nova_b200_ctx *x, const JS &js, const LaunchShape &ls, int width, uint32_t total,
                                  uint32_t cap, LoopStats &st) {
  if (width == 8) return run_persistent<8>(x, js, ls, total, cap, st);
  if (width == 1) return run_persistent<1>(x, js, ls, total, cap, st);
  return run_persistent<2>(x, js, ls, total, cap, st);
}

struct Piece {
  nova_b200_ctx *ctx; /* the job's context: scene, BVH, film */
  const nova_b200_frame *f;
  uint32_t begin, count;
};

/* The frame's own fields (the scene and BVH are checked by validate_frame). */
nova_b200_status validate_frame_fields(nova_b200_ctx *c, const nova_b200_frame *f) {
  using namespace nbctx;
  if (!f) return fail(c, NOVA_B200_INVALID_ARGUMENT, "frame is null%s");
  if (f->width <= 0 || f->height <= 0 || f->spp_total <= 0 || f->sample_begin < 0 || f->sample_count <= 0 ||
      f->sample_begin + f->sample_count > f->spp_total)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid frame size or sample range%s");
  if (f->max_depth < 0 || f->max_depth > kMaxDepth)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "max_depth must be in 0..48 (Sobol dimensions)%s");
  if ((uint64_t)f->width * f->height * (uint64_t)f->spp_total >= (1ull << 32))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "width * height * spp must stay below 2^32 (Sobol index)%s");
  return NOVA_B200_SUCCESS;
}

nova_b200_status validate_frame(nova_b200_ctx *c, const nova_b200_frame *f) {
  using namespace nbctx;
  if (f && !c->bvh_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  return validate_frame_fields(c, f);
}

/* Pipelined batches: called before a chunk uses job j's scene; blocks until that context's upload
 * and build are done and returns their status. */
using WaitReady = std::function<nova_b200_status(size_t)>;

/* Renders frames (one per job) as one wavefront on the executing context `x`.  Jobs are cut into
 * chunks whose per-path radiance fits the radiance buffer; a job's samples stay in order. */
/* The order frames go into chunks: largest film first.  The films of the last chunk are copied
 * out after its waves end (those of earlier chunks while later ones render), so it holds the
 * smallest; a frame's film does not depend on the chunk it lands in. */
std::vector<uint32_t> chunk_order(const std::vector<const nova_b200_frame *> &frames) {
  std::vector<uint32_t> ord(frames.size());
  for (uint32_t j = 0; j < (uint32_t)ord.size(); j++) ord[j] = j;
  std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
    return (uint64_t)frames[a]->width * frames[a]->height > (uint64_t)frames[b]->width * frames[b]->height;
  });
  return ord;
}

nova_b200_status render_jobs(nova_b200_ctx *x, const std::vector<nova_b200_ctx *> &ctxs,
                             const std::vector<const nova_b200_frame *> &frames, float *const *films_host,
                             float *const *films_device, nova_b200_render_stats *stats,
                             const WaitReady *wait_ready = nullptr, int pipelined_width = 0,
                             uint32_t first_chunk_jobs = kParamJobs) {
  using namespace nbctx;
  x->cancel.store(false); /* a cancel applies to the call in progress */
  if (x->h_cancel_map) *x->h_cancel_map = 0;
  const size_t nj = ctxs.size();
  const int width = wait_ready ? pipelined_width : ctxs[0]->bvh_width;
  uint64_t max_np = 0, total = 0;
  for (size_t j = 0; j < nj; j++) {
    if (ctxs[j]->device != x->device)
      return fail(x, NOVA_B200_INVALID_ARGUMENT, "all contexts of a batch must use the same device%s");
    if (!wait_ready && ctxs[j]->bvh_width != width)
      return fail(x, NOVA_B200_INVALID_ARGUMENT, "all scenes of a batch must use the same BVH width%s");
    const uint64_t np = (uint64_t)frames[j]->width * frames[j]->height;
    max_np = std::max(max_np, np);
    total += np * (uint64_t)frames[j]->sample_count;
  }
  const uint64_t cap_entries = kRadianceCapBytes / sizeof(float4);
  const uint64_t radiance = std::max<uint64_t>(max_np, std::min<uint64_t>(total, cap_entries));
  const nova_b200_tuning &tu = x->tuning;
  const uint32_t qc = tu.queue_capacity ? tu.queue_capacity : kQueueCapDefault;
  const uint32_t cap = (uint32_t)std::min<uint64_t>(qc, std::max<uint64_t>(radiance, 1024));
  const LaunchShape ls{cap, tu.trace_block ? tu.trace_block : 128u, tu.shade_block ? tu.shade_block : 128u,
                       tu.trace_mode, tu.wait_limit_us ? tu.wait_limit_us : 1000000u};
  nova_b200_status st = ensure_wave_buffers(x, cap, radiance);
  if (st != NOVA_B200_SUCCESS) return st;
  x->primal_valid = false; /* this render overwrites the radiance buffer */
  for (size_t j = 0; j < nj; j++) {
    nova_b200_ctx *c = ctxs[j];
    if ((st = ensure_film(c, frames[j]->width, frames[j]->height)) != NOVA_B200_SUCCESS) return st;
    if (frames[j]->reset) {
      NB_CUDA(x, cudaMemsetAsync(c->d_film_acc, 0, (size_t)frames[j]->width * frames[j]->height * sizeof(float4),
                                 x->stream),
              "memset(film)");
      c->film_samples = 0;
    }
  }
  /* scene uploads and film clears of other contexts ran on their own streams (pipelined: each
   * context's upload and build end with a synchronisation of its stream, and the chunk loop waits
   * for them) */
  if (!wait_ready)
    for (size_t j = 0; j < nj; j++)
      if (ctxs[j] != x) NB_CUDA(x, cudaStreamSynchronize(ctxs[j]->stream), "sync batch context");
  /* cut the work into chunks of at most `radiance` paths and kParamJobs frame pieces */
  std::vector<std::vector<Piece>> chunks(1);
  uint64_t in_chunk = 0;
  const std::vector<uint32_t> ord = chunk_order(frames);
  for (size_t q = 0; q < nj; q++) {
    const size_t j = ord[q];
    const nova_b200_frame *f = frames[j];
    const uint64_t np = (uint64_t)f->width * f->height;
    uint32_t s = 0;
    while (s < (uint32_t)f->sample_count) {
      uint64_t room = (radiance - in_chunk) / np;
      if (room == 0 || chunks.back().size() == (chunks.size() == 1 ? first_chunk_jobs : kParamJobs)) {
        chunks.emplace_back();
        in_chunk = 0;
        room = radiance / np;
      }
      const uint32_t take = (uint32_t)std::min<uint64_t>(room, (uint64_t)f->sample_count - s);
      chunks.back().push_back(Piece{ctxs[j], f, (uint32_t)f->sample_begin + s, take});
      in_chunk += np * take;
      s += take;
    }
  }
  /* A frame's film is final after its last chunk: with several chunks, device films and pinned host
   * films of finished frames are copied out on a second stream while later chunks render. */
  const size_t nc = chunks.size();
  std::vector<size_t> last_chunk(nj, 0);
  std::vector<char> early(nj, 0);
  if (nc > 1) {
    for (size_t ci = 0; ci < nc; ci++)
      for (const Piece &P : chunks[ci])
        for (size_t j = 0; j < nj; j++)
          if (ctxs[j] == P.ctx) last_chunk[j] = ci;
    for (size_t j = 0; j < nj; j++) {
      bool pinned = false;
      if (films_host && films_host[j]) {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, films_host[j]) == cudaSuccess)
          pinned = pa.type == cudaMemoryTypeHost;
        else
          cudaGetLastError(); /* not a pointer the runtime knows: treated as pageable */
      }
      const bool host_ok = !(films_host && films_host[j]) || pinned;
      early[j] = host_ok && last_chunk[j] + 1 < nc ? 1 : 0;
    }
    if (!x->copy_stream) {
      NB_CUDA(x, cudaStreamCreateWithFlags(&x->copy_stream, cudaStreamNonBlocking), "film copy stream");
      NB_CUDA(x, cudaEventCreateWithFlags(&x->ev_copy, cudaEventDisableTiming), "film copy event");
    }
  }
  struct CopiesDone { /* every return waits for the film copies already issued */
    cudaStream_t s;
    ~CopiesDone() {
      if (s) cudaStreamSynchronize(s);
    }
  } copies_done{nc > 1 ? x->copy_stream : nullptr};
  auto copy_film = [&](size_t j, cudaStream_t stream) -> nova_b200_status {
    const size_t bytes = (size_t)frames[j]->width * frames[j]->height * 4 * sizeof(float);
    if (films_device && films_device[j])
      NB_CUDA(x, cudaMemcpyAsync(films_device[j], ctxs[j]->d_film_out, bytes, cudaMemcpyDeviceToDevice, stream),
              "copy film");
    if (films_host && films_host[j])
      NB_CUDA(x, cudaMemcpyAsync(films_host[j], ctxs[j]->d_film_out, bytes, cudaMemcpyDeviceToHost, stream),
              "copy film");
    return NOVA_B200_SUCCESS;
  };
  nova_b200_render_stats sum{};
  LoopStats loop;
  NB_CUDA(x, cudaEventRecord(x->ev_begin, x->stream), "event");
  std::vector<Job> hj(kParamJobs);
  ManyJobs many{};
  for (size_t ci = 0; ci < nc; ci++) {
    const auto &chunk = chunks[ci];
    if (x->cancel.load()) return fail(x, NOVA_B200_RENDERER_EXCEPTION, "render cancelled%s");
    if (chunk.empty()) continue;
    if (wait_ready)
      for (const Piece &P : chunk)
        for (size_t j = 0; j < nj; j++)
          if (ctxs[j] == P.ctx && (st = (*wait_ready)(j)) != NOVA_B200_SUCCESS) return st;
    uint32_t pb = 0;
    for (size_t k = 0; k < chunk.size(); k++) {
      const Piece &P = chunk[k];
      Job &J = hj[k];
      J = Job{};
      J.sc = P.ctx->scene;
      RenderParams &rp = J.rp;
      rp.W = P.f->width, rp.H = P.f->height, rp.NP = (uint32_t)((uint64_t)P.f->width * P.f->height);
      rp.count = P.count;
      rp.begin = P.begin;
      rp.spp_total = (uint32_t)P.f->spp_total;
      rp.max_depth = P.f->max_depth;
      rp.seed = P.f->seed;
      rp.rr_start = P.f->rr_start;
      std::copy(P.f->inv_P, P.f->inv_P + 16, rp.inv_P);
      std::copy(P.f->inv_V, P.f->inv_V + 16, rp.inv_V);
      rp.vinv = P.f->vertical_invert;
      set_tiles(rp, tu);
      J.path_begin = pb;
      J.n_paths = rp.NP * P.count;
      pb += J.n_paths;
    }
    const bool single = chunk.size() == 1;
    OneJob one{};
    if (single) {
      one.j = hj[0];
    } else {
      many = ManyJobs{};
      many.n = (uint32_t)chunk.size();
      std::copy(hj.begin(), hj.begin() + chunk.size(), many.j);
    }
    if (ls.trace_mode == 3) { /* the persistent wavefront: one launch runs every wave of the chunk */
      st = single ? run_persistent_w(x, one, ls, width, pb, cap, loop) : run_persistent_w(x, many, ls, width, pb, cap, loop);
      if (st != NOVA_B200_SUCCESS) return st;
    } else {
      if (!single && (st = capture_graphs(x, many, ls, width)) != NOVA_B200_SUCCESS) return st;
      auto launch = [&](int slot) {
        if (!single) return cudaGraphLaunch(x->graph_exec[slot], x->stream);
        enqueue_group(x, one, ls, width, slot, false);
        return cudaGetLastError();
      };
      if ((st = run_waves(x, pb, cap, launch, loop)) != NOVA_B200_SUCCESS) return st;
    }
    sum.paths += pb;
    for (size_t k = 0; k < chunk.size(); k++) {
      const Piece &P = chunk[k];
      nova_b200_ctx *c = P.ctx;
      c->film_samples += P.count;
      const uint32_t NP = hj[k].rp.NP;
      k_resolve<<<(NP + 255) / 256, 256, 0, x->stream>>>(x->d_radiance + hj[k].path_begin, NP, P.count, c->d_film_acc,
                                                         (float)c->film_samples, c->d_film_out, P.f->width,
                                                         P.f->height, P.f->vertical_invert);
      sum.kernels++;
    }
    bool any = false;
    for (size_t j = 0; j < nj; j++) any = any || (early[j] && last_chunk[j] == ci);
    if (any) {
      NB_CUDA(x, cudaEventRecord(x->ev_copy, x->stream), "event");
      NB_CUDA(x, cudaStreamWaitEvent(x->copy_stream, x->ev_copy, 0), "event");
      for (size_t j = 0; j < nj; j++)
        if (early[j] && last_chunk[j] == ci && (st = copy_film(j, x->copy_stream)) != NOVA_B200_SUCCESS) return st;
    }
  }
  NB_CUDA(x, cudaGetLastError(), "render kernels");
  NB_CUDA(x, cudaEventRecord(x->ev_end, x->stream), "event");
  for (size_t j = 0; j < nj; j++)
    if (!early[j] && (st = copy_film(j, x->stream)) != NOVA_B200_SUCCESS) return st;
  NB_CUDA(x, cudaStreamSynchronize(x->stream), "render");
  if (x->copy_stream) NB_CUDA(x, cudaStreamSynchronize(x->copy_stream), "film copies");
  if (nj == 1 && chunks.size() == 1 && chunks[0].size() == 1) {
    x->primal_valid = true;
    x->primal_frame = *frames[0];
    x->primal_albedo = x->scene.diff_albedo;
    x->primal_rough = x->scene.diff_rough;
  }
  float total_ms = 0.f;
  cudaEventElapsedTime(&total_ms, x->ev_begin, x->ev_end);
  loop.add_to(sum);
  sum.device_ms = total_ms;
  if (stats) *stats = sum;
  return NOVA_B200_SUCCESS;
}

}  // namespace

nova_b200_status nb_render(nova_b200_ctx *c, const nova_b200_frame *f, float *film_host, float *film_device,
                           nova_b200_render_stats *stats) {
  nova_b200_status st = validate_frame(c, f);
  if (st != NOVA_B200_SUCCESS) return st;
  cudaSetDevice(c->device);
  return render_jobs(c, {c}, {f}, &film_host, &film_device, stats);
}

/* Upload, build and render a batch in one pipelined call: up to 16 host threads upload and build
 * the contexts in batch order (each on its own stream), and the calling thread renders on ctxs[0],
 * starting each chunk as soon as the contexts of its frames are built, so the later scenes' copies
 * and builds overlap the first chunks' waves.  Same result as the three calls one after another. */
nova_b200_status nb_upload_build_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                              const nova_b200_frame *frames, uint32_t n,
                                              const nova_b200_bvh_options *opts, float *const *films_host,
                                              float *const *films_device, nova_b200_render_stats *stats) {
  using namespace nbctx;
  if (!ctxs || !ctxs[0]) return NOVA_B200_INVALID_ARGUMENT;
  nova_b200_ctx *x = ctxs[0];
  if (!descs || !frames || n == 0) return fail(x, NOVA_B200_INVALID_ARGUMENT, "empty batch%s");
  const int width = opts && opts->width ? opts->width : 2;
  std::vector<nova_b200_ctx *> cs(n);
  std::vector<const nova_b200_frame *> fs(n);
  for (uint32_t j = 0; j < n; j++) {
    if (!ctxs[j]) return fail(x, NOVA_B200_INVALID_ARGUMENT, "null context in batch%s");
    if (ctxs[j]->device != x->device)
      return fail(x, NOVA_B200_INVALID_ARGUMENT, "all contexts of a batch must use the same device%s");
    nova_b200_status st = validate_frame_fields(ctxs[j], &frames[j]);
    if (st != NOVA_B200_SUCCESS) {
      x->error = ctxs[j]->error;
      return st;
    }
    for (uint32_t k = 0; k < j; k++)
      if (ctxs[k] == ctxs[j]) return fail(x, NOVA_B200_INVALID_ARGUMENT, "a context appears twice in a batch%s");
    cs[j] = ctxs[j];
    fs[j] = &frames[j];
  }
  constexpr int kPending = -1;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<int> done(n, kPending);
  std::atomic<uint32_t> next{0};
  std::atomic<bool> stop{false};
  /* scenes are built in the order chunks render them, the executing context's own first (its stream
   * carries the render) */
  std::vector<uint32_t> ord = chunk_order(fs);
  std::rotate(ord.begin(), std::find(ord.begin(), ord.end(), 0u), std::find(ord.begin(), ord.end(), 0u) + 1);
  auto work = [&] {
    for (uint32_t q; (q = next.fetch_add(1)) < n;) {
      const uint32_t k = ord[q];
      nova_b200_status st = stop.load() ? NOVA_B200_RENDERER_EXCEPTION : nova_b200_upload_scene(cs[k], &descs[k]);
      if (st == NOVA_B200_SUCCESS) st = nova_b200_build_bvh(cs[k], opts);
      {
        std::lock_guard<std::mutex> lock(mu);
        done[k] = (int)st;
      }
      cv.notify_all();
    }
  };
  const unsigned nt = std::max(1u, std::min(std::min(n, 16u), std::max(1u, std::thread::hardware_concurrency())));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; t++) pool.emplace_back(work);
  const WaitReady wait_ready = [&](size_t j) -> nova_b200_status {
    nova_b200_status st;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv.wait(lock, [&] { return done[j] != kPending; });
      st = (nova_b200_status)done[j];
    }
    if (st != NOVA_B200_SUCCESS) {
      if (cs[j] != x) x->error = cs[j]->error;
      return st;
    }
    if (cs[j]->bvh_width != width)
      return fail(x, NOVA_B200_INVALID_ARGUMENT, "all scenes of a batch must use the same BVH width%s");
    return NOVA_B200_SUCCESS;
  };
  /* the executing context's own scene must be in place before its stream renders */
  nova_b200_status st = wait_ready(0);
  if (st == NOVA_B200_SUCCESS) {
    cudaSetDevice(x->device);
    /* the first chunk holds only the frames whose scenes the first round of threads builds, so its
     * waves start while the rest build */
    st = render_jobs(x, cs, fs, films_host, films_device, stats, &wait_ready, width, std::min<uint32_t>(nt, kParamJobs));
  }
  stop.store(st != NOVA_B200_SUCCESS); /* a failed render skips the uploads not started yet */
  for (auto &t : pool) t.join();
  if (st == NOVA_B200_SUCCESS)
    for (uint32_t k = 0; k < n; k++)
      if (done[k] != (int)NOVA_B200_SUCCESS) {
        if (k != 0) x->error = cs[k]->error;
        return (nova_b200_status)done[k];
      }
  return st;
}

nova_b200_status nb_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_frame *frames, uint32_t n,
                                 float *const *films_host, float *const *films_device, nova_b200_render_stats *stats) {
  using namespace nbctx;
  if (!ctxs || !ctxs[0]) return NOVA_B200_INVALID_ARGUMENT;
  nova_b200_ctx *x = ctxs[0];
  if (!frames || n == 0) return fail(x, NOVA_B200_INVALID_ARGUMENT, "empty batch%s");
  std::vector<nova_b200_ctx *> cs(n);
  std::vector<const nova_b200_frame *> fs(n);
  for (uint32_t j = 0; j < n; j++) {
    if (!ctxs[j]) return fail(x, NOVA_B200_INVALID_ARGUMENT, "null context in batch%s");
    nova_b200_status st = validate_frame(ctxs[j], &frames[j]);
    if (st != NOVA_B200_SUCCESS) {
      x->error = ctxs[j]->error;
      return st;
    }
    for (uint32_t k = 0; k < j; k++)
      if (ctxs[k] == ctxs[j]) return fail(x, NOVA_B200_INVALID_ARGUMENT, "a context appears twice in a batch%s");
    cs[j] = ctxs[j];
    fs[j] = &frames[j];
  }
  cudaSetDevice(x->device);
  return render_jobs(x, cs, fs, films_host, films_device, stats);
}

/* The frame fields that decide every path of a render (reset and vertical_invert do not). */
bool same_paths(const nova_b200_frame &a, const nova_b200_frame &b) {
  return a.width == b.width && a.height == b.height && a.spp_total == b.spp_total &&
         a.sample_begin == b.sample_begin && a.sample_count == b.sample_count && a.max_depth == b.max_depth &&
         a.seed == b.seed && a.rr_start == b.rr_start && std::memcmp(a.inv_P, b.inv_P, sizeof(a.inv_P)) == 0 &&
         std::memcmp(a.inv_V, b.inv_V, sizeof(a.inv_V)) == 0;
}

nova_b200_status nb_backward(nova_b200_ctx *c, const nova_b200_frame *f, const float *d_image, float *grad_albedo,
                             float *grad_roughness, uint32_t flags, nova_b200_render_stats *stats) {
  using namespace nbctx;
  nova_b200_status st = validate_frame(c, f);
  if (st != NOVA_B200_SUCCESS) return st;
  if (!d_image) return fail(c, NOVA_B200_INVALID_ARGUMENT, "d_image is null%s");
  cudaSetDevice(c->device);
  const uint32_t NP = (uint32_t)((uint64_t)f->width * f->height);
  const uint64_t total = (uint64_t)NP * (uint64_t)f->sample_count;
  const uint64_t radiance = std::max<uint64_t>(NP, std::min<uint64_t>(total, kRadianceCapBytes / sizeof(float4)));
  const nova_b200_tuning &tu = c->tuning;
  const uint32_t qc = tu.queue_capacity ? tu.queue_capacity : kQueueCapDefault;
  const uint32_t cap = (uint32_t)std::min<uint64_t>(qc, std::max<uint64_t>(radiance, 1024));
  const LaunchShape ls{cap, tu.trace_block ? tu.trace_block : 128u, tu.shade_block ? tu.shade_block : 128u,
                       tu.trace_mode == 3 ? 0u : tu.trace_mode, 0u}; /* the replay keeps the per-wave kernels */
  if ((st = ensure_wave_buffers(c, cap, radiance)) != NOVA_B200_SUCCESS) return st;
  if (c->adj_cap < c->queue_cap) {
    cudaFree(c->d_adj);
    c->d_adj = nullptr;
    c->adj_cap = 0;
    NB_CUDA(c, cudaMalloc(&c->d_adj, sizeof(float4) * 4 * (size_t)c->queue_cap), "cudaMalloc(adjoint queues)");
    c->adj_cap = c->queue_cap;
  }
  AdjArgs adj;
  const size_t qcap = c->adj_cap;
  adj.qa = AdjQueue{c->d_adj, c->d_adj + qcap};
  adj.qb = AdjQueue{c->d_adj + 2 * qcap, c->d_adj + 3 * qcap};
  adj.d_image = reinterpret_cast<const float4 *>(d_image);
  adj.g_alb = grad_albedo;
  adj.g_rough = grad_roughness;
  const int width = c->bvh_width;
  nova_b200_render_stats sum{};
  LoopStats primal, replay;
  NB_CUDA(c, cudaEventRecord(c->ev_begin, c->stream), "event");
  const uint32_t per_chunk = (uint32_t)std::max<uint64_t>(1, radiance / NP);
  const bool reuse = (flags & NOVA_B200_BACKWARD_REUSE_PRIMAL) && c->primal_valid &&
                     per_chunk >= (uint32_t)f->sample_count && same_paths(c->primal_frame, *f) &&
                     c->primal_albedo == c->scene.diff_albedo && c->primal_rough == c->scene.diff_rough;
  if (!reuse) c->primal_valid = false; /* the radiance pass below overwrites the buffer (and may stop midway) */
  c->cancel.store(false);              /* a cancel applies to the call in progress */
  for (uint32_t s0 = 0; s0 < (uint32_t)f->sample_count; s0 += per_chunk) {
    const uint32_t take = std::min<uint32_t>(per_chunk, (uint32_t)f->sample_count - s0);
    OneJob one{};
    Job &J = one.j;
    J.sc = c->scene;
    RenderParams &rp = J.rp;
    rp.W = f->width, rp.H = f->height, rp.NP = NP;
    rp.count = (uint32_t)f->sample_count; /* the image averages all of the frame's samples */
    rp.begin = (uint32_t)f->sample_begin + s0;
    rp.spp_total = (uint32_t)f->spp_total;
    rp.max_depth = f->max_depth;
    rp.seed = f->seed;
    rp.rr_start = f->rr_start;
    std::copy(f->inv_P, f->inv_P + 16, rp.inv_P);
    std::copy(f->inv_V, f->inv_V + 16, rp.inv_V);
    rp.vinv = f->vertical_invert;
    set_tiles(rp, tu);
    J.path_begin = 0;
    J.n_paths = NP * take;
    /* primal: each path's radiance into the radiance buffer */
    auto fwd = [&](int slot) {
      enqueue_group(c, one, ls, width, slot, false);
      return cudaGetLastError();
    };
    if (!reuse && (st = run_waves(c, J.n_paths, cap, fwd, primal)) != NOVA_B200_SUCCESS) return st;
    /* replay with the adjoint */
    auto bwd = [&](int slot) {
      if (width == 8)
        enqueue_waves<OneJob, 8, true>(c, one, ls, slot, false, &adj);
      else if (width == 1)
        enqueue_waves<OneJob, 1, true>(c, one, ls, slot, false, &adj);
      else
        enqueue_waves<OneJob, 2, true>(c, one, ls, slot, false, &adj);
      return cudaGetLastError();
    };
    if ((st = run_waves(c, J.n_paths, cap, bwd, replay)) != NOVA_B200_SUCCESS) return st;
    sum.paths += J.n_paths;
  }
  NB_CUDA(c, cudaEventRecord(c->ev_end, c->stream), "event");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "backward");
  float total_ms = 0.f;
  cudaEventElapsedTime(&total_ms, c->ev_begin, c->ev_end);
  primal.add_to(sum);
  replay.add_to(sum);
  sum.device_ms = total_ms;
  if (stats) *stats = sum;
  /* a one-pass backward leaves this frame's radiance in the buffer */
  c->primal_valid = per_chunk >= (uint32_t)f->sample_count;
  c->primal_frame = *f;
  c->primal_albedo = c->scene.diff_albedo;
  c->primal_rough = c->scene.diff_rough;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nb_trace(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, int32_t *prim, float *t,
                          float *u, float *v) {
  using namespace nbctx;
  if (!c->bvh_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  if (n == 0) return NOVA_B200_SUCCESS;
  if (!o || !d || !prim || !t || !u || !v) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  cudaSetDevice(c->device);
  k_trace_api<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(c->scene, n, o, d, prim, t, u, v);
  NB_CUDA(c, cudaGetLastError(), "k_trace_api");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "trace");
  return NOVA_B200_SUCCESS;
}

nova_b200_status nb_scatter(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, const int32_t *prim,
                            const float *t, const float *u, const float *v, const uint32_t *index,
                            const int32_t *bounce, uint32_t seed, float *out_o, float *out_d, float *weight,
                            float *emissive, int32_t *valid) {
  using namespace nbctx;
  if (!c->bvh_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  if (n == 0) return NOVA_B200_SUCCESS;
  if (!o || !d || !prim || !t || !u || !v || !index || !bounce || !out_o || !out_d || !weight || !emissive || !valid)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  cudaSetDevice(c->device);
  k_scatter_api<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(c->scene, n, o, d, prim, t, u, v, index, bounce,
                                                                     seed, out_o, out_d, weight, emissive, valid);
  NB_CUDA(c, cudaGetLastError(), "k_scatter_api");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "scatter");
  return NOVA_B200_SUCCESS;
}

nova_b200_status nb_sobol(nova_b200_ctx *c, uint64_t n, const uint32_t *idx, const uint32_t *dim, uint32_t seed,
                          float *out) {
  using namespace nbctx;
  if (n == 0) return NOVA_B200_SUCCESS;
  if (!idx || !dim || !out) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  cudaSetDevice(c->device);
  k_sobol_api<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_sobol, n, idx, dim, seed, out);
  NB_CUDA(c, cudaGetLastError(), "k_sobol_api");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "sobol");
  return NOVA_B200_SUCCESS;
}
