/* Wavefront path tracer: the reference's PathIntegrator::Li (integrator/Integrator.cpp:60-99) as
 * four sm_100a kernels over a path queue in HBM.
 *
 *   k_raygen   camera rays for new paths (Integrator.h:66-85 with the OptiX raygen's sample index
 *              (x * H + y) * spp + s, integrator_optix.cu:43; Sobol dimensions 0 and 1 jitter NDC)
 *   k_trace    closest hit per queued ray (traverse.cuh); a miss finishes its path with the
 *              environment lookup, hits go to a compact hit list
 *   k_shade    per hit: principled scatter (Sobol dimensions 2 + 4b .. 5 + 4b at
 *              bounce b), throughput update, spawned ray appended to the next queue with
 *              warp-aggregated atomics; after the last allowed scatter the spawned direction looks
 *              up the environment directly (the reference traces that ray but discards the hit,
 *              Integrator.cpp:94-98)
 *   k_resolve  per pixel, adds the per-path radiance of this call's samples to the running sum in
 *              sample order and writes sum / samples (writeFramebuffer, api/engine.cpp:351-363)
 *
 * The recursive estimator e_0 + c_0 (e_1 + c_1 (... env)) is evaluated forward as
 * sum_k beta_k e_k + beta_K env with beta_k = c_0 ... c_{k-1}; a path whose result is not finite
 * contributes 0 (DENAN, Integrator.cpp:92).  Path state: origin + path id, direction + bounce,
 * throughput (3 x 16 B); hits 16 B + 4 B slot; per-path radiance 16 B, written once.
 */
#include <algorithm>
#include <cfloat>

#include "context.cuh"
#include "shading.cuh"
#include "traverse.cuh"

namespace {

using namespace nb;

constexpr uint32_t kQueueCap = 1u << 22;
constexpr size_t kRadianceCapBytes = 4ull << 30;
constexpr unsigned kRRDimBase = 200; /* Russian roulette decisions use Sobol dimension 200 + bounce */
constexpr int kMaxDepth = 48;        /* 2 + 4 (depth + 1) Sobol dimensions must stay below 200 */

struct RenderParams {
  int32_t W, H;
  uint32_t NP;       /* pixels */
  uint32_t count;    /* samples traced by this chunk */
  uint32_t begin;    /* first sample of this chunk */
  uint32_t spp_total;
  int32_t max_depth;
  uint32_t seed;
  int32_t rr_start;
  float inv_P[16], inv_V[16];
};

struct Queue {
  float4 *o, *d, *beta;
};

__device__ __forceinline__ uint32_t sample_index(const RenderParams &rp, uint32_t p) {
  const uint32_t s_local = p / rp.NP, pix = p - s_local * rp.NP;
  const uint32_t y = pix / (uint32_t)rp.W, x = pix - y * (uint32_t)rp.W;
  return ((uint32_t)x * (uint32_t)rp.H + y) * rp.spp_total + (rp.begin + s_local);
}

__global__ void __launch_bounds__(256) k_raygen(Queue q, uint32_t off, uint64_t first, uint32_t n_new, RenderParams rp,
                                                DevScene sc, float4 *L) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_new) return;
  const uint32_t p = (uint32_t)(first + i);
  const uint32_t s_local = p / rp.NP, pix = p - s_local * rp.NP;
  const int y = (int)(pix / (uint32_t)rp.W), x = (int)(pix - (uint32_t)y * (uint32_t)rp.W);
  const uint32_t index = ((uint32_t)x * (uint32_t)rp.H + (uint32_t)y) * rp.spp_total + (rp.begin + s_local);
  const float r0 = sobol_sample(sc.sobol_dv, index, 0, rp.seed);
  const float r1 = sobol_sample(sc.sobol_dv, index, 1, rp.seed);
  const float dx = r0 * 0.0005f, dy = r1 * 0.0005f; /* RAND_DX / RAND_DY, Integrator.h:54-55 */
  const int ys = rp.H - y;                          /* screen row, Integrator.h:84 */
  const float ndc_x = (float)(2 * x - rp.W) / (float)rp.W;
  const float ndc_y = (float)(rp.H - 2 * ys) / (float)rp.H;
  const float nx = ndc_x + dx, ny = ndc_y + dy;
  const M4 iP = m4_load(rp.inv_P), iV = m4_load(rp.inv_V);
  V4 o = mul(iP, V4{nx, ny, -1.f, 1.f});
  o = o / o.w;
  o = mul(iV, V4{o.x, o.y, o.z, 1.f});
  V4 d = mul(iP, V4{nx, ny, -1.f, 0.f});
  d = normalize(mul(iV, V4{d.x, d.y, -1.f, 0.f}));
  q.o[off + i] = make_float4(o.x, o.y, o.z, __uint_as_float(p));
  q.d[off + i] = make_float4(d.x, d.y, d.z, __int_as_float(0));
  q.beta[off + i] = make_float4(1.f, 1.f, 1.f, 0.f);
  if (sc.has_emissive) L[p] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__device__ __forceinline__ float4 finite_or_zero(V3 L, float alpha) {
  if (!finite3(L)) return make_float4(0.f, 0.f, 0.f, 0.f);
  return make_float4(L.x, L.y, L.z, alpha);
}

/* Writes a finished path's radiance (adds the emission gathered so far when the scene has any). */
__device__ __forceinline__ void finish_path(const DevScene &sc, float4 *L, uint32_t p, float4 result) {
  if (sc.has_emissive) {
    const float4 acc = L[p];
    float4 r = make_float4(acc.x + result.x, acc.y + result.y, acc.z + result.z, result.w);
    if (!isfinite(r.x) || !isfinite(r.y) || !isfinite(r.z)) r = make_float4(0.f, 0.f, 0.f, 0.f);
    L[p] = r;
  } else {
    L[p] = result;
  }
}

/* Closest hit of every queued ray.  A miss finishes its path here (environment lookup,
 * Integrator.cpp:94-98); hits are appended to a compact hit list (warp-aggregated atomics) so
 * the shading kernel only runs on rays that hit. */
template <int WIDTH>
__global__ void __launch_bounds__(128) k_trace(Queue q, uint32_t n, float4 *hits, uint32_t *hit_slot,
                                               unsigned *hit_count, float4 *L, DevScene sc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool is_hit = false;
  TraceResult r{-1, 0.f, 0.f, 0.f};
  if (i < n) {
    const float4 o = q.o[i], d = q.d[i];
    r = trace_closest_w<WIDTH>(sc, V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z});
    if (r.prim < 0) {
      const float4 b4 = q.beta[i];
      const V4 e = env_sample(sc, V3{d.x, d.y, d.z});
      finish_path(sc, L, __float_as_uint(o.w),
                  finite_or_zero(V3{b4.x, b4.y, b4.z} * V3{e.x, e.y, e.z}, (float)__float_as_int(d.w) + e.w));
    } else {
      is_hit = true;
    }
  }
  const unsigned lane = threadIdx.x & 31u;
  const unsigned m = __ballot_sync(0xffffffffu, is_hit);
  unsigned base = 0;
  if (m) {
    if (lane == (unsigned)(__ffs(m) - 1)) base = atomicAdd(hit_count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  }
  if (is_hit) {
    const unsigned slot = base + __popc(m & ((1u << lane) - 1u));
    hits[slot] = make_float4(r.t, r.u, r.v, __int_as_float(r.prim));
    hit_slot[slot] = i;
  }
}

__global__ void __launch_bounds__(128) k_shade(Queue in, const float4 *hits, const uint32_t *hit_slot,
                                               const unsigned *hit_count, Queue out, unsigned *out_count, float4 *L,
                                               RenderParams rp, DevScene sc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < *hit_count;
  bool enq = false;
  float4 no{}, nd{}, nbeta{};
  if (live) {
    const uint32_t slot_in = hit_slot[i];
    const float4 o4 = in.o[slot_in], d4 = in.d[slot_in], b4 = in.beta[slot_in], h = hits[i];
    const uint32_t p = __float_as_uint(o4.w);
    const int bounce = __float_as_int(d4.w);
    const uint32_t index = sample_index(rp, p);
    const V3 ro{o4.x, o4.y, o4.z}, rd{d4.x, d4.y, d4.z};
    V3 beta{b4.x, b4.y, b4.z};
    const int prim = __float_as_int(h.w);
    bool done = false;
    float4 result = make_float4(0.f, 0.f, 0.f, 0.f);
    {
      const uint32_t inst = __ldg(sc.prim_inst + prim);
      const DevInstance &I = sc.instances[inst];
      const HitRecord hr = make_record(sc, ro, rd, I, (uint32_t)prim - I.prim_offset, h.x, h.y, h.z);
      const ScatterResult sr = scatter(sc, rd, hr, sc.materials[I.material], index, 2u + 4u * (unsigned)bounce, rp.seed);
      if (sc.has_emissive && any_nonzero(sr.emissive)) {
        const V3 em = beta * sr.emissive;
        float4 acc = L[p];
        L[p] = make_float4(acc.x + em.x, acc.y + em.y, acc.z + em.z, acc.w);
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
            result = finite_or_zero(beta * V3{e.x, e.y, e.z}, (float)bounce + 1.f + e.w);
            done = true;
          } else {
            enq = true;
            no = make_float4(no3.x, no3.y, no3.z, o4.w);
            nd = make_float4(nd3.x, nd3.y, nd3.z, __int_as_float(bounce + 1));
            nbeta = make_float4(beta.x, beta.y, beta.z, 0.f);
          }
        }
      }
    }
    if (done) finish_path(sc, L, p, result);
  }
  const unsigned lane = threadIdx.x & 31u;
  const unsigned m = __ballot_sync(0xffffffffu, enq);
  unsigned base = 0;
  if (m) {
    if (lane == (unsigned)(__ffs(m) - 1)) base = atomicAdd(out_count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  }
  if (enq) {
    const unsigned slot = base + __popc(m & ((1u << lane) - 1u));
    out.o[slot] = no;
    out.d[slot] = nd;
    out.beta[slot] = nbeta;
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

__global__ void k_sobol_api(const uint32_t *dv, uint64_t n, const uint32_t *idx, const uint32_t *dim, uint32_t seed,
                            float *out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t dm = dim[i];
  out[i] = dm < (uint32_t)kSobolDims ? sobol_sample(dv, idx[i], dm, seed) : __int_as_float(0x7fc00000);
}

nova_b200_status ensure_buffers(nova_b200_ctx *c, uint32_t cap, size_t radiance, int W, int H) {
  if (c->queue_cap < cap) {
    cudaFree(c->d_queue);
    c->d_queue = nullptr;
    c->queue_cap = 0;
    c->queue_bytes = 0;
    const size_t bytes = (size_t)cap * (16 * 7 + 4);
    NB_CUDA(c, cudaMalloc(&c->d_queue, bytes), "cudaMalloc(queue)");
    c->queue_cap = cap;
    c->queue_bytes = bytes;
  }
  if (c->radiance_cap < radiance) {
    cudaFree(c->d_radiance);
    c->d_radiance = nullptr;
    c->radiance_cap = 0;
    NB_CUDA(c, cudaMalloc(&c->d_radiance, radiance * sizeof(float4)), "cudaMalloc(radiance)");
    c->radiance_cap = radiance;
  }
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

}  // namespace

nova_b200_status nb_render(nova_b200_ctx *c, const nova_b200_frame *f, float *film_host, float *film_device,
                           nova_b200_render_stats *stats) {
  using namespace nbctx;
  if (!f) return fail(c, NOVA_B200_INVALID_ARGUMENT, "frame is null%s");
  if (!c->bvh_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  if (f->width <= 0 || f->height <= 0 || f->spp_total <= 0 || f->sample_begin < 0 || f->sample_count <= 0 ||
      f->sample_begin + f->sample_count > f->spp_total)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid frame size or sample range%s");
  if (f->max_depth < 0 || f->max_depth > kMaxDepth)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "max_depth must be in 0..48 (Sobol dimensions)%s");
  const uint64_t NP = (uint64_t)f->width * f->height;
  if (NP * (uint64_t)f->spp_total >= (1ull << 32))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "width * height * spp must stay below 2^32 (Sobol index)%s");
  cudaSetDevice(c->device);
  const size_t cap_entries = kRadianceCapBytes / sizeof(float4);
  const uint32_t chunk_samples = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(f->sample_count, cap_entries / NP));
  const uint64_t max_paths = NP * chunk_samples;
  const uint32_t cap = (uint32_t)std::min<uint64_t>(kQueueCap, max_paths);
  nova_b200_status st = ensure_buffers(c, cap, max_paths, f->width, f->height);
  if (st != NOVA_B200_SUCCESS) return st;
  if (f->reset) {
    NB_CUDA(c, cudaMemsetAsync(c->d_film_acc, 0, NP * sizeof(float4), c->stream), "memset(film)");
    c->film_samples = 0;
  }
  RenderParams rp;
  rp.W = f->width, rp.H = f->height, rp.NP = (uint32_t)NP;
  rp.spp_total = (uint32_t)f->spp_total;
  rp.max_depth = f->max_depth;
  rp.seed = f->seed;
  rp.rr_start = f->rr_start;
  std::copy(f->inv_P, f->inv_P + 16, rp.inv_P);
  std::copy(f->inv_V, f->inv_V + 16, rp.inv_V);
  float4 *base = static_cast<float4 *>(c->d_queue);
  Queue qa{base, base + cap, base + 2 * (size_t)cap}, qb{base + 3 * (size_t)cap, base + 4 * (size_t)cap,
                                                         base + 5 * (size_t)cap};
  float4 *hits = base + 6 * (size_t)cap;
  uint32_t *hit_slot = reinterpret_cast<uint32_t *>(base + 7 * (size_t)cap);
  nova_b200_render_stats s{};
  float t_trace = 0.f, t_shade = 0.f;
  NB_CUDA(c, cudaEventRecord(c->ev_begin, c->stream), "event");
  for (uint32_t done_s = 0; done_s < (uint32_t)f->sample_count; done_s += chunk_samples) {
    const uint32_t cs = std::min<uint32_t>(chunk_samples, (uint32_t)f->sample_count - done_s);
    rp.begin = (uint32_t)f->sample_begin + done_s;
    rp.count = cs;
    const uint64_t paths = NP * cs;
    uint64_t next = 0;
    uint32_t n_active = 0;
    while (next < paths || n_active > 0) {
      const uint32_t n_new = (uint32_t)std::min<uint64_t>(cap - n_active, paths - next);
      if (n_new) {
        k_raygen<<<(n_new + 255) / 256, 256, 0, c->stream>>>(qa, n_active, next, n_new, rp, c->scene, c->d_radiance);
        s.kernels++;
      }
      const uint32_t n = n_active + n_new;
      next += n_new;
      s.traced += n;
      s.segments += n;
      NB_CUDA(c, cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream), "memset");
      NB_CUDA(c, cudaEventRecord(c->ev_a, c->stream), "event");
      if (c->scene.width == 8)
        k_trace<8><<<(n + 127) / 128, 128, 0, c->stream>>>(qa, n, hits, hit_slot, c->d_counters + 1, c->d_radiance,
                                                          c->scene);
      else
        k_trace<2><<<(n + 127) / 128, 128, 0, c->stream>>>(qa, n, hits, hit_slot, c->d_counters + 1, c->d_radiance,
                                                          c->scene);
      NB_CUDA(c, cudaEventRecord(c->ev_b, c->stream), "event");
      k_shade<<<(n + 127) / 128, 128, 0, c->stream>>>(qa, hits, hit_slot, c->d_counters + 1, qb, c->d_counters,
                                                       c->d_radiance, rp, c->scene);
      NB_CUDA(c, cudaEventRecord(c->ev_end, c->stream), "event");
      s.kernels += 2;
      NB_CUDA(c, cudaMemcpyAsync(c->h_counters, c->d_counters, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream),
              "readback");
      NB_CUDA(c, cudaStreamSynchronize(c->stream), "wave");
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, c->ev_a, c->ev_b);
      cudaEventElapsedTime(&b, c->ev_b, c->ev_end);
      t_trace += a;
      t_shade += b;
      n_active = c->h_counters[0];
      std::swap(qa, qb);
      s.waves++;
    }
    c->film_samples += cs;
    k_resolve<<<(uint32_t)((NP + 255) / 256), 256, 0, c->stream>>>(c->d_radiance, (uint32_t)NP, cs, c->d_film_acc,
                                                                   (float)c->film_samples, c->d_film_out, f->width,
                                                                   f->height, f->vertical_invert);
    s.kernels++;
    s.paths += paths;
  }
  NB_CUDA(c, cudaGetLastError(), "render kernels");
  NB_CUDA(c, cudaEventRecord(c->ev_end, c->stream), "event");
  if (film_device)
    NB_CUDA(c, cudaMemcpyAsync(film_device, c->d_film_out, NP * 4 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream),
            "copy film");
  if (film_host)
    NB_CUDA(c, cudaMemcpyAsync(film_host, c->d_film_out, NP * 4 * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
            "copy film");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "render");
  float total = 0.f;
  cudaEventElapsedTime(&total, c->ev_begin, c->ev_end);
  s.device_ms = total;
  s.trace_ms = t_trace;
  s.shade_ms = t_shade;
  if (stats) *stats = s;
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
