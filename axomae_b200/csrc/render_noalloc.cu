/* Allocation-free render: nova_b200_render_noalloc.
 *
 * Some callers cannot call cudaMalloc during a frame: a host loop whose device memory is entirely
 * reserved by another allocator (for example a framework's caching allocator that has claimed the
 * GPU), or a real-time viewport that must not risk a device-wide synchronisation or an allocation
 * failure in the middle of a frame.  This entry point renders with no allocation at all: its only
 * scratch is the file-scope device array below, kNoAllocScratchBytes = 32 MiB.  The caller passes
 * the output film (device memory); the scene and BVH are the ones the context already holds.
 *
 * The scratch holds the radiance of one chunk of paths (pixels x samples, at most
 * kNoAllocPaths = 2 Mi paths): one thread traces one path through every bounce, then a second
 * kernel adds each pixel's samples in sample order and writes the mean.  Every path writes its own
 * scratch slot before the resolve reads it, so nothing has to be cleared between calls; the array
 * keeps the last call's contents.  All calls share the one array, so calls that overlap on the GPU
 * (two contexts, or two streams, rendering at the same time) race on it.
 *
 * Set-up happens in nova_b200_create, on the context's device with that device current
 * (nb_noalloc_prepare below): it makes the CUDA runtime load this file's module (under lazy module
 * loading the 32 MiB array is only allocated then), looks up the array's device address with
 * cudaGetSymbolAddress (in host code the array's name is only a stand-in, not a device address),
 * caches it for that device, and launches the path kernel once over no paths so that the driver
 * reserves the kernel's per-thread local memory (its traversal stack) at that point too.  After
 * that a nova_b200_render_noalloc call launches two kernels and allocates nothing.
 *
 * The per-path arithmetic is the same sequence of device functions as the wavefront kernels
 * (integrator.cu), so the film equals nova_b200_render's for the same sample range.
 */
#include <mutex>

#include "context.cuh"
#include "shading.cuh"
#include "traverse.cuh"

namespace {

using namespace nb;

constexpr size_t kNoAllocScratchBytes = 32ull << 20;
constexpr uint32_t kNoAllocPaths = (uint32_t)(kNoAllocScratchBytes / sizeof(float4));
constexpr int kMaxDevices = 64;
constexpr unsigned kRRDimBase = 200;
constexpr int kMaxDepth = 48;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
float4 *g_scratch_ptr[kMaxDevices] = {};

struct Params {
  int32_t W, H;
  uint32_t first_pixel, n_pix, count, begin, spp_total;
  int32_t max_depth;
  uint32_t seed;
  int32_t rr_start;
  float inv_P[16], inv_V[16];
};

__device__ __forceinline__ float4 finite_or_zero(V3 L, float alpha) {
  if (!finite3(L)) return make_float4(0.f, 0.f, 0.f, 0.f);
  return make_float4(L.x, L.y, L.z, alpha);
}

/* One path per thread, bounce loop in registers (same steps as k_raygen / k_trace / k_shade). */
__global__ void __launch_bounds__(128) k_path_noalloc(DevScene sc, Params rp, float4 *radiance) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rp.n_pix * rp.count) return;
  const uint32_t s_local = i / rp.n_pix, pix = rp.first_pixel + (i - s_local * rp.n_pix);
  const int y = (int)(pix / (uint32_t)rp.W), x = (int)(pix - (uint32_t)y * (uint32_t)rp.W);
  const uint32_t index = ((uint32_t)x * (uint32_t)rp.H + (uint32_t)y) * rp.spp_total + (rp.begin + s_local);
  const float r0 = sobol_sample(sc.sobol_dv, index, 0, rp.seed);
  const float r1 = sobol_sample(sc.sobol_dv, index, 1, rp.seed);
  const float dx = r0 * 0.0005f, dy = r1 * 0.0005f;
  const int ys = rp.H - y;
  const float ndc_x = (float)(2 * x - rp.W) / (float)rp.W;
  const float ndc_y = (float)(rp.H - 2 * ys) / (float)rp.H;
  const float nx = ndc_x + dx, ny = ndc_y + dy;
  const M4 iP = m4_load(rp.inv_P), iV = m4_load(rp.inv_V);
  V4 o4 = mul(iP, V4{nx, ny, -1.f, 1.f});
  o4 = o4 / o4.w;
  o4 = mul(iV, V4{o4.x, o4.y, o4.z, 1.f});
  V4 d4 = mul(iP, V4{nx, ny, -1.f, 0.f});
  d4 = normalize(mul(iV, V4{d4.x, d4.y, -1.f, 0.f}));
  V3 ro{o4.x, o4.y, o4.z}, rd{d4.x, d4.y, d4.z};
  V3 beta{1.f, 1.f, 1.f};
  float4 lacc = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 result = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int bounce = 0;; bounce++) {
    const TraceResult h = trace_closest(sc, ro, rd);
    if (h.prim < 0) {
      const V4 e = env_sample(sc, rd);
      result = finite_or_zero(beta * V3{e.x, e.y, e.z}, (float)bounce + e.w);
      break;
    }
    const uint32_t inst = __ldg(sc.prim_inst + h.prim);
    const DevInstance &I = sc.instances[inst];
    const HitRecord hr = make_record(sc, ro, rd, I, (uint32_t)h.prim - I.prim_offset, h.t, h.u, h.v);
    const ScatterResult sr = scatter(sc, rd, hr, sc.materials[I.material], index, 2u + 4u * (unsigned)bounce, rp.seed,
                                     (uint32_t)h.prim, I.material);
    if (sr.valid && sc.has_emissive && any_nonzero(sr.emissive)) { /* failed scatter: black */
      const V3 em = beta * sr.emissive;
      lacc = make_float4(lacc.x + em.x, lacc.y + em.y, lacc.z + em.z, lacc.w);
    }
    if (!sr.valid) {
      result = make_float4(0.f, 0.f, 0.f, (float)bounce);
      break;
    }
    V3 c = sr.weight;
    if (rp.rr_start >= 0 && bounce >= rp.rr_start) {
      const V3 nbt = beta * c;
      const float q = fmin_std(1.f, fmax_std(0.05f, fmax_std(nbt.x, fmax_std(nbt.y, nbt.z))));
      const float urr = sobol_sample(sc.sobol_dv, index, kRRDimBase + (unsigned)bounce, rp.seed);
      if (!(urr < q)) {
        result = make_float4(0.f, 0.f, 0.f, (float)bounce + 1.f);
        break;
      }
      c = c / q;
    }
    beta = beta * c;
    const float eps = 1e-3f;
    const V3 nd3 = normalize(sr.wi);
    const V3 no3 = hr.position + hr.ng * (eps + eps * fsign(dot(hr.ng, sr.wi)));
    if (bounce + 1 > rp.max_depth) {
      const V4 e = env_sample(sc, nd3);
      result = finite_or_zero(beta * V3{e.x, e.y, e.z}, (float)bounce + 1.f + e.w);
      break;
    }
    ro = no3;
    rd = nd3;
  }
  float4 out = result;
  if (sc.has_emissive) {
    out = make_float4(lacc.x + result.x, lacc.y + result.y, lacc.z + result.z, result.w);
    if (!isfinite(out.x) || !isfinite(out.y) || !isfinite(out.z)) out = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  radiance[i] = out;
}

/* Per pixel: 0 + L_0 + L_1 + ... in sample order, divided by the sample count. */
__global__ void k_resolve_noalloc(const float4 *radiance, Params rp, float *film, int vinv) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= rp.n_pix) return;
  float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint32_t s = 0; s < rp.count; s++) {
    const float4 l = radiance[(size_t)s * rp.n_pix + k];
    a.x += l.x, a.y += l.y, a.z += l.z, a.w += l.w;
  }
  const uint32_t pix = rp.first_pixel + k;
  const uint32_t y = pix / (uint32_t)rp.W, x = pix - y * (uint32_t)rp.W;
  const uint32_t row = vinv ? (uint32_t)rp.H - 1u - y : y;
  const float denom = (float)rp.count;
  reinterpret_cast<float4 *>(film)[(size_t)row * rp.W + x] =
      make_float4(a.x / denom, a.y / denom, a.z / denom, a.w / denom);
}

/* The scratch array's device address on the current device, looked up once per device. */
nova_b200_status scratch_for_device(nova_b200_ctx *c, float4 **out) {
  if (c->device < 0 || c->device >= kMaxDevices) return nbctx::fail(c, NOVA_B200_INVALID_ARGUMENT, "device id%s");
  int current = -1;
  NB_CUDA(c, cudaGetDevice(&current), "cudaGetDevice");
  if (current != c->device) return nbctx::fail(c, NOVA_B200_RENDERER_EXCEPTION, "no-alloc set-up on the wrong device%s");
  std::lock_guard<std::mutex> lk(g_setup_mutex);
  if (!g_scratch_ptr[c->device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return nbctx::cuda_fail(c, e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_ptr[c->device] = static_cast<float4 *>(p);
  }
  *out = g_scratch_ptr[c->device];
  return NOVA_B200_SUCCESS;
}

/* Makes the caller's current device the context's for one call and restores it on return. */
struct DeviceScope {
  int previous = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
    status = cudaSetDevice(device);
  }
  ~DeviceScope() {
    if (previous >= 0) cudaSetDevice(previous);
  }
};

}  // namespace

/* Called by nova_b200_create with the context's device current: module load, scratch address and
 * the driver's local-memory reservation for the path kernel all happen here, not in a render. */
nova_b200_status nb_noalloc_prepare(nova_b200_ctx *c) {
  float4 *scratch = nullptr;
  nova_b200_status st = scratch_for_device(c, &scratch);
  if (st != NOVA_B200_SUCCESS) return st;
  cudaFuncAttributes attr;
  NB_CUDA(c, cudaFuncGetAttributes(&attr, k_path_noalloc), "no-alloc path kernel");
  NB_CUDA(c, cudaFuncGetAttributes(&attr, k_resolve_noalloc), "no-alloc resolve kernel");
  Params none{};  /* n_pix * count = 0: every thread returns before reading the scene */
  k_path_noalloc<<<1, 128, 0, c->stream>>>(c->scene, none, scratch);
  NB_CUDA(c, cudaGetLastError(), "no-alloc set-up launch");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "no-alloc set-up");
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_render_noalloc(nova_b200_ctx *c, const nova_b200_frame *f, float *film_device) {
  using namespace nbctx;
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (!f || !film_device) return fail(c, NOVA_B200_INVALID_ARGUMENT, "frame and film_device are required%s");
  if (!c->bvh_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  if (f->width <= 0 || f->height <= 0 || f->spp_total <= 0 || f->sample_begin < 0 || f->sample_count <= 0 ||
      f->sample_begin + f->sample_count > f->spp_total)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid frame size or sample range%s");
  if (f->max_depth < 0 || f->max_depth > kMaxDepth)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "max_depth must be in 0..48 (Sobol dimensions)%s");
  const uint64_t NP = (uint64_t)f->width * f->height;
  if (NP * (uint64_t)f->spp_total >= (1ull << 32))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "width * height * spp must stay below 2^32 (Sobol index)%s");
  if ((uint64_t)f->sample_count > kNoAllocPaths)
    return fail(c, NOVA_B200_INVALID_ARGUMENT,
                "sample_count exceeds the no-alloc scratch limit of 2097152 paths per pixel chunk%s");
  DeviceScope on_device(c->device);
  NB_CUDA(c, on_device.status, "cudaSetDevice");
  float4 *scratch = nullptr;
  nova_b200_status st = scratch_for_device(c, &scratch);
  if (st != NOVA_B200_SUCCESS) return st;
  Params rp;
  rp.W = f->width, rp.H = f->height;
  rp.count = (uint32_t)f->sample_count;
  rp.begin = (uint32_t)f->sample_begin;
  rp.spp_total = (uint32_t)f->spp_total;
  rp.max_depth = f->max_depth;
  rp.seed = f->seed;
  rp.rr_start = f->rr_start;
  for (int k = 0; k < 16; k++) rp.inv_P[k] = f->inv_P[k], rp.inv_V[k] = f->inv_V[k];
  const uint32_t chunk_pixels = (uint32_t)std::min<uint64_t>(NP, kNoAllocPaths / rp.count);
  for (uint64_t first = 0; first < NP; first += chunk_pixels) {
    rp.first_pixel = (uint32_t)first;
    rp.n_pix = (uint32_t)std::min<uint64_t>(chunk_pixels, NP - first);
    const uint32_t paths = rp.n_pix * rp.count;
    k_path_noalloc<<<(paths + 127) / 128, 128, 0, c->stream>>>(c->scene, rp, scratch);
    k_resolve_noalloc<<<(rp.n_pix + 255) / 256, 256, 0, c->stream>>>(scratch, rp, film_device, f->vertical_invert);
  }
  NB_CUDA(c, cudaGetLastError(), "render_noalloc kernels");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "render_noalloc");
  return NOVA_B200_SUCCESS;
}
