/* AOV integrators: nova_b200_render_aov.
 *
 * The reference's three auxiliary integrators (integrator/NormalIntegrator.cpp,
 * DepthIntegrator.cpp, EmissiveIntegrator.cpp, dispatched by Integrator.cpp:18-48) trace one camera
 * ray per pixel without the sub-pixel jitter and write one value per pixel:
 *   normal    the normal-mapped shading normal of the closest hit (mat_rec.normal, set by
 *             PrincipledMaterial::scatter whether or not the BSDF sample succeeds), (n, 1); 0 on a
 *             miss;
 *   depth     with t the closest-hit distance, near / far the camera planes:
 *             z = 1 - (t - near) / (far - near), d = 2 near far / (far + near - z (far - near)) * 2 - 1,
 *             every channel d / far; every channel far on a miss (DepthIntegrator.cpp:41-47);
 *   emissive  the emission of the closest hit's material, (e, 1), when its scatter succeeds; 0 on a
 *             miss or a failed scatter.  The scatter draws its four Sobol dimensions from 0 with the
 *             sample index set to the pixel's film offset (y W + x) * 4 (generateImageOffset,
 *             Integrator.h:38-42), as the reference's sampler.reset(idx) does.
 * One thread per pixel; the film layout is the one nova_b200_render returns.
 */
#include "context.cuh"
#include "shading.cuh"
#include "traverse.cuh"

namespace {

using namespace nb;

struct AovParams {
  int32_t W, H, vinv, kind;
  uint32_t seed;
  float near_plane, far_plane;
  float inv_P[16], inv_V[16];
};

__global__ void k_aov(DevScene sc, const AovParams p, float4 *out) {
  const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= (uint32_t)p.W * (uint32_t)p.H) return;
  const int y = (int)(pix / (uint32_t)p.W), x = (int)(pix - (uint32_t)y * (uint32_t)p.W);
  const int ys = p.H - y; /* screen row, as the path integrator */
  const float nx = (float)(2 * x - p.W) / (float)p.W;
  const float ny = (float)(p.H - 2 * ys) / (float)p.H;
  const M4 iP = m4_load(p.inv_P), iV = m4_load(p.inv_V);
  V4 o = mul(iP, V4{nx, ny, -1.f, 1.f});
  o = o / o.w;
  o = mul(iV, V4{o.x, o.y, o.z, 1.f});
  V4 d = mul(iP, V4{nx, ny, -1.f, 0.f});
  d = normalize(mul(iV, V4{d.x, d.y, -1.f, 0.f}));
  const V3 ro{o.x, o.y, o.z}, rd{d.x, d.y, d.z};
  const TraceResult h = trace_closest(sc, ro, rd);
  const uint32_t row = p.vinv ? (uint32_t)(p.H - 1 - y) : (uint32_t)y;
  float4 res = make_float4(0.f, 0.f, 0.f, 0.f);
  if (p.kind == NOVA_B200_AOV_DEPTH) {
    const float nr = p.near_plane, fr = p.far_plane;
    if (h.prim < 0) {
      res = make_float4(fr, fr, fr, fr);
    } else {
      float z = 1 - (h.t - nr) / (fr - nr);
      z = (2.0f * nr * fr) / (fr + nr - z * (fr - nr)) * 2.f - 1.f;
      const float v = z / fr;
      res = make_float4(v, v, v, v);
    }
  } else if (h.prim >= 0) {
    const DevInstance &I = sc.instances[__ldg(sc.prim_inst + h.prim)];
    const HitRecord hr = make_record(sc, ro, rd, I, (uint32_t)h.prim - I.prim_offset, h.t, h.u, h.v);
    const DevMaterial &mat = sc.materials[I.material];
    if (p.kind == NOVA_B200_AOV_NORMAL) {
      const V3 ns = shading_normal(sc, hr, mat);
      res = make_float4(ns.x, ns.y, ns.z, 1.f);
    } else {
      const uint32_t index = (row * (uint32_t)p.W + (uint32_t)x) * 4u;
      const ScatterResult sr = scatter(sc, rd, hr, mat, index, 0u, p.seed, (uint32_t)h.prim, I.material);
      if (sr.valid) res = make_float4(sr.emissive.x, sr.emissive.y, sr.emissive.z, 1.f);
    }
  }
  out[(size_t)row * p.W + x] = res;
}

}  // namespace

extern "C" nova_b200_status nova_b200_render_aov(nova_b200_ctx *c, const nova_b200_frame *f, int32_t kind,
                                                 float near_plane, float far_plane, float *film_host,
                                                 float *film_device) {
  using namespace nbctx;
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  if (!f) return fail(c, NOVA_B200_INVALID_ARGUMENT, "frame is null%s");
  if (!c->bvh_ready) return fail(c, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  if (kind != NOVA_B200_AOV_NORMAL && kind != NOVA_B200_AOV_DEPTH && kind != NOVA_B200_AOV_EMISSIVE)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "kind must be NOVA_B200_AOV_NORMAL, _DEPTH or _EMISSIVE%s");
  if (f->width <= 0 || f->height <= 0 || (uint64_t)f->width * f->height >= (1ull << 30))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid frame size%s");
  if (kind == NOVA_B200_AOV_DEPTH && !(far_plane > near_plane))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "far_plane must exceed near_plane%s");
  cudaSetDevice(c->device);
  AovParams p{};
  p.W = f->width, p.H = f->height, p.vinv = f->vertical_invert, p.kind = kind, p.seed = f->seed;
  p.near_plane = near_plane, p.far_plane = far_plane;
  for (int k = 0; k < 16; k++) p.inv_P[k] = f->inv_P[k], p.inv_V[k] = f->inv_V[k];
  const size_t npx = (size_t)f->width * f->height;
  float4 *out = reinterpret_cast<float4 *>(film_device);
  float4 *tmp = nullptr;
  if (!out) {
    NB_CUDA(c, cudaMallocAsync(&tmp, npx * sizeof(float4), c->stream), "cudaMalloc(aov film)");
    out = tmp;
  }
  k_aov<<<(unsigned)((npx + 127) / 128), 128, 0, c->stream>>>(c->scene, p, out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && film_host)
    e = cudaMemcpyAsync(film_host, out, npx * sizeof(float4), cudaMemcpyDeviceToHost, c->stream);
  if (tmp) cudaFreeAsync(tmp, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "render_aov");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "render_aov");
  return NOVA_B200_SUCCESS;
}
