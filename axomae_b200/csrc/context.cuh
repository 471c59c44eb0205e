/* The C-ABI context: owns the device, stream, scene buffers, BVH and render buffers. */
#pragma once
#include <atomic>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/nova_b200.h"
#include "device_scene.cuh"

struct nova_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr; /* batch renders: films of finished frames go out on it */
  cudaEvent_t ev_copy = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr, ev_a = nullptr, ev_b = nullptr;
  std::string error;
  std::atomic<bool> cancel{false}; /* set by nova_b200_cancel from any thread, read by the wave loop */

  /* tables (allocated once) */
  uint32_t *d_sobol = nullptr;
  float *d_acos = nullptr;

  /* scene */
  void *d_arena = nullptr;      /* every scene buffer (textures, meshes, tables) in one pool allocation */
  void *h_stage = nullptr;      /* pinned upload staging for small pieces */
  size_t h_stage_bytes = 0;
  nb::DevScene scene{};
  std::vector<nb::DevInstance> h_instances;
  std::vector<nb::DevMesh> h_meshes;      /* device pointers, host copy of the mesh table */
  uint32_t *d_blas_root = nullptr;        /* two-level BVH: per mesh, its bottom-level root node */
  uint32_t *d_valid = nullptr;   /* global primitive ids that can be hit, ascending (device) */
  uint32_t n_valid = 0;
  uint64_t n_prims = 0;
  uint32_t n_materials = 0;
  bool scene_ready = false;
  bool bvh_ready = false;
  uint32_t n_nodes = 0, n_leaves = 0;
  int bvh_depth = 0;
  int bvh_width = 0;
  double bvh_ms = 0.0;
  uint64_t scene_bytes = 0;

  /* BVH buffers */
  float4 *d_nodes = nullptr;
  float4 *d_tris = nullptr;

  /* render buffers */
  float4 *d_film_acc = nullptr; /* running sum, row-major */
  int film_w = 0, film_h = 0;
  uint64_t film_samples = 0;
  void *d_queue = nullptr;
  size_t queue_bytes = 0;
  uint32_t queue_cap = 0;
  float4 *d_radiance = nullptr;
  size_t radiance_cap = 0; /* float4 entries */
  unsigned *d_counters = nullptr;
  unsigned *h_counters = nullptr; /* pinned */
  float *d_film_out = nullptr;
  size_t film_out_cap = 0;

  /* device-driven wave loop (integrator.cu) */
  void *d_wave = nullptr, *h_wave = nullptr; /* wave counters: device copy; pinned read-back slots 0, 1 + upload slot 2 */
  cudaEvent_t ev_wave[24] = {};              /* per pipeline slot: start, trace end, shade end of each wave */
  cudaEvent_t ev_done[2] = {};               /* per pipeline slot: the slot's counters are in host memory */
  cudaGraphExec_t graph_exec[2] = {};        /* batch chunks: the wave group of each pipeline slot */
  std::vector<char> graph_key;               /* job table, launch shape and width of the graphs */
  nova_b200_tuning tuning{};                 /* launch parameters (zeros: defaults) */

  /* persistent wavefront (tuning.trace_mode 3): its grid barrier, and the cancel flag in mapped host
   * memory that its wave-end step reads */
  void *d_persist = nullptr;
  volatile int *h_cancel_map = nullptr;

  /* adjoint: the replay queues' extra path state (remaining radiance, image adjoint) */
  float4 *d_adj = nullptr;
  uint32_t adj_cap = 0;
  /* the radiance buffer holds every path of this frame (last single render, one pass) */
  bool primal_valid = false;
  nova_b200_frame primal_frame{};
  const float *primal_albedo = nullptr, *primal_rough = nullptr;
};

namespace nbctx {

inline nova_b200_status fail(nova_b200_ctx *c, nova_b200_status st, const char *fmt, const char *detail = "") {
  if (c) {
    char buf[1024];
    std::snprintf(buf, sizeof(buf), fmt, detail);
    c->error = buf;
  }
  return st;
}

inline nova_b200_status cuda_fail(nova_b200_ctx *c, cudaError_t e, const char *where) {
  char buf[1024];
  std::snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
  if (c) c->error = buf;
  return e == cudaErrorMemoryAllocation ? NOVA_B200_OUT_OF_MEMORY : NOVA_B200_RENDERER_EXCEPTION;
}

}  // namespace nbctx

#define NB_CUDA(ctx, call, where)                                       \
  do {                                                                  \
    cudaError_t nb_e_ = (call);                                         \
    if (nb_e_ != cudaSuccess) return nbctx::cuda_fail((ctx), nb_e_, where); \
  } while (0)

/* Defined in integrator.cu / bake.cu, called by the C-ABI entry points in context.cu. */
nova_b200_status nb_render(nova_b200_ctx *c, const nova_b200_frame *f, float *film_host, float *film_device,
                           nova_b200_render_stats *stats);
nova_b200_status nb_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_frame *frames, uint32_t n,
                                 float *const *films_host, float *const *films_device, nova_b200_render_stats *stats);
nova_b200_status nb_upload_build_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                              const nova_b200_frame *frames, uint32_t n,
                                              const nova_b200_bvh_options *opts, float *const *films_host,
                                              float *const *films_device, nova_b200_render_stats *stats);
nova_b200_status nb_backward(nova_b200_ctx *c, const nova_b200_frame *f, const float *d_image, float *grad_albedo,
                             float *grad_roughness, uint32_t flags, nova_b200_render_stats *stats);
nova_b200_status nb_trace(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, int32_t *prim, float *t,
                          float *u, float *v);
nova_b200_status nb_scatter(nova_b200_ctx *c, uint64_t n, const float *o, const float *d, const int32_t *prim,
                            const float *t, const float *u, const float *v, const uint32_t *index,
                            const int32_t *bounce, uint32_t seed, float *out_o, float *out_d, float *weight,
                            float *emissive, int32_t *valid);
nova_b200_status nb_sobol(nova_b200_ctx *c, uint64_t n, const uint32_t *idx, const uint32_t *dim, uint32_t seed,
                          float *out);
nova_b200_status nb_bake_texunit(nova_b200_ctx *c, const float *src, int32_t sw, int32_t sh, int32_t ch, int32_t ow,
                                 int32_t oh, int32_t samples, float *out);
nova_b200_status nb_bake(nova_b200_ctx *c, const float *src, int32_t sw, int32_t sh, int32_t ch, int32_t ow,
                         int32_t oh, int32_t samples, float *out);
/* Defined in render_noalloc.cu: loads the no-alloc kernels' module on the context's device, takes
 * the scratch array's address and reserves the path kernel's local memory (called at create). */
nova_b200_status nb_noalloc_prepare(nova_b200_ctx *c);
