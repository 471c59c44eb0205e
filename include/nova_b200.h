/* nova_b200.h — C ABI of the B200 (sm_100a) implementation of the Nova path-tracing hot path.
 *
 * This is the boundary a Nova render call binds to.  It replaces the reference's GPU backend
 * plug-in point and the render dispatch that drives it (HamilcarR/Axomae, corelib/nova):
 *
 *   DeviceAcceleratorInterface::make / build / cleanup / copyParamsToDevice / getIntersectorObject
 *       aggregate/device_acceleration_interface.h:20-36, factory api/device_accelerator_factory.cpp:9-18
 *   DeviceIntersectorInterface::traverse        aggregate/device_acceleration_interface.h:11-15
 *   Engine::buildScene / buildAcceleration      api_engine.h:68-82, api/engine.cpp:201,235
 *   NvEngineInstance::renderGpu + writeFramebuffer (progressive running-mean film)
 *                                               api/engine.cpp:457-496, :351-363
 *   Engine::getRenderEngineError                api_engine.h:185
 *   TextureOperations<float>::computeDiffuseIrradiance (irradiance bake)
 *                                               sources/processing/TextureProcessing.cpp:10-64,
 *                                               sources/processing/cuda/CubemapProcessing.cu:244-284
 *
 * Conventions: plain C types only; every call returns a status whose values are the reference's
 * nova::ERROR_STATE enumerators (api_common.h:7-27); no exception crosses the ABI.  A context owns
 * all device memory it allocates and one CUDA stream; it is not thread-safe (one caller thread).
 * Scene data is copied to the device by nova_b200_upload_scene, so caller buffers may be released
 * afterwards (the reference keeps non-owning spans; api/geometry.cpp:17-70).
 */
#ifndef NOVA_B200_H
#define NOVA_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: identical numbering to nova::ERROR_STATE (api_common.h:7-27). */
typedef enum {
  NOVA_B200_SUCCESS = 0,
  NOVA_B200_INVALID_ENGINE_STATE = 1,
  NOVA_B200_INVALID_BUFFER_STATE = 2,
  NOVA_B200_INVALID_CHANNEL_DESCRIPTOR = 3,
  NOVA_B200_INVALID_SCENE_TYPE = 4,
  NOVA_B200_INVALID_TRANSFORM_TYPE = 5,
  NOVA_B200_RENDER_BUFFER_NOT_INITIALIZED = 6,
  NOVA_B200_RENDER_OPTIONS_NOT_INITIALIZED = 7,
  NOVA_B200_RENDER_ENGINE_NOT_INITIALIZED = 8,
  NOVA_B200_SCENE_NOT_PROCESSED = 9,
  NOVA_B200_NOT_GPU_BUILD = 10,
  NOVA_B200_OUT_OF_MEMORY = 11,
  NOVA_B200_MULTIPLE_INTEGRATORS_NOT_SUPPORTED = 12,
  NOVA_B200_THREADPOOL_CREATION_ERROR = 13,
  NOVA_B200_THREADPOOL_NOT_INITIALIZED = 14,
  NOVA_B200_INVALID_ARGUMENT = 15,
  NOVA_B200_RENDERER_EXCEPTION = 16
} nova_b200_status;

typedef struct nova_b200_ctx nova_b200_ctx;

/* Triangle mesh in object space: the reference's Object3D spans (internal/geometry/Object3D.h:384-394).
 * positions / normals / tangents / bitangents: 3 floats per vertex; uv: 2; indices: 3 per triangle. */
typedef struct {
  const float *vertices;
  const float *normals;
  const float *tangents;
  const float *bitangents;
  const float *uv;
  const uint32_t *indices;
  uint32_t n_verts;
  uint32_t n_tris;
} nova_b200_mesh;

/* One placed mesh with its transform record transform4x4_t {m, inv, n} (internal/common/math/utils_3D.h:84-96),
 * column-major like glm, and its material (one material per mesh, api/engine.cpp:177-184). */
typedef struct {
  uint32_t mesh;
  uint32_t material;
  float m[16];
  float inv[16];
  float n[9];
} nova_b200_instance;

/* PrincipledMaterial inputs (material/NovaMaterials.h:45-137): u8 texture indices or -1, eta, k. */
typedef struct {
  int32_t albedo;
  int32_t metallic; /* roughness = green, metal = blue (NovaMaterials.h:116-117) */
  int32_t normalmap;
  int32_t emissive;
  float eta[3];
  float k[3];
  float anisotropy;
} nova_b200_material;

/* Texture: exactly one of u8_pixels (32-bit packed 8-bit RGBA/BGRA texels) or f32_pixels. */
typedef struct {
  const uint32_t *u8_pixels;
  const float *f32_pixels;
  int32_t width, height, channels;
  int32_t is_rgba, invert_u, invert_v;
} nova_b200_texture;

typedef struct {
  const nova_b200_mesh *meshes;
  uint32_t n_meshes;
  const nova_b200_instance *instances;
  uint32_t n_instances;
  const nova_b200_material *materials;
  uint32_t n_materials;
  const nova_b200_texture *textures;
  uint32_t n_textures;
  int32_t envmap; /* index of a 4-channel f32 texture (api/engine.cpp:273-290) */
} nova_b200_scene_desc;

/* Acceleration-structure build options. */
typedef struct {
  int32_t max_leaf_size; /* 1..16 (1..4 for width 8); 0 = default (8, or 4 for width 8) */
  int32_t bins;          /* SAH bins per axis, 4..32; 0 = default (16) */
  int32_t width;         /* 2: binary BVH (default, fastest measured); 8: compressed 8-wide BVH; 0 = 2 */
  int32_t small_subtree; /* nodes of at most this many triangles are built whole by one thread block
                            (64..65536; 0 = default 256); a build-speed knob, the tree is the same
                            kind either way */
} nova_b200_bvh_options;

/* One render call.  Samples [sample_begin, sample_begin + sample_count) of every pixel are traced and
 * added to the context's accumulation film; the returned image is the running mean over all samples
 * accumulated since the last reset (writeFramebuffer, api/engine.cpp:351-363).  The sample index of
 * pixel (x, y), sample s is (x * height + y) * spp_total + s (integrator_optix.cu:43). */
typedef struct {
  int32_t width, height;
  int32_t spp_total;    /* samples per pixel of the whole render (index mapping) */
  int32_t sample_begin;
  int32_t sample_count;
  int32_t max_depth;    /* scatter events per path = max_depth + 1 (integrator/Integrator.cpp:71) */
  uint32_t seed;        /* Sobol / Owen scrambling seed */
  int32_t rr_start;     /* Russian roulette from this bounce on; -1 = off (the reference has none) */
  int32_t reset;        /* 1: clear the accumulation film first */
  int32_t vertical_invert;
  float inv_P[16];      /* camera inverse projection / view, column-major (camera/nova_camera.h) */
  float inv_V[16];
} nova_b200_frame;

/* Counters of the last render call. */
typedef struct {
  uint64_t paths;      /* camera paths traced */
  uint64_t segments;   /* ray segments of the reference estimator (Li evaluations) */
  uint64_t traced;     /* closest-hit queries issued on the device */
  uint64_t waves;      /* wavefront iterations */
  double device_ms;    /* device time of the render (CUDA events) */
  double trace_ms;     /* device time inside the closest-hit kernel */
  double shade_ms;     /* device time inside the shading kernel */
  uint64_t kernels;    /* kernels launched */
  /* The device status word of the call.  nonfinite: path radiance values that came out NaN or
   * infinite and were written as 0, as the reference's DENAN does (integrator/Integrator.cpp:92); the
   * render succeeds.  bad_index: hits whose primitive, instance or material id lies outside the
   * scene's tables (not reachable through validated uploads; it guards against corrupted device
   * memory): the path ends black, the loop stops after the current wave group and the call returns
   * RENDERER_EXCEPTION, which the engine facade reports as exception::GENERAL_GPU_ERROR. */
  uint64_t nonfinite;
  uint64_t bad_index;
  /* With tuning.trace_mode 2: inner nodes visited and triangles tested by the closest-hit kernel
   * (binary BVH: one 64-byte node per visit; 8-wide: one 80-byte node; 48 bytes per triangle). */
  uint64_t node_visits;
  uint64_t tri_tests;
} nova_b200_render_stats;

/* Context lifecycle: DeviceAcceleratorInterface::make (api/device_accelerator_factory.cpp:9) and
 * cleanup (aggregate/device_acceleration_interface.h:25); destroy frees everything the context holds.
 * create also loads the allocation-free render's kernels on that device, which takes their static
 * 32 MiB scratch array and the path kernel's local memory once per device (see
 * nova_b200_render_noalloc).  Entry points make the context's device current and leave it so, except
 * nova_b200_render_noalloc, which restores the caller's current device. */
nova_b200_status nova_b200_create(nova_b200_ctx **ctx, int32_t device);
nova_b200_status nova_b200_destroy(nova_b200_ctx *ctx);

/* Copies a scene to device memory: Engine::buildScene (api/engine.cpp:201-233). */
nova_b200_status nova_b200_upload_scene(nova_b200_ctx *ctx, const nova_b200_scene_desc *scene);

/* Builds the device BVH (binned SAH on the GPU): Engine::buildAcceleration (api/engine.cpp:235)
 * and DeviceAcceleratorInterface::build (aggregate/device_acceleration_interface.h:24). */
nova_b200_status nova_b200_build_bvh(nova_b200_ctx *ctx, const nova_b200_bvh_options *opts);

/* AOV integrators (integrator/NormalIntegrator.cpp, DepthIntegrator.cpp, EmissiveIntegrator.cpp;
 * the integrator_flag bits of api_common.h:30-47): one unjittered camera ray per pixel, one value per
 * pixel.  NORMAL: the closest hit's normal-mapped shading normal, (n, 1), 0 on a miss.  DEPTH: from
 * the closest-hit distance and the camera's near / far planes, the reference's normalised depth / far
 * in every channel, far on a miss.  EMISSIVE: the hit material's emission, (e, 1), when its BSDF
 * sample succeeds (Sobol dimensions 0-3 of index pixel_offset * 4), else 0.  The frame supplies the
 * size, camera, seed and vertical_invert; its sample fields are not used.  film_host / film_device
 * (width * height * 4 floats) receive the image; either may be NULL. */
#define NOVA_B200_AOV_NORMAL 1
#define NOVA_B200_AOV_DEPTH 2
#define NOVA_B200_AOV_EMISSIVE 4
nova_b200_status nova_b200_render_aov(nova_b200_ctx *ctx, const nova_b200_frame *frame, int32_t kind,
                                      float near_plane, float far_plane, float *film_host, float *film_device);

/* Uploads / builds many contexts at once (no counterpart in the reference): the per-context calls
 * run on up to 16 host threads, each on its context's stream, so the host work and the GPU builds
 * of different scenes overlap.  Every context must be distinct; the first failing status is
 * returned and its message is available from ctxs[0]. */
nova_b200_status nova_b200_upload_scene_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                              uint32_t n);
nova_b200_status nova_b200_build_bvh_batch(nova_b200_ctx *const *ctxs, uint32_t n, const nova_b200_bvh_options *opts);
/* Both at once: each host thread uploads a context's scene and then builds its BVH, so the copies of
 * one scene overlap the build kernels of another.  Equal to nova_b200_upload_scene_batch followed by
 * nova_b200_build_bvh_batch; opts may be NULL (defaults). */
nova_b200_status nova_b200_upload_build_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                              uint32_t n, const nova_b200_bvh_options *opts);

/* Renders one frame batch (renderGpu, api/engine.cpp:457-496).  film_host (width*height*4 floats,
 * pageable or pinned) and/or film_device (a device pointer) receive the running-mean RGBA image;
 * either may be NULL.  stats may be NULL. */
nova_b200_status nova_b200_render(nova_b200_ctx *ctx, const nova_b200_frame *frame, float *film_host,
                                  float *film_device, nova_b200_render_stats *stats);

/* Renders n frames of n different contexts (scenes) as one wavefront on ctxs[0]'s device, stream
 * and path buffers: the batched form of renderGpu for many cameras and scenes of uneven size, sample
 * count and depth (no counterpart in the reference, which renders one engine at a time).  Every
 * frame follows the semantics of nova_b200_render on its own context (sample range, running-mean
 * film, reset) and produces the same film bit for bit.  films_host / films_device may be NULL or
 * hold n pointers (entries may be NULL).  All contexts must share a device and a BVH width.  When
 * the batch takes several chunks (more than 104 frames, or more paths than one radiance buffer
 * holds), the films of frames finished in an earlier chunk are copied out on a second stream while
 * later chunks render, if they are device or pinned host buffers; pageable ones are written at the
 * end.  Chunks take the frames largest film first (so the films left to copy after the last chunk
 * are the smallest); a film does not depend on its chunk.  The call returns after every copy. */
nova_b200_status nova_b200_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_frame *frames, uint32_t n,
                                        float *const *films_host, float *const *films_device,
                                        nova_b200_render_stats *stats);

/* Upload, build and render in one call (no counterpart in the reference): up to 16 host threads
 * upload each context's scene and build its BVH (opts may be NULL) in the order the chunks render
 * them (ctxs[0]'s scene first: its stream carries the render), while the calling
 * thread renders the frames as nova_b200_render_batch does, starting each chunk of the wavefront as
 * soon as the scenes of its frames are built; the later scenes' copies and builds overlap the first
 * chunks.  Scenes, BVHs and films equal those of nova_b200_upload_scene_batch,
 * nova_b200_build_bvh_batch and nova_b200_render_batch called one after another.  The first failing
 * status is returned (its message from ctxs[0]); an upload or build that fails fails the call. */
nova_b200_status nova_b200_upload_build_render_batch(nova_b200_ctx *const *ctxs, const nova_b200_scene_desc *descs,
                                                     const nova_b200_frame *frames, uint32_t n,
                                                     const nova_b200_bvh_options *opts, float *const *films_host,
                                                     float *const *films_device, nova_b200_render_stats *stats);

/* Allocation-free variant of nova_b200_render, for callers that cannot call cudaMalloc during a
 * frame: a host loop whose device memory is entirely reserved by another allocator (a framework's
 * caching allocator that has claimed the GPU), or a real-time loop that must not risk an allocation
 * failure or a device-wide synchronisation mid-frame.  No counterpart in the reference.  Renders
 * samples [sample_begin, sample_begin + sample_count) of every pixel and writes their mean RGBA
 * to film_device (width*height*4 floats, device memory); the context's accumulation film and
 * frame->reset are not used.  Its only scratch is a static 32 MiB device array shared by every
 * call, so calls that overlap on the GPU race; sample_count is limited to 2097152 and larger
 * values are rejected with INVALID_ARGUMENT.  The array, the kernels and the path kernel's local
 * memory are all taken by nova_b200_create on the context's device, so this call allocates
 * nothing.  It runs on the context's stream and returns after that stream has finished: the caller
 * must finish its own work on film_device (on any other stream) before the call.  The caller's
 * current device is restored on return. */
nova_b200_status nova_b200_render_noalloc(nova_b200_ctx *ctx, const nova_b200_frame *frame, float *film_device);

/* Closest-hit queries for n world-space rays held in DEVICE memory (3 floats each): the intersector
 * of DeviceIntersectorInterface::traverse (aggregate/device_acceleration_interface.h:14) /
 * GenericHostAccelerator::hit (aggregate/acceleration_interface.h:29).
 * prim = global primitive index (-1 on miss), t / u / v = Moller-Trumbore distance and barycentrics. */
nova_b200_status nova_b200_trace(nova_b200_ctx *ctx, uint64_t n, const float *orig_dev, const float *dir_dev,
                                 int32_t *prim_dev, float *t_dev, float *u_dev, float *v_dev);
/* The same for rays in host memory: copies them to the device, traces, copies the hits back. */
nova_b200_status nova_b200_trace_host(nova_b200_ctx *ctx, uint64_t n, const float *orig_host, const float *dir_host,
                                      int32_t *prim_host, float *t_host, float *u_host, float *v_host);

/* One shading event for each of n given hits, all buffers in DEVICE memory: the hit record
 * (Embree fillHitStructure semantics, aggregate/api/embree/embree.cpp:360-412), the principled
 * scatter (material/NovaMaterials.h:89-137) with Sobol dimensions 2 + 4 * bounce .. 5 + 4 * bounce of
 * sample `index`, and the spawned ray (ray/Ray.h:22-27) -- the per-hit step of the path integrator.
 * Inputs: ray origin / direction (3 floats each), the hit (global primitive, t, u, v, as returned by
 * nova_b200_trace), the Sobol sample index and bounce per hit, the seed.  Outputs: the next ray's
 * origin and direction (3 floats each), the path weight f * |cos| / pdf and the emission (3 floats
 * each), valid = 1 (scattered), 0 (scatter failed: the path ends black) or -1 (prim or bounce out of
 * range; nothing else written). */
nova_b200_status nova_b200_scatter(nova_b200_ctx *ctx, uint64_t n, const float *orig_dev, const float *dir_dev,
                                   const int32_t *prim_dev, const float *t_dev, const float *u_dev, const float *v_dev,
                                   const uint32_t *index_dev, const int32_t *bounce_dev, uint32_t seed,
                                   float *next_orig_dev, float *next_dir_dev, float *weight_dev, float *emissive_dev,
                                   int32_t *valid_dev);

/* Differentiable rendering (extension; no counterpart in the reference).  Parameters: per-triangle
 * RGB albedo (3 floats per global triangle, replacing the albedo texture) and per-material
 * roughness (1 float per material, replacing the metallic texture's roughness channel), both in
 * caller-owned DEVICE memory that must stay valid while the context renders; NULL keeps the
 * texture.  Every render of the context uses them (nova_b200_render is the forward pass).  A new
 * upload_scene clears them. */
nova_b200_status nova_b200_set_diff_params(nova_b200_ctx *ctx, const float *albedo_dev, const float *roughness_dev);

/* Replay adjoint (path-replay backpropagation): given d_image = dLoss/dImage (width*height*4
 * floats in DEVICE memory, laid out like the film nova_b200_render returns for this frame; alpha
 * ignored) for the image of `frame` rendered alone (reset = 1), adds dLoss/dAlbedo (3 floats per
 * triangle) to grad_albedo_dev and dLoss/dRoughness (1 float per material) to grad_roughness_dev
 * (either may be NULL).  No tape is stored: each path is recomputed from its Sobol index, once
 * for its radiance and once to push the adjoint through its vertices, where the derivative of the
 * sampled lobe's f (its sampling density held fixed) is applied.  The film is not touched.  The
 * call runs on the context's own stream: the caller finishes its writes of d_image and of the
 * gradient buffers (on its own streams) before the call. */
#define NOVA_B200_BACKWARD_REUSE_PRIMAL 1u /* see nova_b200_backward */

/* flags: NOVA_B200_BACKWARD_REUSE_PRIMAL skips the radiance pass when the context's last render was
 * nova_b200_render of this same frame with the same parameter buffers (one pass over the radiance
 * buffer, nothing rendered on the context since): the paths' radiance is still in the context's
 * radiance buffer.  The caller guarantees the parameters' contents did not change in between;
 * when the context cannot reuse the buffer it recomputes it. */
nova_b200_status nova_b200_backward(nova_b200_ctx *ctx, const nova_b200_frame *frame, const float *d_image_dev,
                                    float *grad_albedo_dev, float *grad_roughness_dev, uint32_t flags,
                                    nova_b200_render_stats *stats);

/* Launch parameters of the wavefront (no counterpart in the reference, whose CPU path has tiles and
 * threads only).  They change speed, never results: every tuning renders the same image, bit for
 * bit.  A batch render uses the tuning of its first context. */
typedef struct {
  uint32_t queue_capacity; /* rays per wave, 65536 .. 67108864; 0 = default (8388608) */
  uint32_t trace_block;    /* threads per block of the trace kernel: 32, 64, 96 or 128; 0 = 128 */
  uint32_t shade_block;    /* threads per block of the shade kernel: 32, 64, 96 or 128; 0 = 128 */
  uint32_t tile_w, tile_h; /* consecutive paths walk tile_w x tile_h pixel tiles (tile_w * tile_h a
                              multiple of 32, both <= 64); 0 x 0 = default 8 x 4; 1 x 1 = image rows */
  int32_t bvh_width;       /* reported by nova_b200_autotune: the BVH width it left the contexts
                              built with (0: not tuned); ignored by nova_b200_set_tuning */
  uint32_t trace_mode;     /* 0: one ray per thread (default); 1: persistent warps that hand out rays
                              as their lanes finish (binary BVH only; the 8-wide BVH ignores it);
                              2: as 0, and the render stats count the traversal's node visits and
                              triangle tests (a measurement mode; the autotuner never picks it);
                              3: the persistent wavefront: one cooperative launch runs every wave of a
                              chunk (refill, trace, shade, wave end) with grid barriers between the
                              phases; the backward pass keeps the per-wave kernels */
  uint32_t wait_limit_us;  /* trace_mode 3: the longest a grid barrier may wait, in microseconds (0 =
                              1000000); a wait past it ends the render with RENDERER_EXCEPTION */
} nova_b200_tuning;

/* tuning = NULL restores the defaults. */
nova_b200_status nova_b200_set_tuning(nova_b200_ctx *ctx, const nova_b200_tuning *tuning);
nova_b200_status nova_b200_get_tuning(nova_b200_ctx *ctx, nova_b200_tuning *tuning);

#define NOVA_B200_TUNE_BVH_WIDTH 1u /* also try the 8-wide BVH (rebuilds every context's BVH) */

/* Autotuner for a batch (or a single frame, n = 1): times probe renders of the given frames with
 * a reduced sample count under candidate tunings (queue capacity, block sizes, pixel tiles and,
 * with NOVA_B200_TUNE_BVH_WIDTH, the BVH width), applies the fastest to every context and writes
 * it to *best.  The tuning fields never change a result bit; the BVH width can change which of two
 * triangles hit at exactly the same distance is reported.  Results are cached in the text file cache_path (NULL: no cache) under a key of
 * device, frame count, path count, depth and BVH width; a cached entry is applied without probing.
 * The probe renders reset the contexts' accumulation films. */
nova_b200_status nova_b200_autotune(nova_b200_ctx *const *ctxs, const nova_b200_frame *frames, uint32_t n,
                                    const char *cache_path, uint32_t flags, nova_b200_tuning *best);

/* Sobol + Owen samples (math_random.h:73-98 SobolGenerator::generate) for n (index, dimension)
 * pairs in device memory. */
nova_b200_status nova_b200_sobol(nova_b200_ctx *ctx, uint64_t n, const uint32_t *index_dev, const uint32_t *dim_dev,
                                 uint32_t seed, float *out_dev);

/* Diffuse irradiance bake of an equirectangular f32 map (TextureProcessing.cpp:10-64 semantics).
 * src_dev: src_w*src_h*channels floats; out_dev: out_w*out_h*channels floats (power-of-two sizes). */
nova_b200_status nova_b200_bake_irradiance(nova_b200_ctx *ctx, const float *src_dev, int32_t src_w, int32_t src_h,
                                           int32_t channels, int32_t out_w, int32_t out_h, int32_t samples,
                                           float *out_dev);
/* The same bake with the semantics of the reference's CUDA kernel, the path its command line takes
 * with --gpu: GPU_compute_irradiance (sources/processing/cuda/CubemapProcessing.cu:244-284, kernel
 * :129-175).  The hash is seeded with the output texel's indices, directions map to uv with the
 * exact acos / atan2f, and the source (RGB or RGBA, made RGBA with alpha 1 as
 * TextureProcessing.cpp:24-32 does) is read through a float4 texture object with hardware bilinear
 * filtering and wrap addressing.  out_dev: out_w*out_h*4 floats, alpha 1.  Power-of-two output
 * sizes; the source must fit a 2D texture. */
nova_b200_status nova_b200_bake_irradiance_texunit(nova_b200_ctx *ctx, const float *src_dev, int32_t src_w,
                                                   int32_t src_h, int32_t channels, int32_t out_w, int32_t out_h,
                                                   int32_t samples, float *out_dev);

/* ---- Film outputs (device buffers, the context's device and stream) ---------------------------
 *
 * Progressive accumulation: Engine::writeFramebuffer (corelib/nova/api/engine.cpp:351-363).
 * accumulator += partial; final = accumulator / (frame_index + 1) (final may be NULL).  n floats,
 * buffers 16-byte aligned. */
nova_b200_status nova_b200_film_accumulate(nova_b200_ctx *ctx, const float *partial_dev, float *accumulator_dev,
                                           float *final_dev, uint64_t n, uint32_t frame_index);
/* The editor's display value: NovaRenderer::copyBufferToPbo (sources/renderer/nova/NovaRenderer_draw.cpp:35-45).
 * old = accumulated / (current_frame + 1); display = old + 0.8 (partial - old).  n floats. */
nova_b200_status nova_b200_display_blend(nova_b200_ctx *ctx, const float *partial_dev, const float *accumulated_dev,
                                         float *display_dev, uint64_t n, uint32_t current_frame);
/* A film resampled to another size: NovaRenderer::getSnapshotFloat (sources/renderer/nova/NovaRenderer.cpp:139-153)
 * with TextureOperations::processTexture (sources/processing/TextureProcessing.h:157-250).  dst holds
 * dst_width * dst_height * channels floats; channels 0-2 of each pixel are written, channel 3 is left
 * as it is.  dst_height <= 65535. */
nova_b200_status nova_b200_snapshot(nova_b200_ctx *ctx, const float *film_dev, int32_t width, int32_t height,
                                    int32_t channels, float *dst_dev, int32_t dst_width, int32_t dst_height);

/* ---- Radiance .hdr files (the bake CLI's input and output, the render saved to disk) -----------
 *
 * Size of a .hdr file: the header checks of IO::Loader::loadHdrEnvmap / loadRadianceFile
 * (sources/IO/Loader_image.cpp:64-90, 146-160).  ctx may be NULL (no error text then). */
nova_b200_status nova_b200_hdr_info(nova_b200_ctx *ctx, const char *path, int32_t *width, int32_t *height);
/* Reads a .hdr file as width * height * 4 floats, RGB and alpha 1: IO::Loader::loadRadianceFile
 * (Loader_image.cpp:146-192).  The RGBE pixels are decoded on the device.  rgba_host and / or
 * rgba_device (16-byte aligned) receive the image; capacity is their size in floats.  OpenEXR files
 * are rejected (INVALID_ARGUMENT). */
nova_b200_status nova_b200_hdr_read(nova_b200_ctx *ctx, const char *path, float *rgba_host, float *rgba_device,
                                    uint64_t capacity);
/* Writes path + ".hdr": IO::Loader::writeHdr (Loader_image.cpp:50-62).  pixels: width * height *
 * channels floats (1-4 channels; 1 or 2 write the first channel as grey) on the host or on the
 * device; encoded to RGBE on the device, rows run-length packed for widths in [8, 32768).  flip
 * writes the rows bottom-up.  height <= 65535. */
nova_b200_status nova_b200_hdr_write(nova_b200_ctx *ctx, const char *path, const float *pixels_host,
                                     const float *pixels_device, int32_t width, int32_t height, int32_t channels,
                                     int32_t flip);
/* The bake command's work: API::bakeTexture (sources/controller/cmd/API.cpp:44-62, options of
 * ProgramOptionsManager.cpp:76-79, 116-137) without the viewer it opens.  Reads the Radiance map
 * path_in (RGBA, alpha 1), bakes the diffuse irradiance map of out_width x out_height texels (powers
 * of two) with `samples` samples per texel on the device, writes path_out + ".hdr" (alpha 0, as the
 * reference leaves it).  type must be "irradiance" (the only type the reference bakes). */
nova_b200_status nova_b200_bake_texture(nova_b200_ctx *ctx, const char *type, int32_t out_width, int32_t out_height,
                                        int32_t samples, const char *path_in, const char *path_out);
/* The same with flags: NOVA_B200_BAKE_GPU_KERNEL bakes with nova_b200_bake_irradiance_texunit, the
 * reference's `--gpu` path (ProgramOptionsManager.cpp:39-40,69 sets CONF_USE_CUDA, which
 * API.cpp:52 passes to computeDiffuseIrradiance); its output alpha is 1. */
#define NOVA_B200_BAKE_GPU_KERNEL 1u
nova_b200_status nova_b200_bake_texture_flags(nova_b200_ctx *ctx, const char *type, int32_t out_width,
                                              int32_t out_height, int32_t samples, const char *path_in,
                                              const char *path_out, uint32_t flags);
/* Device time in ms of the kernel of the last film_accumulate / display_blend / snapshot /
 * hdr_read / hdr_write call (CUDA events).  No counterpart in the reference. */
nova_b200_status nova_b200_last_call_ms(nova_b200_ctx *ctx, float *device_ms);

/* Stops the render, render_batch or backward call running on this context (for a batch: on its
 * first context) from another thread: NvEngineInstance::stopRender's is_rendering flag
 * (api/engine.cpp:577-586).  The wave loop checks it after every group of four waves and between
 * chunks; the call then waits for the group still in flight and returns RENDERER_EXCEPTION
 * ("render cancelled") without writing the film (a batch spanning several chunks has already
 * written the films of frames that finished in an earlier chunk, when they are device or pinned
 * host buffers).  The accumulation film keeps the chunks finished before the stop, so the next
 * frame should set reset.  A cancel applies to the call in progress:
 * each render / backward call clears it when it starts.  No counterpart call in the reference. */
nova_b200_status nova_b200_cancel(nova_b200_ctx *ctx);

/* Last error message: Engine::getRenderEngineError (api_engine.h:185).  buf holds 1024 chars. */
void nova_b200_get_error(nova_b200_ctx *ctx, char buf[1024], size_t *size);

/* Scene / BVH statistics: triangles, instances, BVH nodes, BVH leaves, device bytes held. */
nova_b200_status nova_b200_scene_info(nova_b200_ctx *ctx, uint64_t *triangles, uint64_t *instances, uint64_t *nodes,
                                      uint64_t *leaves, uint64_t *device_bytes);

/* Waits for all work of the context's stream. */
nova_b200_status nova_b200_synchronize(nova_b200_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* NOVA_B200_H */
