/* nova_b200_api.hpp — the Nova engine API of HamilcarR/Axomae (corelib/nova/api_*.h) re-stated over
 * the B200 C ABI (nova_b200.h), as a host C++ library (libnova_b200_engine.so).
 *
 * A Nova caller (the editor bridge sources/renderer/nova/nova_bake_image.cpp:156-198, or any code
 * written against nova::Engine) keeps its calls: the class names, method names, argument meaning,
 * ERROR_STATE values and factories are the reference's.  What changes is below the facade: scenes go
 * to the device through nova_b200_upload_scene / nova_b200_build_bvh, frames render with
 * nova_b200_render (one sample per frame into the render buffer's partial buffer, then added to its
 * accumulator as Engine::writeFramebuffer does; the render buffers are host memory, as the
 * reference's are), and the AOV passes with nova_b200_render_aov.  Differences, all stated where
 * they apply:
 *   - spans are std::span (the reference's axstd::span); matrices and vectors are float arrays, as
 *     in the reference's signatures (glm stays out of the interface);
 *   - OpenGL interop (registerInterop*, setInteropID, useInterops(true)) is not available on a
 *     compute-only B200 host: those calls return NOT_GPU_BUILD and change nothing;
 *   - RenderOptions::useGpu(false) is accepted, but startRender() then fails with
 *     INVALID_ENGINE_STATE: this library renders on the GPU only (no CPU fallback);
 *   - Engine::getResrcManager (marked for removal in the reference) is not part of the facade.
 *
 * The device accelerator plug-in point (aggregate/device_acceleration_interface.h:11-38) is
 * re-stated in nova::aggregate: DeviceAcceleratorInterface::make() returns the B200 accelerator.
 */
#ifndef NOVA_B200_API_HPP
#define NOVA_B200_API_HPP
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <span>
#include <vector>

namespace nova {

/* api_common.h:7-27, same numbering as nova_b200_status */
enum ERROR_STATE {
  SUCCESS,
  INVALID_ENGINE_STATE,
  INVALID_BUFFER_STATE,
  INVALID_CHANNEL_DESCRIPTOR,
  INVALID_SCENE_TYPE,
  INVALID_TRANSFORM_TYPE,
  RENDER_BUFFER_NOT_INITIALIZED,
  RENDER_OPTIONS_NOT_INITIALIZED,
  RENDER_ENGINE_NOT_INITIALIZED,
  SCENE_NOT_PROCESSED,
  NOT_GPU_BUILD,
  OUT_OF_MEMORY,
  MULTIPLE_INTEGRATORS_NOT_SUPPORTED,
  THREADPOOL_CREATION_ERROR,
  THREADPOOL_NOT_INITIALIZED,
  INVALID_ARGUMENT,
  RENDERER_EXCEPTION,
};

namespace exception {
/* engine/nova_exception.h:13-31: one bit per render error, numbered as in the reference. */
enum ERROR : uint64_t {
  NOERR = 0,
  INVALID_INTEGRATOR = 1ULL << 0,
  INVALID_RENDER_MODE = 1ULL << 1,
  INVALID_SAMPLER_DIM = 1ULL << 2,
  SAMPLER_INIT_ERROR = 1ULL << 3,
  SAMPLER_DOMAIN_EXHAUSTED = 1ULL << 4,
  SAMPLER_INVALID_ALLOC = 1ULL << 5,
  SAMPLER_INVALID_ARG = 1ULL << 6,
  INVALID_RENDERBUFFER_STATE = 1ULL << 7,
  INVALID_ENGINE_INSTANCE = 1ULL << 8,
  INVALID_RENDERBUFFER_DIM = 1ULL << 9,
  GENERAL_GPU_ERROR = 1ULL << 31,
  GENERAL_ERROR = 1ULL << 32,
};

/* NovaException (engine/nova_exception.h:33-61, nova_exception.cpp): a set of ERROR bits that any
 * thread may add to.  A copy carries the bits; a move takes them and leaves the source empty. */
class NovaException {
  std::atomic<uint64_t> flags_{NOERR};

 public:
  NovaException() = default;
  NovaException(const NovaException &o) noexcept : flags_(o.getErrorFlag()) {}
  NovaException(NovaException &&o) noexcept : flags_(o.flags_.exchange(NOERR, std::memory_order_relaxed)) {}
  NovaException &operator=(const NovaException &o) noexcept {
    if (this != &o) flags_.store(o.getErrorFlag(), std::memory_order_relaxed);
    return *this;
  }
  NovaException &operator=(NovaException &&o) noexcept {
    if (this != &o) flags_.store(o.flags_.exchange(NOERR, std::memory_order_relaxed), std::memory_order_relaxed);
    return *this;
  }
  [[nodiscard]] bool errorCheck() const { return getErrorFlag() != NOERR; }
  [[nodiscard]] uint64_t getErrorFlag() const { return flags_.load(std::memory_order_relaxed); }
  void addErrorType(uint64_t errors) { flags_.fetch_or(errors, std::memory_order_relaxed); }
  /* adds another exception's bits to these */
  void merge(uint64_t other_flags) { flags_.fetch_or(other_flags, std::memory_order_relaxed); }
  /* every set bit as its own ERROR, lowest first ({NOERR} when none is); bits 0 to 62 */
  [[nodiscard]] std::vector<ERROR> getErrorList() const {
    const uint64_t f = getErrorFlag();
    if (f == NOERR) return {NOERR};
    std::vector<ERROR> out;
    for (unsigned bit = 0; bit < 63; bit++)
      if (f & (1ULL << bit)) out.push_back(static_cast<ERROR>(1ULL << bit));
    return out;
  }
};
}  // namespace exception

namespace integrator {
/* api_common.h:29-48: integrator bits 0-7, render-pass bits 8-13 */
enum TYPE : int {
  PATH = 1 << 0,
  BIPATH = 1 << 1,
  SPECTRAL = 1 << 2,
  METROPOLIS = 1 << 3,
  PHOTON = 1 << 4,
  MARCHING = 1 << 5,
  HYBRID = 1 << 6,
  VOXEL = 1 << 7,
  COMBINED = 1 << 8,
  NORMAL = 1 << 9,
  DEPTH = 1 << 10,
  SPECULAR = 1 << 11,
  DIFFUSE = 1 << 12,
  EMISSIVE = 1 << 13,
};
}  // namespace integrator

namespace texture {
enum FORMAT { UINT8X4, FLOATX4 };
enum CHANNEL_TYPE { COLOR, DEPTH, NORMAL };
}  // namespace texture

namespace mesh {
enum TYPE { TRIANGLE, SPHERE, BOX, NURB };
}  // namespace mesh

class Camera;
class Scene;
class Transform;
class Engine;
class Trimesh;
class Material;
class Texture;
class RenderBuffer;
class RenderOptions;
class EngineUserCallbackHandler;

using RenderBufferPtr = std::unique_ptr<RenderBuffer>;
using EnginePtr = std::unique_ptr<Engine>;
using RenderOptionsPtr = std::unique_ptr<RenderOptions>;
using TransformPtr = std::unique_ptr<Transform>;
using TexturePtr = std::unique_ptr<Texture>;
using ScenePtr = std::unique_ptr<Scene>;
using TrimeshPtr = std::unique_ptr<Trimesh>;
using CameraPtr = std::unique_ptr<Camera>;
using MaterialPtr = std::unique_ptr<Material>;
using EngineUserCallbackHandlerPtr = std::unique_ptr<EngineUserCallbackHandler>;
using CsteTriMeshCollection = std::span<const TrimeshPtr>;
using CsteCameraCollection = std::span<const CameraPtr>;
using CsteMaterialCollection = std::span<const MaterialPtr>;
using CsteTextureCollection = std::span<const TexturePtr>;
using CsteFloatView = std::span<const float>;
using FloatView = std::span<float>;

/* api_datastructures.h */
template <class T>
struct RenderBuffers {
  T *partial_buffer;
  T *depth_buffer;
  T *normal_buffer;
  size_t color_buffers_pitch{};
  size_t depth_buffers_pitch{};
  size_t normal_buffers_pitch{};
  size_t byte_size_color_buffers{};
  size_t byte_size_depth_buffers{};
  int channels{};
};
using HdrBufferStruct = RenderBuffers<float>;

/* api_transform.h: a column-major 4x4 matrix with glm's composition order (M = M * op). */
class Transform {
 public:
  virtual ~Transform() = default;
  virtual void clone(const Transform &other) = 0;
  virtual void setTransformMatrix(const float transform[16]) = 0;
  virtual void rotateQuat(float x, float y, float z, float w) = 0;
  virtual void rotateEuler(float angle, float x, float y, float z) = 0;
  virtual void reset() = 0;
  virtual void getTransformMatrix(float transform[16]) const = 0;
  virtual void translate(float x, float y, float z) = 0;
  virtual void scale(float scale) = 0;
  virtual void scale(float x, float y, float z) = 0;
  virtual void setTranslation(float x, float y, float z) = 0;
  virtual void getTranslation(float translation[3]) const = 0;
  virtual void setScale(float x, float y, float z) = 0;
  virtual void getScale(float scale[3]) const = 0;
  virtual void getRotation(float rotation[4]) const = 0;
  virtual void setRotation(const float rotation[4]) = 0;
  virtual void multiply(const Transform &other) = 0;
  virtual void invert(float inverse[16]) const = 0;
  virtual void transpose(float result[16]) const = 0;
  virtual void transposeInvert(float result[9]) const = 0;
};
TransformPtr create_transform();

/* api_geometry.h: non-owning views of the caller's attribute buffers (the caller keeps them alive
 * until buildScene() has copied them to the device). */
class AbstractMesh {
 public:
  virtual ~AbstractMesh() = default;
  virtual ERROR_STATE registerTransform(TransformPtr transform) = 0;
  virtual const Transform &getTransform() const = 0;
};

class Trimesh : public AbstractMesh {
 public:
  virtual ERROR_STATE registerBufferVertices(float *vert, size_t num) = 0;
  virtual ERROR_STATE registerBufferNormals(float *normals, size_t num) = 0;
  virtual ERROR_STATE registerBufferTangents(float *tangents, size_t num) = 0;
  virtual ERROR_STATE registerBufferBitangents(float *bitangents, size_t num) = 0;
  virtual ERROR_STATE registerBufferColors(float *colors, size_t num) = 0;
  virtual ERROR_STATE registerBufferUVs(float *uv, size_t num) = 0;
  virtual ERROR_STATE registerBufferIndices(unsigned *indices, size_t num) = 0;
  virtual ERROR_STATE registerInteropVertices(uint32_t vbo_id) = 0;
  virtual ERROR_STATE registerInteropNormals(uint32_t vbo_id) = 0;
  virtual ERROR_STATE registerInteropTangents(uint32_t vbo_id) = 0;
  virtual ERROR_STATE registerInteropBitangents(uint32_t vbo_id) = 0;
  virtual ERROR_STATE registerInteropColors(uint32_t vbo_id) = 0;
  virtual ERROR_STATE registerInteropUVs(uint32_t vbo_id) = 0;
  virtual ERROR_STATE registerInteropIndices(uint32_t vbo_id) = 0;
  virtual std::span<float> getVertices() const = 0;
  virtual std::span<float> getNormals() const = 0;
  virtual std::span<float> getTangents() const = 0;
  virtual std::span<float> getBitangents() const = 0;
  virtual std::span<float> getColors() const = 0;
  virtual std::span<float> getUVs() const = 0;
  virtual std::span<unsigned> getIndices() const = 0;
  virtual uint32_t getInteropVertices() const = 0;
  virtual uint32_t getInteropNormals() const = 0;
  virtual uint32_t getInteropTangents() const = 0;
  virtual uint32_t getInteropBitangents() const = 0;
  virtual uint32_t getInteropColors() const = 0;
  virtual uint32_t getInteropUVs() const = 0;
  virtual uint32_t getInteropIndices() const = 0;
};
TrimeshPtr create_trimesh();

/* api_texture.h: a non-owning view of 32-bit packed u8 RGBA texels or float texels. */
class Texture {
 public:
  virtual ~Texture() = default;
  template <class T>
  ERROR_STATE setTextureBuffer(const T *data) {
    return setData(data);
  }
  virtual ERROR_STATE setWidth(unsigned w) = 0;
  virtual ERROR_STATE setHeight(unsigned h) = 0;
  virtual ERROR_STATE setChannels(unsigned c) = 0;
  virtual ERROR_STATE setInteropID(uint32_t texture_id) = 0;
  virtual ERROR_STATE invertY() = 0;
  virtual ERROR_STATE invertX() = 0;
  virtual const void *getTextureBuffer() const = 0;
  virtual unsigned getWidth() const = 0;
  virtual unsigned getHeight() const = 0;
  virtual unsigned getChannels() const = 0;
  virtual uint32_t getInteropID() const = 0;
  virtual bool getInvertY() const = 0;
  virtual bool getInvertX() const = 0;
  virtual texture::FORMAT getFormat() const = 0;

 protected:
  virtual ERROR_STATE setData(const uint32_t *buffer) = 0;
  virtual ERROR_STATE setData(const float *buffer) = 0;
};
TexturePtr create_texture();

/* api_material.h: the principled material's texture pack and refraction parameters.  The device
 * shading reads albedo, metallic (roughness = green, metal = blue), normal and emissive
 * (NovaMaterials.h:116-117); roughness, opacity, specular and ambient-occlusion textures are kept
 * for the caller but not read, as in the reference's principled material. */
class Material {
 public:
  virtual ~Material() = default;
  virtual ERROR_STATE registerAlbedo(TexturePtr texture) = 0;
  virtual ERROR_STATE registerNormal(TexturePtr texture) = 0;
  virtual ERROR_STATE registerMetallic(TexturePtr texture) = 0;
  virtual ERROR_STATE registerEmissive(TexturePtr texture) = 0;
  virtual ERROR_STATE registerRoughness(TexturePtr texture) = 0;
  virtual ERROR_STATE registerOpacity(TexturePtr texture) = 0;
  virtual ERROR_STATE registerSpecular(TexturePtr texture) = 0;
  virtual ERROR_STATE registerAmbientOcclusion(TexturePtr texture) = 0;
  virtual ERROR_STATE setRefractiveIndex(const float eta[3]) = 0;
  virtual ERROR_STATE setRefractiveIndex(const float eta[3], const float k[3]) = 0;
  virtual ERROR_STATE setAnisotropyFactor(float anisotropy) = 0;
  virtual Texture *getAlbedo() = 0;
  virtual const Texture *getAlbedo() const = 0;
  virtual Texture *getNormal() = 0;
  virtual const Texture *getNormal() const = 0;
  virtual Texture *getMetallic() = 0;
  virtual const Texture *getMetallic() const = 0;
  virtual Texture *getEmissive() = 0;
  virtual const Texture *getEmissive() const = 0;
  virtual Texture *getRoughness() = 0;
  virtual const Texture *getRoughness() const = 0;
  virtual Texture *getOpacity() = 0;
  virtual const Texture *getOpacity() const = 0;
  virtual Texture *getSpecular() = 0;
  virtual const Texture *getSpecular() const = 0;
  virtual Texture *getAmbientOcclusion() = 0;
  virtual const Texture *getAmbientOcclusion() const = 0;
  virtual void getRefractiveIndex(float eta[3], float k[3]) const = 0;
  virtual float getAnisotropyFactor() const = 0;
};
MaterialPtr create_material();

/* api_camera.h */
class Camera {
 public:
  virtual ~Camera() = default;
  virtual ERROR_STATE setUpVector(const float up[3]) = 0;
  virtual ERROR_STATE setMatrices(const float projection_matrix[16], const float view_matrix[16]) = 0;
  virtual ERROR_STATE setPosition(const float pos[3]) = 0;
  virtual ERROR_STATE setDirection(const float dir[3]) = 0;
  virtual ERROR_STATE setClipPlaneFar(float far_plane) = 0;
  virtual ERROR_STATE setClipPlaneNear(float near_plane) = 0;
  virtual ERROR_STATE setResolutionWidth(unsigned width) = 0;
  virtual ERROR_STATE setResolutionHeight(unsigned height) = 0;
  virtual ERROR_STATE setFov(float fov) = 0;
  virtual ERROR_STATE getUpVector(float up[3]) const = 0;
  virtual ERROR_STATE getProjectionMatrix(float proj[16]) const = 0;
  virtual ERROR_STATE getViewMatrix(float view[16]) const = 0;
  virtual ERROR_STATE getInverseProjectionMatrix(float proj[16]) const = 0;
  virtual ERROR_STATE getInverseViewMatrix(float proj[16]) const = 0;
  virtual ERROR_STATE getProjectionViewMatrix(float proj[16]) const = 0;
  virtual ERROR_STATE getInverseProjectionViewMatrix(float proj[16]) const = 0;
  virtual ERROR_STATE getPosition(float pos[3]) const = 0;
  virtual ERROR_STATE getDirection(float dir[3]) const = 0;
  virtual float getClipPlaneFar() const = 0;
  virtual float getClipPlaneNear() const = 0;
  virtual unsigned getResolutionWidth() const = 0;
  virtual unsigned getResolutionHeight() const = 0;
  virtual float getFov() const = 0;
};
CameraPtr create_camera();

/* api_renderoptions.h */
class RenderOptions {
 public:
  virtual ~RenderOptions() = default;
  virtual void setAliasingSamples(unsigned s) = 0;
  virtual unsigned getAliasingSamples() const = 0;
  virtual void setMaxDepth(unsigned depth) = 0;
  virtual unsigned getMaxDepth() const = 0;
  virtual void setMaxSamples(unsigned samples) = 0;
  virtual unsigned getMaxSamples() const = 0;
  virtual void setSamplesIncrement(unsigned inc) = 0;
  virtual unsigned getSamplesIncrement() const = 0;
  virtual void setTileDimension(unsigned width, unsigned height) = 0;
  virtual unsigned getTileDimensionWidth() const = 0;
  virtual unsigned getTileDimensionHeight() const = 0;
  virtual ERROR_STATE setIntegratorFlag(int flag) = 0;
  virtual int getIntegratorFlag() const = 0;
  virtual ERROR_STATE useGpu(bool use) = 0;
  virtual bool isUsingGpu() const = 0;
  virtual ERROR_STATE useInterops(bool use) = 0;
  virtual bool isUsingInterops() const = 0;
  virtual void flipV() = 0;
  virtual bool isFlippedV() const = 0;
};
RenderOptionsPtr create_renderoptions();

/* api_renderbuffer.h: host buffers the engine fills after every frame. */
struct Framebuffer {
  FloatView color_buffer{};
  unsigned color_buffer_channels{};
  unsigned color_buffer_width{};
  unsigned color_buffer_height{};
  FloatView depth_buffer{};
  unsigned depth_buffer_width{};
  unsigned depth_buffer_height{};
  FloatView normal_buffer{};
  unsigned normal_buffer_channels{};
  unsigned normal_buffer_width{};
  unsigned normal_buffer_height{};
};
struct frgba_s {
  float r, g, b, a;
};
struct frgb_s {
  float r, g, b;
};

class RenderBuffer {
 public:
  virtual ~RenderBuffer() = default;
  virtual ERROR_STATE preallocate(unsigned width, unsigned height) = 0;
  virtual ERROR_STATE resize(unsigned width, unsigned height) = 0;
  virtual ERROR_STATE resetBuffers() = 0;
  virtual HdrBufferStruct getRenderBuffers() const = 0;
  virtual FloatView backBuffer() = 0;
  virtual FloatView frontBuffer() = 0;
  virtual void swapBackBuffer() = 0;
  virtual FloatView getAccumulator() const = 0;
  virtual Framebuffer getFramebuffer() const = 0;
  virtual unsigned getWidth() const = 0;
  virtual unsigned getHeight() const = 0;
  virtual unsigned getChannel(texture::CHANNEL_TYPE type) const = 0;
  virtual frgba_s sampleColor(unsigned x, unsigned y) const = 0;
  virtual frgb_s sampleNormal(unsigned x, unsigned y) const = 0;
  virtual float sampleDepth(unsigned x, unsigned y) const = 0;
};
RenderBufferPtr create_renderbuffer();

/* api_scene.h: one material per mesh (api/engine.cpp:177-184), environment maps, cameras. */
class Scene {
 public:
  virtual ~Scene() = default;
  virtual ERROR_STATE addMesh(TrimeshPtr mesh, MaterialPtr material) = 0;
  virtual unsigned addEnvmap(TexturePtr envmap_texture) = 0;
  virtual ERROR_STATE useEnvmap(unsigned id) = 0;
  virtual Texture *getEnvmap(unsigned id) = 0;
  virtual const Texture *getEnvmap(unsigned id) const = 0;
  virtual void clearEnvmaps() = 0;
  virtual int getCurrentEnvmapId() const = 0;
  virtual ERROR_STATE setRootTransform(TransformPtr transform) = 0;
  virtual unsigned addCamera(CameraPtr camera) = 0;
  virtual void clearCameras() = 0;
  virtual ERROR_STATE useCamera(unsigned id) = 0;
  virtual int getCurrentCameraId() const = 0;
  virtual Camera *getCamera(unsigned id) = 0;
  virtual void cleanup() = 0;
  virtual const Camera *getCamera(unsigned id) const = 0;
  virtual unsigned getPrimitivesNum(mesh::TYPE type) const = 0;
  virtual unsigned getMeshesNum(mesh::TYPE type) const = 0;
  virtual CsteTriMeshCollection getTriangleMeshCollection() const = 0;
  virtual CsteMaterialCollection getMaterialCollection(mesh::TYPE type) const = 0;
  virtual CsteCameraCollection getCameraCollection() const = 0;
  virtual CsteTextureCollection getEnvmapCollection() const = 0;
};
ScenePtr create_scene();

/* api_engine.h */
class EngineUserCallbackHandler {
 public:
  virtual ~EngineUserCallbackHandler() = default;
  virtual void framePreRenderRoutine() = 0;
  virtual void framePostRenderRoutine() = 0;
};

class Engine {
 public:
  virtual ~Engine() = default;
  virtual ERROR_STATE buildScene() = 0;
  virtual ERROR_STATE setScene(ScenePtr scene) = 0;
  virtual const Scene *getScene() const = 0;
  virtual Scene *getScene() = 0;
  virtual ERROR_STATE buildAcceleration() = 0;
  virtual ERROR_STATE setRenderBuffers(RenderBufferPtr render_buffer) = 0;
  virtual const RenderBuffer *getRenderBuffers() const = 0;
  virtual RenderBuffer *getRenderBuffers() = 0;
  virtual ERROR_STATE cleanup() = 0;
  virtual ERROR_STATE setRenderOptions(RenderOptionsPtr opts) = 0;
  virtual const RenderOptions *getRenderOptions() const = 0;
  virtual RenderOptions *getRenderOptions() = 0;
  virtual ERROR_STATE stopRender() = 0;
  virtual ERROR_STATE startRender() = 0;
  virtual void setUserCallback(EngineUserCallbackHandlerPtr user_callback) = 0;
  /* true from startRender() until stopRender() (after the last frame too, as in the reference), or
   * until a frame fails */
  virtual bool isRendering() const = 0;
  virtual ERROR_STATE prepareRender() = 0;
  virtual void getRenderEngineError(char error_log[1024], size_t &size) = 0;
  virtual unsigned getFrameIndex() const = 0;
};

/* The engine on device `device` (the reference's create_engine() takes no argument: device 0). */
EnginePtr create_engine();
EnginePtr create_engine(int device);
/* api_engine.h:193-196 read the engine's exception manager; here the engine holds the errors of its
 * last startRender() and render: what the start checks found (INVALID_INTEGRATOR without the PATH
 * bit, INVALID_RENDER_MODE without a pass, INVALID_RENDERBUFFER_DIM / _STATE for unsized buffers),
 * then the failure of a frame (GENERAL_GPU_ERROR for a device failure, INVALID_RENDERBUFFER_STATE,
 * GENERAL_ERROR otherwise).  startRender() clears them. */
uint64_t get_error_status(const Engine &engine);
std::vector<exception::ERROR> get_error_list(const Engine &engine);

/* The reference sizes its CPU thread pool here; the B200 engine renders on its own host thread and
 * the device, so this only checks the argument (0 -> THREADPOOL_CREATION_ERROR). */
ERROR_STATE init_threads(unsigned number_threads);

/* gpu/nova_gpu.h:20-29, reduced to what a traversal launch of the B200 backend reads. */
struct camera_matrices_s {
  float inv_P[16];
  float inv_V[16];
};
struct device_traversal_param_s {
  HdrBufferStruct render_buffers;
  camera_matrices_s camera;
  uint32_t width, height, depth, current_envmap_index, sample_index, sample_max;
};

namespace aggregate {

/* One mesh of primitive_aggregate_data_s: the Object3D spans (internal/geometry/Object3D.h:384-394)
 * and its transform record (utils_3D.h:84-96: m, inv, n), plus the material index the primitives
 * of this mesh use, and the scene's materials, textures and environment map (the resource
 * managers' views in the reference's mesh_geometry / primitive_list_view). */
struct mesh_view_s {
  std::span<const float> vertices, normals, tangents, bitangents, uv;
  std::span<const unsigned> indices;
  float m[16], inv[16], n[9];
  uint32_t material;
};
struct material_view_s {
  int32_t albedo, metallic, normalmap, emissive; /* texture indices or -1 */
  float eta[3], k[3];
  float anisotropy;
};
struct texture_view_s {
  const uint32_t *u8_pixels;
  const float *f32_pixels;
  int32_t width, height, channels;
  int32_t invert_u, invert_v;
};
struct primitive_aggregate_data_s {
  std::span<const mesh_view_s> meshes;
  std::span<const material_view_s> materials;
  std::span<const texture_view_s> textures;
  int32_t envmap;
};

/* aggregate/device_acceleration_interface.h:11-38 */
class DeviceIntersectorInterface {
 public:
  virtual ~DeviceIntersectorInterface() = default;
  virtual void traverse(const device_traversal_param_s &params) const = 0;
};

class DeviceAcceleratorInterface {
 public:
  virtual ~DeviceAcceleratorInterface() = default;
  virtual void build(primitive_aggregate_data_s primitive_data_list) = 0;
  virtual void cleanup() = 0;
  virtual unsigned getMaxRecursiveDepth() const = 0;
  virtual void copyParamsToDevice(const device_traversal_param_s &params) const = 0;
  /* The B200 intersector shares the accelerator's device scene and stays valid after the
   * accelerator's cleanup() or destruction. */
  virtual std::unique_ptr<DeviceIntersectorInterface> getIntersectorObject() const = 0;
  /* The B200 accelerator on device 0 (api/device_accelerator_factory.cpp:9-18). */
  static std::unique_ptr<DeviceAcceleratorInterface> make();
};

/* The B200 accelerator's extra queries, beyond the interface: the status of the last build, its
 * error text, and closest hits of rays in host memory (nova_b200_trace_host: 3 floats of origin and
 * of direction per ray in, primitive id (-1 on a miss), t, u, v out) for callers that cast their
 * own rays. */
class B200Accelerator : public DeviceAcceleratorInterface {
 public:
  virtual ERROR_STATE lastStatus() const = 0;
  virtual void getError(char error_log[1024], size_t &size) const = 0;
  virtual ERROR_STATE closestHits(uint64_t n, const float *orig_dev, const float *dir_dev, int32_t *prim_dev,
                                  float *t_dev, float *u_dev, float *v_dev) const = 0;
};

}  // namespace aggregate
}  // namespace nova

#endif  // NOVA_B200_API_HPP
