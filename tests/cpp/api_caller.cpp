/* A Nova caller, written once against the nova:: scene / camera / transform / material / texture /
 * render-option / render-buffer API, that compiles unchanged against both
 *   - the reference's own API headers (corelib/nova/api_{common,camera,transform,geometry,material,
 *     texture,scene,renderoptions,renderbuffer}.h; syntax only, there is nothing to link), and
 *   - this library's restatement (include/nova_b200_api.hpp), where it also links and runs.
 * Every method of those classes is called with the argument types the reference declares, so a
 * method missing here, renamed or with another parameter list fails the build on one side; the
 * same holds for the render's error bits (engine/nova_exception.h, NovaException).  The
 * engine class itself (api_engine.h) cannot be compiled here: it pulls in the reference's renderer,
 * which needs glm.  The enum values are printed so that the two sides can be compared.
 * Built by tests/cpp/Makefile: `api_caller` (this library) always, `api_caller_ref` (the reference's
 * headers, from the reference tree where it lies) where that tree is present. */
#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include <memory>
#include <utility>
#include <vector>

#ifdef NOVA_API_REFERENCE
#  include <api_camera.h>
#  include <api_common.h>
#  include <api_geometry.h>
#  include <api_material.h>
#  include <api_renderbuffer.h>
#  include <api_renderoptions.h>
#  include <api_scene.h>
#  include <api_texture.h>
#  include <api_transform.h>
#  include <engine/nova_exception.h>
#else
#  include "../../include/nova_b200_api.hpp"
#endif

namespace {

[[maybe_unused]] int use_camera(nova::Camera &c) {
  const float v3[3] = {0.f, 1.f, 0.f};
  float o3[3], o16[16];
  const float m16[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  int bad = 0;
  bad += c.setUpVector(v3) != nova::SUCCESS;
  bad += c.setMatrices(m16, m16) != nova::SUCCESS;
  bad += c.setPosition(v3) != nova::SUCCESS;
  bad += c.setDirection(v3) != nova::SUCCESS;
  bad += c.setClipPlaneFar(100.f) != nova::SUCCESS;
  bad += c.setClipPlaneNear(0.1f) != nova::SUCCESS;
  bad += c.setResolutionWidth(64u) != nova::SUCCESS;
  bad += c.setResolutionHeight(32u) != nova::SUCCESS;
  bad += c.setFov(60.f) != nova::SUCCESS;
  bad += c.getUpVector(o3) != nova::SUCCESS;
  bad += c.getProjectionMatrix(o16) != nova::SUCCESS;
  bad += c.getViewMatrix(o16) != nova::SUCCESS;
  bad += c.getInverseProjectionMatrix(o16) != nova::SUCCESS;
  bad += c.getInverseViewMatrix(o16) != nova::SUCCESS;
  bad += c.getProjectionViewMatrix(o16) != nova::SUCCESS;
  bad += c.getInverseProjectionViewMatrix(o16) != nova::SUCCESS;
  bad += c.getPosition(o3) != nova::SUCCESS;
  bad += c.getDirection(o3) != nova::SUCCESS;
  const nova::Camera &cc = c;
  bad += cc.getClipPlaneFar() != 100.f;
  bad += cc.getClipPlaneNear() != 0.1f;
  bad += cc.getResolutionWidth() != 64u;
  bad += cc.getResolutionHeight() != 32u;
  bad += cc.getFov() != 60.f;
  return bad;
}

[[maybe_unused]] int use_transform(nova::Transform &t, const nova::Transform &other) {
  const float m16[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 2, 3, 4, 1};
  const float q[4] = {0.f, 0.f, 0.f, 1.f};
  float o16[16], o9[9], o4[4], o3[3];
  t.clone(other);
  t.setTransformMatrix(m16);
  t.rotateQuat(0.f, 0.f, 0.f, 1.f);
  t.rotateEuler(0.f, 0.f, 1.f, 0.f);
  t.reset();
  t.getTransformMatrix(o16);
  t.translate(1.f, 2.f, 3.f);
  t.scale(2.f);
  t.scale(1.f, 1.f, 1.f);
  t.setTranslation(1.f, 2.f, 3.f);
  t.getTranslation(o3);
  t.setScale(1.f, 1.f, 1.f);
  t.getScale(o3);
  t.getRotation(o4);
  t.setRotation(q);
  t.multiply(other);
  t.invert(o16);
  t.transpose(o16);
  t.transposeInvert(o9);
  return o3[0] != 1.f;
}

[[maybe_unused]] int use_trimesh(nova::Trimesh &m, std::vector<float> &f, std::vector<unsigned> &idx, nova::TransformPtr tr) {
  int bad = 0;
  bad += m.registerBufferVertices(f.data(), f.size()) != nova::SUCCESS;
  bad += m.registerBufferNormals(f.data(), f.size()) != nova::SUCCESS;
  bad += m.registerBufferTangents(f.data(), f.size()) != nova::SUCCESS;
  bad += m.registerBufferBitangents(f.data(), f.size()) != nova::SUCCESS;
  bad += m.registerBufferColors(f.data(), f.size()) != nova::SUCCESS;
  bad += m.registerBufferUVs(f.data(), f.size()) != nova::SUCCESS;
  bad += m.registerBufferIndices(idx.data(), idx.size()) != nova::SUCCESS;
  const uint32_t vbo = 7;
  /* GL buffers: the reference registers them in a GL build, this library has none */
  m.registerInteropVertices(vbo), m.registerInteropNormals(vbo), m.registerInteropTangents(vbo);
  m.registerInteropBitangents(vbo), m.registerInteropColors(vbo), m.registerInteropUVs(vbo);
  m.registerInteropIndices(vbo);
  const nova::Trimesh &cm = m;
  bad += cm.getVertices().size() != f.size() || cm.getNormals().size() != f.size();
  bad += cm.getTangents().size() != f.size() || cm.getBitangents().size() != f.size();
  bad += cm.getColors().size() != f.size() || cm.getUVs().size() != f.size();
  bad += cm.getIndices().size() != idx.size();
  uint32_t ids = cm.getInteropVertices() + cm.getInteropNormals() + cm.getInteropTangents() +
                 cm.getInteropBitangents() + cm.getInteropColors() + cm.getInteropUVs() + cm.getInteropIndices();
  (void)ids;
  bad += m.registerTransform(std::move(tr)) != nova::SUCCESS;
  float o16[16];
  cm.getTransform().getTransformMatrix(o16);
  return bad;
}

[[maybe_unused]] int use_texture(nova::Texture &t, const std::vector<uint32_t> &px, const std::vector<float> &fpx) {
  int bad = 0;
  bad += t.setWidth(2u) != nova::SUCCESS;
  bad += t.setHeight(2u) != nova::SUCCESS;
  bad += t.setChannels(4u) != nova::SUCCESS;
  bad += t.setTextureBuffer(px.data()) != nova::SUCCESS;
  bad += t.getFormat() != nova::texture::UINT8X4;
  bad += t.setTextureBuffer(fpx.data()) != nova::SUCCESS;
  bad += t.getFormat() != nova::texture::FLOATX4;
  bad += t.setTextureBuffer(px.data()) != nova::SUCCESS;
  t.setInteropID(3u);
  bad += t.invertY() != nova::SUCCESS;
  bad += t.invertX() != nova::SUCCESS;
  const nova::Texture &ct = t;
  bad += ct.getTextureBuffer() == nullptr;
  bad += ct.getWidth() != 2u || ct.getHeight() != 2u || ct.getChannels() != 4u;
  unsigned gl = ct.getInteropID();
  (void)gl;
  bad += !ct.getInvertY() || !ct.getInvertX();
  return bad;
}

[[maybe_unused]] int use_material(nova::Material &m, nova::TexturePtr (*tex)()) {
  const float eta[3] = {1.5f, 1.5f, 1.5f}, k[3] = {0.f, 0.f, 0.f};
  int bad = 0;
  bad += m.registerAlbedo(tex()) != nova::SUCCESS;
  bad += m.registerNormal(tex()) != nova::SUCCESS;
  bad += m.registerMetallic(tex()) != nova::SUCCESS;
  bad += m.registerEmissive(tex()) != nova::SUCCESS;
  bad += m.registerRoughness(tex()) != nova::SUCCESS;
  bad += m.registerOpacity(tex()) != nova::SUCCESS;
  bad += m.registerSpecular(tex()) != nova::SUCCESS;
  bad += m.registerAmbientOcclusion(tex()) != nova::SUCCESS;
  bad += m.setRefractiveIndex(eta) != nova::SUCCESS;
  bad += m.setRefractiveIndex(eta, k) != nova::SUCCESS;
  bad += m.setAnisotropyFactor(0.25f) != nova::SUCCESS;
  const nova::Material &cm = m;
  bad += !m.getAlbedo() || !cm.getAlbedo() || !m.getNormal() || !cm.getNormal();
  bad += !m.getMetallic() || !cm.getMetallic() || !m.getEmissive() || !cm.getEmissive();
  bad += !m.getRoughness() || !cm.getRoughness() || !m.getOpacity() || !cm.getOpacity();
  bad += !m.getSpecular() || !cm.getSpecular() || !m.getAmbientOcclusion() || !cm.getAmbientOcclusion();
  float e[3], kk[3];
  cm.getRefractiveIndex(e, kk);
  bad += e[0] != 1.5f || cm.getAnisotropyFactor() != 0.25f;
  return bad;
}

[[maybe_unused]] int use_scene(nova::Scene &s, nova::TrimeshPtr mesh, nova::MaterialPtr mat, nova::TexturePtr env, nova::CameraPtr cam,
              nova::TransformPtr root) {
  int bad = 0;
  bad += s.addMesh(std::move(mesh), std::move(mat)) != nova::SUCCESS;
  const unsigned e = s.addEnvmap(std::move(env));
  bad += s.useEnvmap(e) != nova::SUCCESS;
  bad += s.getEnvmap(e) == nullptr;
  const nova::Scene &cs = s;
  bad += cs.getEnvmap(e) == nullptr || cs.getCurrentEnvmapId() != (int)e;
  bad += s.setRootTransform(std::move(root)) != nova::SUCCESS;
  const unsigned c = s.addCamera(std::move(cam));
  bad += s.useCamera(c) != nova::SUCCESS || cs.getCurrentCameraId() != (int)c;
  bad += s.getCamera(c) == nullptr || cs.getCamera(c) == nullptr;
  bad += cs.getPrimitivesNum(nova::mesh::TRIANGLE) != 1 || cs.getMeshesNum(nova::mesh::TRIANGLE) != 1;
  nova::CsteTriMeshCollection meshes = cs.getTriangleMeshCollection();
  nova::CsteMaterialCollection mats = cs.getMaterialCollection(nova::mesh::TRIANGLE);
  nova::CsteCameraCollection cams = cs.getCameraCollection();
  nova::CsteTextureCollection envs = cs.getEnvmapCollection();
  bad += meshes.size() != 1 || mats.size() != 1 || cams.size() != 1 || envs.size() != 1;
  s.clearEnvmaps();
  s.clearCameras();
  s.cleanup();
  bad += cs.getMeshesNum(nova::mesh::TRIANGLE) != 0;
  return bad;
}

[[maybe_unused]] int use_options(nova::RenderOptions &o) {
  int bad = 0;
  o.setAliasingSamples(4u);
  o.setMaxDepth(6u);
  o.setMaxSamples(16u);
  o.setSamplesIncrement(1u);
  o.setTileDimension(20u, 10u);
  bad += o.setIntegratorFlag(nova::integrator::PATH | nova::integrator::COMBINED) != nova::SUCCESS;
  bad += o.useGpu(true) != nova::SUCCESS;
  o.useInterops(false);
  o.flipV();
  const nova::RenderOptions &co = o;
  bad += co.getAliasingSamples() != 4u || co.getMaxDepth() != 6u || co.getMaxSamples() != 16u;
  bad += co.getSamplesIncrement() != 1u || co.getTileDimensionWidth() != 20u || co.getTileDimensionHeight() != 10u;
  bad += co.getIntegratorFlag() != (nova::integrator::PATH | nova::integrator::COMBINED);
  bad += !co.isUsingGpu() || co.isUsingInterops() || !co.isFlippedV();
  return bad;
}

[[maybe_unused]] int use_renderbuffer(nova::RenderBuffer &b) {
  int bad = 0;
  bad += b.preallocate(8u, 8u) != nova::SUCCESS;
  bad += b.resize(4u, 3u) != nova::SUCCESS;
  bad += b.resetBuffers() != nova::SUCCESS;
  nova::HdrBufferStruct h = b.getRenderBuffers();
  bad += h.partial_buffer == nullptr || h.channels != 4;
  nova::FloatView back = b.backBuffer(), front = b.frontBuffer();
  b.swapBackBuffer();
  const nova::RenderBuffer &cb = b;
  nova::FloatView acc = cb.getAccumulator();
  nova::Framebuffer fb = cb.getFramebuffer();
  bad += back.size() != 48 || front.size() != 48 || acc.size() != 48 || fb.color_buffer_width != 4u;
  bad += cb.getWidth() != 4u || cb.getHeight() != 3u || cb.getChannel(nova::texture::COLOR) != 4u;
  nova::frgba_s c = cb.sampleColor(1u, 2u);
  nova::frgb_s n = cb.sampleNormal(1u, 2u);
  float d = cb.sampleDepth(1u, 2u);
  bad += c.r != 0.f || n.r != 0.f || d != d;
  return bad;
}

[[maybe_unused]] int use_exception() {
  namespace ex = nova::exception;
  ex::NovaException e;
  e.addErrorType(ex::SAMPLER_INIT_ERROR | ex::INVALID_SAMPLER_DIM);
  e.merge(ex::GENERAL_ERROR);
  ex::NovaException copy(e), moved(std::move(copy));
  copy = moved;
  moved = std::move(copy);
  std::vector<ex::ERROR> list = moved.getErrorList();
  return !moved.errorCheck() || moved.getErrorFlag() != (ex::SAMPLER_INIT_ERROR | ex::INVALID_SAMPLER_DIM | ex::GENERAL_ERROR) ||
         list.size() != 3;
}

void print_enums() {
  std::printf("ERROR_STATE");
  for (int v : {nova::SUCCESS, nova::INVALID_ENGINE_STATE, nova::INVALID_BUFFER_STATE, nova::INVALID_CHANNEL_DESCRIPTOR,
                nova::INVALID_SCENE_TYPE, nova::INVALID_TRANSFORM_TYPE, nova::RENDER_BUFFER_NOT_INITIALIZED,
                nova::RENDER_OPTIONS_NOT_INITIALIZED, nova::RENDER_ENGINE_NOT_INITIALIZED, nova::SCENE_NOT_PROCESSED,
                nova::NOT_GPU_BUILD, nova::OUT_OF_MEMORY, nova::MULTIPLE_INTEGRATORS_NOT_SUPPORTED,
                nova::THREADPOOL_CREATION_ERROR, nova::THREADPOOL_NOT_INITIALIZED, nova::INVALID_ARGUMENT,
                nova::RENDERER_EXCEPTION})
    std::printf(" %d", v);
  std::printf("\nintegrator");
  for (int v : {nova::integrator::PATH, nova::integrator::BIPATH, nova::integrator::SPECTRAL, nova::integrator::METROPOLIS,
                nova::integrator::PHOTON, nova::integrator::MARCHING, nova::integrator::HYBRID, nova::integrator::VOXEL,
                nova::integrator::COMBINED, nova::integrator::NORMAL, nova::integrator::DEPTH, nova::integrator::SPECULAR,
                nova::integrator::DIFFUSE, nova::integrator::EMISSIVE})
    std::printf(" %d", v);
  std::printf("\ntexture");
  for (int v : {(int)nova::texture::UINT8X4, (int)nova::texture::FLOATX4, (int)nova::texture::COLOR,
                (int)nova::texture::DEPTH, (int)nova::texture::NORMAL})
    std::printf(" %d", v);
  std::printf("\nmesh");
  for (int v : {nova::mesh::TRIANGLE, nova::mesh::SPHERE, nova::mesh::BOX, nova::mesh::NURB}) std::printf(" %d", v);
  std::printf("\nexception");
  namespace ex = nova::exception;
  for (unsigned long long v :
       {(unsigned long long)ex::NOERR, (unsigned long long)ex::INVALID_INTEGRATOR, (unsigned long long)ex::INVALID_RENDER_MODE,
        (unsigned long long)ex::INVALID_SAMPLER_DIM, (unsigned long long)ex::SAMPLER_INIT_ERROR,
        (unsigned long long)ex::SAMPLER_DOMAIN_EXHAUSTED, (unsigned long long)ex::SAMPLER_INVALID_ALLOC,
        (unsigned long long)ex::SAMPLER_INVALID_ARG, (unsigned long long)ex::INVALID_RENDERBUFFER_STATE,
        (unsigned long long)ex::INVALID_ENGINE_INSTANCE, (unsigned long long)ex::INVALID_RENDERBUFFER_DIM,
        (unsigned long long)ex::GENERAL_GPU_ERROR, (unsigned long long)ex::GENERAL_ERROR})
    std::printf(" %llu", v);
  std::printf("\n");
}

}  // namespace

#ifdef NOVA_API_REFERENCE
/* Against the reference's headers there is nothing to link the factories to: the calls above are
 * compiled (type-checked) and the enum values printed. */
int main() {
  print_enums();
  return 0;
}
#else
int main() {
  print_enums();
  std::vector<float> f(9, 0.5f);
  std::vector<unsigned> idx = {0, 1, 2};
  std::vector<uint32_t> px(4, 0xff0000ffu);
  std::vector<float> fpx(16, 1.f);
  auto make_tex = []() -> nova::TexturePtr {
    static const std::vector<uint32_t> p(4, 0xffffffffu);
    nova::TexturePtr t = nova::create_texture();
    t->setWidth(2u), t->setHeight(2u), t->setChannels(4u), t->setTextureBuffer(p.data());
    return t;
  };
  int bad = 0;
  nova::CameraPtr cam = nova::create_camera();
  bad += use_camera(*cam);
  nova::TransformPtr tr = nova::create_transform(), other = nova::create_transform();
  bad += use_transform(*tr, *other);
  nova::TrimeshPtr mesh = nova::create_trimesh();
  bad += use_trimesh(*mesh, f, idx, nova::create_transform());
  nova::TexturePtr tex = nova::create_texture();
  bad += use_texture(*tex, px, fpx);
  nova::MaterialPtr mat = nova::create_material();
  bad += use_material(*mat, +make_tex);
  nova::ScenePtr scene = nova::create_scene();
  bad += use_scene(*scene, std::move(mesh), std::move(mat), make_tex(), std::move(cam), std::move(tr));
  nova::RenderOptionsPtr opts = nova::create_renderoptions();
  bad += use_options(*opts);
  nova::RenderBufferPtr rb = nova::create_renderbuffer();
  bad += use_renderbuffer(*rb);
  bad += use_exception();
  std::printf("api caller: %d failed checks\n", bad);
  return bad ? 1 : 0;
}
#endif
