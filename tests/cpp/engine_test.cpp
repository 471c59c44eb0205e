/* Tests of the Nova engine API (include/nova_b200_api.hpp, libnova_b200_engine.so), driven the way a
 * Nova caller drives nova::Engine.
 *
 *   engine_test cpu            API logic that needs no GPU: transforms, cameras, options, render
 *                              buffers, scenes, engine error codes
 *   engine_test accel          the reference's acceleration tests (tests/unit_test/corelib/nova/
 *                              aggregate/acceleration_interfaceTest.cpp: intersect_inside,
 *                              intersect_outside_front, nointersect_outside_back,
 *                              nointersect_outside_back_translated) on the B200 device accelerator
 *   engine_test render <dir>   a progressive engine render against a one-shot C-ABI render of the
 *                              same scene (bit for bit), a NORMAL pass against nova_b200_render_aov,
 *                              error paths; the scene and image are written to <dir> for the oracle
 *
 * Exit status 0 when every check passes; each failed check prints its line.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nova_b200.h"
#include "../../include/nova_b200_api.hpp"

namespace {

int g_failures = 0;
#define CHECK(cond)                                                               \
  do {                                                                            \
    if (!(cond)) {                                                                \
      std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
      g_failures++;                                                               \
    }                                                                             \
  } while (0)

bool close(float a, float b, float tol = 1e-5f) { return std::fabs(a - b) <= tol * (1.f + std::fabs(b)); }

/* column-major helpers for the tests' own cameras (double precision, rounded once) */
void mat_mul(const float *a, const float *b, float *o) {
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += (double)a[k * 4 + r] * b[c * 4 + k];
      o[c * 4 + r] = (float)s;
    }
}
bool is_identity(const float *m, float tol) {
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++)
      if (std::fabs(m[c * 4 + r] - (r == c ? 1.f : 0.f)) > tol) return false;
  return true;
}
void perspective(float fovy_deg, float aspect, float n, float f, float *P) {
  std::memset(P, 0, 64);
  const double t = 1.0 / std::tan(fovy_deg * M_PI / 360.0);
  P[0] = (float)(t / aspect), P[5] = (float)t;
  P[10] = (float)(-(f + n) / (f - n)), P[11] = -1.f, P[14] = (float)(-2.0 * f * n / (f - n));
}
void look_at(const double e[3], const double c[3], const double up[3], float *V) {
  double f[3] = {c[0] - e[0], c[1] - e[1], c[2] - e[2]};
  double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (double &x : f) x /= fl;
  double s[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
  double sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
  for (double &x : s) x /= sl;
  double u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
  std::memset(V, 0, 64);
  for (int k = 0; k < 3; k++) V[k * 4 + 0] = (float)s[k], V[k * 4 + 1] = (float)u[k], V[k * 4 + 2] = (float)-f[k];
  V[12] = (float)-(s[0] * e[0] + s[1] * e[1] + s[2] * e[2]);
  V[13] = (float)-(u[0] * e[0] + u[1] * e[1] + u[2] * e[2]);
  V[14] = (float)(f[0] * e[0] + f[1] * e[1] + f[2] * e[2]);
  V[15] = 1.f;
}

uint32_t rgba8(int r, int g, int b, int a = 255) {
  return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16) | ((uint32_t)a << 24);
}

/* ---- geometry fixtures: a mesh with every attribute the device path reads ---------------- */

struct MeshData {
  std::vector<float> v, n, t, b, uv;
  std::vector<unsigned> idx;
  void vertex(double px, double py, double pz, double nx, double ny, double nz, double u, double w) {
    v.insert(v.end(), {(float)px, (float)py, (float)pz});
    n.insert(n.end(), {(float)nx, (float)ny, (float)nz});
    /* tangent: any unit vector orthogonal to n; bitangent = n x t */
    double tx = -nz, ty = 0, tz = nx;
    if (std::fabs(nx) < 1e-6 && std::fabs(nz) < 1e-6) tx = 1, ty = 0, tz = 0;
    const double tl = std::sqrt(tx * tx + ty * ty + tz * tz);
    tx /= tl, ty /= tl, tz /= tl;
    t.insert(t.end(), {(float)tx, (float)ty, (float)tz});
    b.insert(b.end(), {(float)(ny * tz - nz * ty), (float)(nz * tx - nx * tz), (float)(nx * ty - ny * tx)});
    uv.insert(uv.end(), {(float)u, (float)w});
  }
};

/* axis-aligned box [-h, h]^3 around c: 4 vertices and 2 triangles per face, outward normals */
MeshData box(double cx, double cy, double cz, double h) {
  MeshData m;
  for (int axis = 0; axis < 3; axis++)
    for (int sgn = -1; sgn <= 1; sgn += 2) {
      const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
      const unsigned base = (unsigned)(m.v.size() / 3);
      for (int k = 0; k < 4; k++) {
        double p[3], nrm[3] = {0, 0, 0};
        p[axis] = sgn * h;
        p[a1] = (k & 1) ? h : -h;
        p[a2] = (k & 2) ? h : -h;
        nrm[axis] = sgn;
        m.vertex(cx + p[0], cy + p[1], cz + p[2], nrm[0], nrm[1], nrm[2], (k & 1) ? 1 : 0, (k & 2) ? 1 : 0);
      }
      m.idx.insert(m.idx.end(), {base, base + 1, base + 3, base, base + 3, base + 2});
    }
  return m;
}

MeshData sphere(double cx, double cy, double cz, double r, int su, int sv) {
  MeshData m;
  for (int j = 0; j <= sv; j++)
    for (int i = 0; i <= su; i++) {
      const double th = M_PI * j / sv, ph = 2 * M_PI * i / su;
      const double nx = std::sin(th) * std::cos(ph), ny = std::cos(th), nz = std::sin(th) * std::sin(ph);
      m.vertex(cx + r * nx, cy + r * ny, cz + r * nz, nx, ny, nz, (double)i / su, (double)j / sv);
    }
  for (int j = 0; j < sv; j++)
    for (int i = 0; i < su; i++) {
      const unsigned a = j * (su + 1) + i, b = a + su + 1;
      m.idx.insert(m.idx.end(), {a, b, a + 1, a + 1, b, b + 1});
    }
  return m;
}

MeshData ground(double size, double y) {
  MeshData m;
  m.vertex(-size, y, -size, 0, 1, 0, 0, 0);
  m.vertex(size, y, -size, 0, 1, 0, 1, 0);
  m.vertex(-size, y, size, 0, 1, 0, 0, 1);
  m.vertex(size, y, size, 0, 1, 0, 1, 1);
  m.idx = {0, 2, 1, 1, 2, 3};
  return m;
}

nova::aggregate::mesh_view_s view_of(const MeshData &d, const float m[16], const float inv[16], const float n[9]) {
  nova::aggregate::mesh_view_s x{};
  x.vertices = d.v, x.normals = d.n, x.tangents = d.t, x.bitangents = d.b, x.uv = d.uv, x.indices = d.idx;
  std::memcpy(x.m, m, 64), std::memcpy(x.inv, inv, 64), std::memcpy(x.n, n, 36);
  x.material = 0;
  return x;
}

/* ---- cpu ----------------------------------------------------------------------------------- */

void test_transform() {
  auto t = nova::create_transform();
  float m[16], inv[16], p[16];
  t->translate(1, 2, 3);
  t->getTransformMatrix(m);
  CHECK(m[12] == 1.f && m[13] == 2.f && m[14] == 3.f && m[0] == 1.f);
  t->scale(2.f);
  t->getTransformMatrix(m);
  CHECK(m[0] == 2.f && m[5] == 2.f && m[10] == 2.f && m[12] == 1.f); /* M * S keeps the translation */
  t->rotateEuler((float)(M_PI / 2), 0, 0, 1);
  t->getTransformMatrix(m);
  CHECK(close(m[0], 0.f, 1e-6f) && close(m[1], 2.f)); /* x axis -> y axis, scaled */
  t->invert(inv);
  mat_mul(m, inv, p);
  CHECK(is_identity(p, 1e-5f));
  float s[3], tr[3];
  t->getScale(s);
  t->getTranslation(tr);
  CHECK(close(s[0], 2.f) && close(s[1], 2.f) && close(s[2], 2.f) && tr[0] == 1.f && tr[2] == 3.f);
  /* setTranslation keeps the scale and drops the rotation: S * T (api/transform.cpp) */
  t->setTranslation(5, 6, 7);
  t->getTransformMatrix(m);
  CHECK(close(m[0], 2.f) && close(m[1], 0.f, 1e-6f) && close(m[12], 10.f) && close(m[13], 12.f) && close(m[14], 14.f));
  auto q = nova::create_transform();
  const float rot[4] = {0.f, 0.f, (float)std::sin(M_PI / 8), (float)std::cos(M_PI / 8)};
  q->rotateQuat(rot[0], rot[1], rot[2], rot[3]);
  float got[4];
  q->getRotation(got);
  for (int k = 0; k < 4; k++) CHECK(close(got[k], rot[k], 1e-5f));
  auto d = nova::create_transform();
  d->scale(2, 4, 8);
  float n9[9];
  d->transposeInvert(n9);
  CHECK(close(n9[0], 0.5f) && close(n9[4], 0.25f) && close(n9[8], 0.125f) && n9[1] == 0.f);
  auto c = nova::create_transform();
  c->clone(*t);
  float cm[16];
  c->getTransformMatrix(cm);
  t->getTransformMatrix(m);
  CHECK(std::memcmp(cm, m, 64) == 0);
  c->reset();
  c->getTransformMatrix(cm);
  CHECK(is_identity(cm, 0.f));
  /* multiply: M * other */
  auto a = nova::create_transform(), b = nova::create_transform();
  a->translate(1, 0, 0);
  b->scale(3.f);
  a->multiply(*b);
  a->getTransformMatrix(m);
  CHECK(m[0] == 3.f && m[12] == 1.f);
  float tp[16];
  a->transpose(tp);
  CHECK(tp[3] == 1.f && tp[12] == 0.f);
}

void test_camera() {
  auto cam = nova::create_camera();
  float P[16], V[16], got[16], prod[16];
  perspective(60.f, 4.f / 3.f, 0.1f, 100.f, P);
  const double e[3] = {1, 2, 5}, c[3] = {0, 0.5, 0}, up[3] = {0, 1, 0};
  look_at(e, c, up, V);
  CHECK(cam->setMatrices(P, V) == nova::SUCCESS);
  cam->getInverseProjectionMatrix(got);
  mat_mul(P, got, prod);
  CHECK(is_identity(prod, 1e-5f));
  cam->getInverseViewMatrix(got);
  mat_mul(V, got, prod);
  CHECK(is_identity(prod, 1e-5f));
  float pv[16], ref[16];
  cam->getProjectionViewMatrix(pv);
  mat_mul(P, V, ref);
  for (int k = 0; k < 16; k++) CHECK(close(pv[k], ref[k], 1e-5f));
  cam->setClipPlaneNear(0.5f);
  cam->setClipPlaneFar(50.f);
  cam->setResolutionWidth(320);
  CHECK(cam->getClipPlaneNear() == 0.5f && cam->getClipPlaneFar() == 50.f && cam->getResolutionWidth() == 320);
}

void test_options_and_buffers() {
  auto o = nova::create_renderoptions();
  CHECK(o->setIntegratorFlag(nova::integrator::PATH | nova::integrator::BIPATH) ==
        nova::MULTIPLE_INTEGRATORS_NOT_SUPPORTED);
  CHECK(o->setIntegratorFlag(nova::integrator::PATH | nova::integrator::COMBINED) == nova::SUCCESS);
  CHECK(o->getIntegratorFlag() == (nova::integrator::PATH | nova::integrator::COMBINED));
  CHECK(o->useInterops(true) == nova::NOT_GPU_BUILD && !o->isUsingInterops());
  CHECK(o->useGpu(true) == nova::SUCCESS && o->isUsingGpu());
  CHECK(!o->isFlippedV());
  o->flipV();
  CHECK(o->isFlippedV());
  o->setTileDimension(20, 10);
  CHECK(o->getTileDimensionWidth() == 20 && o->getTileDimensionHeight() == 10);

  auto rb = nova::create_renderbuffer();
  CHECK(rb->resize(4, 3) == nova::SUCCESS);
  CHECK(rb->getWidth() == 4 && rb->getHeight() == 3);
  const nova::HdrBufferStruct h = rb->getRenderBuffers();
  CHECK(h.channels == 4 && h.color_buffers_pitch == 4 * 4 * sizeof(float) && h.byte_size_color_buffers == 48 * 4);
  CHECK(rb->getAccumulator().size() == 48 && rb->backBuffer().size() == 48);
  CHECK(rb->getChannel(nova::texture::DEPTH) == 1 && rb->getChannel(nova::texture::NORMAL) == 3);
  float *back = rb->backBuffer().data(), *front = rb->frontBuffer().data();
  CHECK(back != front);
  back[(1 * 3 + 2) * 4] = 7.f; /* pixel (x = 1, y = 2) in the reference's (x * height + y) order */
  rb->swapBackBuffer();
  CHECK(rb->frontBuffer().data() == back && rb->sampleColor(1, 2).r == 7.f);
  CHECK(rb->resetBuffers() == nova::SUCCESS && rb->frontBuffer()[(1 * 3 + 2) * 4] == 0.f);
}

void test_scene() {
  auto s = nova::create_scene();
  CHECK(s->addMesh(nullptr, nova::create_material()) == nova::INVALID_ARGUMENT);
  MeshData b = box(0, 0, 0, 1);
  auto m = nova::create_trimesh();
  CHECK(m->registerBufferVertices(b.v.data(), b.v.size()) == nova::SUCCESS);
  CHECK(m->registerBufferIndices(b.idx.data(), b.idx.size()) == nova::SUCCESS);
  CHECK(m->registerInteropVertices(3) == nova::NOT_GPU_BUILD);
  CHECK(s->addMesh(std::move(m), nova::create_material()) == nova::SUCCESS);
  CHECK(s->getMeshesNum(nova::mesh::TRIANGLE) == 1 && s->getPrimitivesNum(nova::mesh::TRIANGLE) == 12);
  CHECK(s->getMeshesNum(nova::mesh::SPHERE) == 0);
  CHECK(s->addEnvmap(nova::create_texture()) == 0 && s->addEnvmap(nova::create_texture()) == 1);
  CHECK(s->useEnvmap(5) == nova::INVALID_ARGUMENT && s->useEnvmap(1) == nova::SUCCESS && s->getCurrentEnvmapId() == 1);
  CHECK(s->addCamera(nova::create_camera()) == 0 && s->useCamera(0) == nova::SUCCESS);
  CHECK(s->getCamera(3) == nullptr && s->getCamera(0) != nullptr);
  s->cleanup();
  CHECK(s->getMeshesNum(nova::mesh::TRIANGLE) == 0 && s->getCurrentCameraId() == -1);
  auto t = nova::create_texture();
  const uint32_t px[4] = {1, 2, 3, 4};
  CHECK(t->setTextureBuffer(px) == nova::SUCCESS && t->getFormat() == nova::texture::UINT8X4);
  const float fpx[4] = {1, 2, 3, 4};
  CHECK(t->setTextureBuffer(fpx) == nova::SUCCESS && t->getFormat() == nova::texture::FLOATX4);
  CHECK(t->setInteropID(5) == nova::NOT_GPU_BUILD);
}

void test_engine_errors_without_device() {
  auto e = nova::create_engine();
  CHECK(e->setScene(nullptr) == nova::INVALID_ARGUMENT);
  CHECK(e->buildScene() == nova::INVALID_SCENE_TYPE);
  CHECK(e->buildAcceleration() == nova::SCENE_NOT_PROCESSED);
  CHECK(e->startRender() == nova::RENDER_OPTIONS_NOT_INITIALIZED);
  CHECK(e->setRenderOptions(nullptr) == nova::INVALID_ARGUMENT);
  CHECK(e->setRenderOptions(nova::create_renderoptions()) == nova::SUCCESS);
  CHECK(e->startRender() == nova::RENDER_BUFFER_NOT_INITIALIZED);
  CHECK(nova::get_error_status(*e) == nova::exception::INVALID_RENDERBUFFER_STATE);
  CHECK(e->setRenderBuffers(nullptr) == nova::INVALID_BUFFER_STATE);
  CHECK(e->setRenderBuffers(nova::create_renderbuffer()) == nova::SUCCESS);
  CHECK(e->prepareRender() == nova::SUCCESS);
  CHECK(e->startRender() == nova::SCENE_NOT_PROCESSED);
  CHECK(nova::get_error_status(*e) == nova::exception::NOERR); /* each start clears the bits */
  CHECK(nova::get_error_list(*e) == std::vector<nova::exception::ERROR>{nova::exception::NOERR});
  CHECK(!e->isRendering() && e->getFrameIndex() == 0);
  CHECK(e->stopRender() == nova::SUCCESS && e->getFrameIndex() == 1); /* as the reference's stopRender */
  CHECK(e->cleanup() == nova::INVALID_ENGINE_STATE);                  /* no scene */
  CHECK(nova::init_threads(0) == nova::THREADPOOL_CREATION_ERROR && nova::init_threads(8) == nova::SUCCESS);
  char log[1024];
  size_t n = 0;
  e->getRenderEngineError(log, n);
  CHECK(n > 0 && std::strstr(log, "buildScene") != nullptr); /* the last failure: buildAcceleration() */
}

/* The reference's nova_exception tests (tests/unit_test/corelib/nova/engine/nova_exceptionTest.cpp). */
bool has(const std::vector<nova::exception::ERROR> &list, nova::exception::ERROR e) {
  return std::find(list.begin(), list.end(), e) != list.end();
}

void test_nova_exception() {
  namespace ex = nova::exception;
  {
    ex::NovaException e; /* get_error_list */
    e.addErrorType(ex::SAMPLER_INIT_ERROR | ex::INVALID_SAMPLER_DIM);
    const auto list = e.getErrorList();
    CHECK(has(list, ex::SAMPLER_INIT_ERROR) && has(list, ex::INVALID_SAMPLER_DIM) && list.size() == 2);
  }
  {
    ex::NovaException e; /* add_error_type */
    e.addErrorType(ex::SAMPLER_INIT_ERROR);
    e.addErrorType(ex::INVALID_SAMPLER_DIM);
    CHECK((e.getErrorFlag() & ex::SAMPLER_INIT_ERROR) && (e.getErrorFlag() & ex::INVALID_SAMPLER_DIM) && e.errorCheck());
  }
  {
    ex::NovaException origin, target; /* copy_constructor: the copy carries the bits, the source keeps them */
    origin.addErrorType(ex::INVALID_INTEGRATOR | ex::SAMPLER_INIT_ERROR | ex::INVALID_RENDER_MODE);
    target = origin;
    const auto list = target.getErrorList();
    CHECK(has(list, ex::INVALID_INTEGRATOR) && has(list, ex::SAMPLER_INIT_ERROR) && has(list, ex::INVALID_RENDER_MODE));
    CHECK(!has(list, ex::INVALID_SAMPLER_DIM) && origin.getErrorFlag() == target.getErrorFlag());
    ex::NovaException copied(origin);
    CHECK(copied.getErrorFlag() == origin.getErrorFlag());
  }
  {
    ex::NovaException origin, target; /* move_constructor: the bits move, the source is left empty */
    origin.addErrorType(ex::INVALID_INTEGRATOR | ex::SAMPLER_INIT_ERROR | ex::INVALID_RENDER_MODE);
    target = std::move(origin);
    const auto list = target.getErrorList();
    CHECK(has(list, ex::INVALID_INTEGRATOR) && has(list, ex::SAMPLER_INIT_ERROR) && has(list, ex::INVALID_RENDER_MODE));
    CHECK(!has(list, ex::INVALID_SAMPLER_DIM));
    ex::NovaException moved(std::move(target));
    CHECK(moved.getErrorList().size() == 3 && !target.errorCheck()); /* NOLINT: use after move is the point */
  }
  {
    ex::NovaException origin, target; /* merge */
    origin.addErrorType(ex::SAMPLER_INIT_ERROR | ex::INVALID_SAMPLER_DIM);
    target.addErrorType(ex::SAMPLER_INVALID_ARG | ex::SAMPLER_INVALID_ALLOC);
    target.merge(origin.getErrorFlag());
    const auto list = target.getErrorList();
    CHECK(has(list, ex::SAMPLER_INIT_ERROR) && has(list, ex::INVALID_SAMPLER_DIM) && has(list, ex::SAMPLER_INVALID_ARG) &&
          has(list, ex::SAMPLER_INVALID_ALLOC) && !has(list, ex::INVALID_RENDER_MODE));
  }
  {
    ex::NovaException e; /* no error: {NOERR}; the two high bits are listed like the others */
    CHECK(e.getErrorList() == std::vector<ex::ERROR>{ex::NOERR} && !e.errorCheck());
    e.addErrorType(ex::GENERAL_ERROR | ex::GENERAL_GPU_ERROR);
    CHECK(e.getErrorList() == (std::vector<ex::ERROR>{ex::GENERAL_GPU_ERROR, ex::GENERAL_ERROR}));
  }
}

/* ---- accel --------------------------------------------------------------------------------- */

struct Lcg {
  uint64_t s;
  float next(float lo, float hi) {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return lo + (hi - lo) * (float)((s >> 40) * (1.0 / 16777216.0));
  }
};

const float kIdentity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
const float kIdentity9[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

struct CubeAccel {
  MeshData cube = box(0, 0, 0, 1);
  std::vector<float> env = std::vector<float>(2 * 2 * 4, 1.f);
  std::unique_ptr<nova::aggregate::DeviceAcceleratorInterface> acc;
  explicit CubeAccel(float tx) {
    float m[16], inv[16];
    std::memcpy(m, kIdentity, 64), std::memcpy(inv, kIdentity, 64);
    m[12] = tx, inv[12] = -tx;
    nova::aggregate::mesh_view_s mv = view_of(cube, m, inv, kIdentity9);
    nova::aggregate::material_view_s mat{-1, -1, -1, -1, {0, 0, 0}, {0, 0, 0}, 0.f};
    nova::aggregate::texture_view_s tex{nullptr, env.data(), 2, 2, 4, 0, 0};
    acc = nova::aggregate::DeviceAcceleratorInterface::make();
    acc->build(nova::aggregate::primitive_aggregate_data_s{{&mv, 1}, {&mat, 1}, {&tex, 1}, 0});
  }
  nova::aggregate::B200Accelerator &b200() { return dynamic_cast<nova::aggregate::B200Accelerator &>(*acc); }
  /* hits of rays from `eye` towards `dirs` */
  std::vector<int32_t> hits(const float eye[3], const std::vector<float> &dirs) {
    const size_t n = dirs.size() / 3;
    std::vector<float> o(3 * n), t(n), u(n), v(n);
    std::vector<int32_t> prim(n);
    for (size_t i = 0; i < n; i++) o[3 * i] = eye[0], o[3 * i + 1] = eye[1], o[3 * i + 2] = eye[2];
    CHECK(b200().closestHits(n, o.data(), dirs.data(), prim.data(), t.data(), u.data(), v.data()) == nova::SUCCESS);
    return prim;
  }
};

/* directions through a camera at `eye` looking along +z or -z, spread over +-0.5 of the forward axis */
std::vector<float> frustum_dirs(Lcg &g, float fz, int n) {
  std::vector<float> d;
  for (int i = 0; i < n; i++) {
    const float x = 0.5f * g.next(-1.f, 1.f), y = 0.5f * g.next(-1.f, 1.f);
    const float l = std::sqrt(x * x + y * y + 1.f);
    d.insert(d.end(), {x / l, y / l, fz / l});
  }
  return d;
}

void test_accel() {
  Lcg g{7};
  {
    CubeAccel c(0.f);
    CHECK(c.b200().lastStatus() == nova::SUCCESS);
    /* intersect_inside: from the centre every direction hits a face */
    std::vector<float> d;
    for (int i = 0; i < 100; i++) {
      float x = g.next(-2.f, 2.f), y = g.next(-2.f, 2.f), z = g.next(-2.f, 2.f);
      const float l = std::sqrt(x * x + y * y + z * z) + 1e-6f;
      d.insert(d.end(), {x / l, y / l, z / l});
    }
    const float centre[3] = {0, 0, 0};
    for (int32_t p : c.hits(centre, d)) CHECK(p >= 0);
    /* intersect_outside_front: in front of the cube, looking at it */
    const float front[3] = {0, 0, -2};
    for (int32_t p : c.hits(front, frustum_dirs(g, 1.f, 100))) CHECK(p >= 0);
    /* nointersect_outside_back: just outside a face, looking away */
    const float back[3] = {0, 0, -1.0001f};
    for (int32_t p : c.hits(back, frustum_dirs(g, -1.f, 100))) CHECK(p < 0);
    /* the intersector renders a frame into the caller's partial buffer (renderGpu's traverse) */
    std::vector<float> film(8 * 6 * 4, -1.f);
    nova::device_traversal_param_s prm{};
    prm.render_buffers.partial_buffer = film.data();
    float P[16], V[16];
    perspective(60.f, 8.f / 6.f, 0.1f, 100.f, P);
    const double e[3] = {0, 0, -4}, ctr[3] = {0, 0, 0}, up[3] = {0, 1, 0};
    look_at(e, ctr, up, V);
    auto cam = nova::create_camera();
    cam->setMatrices(P, V);
    cam->getInverseProjectionMatrix(prm.camera.inv_P);
    cam->getInverseViewMatrix(prm.camera.inv_V);
    prm.width = 8, prm.height = 6, prm.depth = 2, prm.sample_index = 0, prm.sample_max = 1;
    c.acc->copyParamsToDevice(prm);
    auto intersector = c.acc->getIntersectorObject();
    intersector->traverse(prm);
    bool all_finite = true, any_written = false;
    for (float x : film) all_finite &= std::isfinite(x), any_written |= x != -1.f;
    CHECK(all_finite && any_written);
    CHECK(c.acc->getMaxRecursiveDepth() >= 16);
    /* an intersector outlives its accelerator's cleanup: it renders the same frame again */
    std::vector<float> first = film;
    c.acc->cleanup();
    CHECK(c.b200().lastStatus() == nova::RENDER_ENGINE_NOT_INITIALIZED);
    std::fill(film.begin(), film.end(), -1.f);
    intersector->traverse(prm);
    CHECK(std::memcmp(film.data(), first.data(), film.size() * 4) == 0);
  }
  {
    /* nointersect_outside_back_translated: the cube 3 units to the right of the view */
    CubeAccel c(3.f);
    const float eye[3] = {0, 0, -1};
    for (int32_t p : c.hits(eye, frustum_dirs(g, 1.f, 100))) CHECK(p < 0);
  }
}

/* ---- render -------------------------------------------------------------------------------- */

struct SceneData {
  std::vector<MeshData> meshes;
  std::vector<std::vector<uint32_t>> u8;    /* 2x2 material textures */
  std::vector<float> env;                   /* 16 x 8 float environment */
  struct Mat {
    int albedo, metallic, normal;
    float eta[3];
  };
  std::vector<Mat> mats;
};

SceneData make_scene() {
  SceneData s;
  s.meshes.push_back(ground(6.0, 0.0));
  s.meshes.push_back(sphere(-1.3, 0.7, 0.0, 0.7, 24, 12));
  s.meshes.push_back(sphere(0.2, 0.6, 0.8, 0.6, 24, 12));
  s.meshes.push_back(box(1.6, 0.5, -0.4, 0.5));
  auto solid = [&](uint32_t c) {
    s.u8.push_back(std::vector<uint32_t>(4, c));
    return (int)s.u8.size() - 1;
  };
  const int flat = solid(rgba8(128, 128, 255));
  /* ground: diffuse grey; sphere 1: rough diffuse red; sphere 2: glossy conductor; box: dielectric */
  s.mats.push_back({solid(rgba8(160, 160, 150)), solid(rgba8(0, 230, 0)), flat, {0, 0, 0}});
  s.mats.push_back({solid(rgba8(200, 60, 40)), solid(rgba8(0, 180, 0)), flat, {0, 0, 0}});
  s.mats.push_back({solid(rgba8(220, 200, 120)), solid(rgba8(0, 70, 255)), flat, {0, 0, 0}});
  s.mats.push_back({solid(rgba8(250, 250, 250)), solid(rgba8(0, 20, 0)), flat, {1.5f, 1.5f, 1.5f}});
  for (int j = 0; j < 8; j++)
    for (int i = 0; i < 16; i++) {
      const float sky = 0.4f + 1.2f * (float)(8 - j) / 8.f;
      s.env.insert(s.env.end(), {sky * 0.8f, sky * 0.9f, sky * (1.0f + 0.05f * (float)i), 1.f});
    }
  return s;
}

void write_bin(const std::string &path, const void *p, size_t bytes) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "cannot write %s\n", path.c_str());
    g_failures++;
    return;
  }
  std::fwrite(p, 1, bytes, f);
  std::fclose(f);
}

void test_render(const std::string &dir) {
  constexpr unsigned W = 64, H = 48, SPP = 8, DEPTH = 4;
  SceneData sd = make_scene();
  /* textures as nova::Texture objects (shared by pointer between materials is not needed here) */
  auto make_u8 = [&](int k) {
    auto t = nova::create_texture();
    t->setTextureBuffer(sd.u8[k].data());
    t->setWidth(2), t->setHeight(2), t->setChannels(4);
    return t;
  };
  auto scene = nova::create_scene();
  for (size_t i = 0; i < sd.meshes.size(); i++) {
    MeshData &m = sd.meshes[i];
    auto tm = nova::create_trimesh();
    tm->registerBufferVertices(m.v.data(), m.v.size());
    tm->registerBufferNormals(m.n.data(), m.n.size());
    tm->registerBufferTangents(m.t.data(), m.t.size());
    tm->registerBufferBitangents(m.b.data(), m.b.size());
    tm->registerBufferUVs(m.uv.data(), m.uv.size());
    tm->registerBufferIndices(m.idx.data(), m.idx.size());
    auto mat = nova::create_material();
    mat->registerAlbedo(make_u8(sd.mats[i].albedo));
    mat->registerMetallic(make_u8(sd.mats[i].metallic));
    mat->registerNormal(make_u8(sd.mats[i].normal));
    mat->setRefractiveIndex(sd.mats[i].eta);
    CHECK(scene->addMesh(std::move(tm), std::move(mat)) == nova::SUCCESS);
  }
  auto env = nova::create_texture();
  env->setTextureBuffer(sd.env.data());
  env->setWidth(16), env->setHeight(8), env->setChannels(4);
  scene->useEnvmap(scene->addEnvmap(std::move(env)));
  float P[16], V[16];
  perspective(55.f, (float)W / H, 0.1f, 100.f, P);
  const double e[3] = {0.3, 2.2, 5.5}, c[3] = {0.0, 0.5, 0.0}, up[3] = {0, 1, 0};
  look_at(e, c, up, V);
  auto cam = nova::create_camera();
  cam->setMatrices(P, V);
  cam->setClipPlaneNear(0.1f), cam->setClipPlaneFar(100.f);
  scene->useCamera(scene->addCamera(std::move(cam)));

  auto engine = nova::create_engine();
  auto opts = nova::create_renderoptions();
  opts->setMaxSamples(SPP), opts->setMaxDepth(DEPTH);
  CHECK(opts->setIntegratorFlag(nova::integrator::PATH | nova::integrator::COMBINED) == nova::SUCCESS);
  auto rb = nova::create_renderbuffer();
  CHECK(rb->resize(W, H) == nova::SUCCESS);
  CHECK(engine->setScene(std::move(scene)) == nova::SUCCESS);
  CHECK(engine->setRenderOptions(std::move(opts)) == nova::SUCCESS);
  CHECK(engine->setRenderBuffers(std::move(rb)) == nova::SUCCESS);
  CHECK(engine->startRender() == nova::SCENE_NOT_PROCESSED);
  CHECK(engine->buildScene() == nova::SUCCESS);
  CHECK(engine->buildAcceleration() == nova::SUCCESS);
  CHECK(engine->prepareRender() == nova::SUCCESS);
  /* the CPU path is not part of this library */
  CHECK(engine->startRender() == nova::INVALID_ENGINE_STATE);
  char log[1024];
  size_t n = 0;
  engine->getRenderEngineError(log, n);
  CHECK(std::strstr(log, "GPU") != nullptr);
  engine->getRenderOptions()->useGpu(true);

  struct Counter : nova::EngineUserCallbackHandler {
    int *pre, *post;
    Counter(int *a, int *b) : pre(a), post(b) {}
    void framePreRenderRoutine() override { (*pre)++; }
    void framePostRenderRoutine() override { (*post)++; }
  };
  int pre = 0, post = 0;
  engine->setUserCallback(std::make_unique<Counter>(&pre, &post));
  CHECK(engine->startRender() == nova::SUCCESS);
  const auto t0 = std::chrono::steady_clock::now();
  while (engine->getFrameIndex() < SPP && std::chrono::steady_clock::now() - t0 < std::chrono::seconds(120))
    std::this_thread::sleep_for(std::chrono::milliseconds(2));
  CHECK(engine->getFrameIndex() == SPP && engine->isRendering());
  CHECK(engine->stopRender() == nova::SUCCESS && !engine->isRendering());
  CHECK(nova::get_error_status(*engine) == nova::exception::NOERR);
  CHECK(pre == (int)SPP && post == (int)SPP);
  engine->getRenderEngineError(log, n);
  std::vector<float> image(engine->getRenderBuffers()->frontBuffer().begin(),
                           engine->getRenderBuffers()->frontBuffer().end());

  /* the same scene through the C ABI, all samples in one call: the progressive mean of one-sample
   * frames equals it bit for bit (samples are summed in sample order either way) */
  nova_b200_ctx *ctx = nullptr;
  CHECK(nova_b200_create(&ctx, 0) == NOVA_B200_SUCCESS);
  std::vector<nova_b200_mesh> meshes;
  std::vector<nova_b200_instance> insts;
  std::vector<nova_b200_material> mats;
  std::vector<nova_b200_texture> texs;
  for (auto &t : sd.u8) texs.push_back(nova_b200_texture{t.data(), nullptr, 2, 2, 4, 1, 0, 0});
  texs.push_back(nova_b200_texture{nullptr, sd.env.data(), 16, 8, 4, 1, 0, 0});
  for (size_t i = 0; i < sd.meshes.size(); i++) {
    MeshData &m = sd.meshes[i];
    meshes.push_back(nova_b200_mesh{m.v.data(), m.n.data(), m.t.data(), m.b.data(), m.uv.data(), m.idx.data(),
                                    (uint32_t)(m.v.size() / 3), (uint32_t)(m.idx.size() / 3)});
    nova_b200_instance x{};
    x.mesh = (uint32_t)i, x.material = (uint32_t)i;
    std::memcpy(x.m, kIdentity, 64), std::memcpy(x.inv, kIdentity, 64), std::memcpy(x.n, kIdentity9, 36);
    insts.push_back(x);
    nova_b200_material mt{};
    mt.albedo = sd.mats[i].albedo, mt.metallic = sd.mats[i].metallic, mt.normalmap = sd.mats[i].normal;
    mt.emissive = -1;
    for (int k = 0; k < 3; k++) mt.eta[k] = sd.mats[i].eta[k];
    mats.push_back(mt);
  }
  nova_b200_scene_desc desc{meshes.data(), (uint32_t)meshes.size(), insts.data(), (uint32_t)insts.size(),
                            mats.data(),   (uint32_t)mats.size(),   texs.data(),  (uint32_t)texs.size(),
                            (int32_t)texs.size() - 1};
  CHECK(nova_b200_upload_scene(ctx, &desc) == NOVA_B200_SUCCESS);
  CHECK(nova_b200_build_bvh(ctx, nullptr) == NOVA_B200_SUCCESS);
  nova_b200_frame f{};
  f.width = W, f.height = H, f.spp_total = SPP, f.sample_begin = 0, f.sample_count = SPP, f.max_depth = DEPTH;
  f.rr_start = -1, f.reset = 1;
  const nova::Camera *ec = engine->getScene()->getCamera(0);
  ec->getInverseProjectionMatrix(f.inv_P);
  ec->getInverseViewMatrix(f.inv_V);
  std::vector<float> direct(W * H * 4);
  CHECK(nova_b200_render(ctx, &f, direct.data(), nullptr, nullptr) == NOVA_B200_SUCCESS);
  size_t mismatched = 0;
  for (size_t i = 0; i < direct.size(); i++) mismatched += std::memcmp(&direct[i], &image[i], 4) != 0;
  CHECK(mismatched == 0);
  if (mismatched) std::fprintf(stderr, "%zu of %zu floats differ from the one-shot render\n", mismatched, direct.size());

  /* the NORMAL pass through the engine equals nova_b200_render_aov */
  CHECK(engine->getRenderOptions()->setIntegratorFlag(nova::integrator::PATH | nova::integrator::NORMAL) ==
        nova::SUCCESS);
  engine->getRenderOptions()->setMaxSamples(1);
  CHECK(engine->startRender() == nova::SUCCESS);
  const auto t1 = std::chrono::steady_clock::now();
  while (engine->getFrameIndex() < 1 && std::chrono::steady_clock::now() - t1 < std::chrono::seconds(60))
    std::this_thread::sleep_for(std::chrono::milliseconds(2));
  CHECK(engine->stopRender() == nova::SUCCESS);
  std::vector<float> normal_engine(engine->getRenderBuffers()->frontBuffer().begin(),
                                   engine->getRenderBuffers()->frontBuffer().end());
  f.spp_total = 1, f.sample_count = 1;
  std::vector<float> normal_direct(W * H * 4);
  CHECK(nova_b200_render_aov(ctx, &f, NOVA_B200_AOV_NORMAL, 0.1f, 100.f, normal_direct.data(), nullptr) ==
        NOVA_B200_SUCCESS);
  CHECK(std::memcmp(normal_engine.data(), normal_direct.data(), normal_direct.size() * 4) == 0);
  /* a frame that fails stops the render and leaves its message */
  CHECK(engine->getRenderOptions()->setIntegratorFlag(nova::integrator::PATH | nova::integrator::COMBINED) ==
        nova::SUCCESS);
  engine->getRenderOptions()->setMaxDepth(100000);
  engine->getRenderOptions()->setMaxSamples(4);
  CHECK(engine->startRender() == nova::SUCCESS);
  const auto t2 = std::chrono::steady_clock::now();
  while (engine->isRendering() && std::chrono::steady_clock::now() - t2 < std::chrono::seconds(60))
    std::this_thread::sleep_for(std::chrono::milliseconds(2));
  CHECK(!engine->isRendering() && engine->getFrameIndex() == 0);
  engine->getRenderEngineError(log, n);
  CHECK(n > 0);
  CHECK(nova::get_error_status(*engine) == nova::exception::GENERAL_ERROR); /* an invalid argument of the frame */
  engine->stopRender();
  CHECK(engine->cleanup() == nova::SUCCESS);
  nova_b200_destroy(ctx);

  /* the scene and image for the oracle: meta, per-mesh attributes, materials, textures, camera */
  std::string meta = std::to_string(W) + " " + std::to_string(H) + " " + std::to_string(SPP) + " " +
                     std::to_string(DEPTH) + " " + std::to_string(sd.meshes.size()) + " " +
                     std::to_string(sd.u8.size()) + "\n";
  for (auto &m : sd.mats)
    meta += std::to_string(m.albedo) + " " + std::to_string(m.metallic) + " " + std::to_string(m.normal) + " " +
            std::to_string(m.eta[0]) + "\n";
  write_bin(dir + "/meta.txt", meta.data(), meta.size());
  for (size_t i = 0; i < sd.meshes.size(); i++) {
    const MeshData &m = sd.meshes[i];
    const std::string p = dir + "/mesh" + std::to_string(i) + "_";
    write_bin(p + "v.bin", m.v.data(), m.v.size() * 4), write_bin(p + "n.bin", m.n.data(), m.n.size() * 4);
    write_bin(p + "t.bin", m.t.data(), m.t.size() * 4), write_bin(p + "b.bin", m.b.data(), m.b.size() * 4);
    write_bin(p + "uv.bin", m.uv.data(), m.uv.size() * 4), write_bin(p + "idx.bin", m.idx.data(), m.idx.size() * 4);
  }
  for (size_t k = 0; k < sd.u8.size(); k++) write_bin(dir + "/tex" + std::to_string(k) + ".bin", sd.u8[k].data(), 16);
  write_bin(dir + "/env.bin", sd.env.data(), sd.env.size() * 4);
  write_bin(dir + "/inv_P.bin", f.inv_P, 64), write_bin(dir + "/inv_V.bin", f.inv_V, 64);
  write_bin(dir + "/image.bin", image.data(), image.size() * 4);
}

}  // namespace

int main(int argc, char **argv) {
  const std::string mode = argc > 1 ? argv[1] : "";
  if (mode == "cpu") {
    test_transform();
    test_camera();
    test_options_and_buffers();
    test_scene();
    test_engine_errors_without_device();
    test_nova_exception();
  } else if (mode == "accel") {
    test_accel();
  } else if (mode == "render" && argc > 2) {
    test_render(argv[2]);
  } else {
    std::fprintf(stderr, "usage: engine_test cpu | accel | render <dir>\n");
    return 2;
  }
  std::printf("%s: %d failed checks\n", mode.c_str(), g_failures);
  return g_failures ? 1 : 0;
}
