/* The Nova engine API (include/nova_b200_api.hpp) over the B200 C ABI (include/nova_b200.h).
 *
 * Host code only: every device operation is a nova_b200_* call.  Scene objects keep non-owning
 * views of the caller's buffers (api/geometry.cpp:17-70, api_texture.h:182) until buildScene()
 * copies them to the device.  The render loop follows NvEngineInstance::renderGpu
 * (corelib/nova/api/engine.cpp:457-496): frame k renders sample k of max_samples into the partial
 * buffer, then writeFramebuffer (:351-363) adds it to the accumulator and writes the running mean
 * to the back buffer, and the buffers swap; the loop runs on its own host thread (the reference uses
 * its thread pool, :555-574) until max_samples frames or stopRender().
 */
#include "../../include/nova_b200_api.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nova_b200.h"

namespace nova {
namespace {

/* ---- column-major 4x4 float matrices, composed like glm (M = M * op) ------------------------ */

struct M4 {
  float a[16]; /* a[col * 4 + row] */
  float &at(int r, int c) { return a[c * 4 + r]; }
  float at(int r, int c) const { return a[c * 4 + r]; }
};

M4 identity() {
  M4 m{};
  for (int i = 0; i < 4; i++) m.at(i, i) = 1.f;
  return m;
}

M4 mul(const M4 &x, const M4 &y) {
  M4 r{};
  for (int c = 0; c < 4; c++)
    for (int rr = 0; rr < 4; rr++) {
      float s = 0.f;
      for (int k = 0; k < 4; k++) s += x.at(rr, k) * y.at(k, c);
      r.at(rr, c) = s;
    }
  return r;
}

/* Inverse by cofactors in double, rounded once to float; a singular matrix gives NaNs, as glm's
 * division by a zero determinant does. */
M4 inverse(const M4 &m) {
  double s[16];
  for (int i = 0; i < 16; i++) s[i] = m.a[i];
  double inv[16];
  inv[0] = s[5] * s[10] * s[15] - s[5] * s[11] * s[14] - s[9] * s[6] * s[15] + s[9] * s[7] * s[14] + s[13] * s[6] * s[11] - s[13] * s[7] * s[10];
  inv[4] = -s[4] * s[10] * s[15] + s[4] * s[11] * s[14] + s[8] * s[6] * s[15] - s[8] * s[7] * s[14] - s[12] * s[6] * s[11] + s[12] * s[7] * s[10];
  inv[8] = s[4] * s[9] * s[15] - s[4] * s[11] * s[13] - s[8] * s[5] * s[15] + s[8] * s[7] * s[13] + s[12] * s[5] * s[11] - s[12] * s[7] * s[9];
  inv[12] = -s[4] * s[9] * s[14] + s[4] * s[10] * s[13] + s[8] * s[5] * s[14] - s[8] * s[6] * s[13] - s[12] * s[5] * s[10] + s[12] * s[6] * s[9];
  inv[1] = -s[1] * s[10] * s[15] + s[1] * s[11] * s[14] + s[9] * s[2] * s[15] - s[9] * s[3] * s[14] - s[13] * s[2] * s[11] + s[13] * s[3] * s[10];
  inv[5] = s[0] * s[10] * s[15] - s[0] * s[11] * s[14] - s[8] * s[2] * s[15] + s[8] * s[3] * s[14] + s[12] * s[2] * s[11] - s[12] * s[3] * s[10];
  inv[9] = -s[0] * s[9] * s[15] + s[0] * s[11] * s[13] + s[8] * s[1] * s[15] - s[8] * s[3] * s[13] - s[12] * s[1] * s[11] + s[12] * s[3] * s[9];
  inv[13] = s[0] * s[9] * s[14] - s[0] * s[10] * s[13] - s[8] * s[1] * s[14] + s[8] * s[2] * s[13] + s[12] * s[1] * s[10] - s[12] * s[2] * s[9];
  inv[2] = s[1] * s[6] * s[15] - s[1] * s[7] * s[14] - s[5] * s[2] * s[15] + s[5] * s[3] * s[14] + s[13] * s[2] * s[7] - s[13] * s[3] * s[6];
  inv[6] = -s[0] * s[6] * s[15] + s[0] * s[7] * s[14] + s[4] * s[2] * s[15] - s[4] * s[3] * s[14] - s[12] * s[2] * s[7] + s[12] * s[3] * s[6];
  inv[10] = s[0] * s[5] * s[15] - s[0] * s[7] * s[13] - s[4] * s[1] * s[15] + s[4] * s[3] * s[13] + s[12] * s[1] * s[7] - s[12] * s[3] * s[5];
  inv[14] = -s[0] * s[5] * s[14] + s[0] * s[6] * s[13] + s[4] * s[1] * s[14] - s[4] * s[2] * s[13] - s[12] * s[1] * s[6] + s[12] * s[2] * s[5];
  inv[3] = -s[1] * s[6] * s[11] + s[1] * s[7] * s[10] + s[5] * s[2] * s[11] - s[5] * s[3] * s[10] - s[9] * s[2] * s[7] + s[9] * s[3] * s[6];
  inv[7] = s[0] * s[6] * s[11] - s[0] * s[7] * s[10] - s[4] * s[2] * s[11] + s[4] * s[3] * s[10] + s[8] * s[2] * s[7] - s[8] * s[3] * s[6];
  inv[11] = -s[0] * s[5] * s[11] + s[0] * s[7] * s[9] + s[4] * s[1] * s[11] - s[4] * s[3] * s[9] - s[8] * s[1] * s[7] + s[8] * s[3] * s[5];
  inv[15] = s[0] * s[5] * s[10] - s[0] * s[6] * s[9] - s[4] * s[1] * s[10] + s[4] * s[2] * s[9] + s[8] * s[1] * s[6] - s[8] * s[2] * s[5];
  const double det = s[0] * inv[0] + s[1] * inv[4] + s[2] * inv[8] + s[3] * inv[12];
  M4 r{};
  for (int i = 0; i < 16; i++) r.a[i] = (float)(inv[i] / det);
  return r;
}

M4 transposed(const M4 &m) {
  M4 r{};
  for (int c = 0; c < 4; c++)
    for (int rr = 0; rr < 4; rr++) r.at(rr, c) = m.at(c, rr);
  return r;
}

M4 translation(float x, float y, float z) {
  M4 m = identity();
  m.at(0, 3) = x, m.at(1, 3) = y, m.at(2, 3) = z;
  return m;
}

M4 scaling(float x, float y, float z) {
  M4 m = identity();
  m.at(0, 0) = x, m.at(1, 1) = y, m.at(2, 2) = z;
  return m;
}

/* rotation matrix of a normalised quaternion (x, y, z, w) */
M4 quat_matrix(float x, float y, float z, float w) {
  const float n = std::sqrt(x * x + y * y + z * z + w * w);
  if (n > 0.f) x /= n, y /= n, z /= n, w /= n;
  M4 m = identity();
  m.at(0, 0) = 1.f - 2.f * (y * y + z * z), m.at(0, 1) = 2.f * (x * y - w * z), m.at(0, 2) = 2.f * (x * z + w * y);
  m.at(1, 0) = 2.f * (x * y + w * z), m.at(1, 1) = 1.f - 2.f * (x * x + z * z), m.at(1, 2) = 2.f * (y * z - w * x);
  m.at(2, 0) = 2.f * (x * z - w * y), m.at(2, 1) = 2.f * (y * z + w * x), m.at(2, 2) = 1.f - 2.f * (x * x + y * y);
  return m;
}

/* rotation by `angle` radians about the (normalised) axis */
M4 axis_rotation(float angle, float x, float y, float z) {
  const float h = 0.5f * angle, s = std::sin(h);
  return quat_matrix(x * s, y * s, z * s, std::cos(h));
}

float column_length(const M4 &m, int c) {
  return std::sqrt(m.at(0, c) * m.at(0, c) + m.at(1, c) * m.at(1, c) + m.at(2, c) * m.at(2, c));
}

/* quaternion (x, y, z, w) of the rotation part, by the largest-diagonal method */
void matrix_quat(const M4 &m, float q[4]) {
  const float t = m.at(0, 0) + m.at(1, 1) + m.at(2, 2);
  float x, y, z, w;
  if (t > 0.f) {
    const float s = std::sqrt(t + 1.f) * 2.f;
    w = 0.25f * s, x = (m.at(2, 1) - m.at(1, 2)) / s, y = (m.at(0, 2) - m.at(2, 0)) / s, z = (m.at(1, 0) - m.at(0, 1)) / s;
  } else if (m.at(0, 0) > m.at(1, 1) && m.at(0, 0) > m.at(2, 2)) {
    const float s = std::sqrt(1.f + m.at(0, 0) - m.at(1, 1) - m.at(2, 2)) * 2.f;
    w = (m.at(2, 1) - m.at(1, 2)) / s, x = 0.25f * s, y = (m.at(0, 1) + m.at(1, 0)) / s, z = (m.at(0, 2) + m.at(2, 0)) / s;
  } else if (m.at(1, 1) > m.at(2, 2)) {
    const float s = std::sqrt(1.f + m.at(1, 1) - m.at(0, 0) - m.at(2, 2)) * 2.f;
    w = (m.at(0, 2) - m.at(2, 0)) / s, x = (m.at(0, 1) + m.at(1, 0)) / s, y = 0.25f * s, z = (m.at(1, 2) + m.at(2, 1)) / s;
  } else {
    const float s = std::sqrt(1.f + m.at(2, 2) - m.at(0, 0) - m.at(1, 1)) * 2.f;
    w = (m.at(1, 0) - m.at(0, 1)) / s, x = (m.at(0, 2) + m.at(2, 0)) / s, y = (m.at(1, 2) + m.at(2, 1)) / s, z = 0.25f * s;
  }
  q[0] = x, q[1] = y, q[2] = z, q[3] = w;
}

/* ---- scene objects ------------------------------------------------------------------------ */

class B200Transform final : public Transform {
  M4 m_ = identity();

 public:
  void clone(const Transform &other) override { other.getTransformMatrix(m_.a); }
  void setTransformMatrix(const float t[16]) override { std::memcpy(m_.a, t, sizeof(m_.a)); }
  void rotateQuat(float x, float y, float z, float w) override { m_ = mul(m_, quat_matrix(x, y, z, w)); }
  void rotateEuler(float angle, float x, float y, float z) override {
    const float len = std::sqrt(x * x + y * y + z * z);
    if (len > 0.f) m_ = mul(m_, axis_rotation(angle, x / len, y / len, z / len));
  }
  void reset() override { m_ = identity(); }
  void getTransformMatrix(float t[16]) const override { std::memcpy(t, m_.a, sizeof(m_.a)); }
  void translate(float x, float y, float z) override { m_ = mul(m_, translation(x, y, z)); }
  void scale(float s) override { m_ = mul(m_, scaling(s, s, s)); }
  void scale(float x, float y, float z) override { m_ = mul(m_, scaling(x, y, z)); }
  /* api/transform.cpp: the new matrix is scale(current scale) then translate, rotation dropped */
  void setTranslation(float x, float y, float z) override {
    const float sx = column_length(m_, 0), sy = column_length(m_, 1), sz = column_length(m_, 2);
    m_ = mul(scaling(sx, sy, sz), translation(x, y, z));
  }
  void getTranslation(float t[3]) const override { t[0] = m_.at(0, 3), t[1] = m_.at(1, 3), t[2] = m_.at(2, 3); }
  void setScale(float x, float y, float z) override {
    const float tx = m_.at(0, 3), ty = m_.at(1, 3), tz = m_.at(2, 3);
    m_ = mul(scaling(x, y, z), translation(tx, ty, tz));
  }
  void getScale(float s[3]) const override {
    s[0] = column_length(m_, 0), s[1] = column_length(m_, 1), s[2] = column_length(m_, 2);
  }
  void getRotation(float q[4]) const override { matrix_quat(m_, q); }
  void setRotation(const float q[4]) override {
    const float tx = m_.at(0, 3), ty = m_.at(1, 3), tz = m_.at(2, 3);
    const float sx = column_length(m_, 0), sy = column_length(m_, 1), sz = column_length(m_, 2);
    m_ = mul(mul(scaling(sx, sy, sz), translation(tx, ty, tz)), quat_matrix(q[0], q[1], q[2], q[3]));
  }
  void multiply(const Transform &other) override {
    M4 o{};
    other.getTransformMatrix(o.a);
    m_ = mul(m_, o);
  }
  void invert(float out[16]) const override { std::memcpy(out, inverse(m_).a, 16 * sizeof(float)); }
  void transpose(float out[16]) const override { std::memcpy(out, transposed(m_).a, 16 * sizeof(float)); }
  /* transpose(mat3(inverse(m))), column-major 3x3 */
  void transposeInvert(float out[9]) const override {
    const M4 inv = inverse(m_);
    for (int c = 0; c < 3; c++)
      for (int r = 0; r < 3; r++) out[c * 3 + r] = inv.at(c, r);
  }
};

class B200Trimesh final : public Trimesh {
  std::span<float> v_, n_, t_, b_, c_, uv_;
  std::span<unsigned> idx_;
  TransformPtr transform_ = create_transform();

 public:
  ERROR_STATE registerTransform(TransformPtr t) override {
    if (!t) return INVALID_ARGUMENT;
    transform_ = std::move(t);
    return SUCCESS;
  }
  const Transform &getTransform() const override { return *transform_; }
  ERROR_STATE registerBufferVertices(float *p, size_t n) override { return set(v_, p, n); }
  ERROR_STATE registerBufferNormals(float *p, size_t n) override { return set(n_, p, n); }
  ERROR_STATE registerBufferTangents(float *p, size_t n) override { return set(t_, p, n); }
  ERROR_STATE registerBufferBitangents(float *p, size_t n) override { return set(b_, p, n); }
  ERROR_STATE registerBufferColors(float *p, size_t n) override { return set(c_, p, n); }
  ERROR_STATE registerBufferUVs(float *p, size_t n) override { return set(uv_, p, n); }
  ERROR_STATE registerBufferIndices(unsigned *p, size_t n) override {
    if (!p && n) return INVALID_ARGUMENT;
    idx_ = std::span<unsigned>(p, n);
    return SUCCESS;
  }
  /* GL buffer objects: no graphics stack on a compute-only host */
  ERROR_STATE registerInteropVertices(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE registerInteropNormals(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE registerInteropTangents(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE registerInteropBitangents(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE registerInteropColors(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE registerInteropUVs(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE registerInteropIndices(uint32_t) override { return NOT_GPU_BUILD; }
  std::span<float> getVertices() const override { return v_; }
  std::span<float> getNormals() const override { return n_; }
  std::span<float> getTangents() const override { return t_; }
  std::span<float> getBitangents() const override { return b_; }
  std::span<float> getColors() const override { return c_; }
  std::span<float> getUVs() const override { return uv_; }
  std::span<unsigned> getIndices() const override { return idx_; }
  uint32_t getInteropVertices() const override { return 0; }
  uint32_t getInteropNormals() const override { return 0; }
  uint32_t getInteropTangents() const override { return 0; }
  uint32_t getInteropBitangents() const override { return 0; }
  uint32_t getInteropColors() const override { return 0; }
  uint32_t getInteropUVs() const override { return 0; }
  uint32_t getInteropIndices() const override { return 0; }

 private:
  static ERROR_STATE set(std::span<float> &s, float *p, size_t n) {
    if (!p && n) return INVALID_ARGUMENT;
    s = std::span<float>(p, n);
    return SUCCESS;
  }
};

class B200Texture final : public Texture {
  const void *data_ = nullptr;
  texture::FORMAT format_ = texture::UINT8X4;
  unsigned w_ = 0, h_ = 0, c_ = 4;
  bool inv_x_ = false, inv_y_ = false;

 public:
  ERROR_STATE setWidth(unsigned w) override { return w_ = w, SUCCESS; }
  ERROR_STATE setHeight(unsigned h) override { return h_ = h, SUCCESS; }
  ERROR_STATE setChannels(unsigned c) override { return c_ = c, SUCCESS; }
  ERROR_STATE setInteropID(uint32_t) override { return NOT_GPU_BUILD; }
  ERROR_STATE invertY() override { return inv_y_ = !inv_y_, SUCCESS; }
  ERROR_STATE invertX() override { return inv_x_ = !inv_x_, SUCCESS; }
  const void *getTextureBuffer() const override { return data_; }
  unsigned getWidth() const override { return w_; }
  unsigned getHeight() const override { return h_; }
  unsigned getChannels() const override { return c_; }
  uint32_t getInteropID() const override { return 0; }
  bool getInvertY() const override { return inv_y_; }
  bool getInvertX() const override { return inv_x_; }
  texture::FORMAT getFormat() const override { return format_; }

 protected:
  ERROR_STATE setData(const uint32_t *b) override {
    if (!b) return INVALID_ARGUMENT;
    data_ = b, format_ = texture::UINT8X4;
    return SUCCESS;
  }
  ERROR_STATE setData(const float *b) override {
    if (!b) return INVALID_ARGUMENT;
    data_ = b, format_ = texture::FLOATX4;
    return SUCCESS;
  }
};

class B200Material final : public Material {
  TexturePtr albedo_, normal_, metallic_, emissive_, roughness_, opacity_, specular_, ao_;
  float eta_[3] = {0, 0, 0}, k_[3] = {0, 0, 0};
  float aniso_ = 0.f;
  static ERROR_STATE put(TexturePtr &slot, TexturePtr t) {
    if (!t) return INVALID_ARGUMENT;
    slot = std::move(t);
    return SUCCESS;
  }

 public:
  ERROR_STATE registerAlbedo(TexturePtr t) override { return put(albedo_, std::move(t)); }
  ERROR_STATE registerNormal(TexturePtr t) override { return put(normal_, std::move(t)); }
  ERROR_STATE registerMetallic(TexturePtr t) override { return put(metallic_, std::move(t)); }
  ERROR_STATE registerEmissive(TexturePtr t) override { return put(emissive_, std::move(t)); }
  ERROR_STATE registerRoughness(TexturePtr t) override { return put(roughness_, std::move(t)); }
  ERROR_STATE registerOpacity(TexturePtr t) override { return put(opacity_, std::move(t)); }
  ERROR_STATE registerSpecular(TexturePtr t) override { return put(specular_, std::move(t)); }
  ERROR_STATE registerAmbientOcclusion(TexturePtr t) override { return put(ao_, std::move(t)); }
  ERROR_STATE setRefractiveIndex(const float eta[3]) override {
    for (int i = 0; i < 3; i++) eta_[i] = eta[i];
    return SUCCESS;
  }
  ERROR_STATE setRefractiveIndex(const float eta[3], const float k[3]) override {
    for (int i = 0; i < 3; i++) eta_[i] = eta[i], k_[i] = k[i];
    return SUCCESS;
  }
  ERROR_STATE setAnisotropyFactor(float a) override { return aniso_ = a, SUCCESS; }
  Texture *getAlbedo() override { return albedo_.get(); }
  const Texture *getAlbedo() const override { return albedo_.get(); }
  Texture *getNormal() override { return normal_.get(); }
  const Texture *getNormal() const override { return normal_.get(); }
  Texture *getMetallic() override { return metallic_.get(); }
  const Texture *getMetallic() const override { return metallic_.get(); }
  Texture *getEmissive() override { return emissive_.get(); }
  const Texture *getEmissive() const override { return emissive_.get(); }
  Texture *getRoughness() override { return roughness_.get(); }
  const Texture *getRoughness() const override { return roughness_.get(); }
  Texture *getOpacity() override { return opacity_.get(); }
  const Texture *getOpacity() const override { return opacity_.get(); }
  Texture *getSpecular() override { return specular_.get(); }
  const Texture *getSpecular() const override { return specular_.get(); }
  Texture *getAmbientOcclusion() override { return ao_.get(); }
  const Texture *getAmbientOcclusion() const override { return ao_.get(); }
  void getRefractiveIndex(float eta[3], float k[3]) const override {
    for (int i = 0; i < 3; i++) eta[i] = eta_[i], k[i] = k_[i];
  }
  float getAnisotropyFactor() const override { return aniso_; }
};

/* api/camera.cpp: the inverses are computed when the matrices are set */
class B200Camera final : public Camera {
  M4 P_ = identity(), V_ = identity(), iP_ = identity(), iV_ = identity(), PV_ = identity(), iPV_ = identity();
  float up_[3] = {0, 1, 0}, pos_[3] = {0, 0, 0}, dir_[3] = {0, 0, -1};
  float near_ = 0.1f, far_ = 1000.f, fov_ = 45.f;
  unsigned w_ = 0, h_ = 0;
  static void copy3(float *d, const float *s) { d[0] = s[0], d[1] = s[1], d[2] = s[2]; }

 public:
  ERROR_STATE setUpVector(const float up[3]) override { return copy3(up_, up), SUCCESS; }
  ERROR_STATE setMatrices(const float p[16], const float v[16]) override {
    std::memcpy(P_.a, p, 64);
    std::memcpy(V_.a, v, 64);
    iP_ = inverse(P_), iV_ = inverse(V_);
    PV_ = mul(P_, V_);
    iPV_ = inverse(PV_);
    return SUCCESS;
  }
  ERROR_STATE setPosition(const float p[3]) override { return copy3(pos_, p), SUCCESS; }
  ERROR_STATE setDirection(const float d[3]) override { return copy3(dir_, d), SUCCESS; }
  ERROR_STATE setClipPlaneFar(float f) override { return far_ = f, SUCCESS; }
  ERROR_STATE setClipPlaneNear(float n) override { return near_ = n, SUCCESS; }
  ERROR_STATE setResolutionWidth(unsigned w) override { return w_ = w, SUCCESS; }
  ERROR_STATE setResolutionHeight(unsigned h) override { return h_ = h, SUCCESS; }
  ERROR_STATE setFov(float f) override { return fov_ = f, SUCCESS; }
  ERROR_STATE getUpVector(float up[3]) const override { return copy3(up, up_), SUCCESS; }
  ERROR_STATE getProjectionMatrix(float o[16]) const override { return std::memcpy(o, P_.a, 64), SUCCESS; }
  ERROR_STATE getViewMatrix(float o[16]) const override { return std::memcpy(o, V_.a, 64), SUCCESS; }
  ERROR_STATE getInverseProjectionMatrix(float o[16]) const override { return std::memcpy(o, iP_.a, 64), SUCCESS; }
  ERROR_STATE getInverseViewMatrix(float o[16]) const override { return std::memcpy(o, iV_.a, 64), SUCCESS; }
  ERROR_STATE getProjectionViewMatrix(float o[16]) const override { return std::memcpy(o, PV_.a, 64), SUCCESS; }
  ERROR_STATE getInverseProjectionViewMatrix(float o[16]) const override {
    return std::memcpy(o, iPV_.a, 64), SUCCESS;
  }
  ERROR_STATE getPosition(float p[3]) const override { return copy3(p, pos_), SUCCESS; }
  ERROR_STATE getDirection(float d[3]) const override { return copy3(d, dir_), SUCCESS; }
  float getClipPlaneFar() const override { return far_; }
  float getClipPlaneNear() const override { return near_; }
  unsigned getResolutionWidth() const override { return w_; }
  unsigned getResolutionHeight() const override { return h_; }
  float getFov() const override { return fov_; }
};

class B200RenderOptions final : public RenderOptions {
  unsigned aa_ = 0, depth_ = 0, samples_ = 0, inc_ = 0, tw_ = 0, th_ = 0;
  int flag_ = 0;
  bool gpu_ = false, flip_ = false;

 public:
  void setAliasingSamples(unsigned s) override { aa_ = s; }
  unsigned getAliasingSamples() const override { return aa_; }
  void setMaxDepth(unsigned d) override { depth_ = d; }
  unsigned getMaxDepth() const override { return depth_; }
  void setMaxSamples(unsigned s) override { samples_ = s; }
  unsigned getMaxSamples() const override { return samples_; }
  void setSamplesIncrement(unsigned i) override { inc_ = i; }
  unsigned getSamplesIncrement() const override { return inc_; }
  void setTileDimension(unsigned w, unsigned h) override { tw_ = w, th_ = h; }
  unsigned getTileDimensionWidth() const override { return tw_; }
  unsigned getTileDimensionHeight() const override { return th_; }
  /* api/renderoption.cpp: at most one of the integrator bits 0-7 */
  ERROR_STATE setIntegratorFlag(int f) override {
    int n = 0;
    for (int i = 0; i <= 7; i++) n += (f >> i) & 1;
    if (n >= 2) return MULTIPLE_INTEGRATORS_NOT_SUPPORTED;
    flag_ = f;
    return SUCCESS;
  }
  int getIntegratorFlag() const override { return flag_; }
  ERROR_STATE useGpu(bool use) override { return gpu_ = use, SUCCESS; }
  bool isUsingGpu() const override { return gpu_; }
  ERROR_STATE useInterops(bool use) override { return use ? NOT_GPU_BUILD : SUCCESS; }
  bool isUsingInterops() const override { return false; }
  void flipV() override { flip_ = !flip_; }
  bool isFlippedV() const override { return flip_; }
};

/* api/renderbuffer.cpp: front / back colour buffers, the partial (one frame) and accumulator
 * buffers, depth and normal buffers; the sample* accessors read the front buffer at
 * (x * height + y) * channels, as the reference's do. */
class B200RenderBuffer final : public RenderBuffer {
  std::vector<float> front_, back_, partial_, accum_, depth_, normal_;
  float *back_ptr_ = nullptr, *front_ptr_ = nullptr;
  unsigned w_ = 0, h_ = 0;
  size_t cap_ = 0;
  static constexpr unsigned kColor = 4, kDepth = 1, kNormal = 3;

 public:
  unsigned getChannel(texture::CHANNEL_TYPE t) const override {
    return t == texture::DEPTH ? kDepth : (t == texture::NORMAL ? kNormal : kColor);
  }
  ERROR_STATE resetBuffers() override {
    for (auto *v : {&front_, &back_, &partial_, &accum_, &depth_, &normal_}) std::fill(v->begin(), v->end(), 0.f);
    return SUCCESS;
  }
  ERROR_STATE preallocate(unsigned w, unsigned h) override {
    try {
      cap_ = (size_t)w * h;
      front_.assign(cap_ * kColor, 0.f), back_.assign(cap_ * kColor, 0.f);
      partial_.assign(cap_ * kColor, 0.f), accum_.assign(cap_ * kColor, 0.f);
      depth_.assign(cap_ * kDepth, 0.f), normal_.assign(cap_ * kNormal, 0.f);
    } catch (...) {
      return OUT_OF_MEMORY;
    }
    back_ptr_ = back_.data(), front_ptr_ = front_.data();
    return SUCCESS;
  }
  ERROR_STATE resize(unsigned w, unsigned h) override {
    ERROR_STATE e = SUCCESS;
    if (cap_ < (size_t)w * h) e = preallocate(w, h);
    w_ = w, h_ = h;
    return e;
  }
  HdrBufferStruct getRenderBuffers() const override {
    HdrBufferStruct b{};
    b.partial_buffer = const_cast<float *>(partial_.data());
    b.depth_buffer = const_cast<float *>(depth_.data());
    b.normal_buffer = const_cast<float *>(normal_.data());
    b.channels = (int)kColor;
    b.byte_size_color_buffers = (size_t)w_ * h_ * kColor * sizeof(float);
    b.byte_size_depth_buffers = (size_t)w_ * h_ * kDepth * sizeof(float);
    b.color_buffers_pitch = (size_t)w_ * kColor * sizeof(float);
    b.depth_buffers_pitch = (size_t)w_ * kDepth * sizeof(float);
    b.normal_buffers_pitch = (size_t)w_ * kNormal * sizeof(float);
    return b;
  }
  FloatView backBuffer() override { return FloatView(back_ptr_, (size_t)w_ * h_ * kColor); }
  FloatView frontBuffer() override { return FloatView(front_ptr_, (size_t)w_ * h_ * kColor); }
  void swapBackBuffer() override { std::swap(back_ptr_, front_ptr_); }
  FloatView getAccumulator() const override {
    return FloatView(const_cast<float *>(accum_.data()), (size_t)w_ * h_ * kColor);
  }
  Framebuffer getFramebuffer() const override {
    Framebuffer f{};
    f.color_buffer = FloatView(front_ptr_, (size_t)w_ * h_ * kColor);
    f.color_buffer_channels = kColor, f.color_buffer_width = w_, f.color_buffer_height = h_;
    f.depth_buffer = FloatView(const_cast<float *>(depth_.data()), (size_t)w_ * h_ * kDepth);
    f.depth_buffer_width = w_, f.depth_buffer_height = h_;
    f.normal_buffer = FloatView(const_cast<float *>(normal_.data()), (size_t)w_ * h_ * kNormal);
    f.normal_buffer_channels = kNormal, f.normal_buffer_width = w_, f.normal_buffer_height = h_;
    return f;
  }
  unsigned getWidth() const override { return w_; }
  unsigned getHeight() const override { return h_; }
  frgba_s sampleColor(unsigned x, unsigned y) const override {
    const size_t i = ((size_t)x * h_ + y) * kColor;
    return frgba_s{front_ptr_[i], front_ptr_[i + 1], front_ptr_[i + 2], front_ptr_[i + 3]};
  }
  frgb_s sampleNormal(unsigned x, unsigned y) const override {
    const size_t i = ((size_t)x * h_ + y) * kNormal;
    return frgb_s{front_ptr_[i], front_ptr_[i + 1], front_ptr_[i + 2]};
  }
  float sampleDepth(unsigned x, unsigned y) const override { return front_ptr_[((size_t)x * h_ + y) * kDepth]; }
};

class B200Scene final : public Scene {
  std::vector<TrimeshPtr> meshes_;
  std::vector<MaterialPtr> materials_;
  std::vector<TexturePtr> envmaps_;
  std::vector<CameraPtr> cameras_;
  TransformPtr root_ = create_transform();
  int envmap_ = -1, camera_ = -1;

 public:
  ERROR_STATE addMesh(TrimeshPtr mesh, MaterialPtr material) override {
    if (!mesh || !material) return INVALID_ARGUMENT;
    meshes_.push_back(std::move(mesh));
    materials_.push_back(std::move(material));
    return SUCCESS;
  }
  unsigned addEnvmap(TexturePtr t) override {
    envmaps_.push_back(std::move(t));
    return (unsigned)envmaps_.size() - 1;
  }
  ERROR_STATE useEnvmap(unsigned id) override {
    if (id >= envmaps_.size()) return INVALID_ARGUMENT;
    envmap_ = (int)id;
    return SUCCESS;
  }
  Texture *getEnvmap(unsigned id) override { return id < envmaps_.size() ? envmaps_[id].get() : nullptr; }
  const Texture *getEnvmap(unsigned id) const override { return id < envmaps_.size() ? envmaps_[id].get() : nullptr; }
  void clearEnvmaps() override { envmaps_.clear(), envmap_ = -1; }
  int getCurrentEnvmapId() const override { return envmap_; }
  ERROR_STATE setRootTransform(TransformPtr t) override {
    if (!t) return INVALID_ARGUMENT;
    root_ = std::move(t);
    return SUCCESS;
  }
  unsigned addCamera(CameraPtr c) override {
    cameras_.push_back(std::move(c));
    return (unsigned)cameras_.size() - 1;
  }
  void clearCameras() override { cameras_.clear(), camera_ = -1; }
  ERROR_STATE useCamera(unsigned id) override {
    if (id >= cameras_.size()) return INVALID_ARGUMENT;
    camera_ = (int)id;
    return SUCCESS;
  }
  int getCurrentCameraId() const override { return camera_; }
  Camera *getCamera(unsigned id) override { return id < cameras_.size() ? cameras_[id].get() : nullptr; }
  const Camera *getCamera(unsigned id) const override { return id < cameras_.size() ? cameras_[id].get() : nullptr; }
  void cleanup() override {
    meshes_.clear(), materials_.clear(), envmaps_.clear(), cameras_.clear();
    envmap_ = camera_ = -1;
  }
  unsigned getPrimitivesNum(mesh::TYPE type) const override {
    if (type != mesh::TRIANGLE) return 0;
    size_t n = 0;
    for (const auto &m : meshes_) n += m->getIndices().size() / 3;
    return (unsigned)n;
  }
  unsigned getMeshesNum(mesh::TYPE type) const override { return type == mesh::TRIANGLE ? (unsigned)meshes_.size() : 0; }
  CsteTriMeshCollection getTriangleMeshCollection() const override { return CsteTriMeshCollection(meshes_); }
  CsteMaterialCollection getMaterialCollection(mesh::TYPE type) const override {
    return type == mesh::TRIANGLE ? CsteMaterialCollection(materials_) : CsteMaterialCollection();
  }
  CsteCameraCollection getCameraCollection() const override { return CsteCameraCollection(cameras_); }
  CsteTextureCollection getEnvmapCollection() const override { return CsteTextureCollection(envmaps_); }
};

/* ---- the C-ABI scene description shared by the engine and the accelerator ----------------- */

std::string status_text(nova_b200_ctx *ctx) {
  char buf[1024] = {0};
  size_t n = 0;
  nova_b200_get_error(ctx, buf, &n);
  return std::string(buf, n);
}

/* Uploads and builds a scene given as aggregate views; returns the status and sets *err. */
ERROR_STATE upload_views(nova_b200_ctx *ctx, const aggregate::primitive_aggregate_data_s &d, std::string *err) {
  if (d.meshes.empty()) return *err = "scene has no meshes", INVALID_SCENE_TYPE;
  std::vector<nova_b200_mesh> meshes(d.meshes.size());
  std::vector<nova_b200_instance> insts(d.meshes.size());
  for (size_t i = 0; i < d.meshes.size(); i++) {
    const aggregate::mesh_view_s &m = d.meshes[i];
    const size_t nv = m.vertices.size() / 3;
    if (nv == 0 || m.indices.size() < 3 || m.normals.size() != 3 * nv || m.tangents.size() != 3 * nv ||
        m.bitangents.size() != 3 * nv || m.uv.size() != 2 * nv)
      return *err = "mesh " + std::to_string(i) +
                    " needs vertices, normals, tangents, bitangents (3 floats per vertex), uv (2) and indices",
             INVALID_ARGUMENT;
    meshes[i] = nova_b200_mesh{m.vertices.data(), m.normals.data(), m.tangents.data(), m.bitangents.data(),
                               m.uv.data(), m.indices.data(), (uint32_t)nv, (uint32_t)(m.indices.size() / 3)};
    nova_b200_instance &x = insts[i];
    x.mesh = (uint32_t)i;
    x.material = m.material;
    std::memcpy(x.m, m.m, sizeof(x.m));
    std::memcpy(x.inv, m.inv, sizeof(x.inv));
    std::memcpy(x.n, m.n, sizeof(x.n));
  }
  std::vector<nova_b200_material> mats(d.materials.size());
  for (size_t i = 0; i < d.materials.size(); i++) {
    const aggregate::material_view_s &s = d.materials[i];
    nova_b200_material &o = mats[i];
    o.albedo = s.albedo, o.metallic = s.metallic, o.normalmap = s.normalmap, o.emissive = s.emissive;
    for (int k = 0; k < 3; k++) o.eta[k] = s.eta[k], o.k[k] = s.k[k];
    o.anisotropy = s.anisotropy;
  }
  std::vector<nova_b200_texture> texs(d.textures.size());
  for (size_t i = 0; i < d.textures.size(); i++) {
    const aggregate::texture_view_s &t = d.textures[i];
    texs[i] = nova_b200_texture{t.u8_pixels, t.f32_pixels, t.width, t.height, t.channels, 1, t.invert_u, t.invert_v};
  }
  nova_b200_scene_desc desc{meshes.data(), (uint32_t)meshes.size(), insts.data(), (uint32_t)insts.size(),
                            mats.data(),   (uint32_t)mats.size(),   texs.data(),  (uint32_t)texs.size(),
                            d.envmap};
  nova_b200_status st = nova_b200_upload_scene(ctx, &desc);
  if (st == NOVA_B200_SUCCESS) st = nova_b200_build_bvh(ctx, nullptr);
  if (st != NOVA_B200_SUCCESS) *err = status_text(ctx);
  return (ERROR_STATE)st;
}

/* Views of a Scene: one instance per mesh with the mesh's transform (api/engine.cpp:155-175), the
 * material's texture pack (api/material.cpp:212-226; albedo, metallic, normal and emissive reach the
 * device), and the current environment map (:273-290).  Textures are shared by pointer. */
struct SceneViews {
  std::vector<aggregate::mesh_view_s> meshes;
  std::vector<aggregate::material_view_s> materials;
  std::vector<aggregate::texture_view_s> textures;
  int32_t envmap = -1;
};

ERROR_STATE scene_views(const Scene &scene, SceneViews &v, std::string *err) {
  std::map<const Texture *, int32_t> tex_index;
  auto texture_of = [&](const Texture *t, bool material_slot, int32_t *out) -> ERROR_STATE {
    *out = -1;
    if (!t) return SUCCESS;
    auto it = tex_index.find(t);
    if (it != tex_index.end()) return *out = it->second, SUCCESS;
    if (!t->getTextureBuffer() || t->getWidth() < 2 || t->getHeight() < 2)
      return *err = "texture without pixels or smaller than 2 x 2", INVALID_CHANNEL_DESCRIPTOR;
    if (material_slot && t->getFormat() != texture::UINT8X4)
      return *err = "material textures must be 8-bit RGBA (api/material.cpp:185)", INVALID_CHANNEL_DESCRIPTOR;
    aggregate::texture_view_s tv{};
    if (t->getFormat() == texture::UINT8X4)
      tv.u8_pixels = static_cast<const uint32_t *>(t->getTextureBuffer());
    else
      tv.f32_pixels = static_cast<const float *>(t->getTextureBuffer());
    tv.width = (int32_t)t->getWidth(), tv.height = (int32_t)t->getHeight(), tv.channels = (int32_t)t->getChannels();
    tv.invert_u = t->getInvertX(), tv.invert_v = t->getInvertY();
    v.textures.push_back(tv);
    *out = (int32_t)v.textures.size() - 1;
    tex_index[t] = *out;
    return SUCCESS;
  };
  const CsteTriMeshCollection meshes = scene.getTriangleMeshCollection();
  const CsteMaterialCollection mats = scene.getMaterialCollection(mesh::TRIANGLE);
  for (size_t i = 0; i < meshes.size(); i++) {
    const Trimesh &m = *meshes[i];
    const Material &mat = *mats[i];
    aggregate::material_view_s mv{};
    ERROR_STATE e;
    if ((e = texture_of(mat.getAlbedo(), true, &mv.albedo)) || (e = texture_of(mat.getMetallic(), true, &mv.metallic)) ||
        (e = texture_of(mat.getNormal(), true, &mv.normalmap)) || (e = texture_of(mat.getEmissive(), true, &mv.emissive)))
      return e;
    mat.getRefractiveIndex(mv.eta, mv.k);
    mv.anisotropy = mat.getAnisotropyFactor();
    v.materials.push_back(mv);
    aggregate::mesh_view_s x{};
    x.vertices = m.getVertices(), x.normals = m.getNormals(), x.tangents = m.getTangents();
    x.bitangents = m.getBitangents(), x.uv = m.getUVs(), x.indices = m.getIndices();
    m.getTransform().getTransformMatrix(x.m);
    m.getTransform().invert(x.inv);
    m.getTransform().transposeInvert(x.n);
    x.material = (uint32_t)i;
    v.meshes.push_back(x);
  }
  const int env = scene.getCurrentEnvmapId();
  const Texture *et = env >= 0 ? scene.getEnvmap((unsigned)env) : nullptr;
  if (!et || et->getFormat() != texture::FLOATX4 || et->getChannels() != 4)
    return *err = "the scene needs a current 4-channel float environment map (api/engine.cpp:273-290)",
           INVALID_SCENE_TYPE;
  ERROR_STATE e = texture_of(et, false, &v.envmap);
  if (e) return e;
  return SUCCESS;
}

/* ---- the engine ---------------------------------------------------------------------------- */

class B200Engine final : public Engine {
  int device_ = 0;
  nova_b200_ctx *ctx_ = nullptr;
  ScenePtr scene_;
  RenderBufferPtr buffers_;
  RenderOptionsPtr options_;
  EngineUserCallbackHandlerPtr callback_;
  bool scene_built_ = false, accel_built_ = false;
  std::atomic<bool> rendering_{false};
  std::atomic<unsigned> frame_index_{0};
  std::thread worker_;
  mutable std::mutex err_mu_;
  std::string error_;
  exception::NovaException errors_; /* the last start's and render's error bits */

  void set_error(const std::string &e) {
    std::lock_guard<std::mutex> g(err_mu_);
    error_ = e;
  }
  ERROR_STATE fail(ERROR_STATE st, const std::string &e) {
    set_error(e);
    return st;
  }
  ERROR_STATE ensure_ctx() {
    if (ctx_) return SUCCESS;
    nova_b200_status st = nova_b200_create(&ctx_, device_);
    if (st != NOVA_B200_SUCCESS) {
      ctx_ = nullptr;
      return fail(RENDER_ENGINE_NOT_INITIALIZED, "no CUDA device " + std::to_string(device_) + " for the B200 engine");
    }
    return SUCCESS;
  }
  void join() {
    if (worker_.joinable()) worker_.join();
  }

  /* one frame: the pass the integrator flag selects (Integrator.cpp:18-48: PATH required; of the
   * pass bits, the last one processed wins the pixel: EMISSIVE, then DEPTH, NORMAL, COMBINED) */
  ERROR_STATE render_frame(unsigned frame, const float inv_P[16], const float inv_V[16], float near_p, float far_p) {
    const unsigned W = buffers_->getWidth(), H = buffers_->getHeight();
    nova_b200_frame f{};
    f.width = (int32_t)W, f.height = (int32_t)H;
    f.spp_total = (int32_t)options_->getMaxSamples();
    f.sample_begin = (int32_t)frame;
    f.sample_count = 1;
    f.max_depth = (int32_t)options_->getMaxDepth();
    f.seed = 0;
    f.rr_start = -1;
    f.reset = 1;
    f.vertical_invert = options_->isFlippedV() ? 1 : 0;
    std::memcpy(f.inv_P, inv_P, 64);
    std::memcpy(f.inv_V, inv_V, 64);
    float *partial = buffers_->getRenderBuffers().partial_buffer;
    const int flag = options_->getIntegratorFlag();
    nova_b200_status st;
    if (flag & integrator::EMISSIVE)
      st = nova_b200_render_aov(ctx_, &f, NOVA_B200_AOV_EMISSIVE, near_p, far_p, partial, nullptr);
    else if (flag & integrator::DEPTH)
      st = nova_b200_render_aov(ctx_, &f, NOVA_B200_AOV_DEPTH, near_p, far_p, partial, nullptr);
    else if (flag & integrator::NORMAL)
      st = nova_b200_render_aov(ctx_, &f, NOVA_B200_AOV_NORMAL, near_p, far_p, partial, nullptr);
    else
      st = nova_b200_render(ctx_, &f, partial, nullptr, nullptr);
    if (st != NOVA_B200_SUCCESS) return fail((ERROR_STATE)st, status_text(ctx_));
    return SUCCESS;
  }

  /* api/engine.cpp:351-363.  Every element is independent, so a large film is split over host
   * threads (the same arithmetic per element: the result does not depend on the split). */
  void write_framebuffer(unsigned frame) {
    const HdrBufferStruct rb = buffers_->getRenderBuffers();
    const FloatView acc = buffers_->getAccumulator();
    const FloatView back = buffers_->backBuffer();
    const float denom = float(frame + 1);
    const float *partial = rb.partial_buffer;
    auto range = [&](size_t b, size_t e) {
      for (size_t i = b; i < e; i++) {
        acc[i] += partial[i];
        back[i] = acc[i] / denom;
      }
    };
    const size_t n = acc.size();
    const unsigned nt = n < (size_t)1 << 20 ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (nt == 1) {
      range(0, n);
      return;
    }
    std::vector<std::thread> pool;
    const size_t step = (n + nt - 1) / nt;
    for (unsigned t = 1; t < nt; t++) pool.emplace_back(range, std::min(n, t * step), std::min(n, (t + 1) * step));
    range(0, std::min(n, step));
    for (auto &th : pool) th.join();
  }

  /* the exception bit of a failed frame's status */
  static uint64_t frame_error_bits(ERROR_STATE e) {
    switch (e) {
      case OUT_OF_MEMORY:
      case RENDERER_EXCEPTION:
      case RENDER_ENGINE_NOT_INITIALIZED: return exception::GENERAL_GPU_ERROR;
      case INVALID_BUFFER_STATE:
      case RENDER_BUFFER_NOT_INITIALIZED: return exception::INVALID_RENDERBUFFER_STATE;
      default: return exception::GENERAL_ERROR;
    }
  }

  void render_loop() {
    const Camera *cam = scene_->getCamera((unsigned)std::max(0, scene_->getCurrentCameraId()));
    float iP[16], iV[16];
    cam->getInverseProjectionMatrix(iP);
    cam->getInverseViewMatrix(iV);
    const float near_p = cam->getClipPlaneNear(), far_p = cam->getClipPlaneFar();
    while (frame_index_.load() < options_->getMaxSamples() && rendering_.load()) {
      if (callback_) callback_->framePreRenderRoutine();
      const unsigned frame = frame_index_.load();
      const ERROR_STATE e = render_frame(frame, iP, iV, near_p, far_p);
      if (callback_) callback_->framePostRenderRoutine();
      if (e != SUCCESS) { /* the error text is kept for getRenderEngineError; the render stops */
        if (rendering_.load()) errors_.addErrorType(frame_error_bits(e)); /* not a stopRender() */
        rendering_.store(false);
        break;
      }
      write_framebuffer(frame);
      buffers_->swapBackBuffer();
      frame_index_.store(frame + 1);
    }
  }

 public:
  explicit B200Engine(int device) : device_(device) {}
  ~B200Engine() override {
    rendering_.store(false);
    join();
    if (ctx_) nova_b200_destroy(ctx_);
  }

  ERROR_STATE setScene(ScenePtr s) override {
    if (!s) return INVALID_ARGUMENT;
    scene_ = std::move(s);
    scene_built_ = accel_built_ = false;
    return SUCCESS;
  }
  const Scene *getScene() const override { return scene_.get(); }
  Scene *getScene() override { return scene_.get(); }

  ERROR_STATE buildScene() override {
    if (!scene_) return fail(INVALID_SCENE_TYPE, "no scene: call setScene() first");
    if (rendering_.load()) return fail(INVALID_ENGINE_STATE, "stop the render before rebuilding the scene");
    ERROR_STATE e = ensure_ctx();
    if (e) return e;
    SceneViews v;
    std::string err;
    if ((e = scene_views(*scene_, v, &err))) return fail(e, err);
    aggregate::primitive_aggregate_data_s d{v.meshes, v.materials, v.textures, v.envmap};
    /* the upload copies everything; the BVH is built with it (buildAcceleration() then only checks) */
    if ((e = upload_views(ctx_, d, &err))) return fail(e, err);
    scene_built_ = accel_built_ = true;
    return SUCCESS;
  }

  ERROR_STATE buildAcceleration() override {
    if (!scene_built_) return fail(SCENE_NOT_PROCESSED, "buildScene() has not succeeded");
    return accel_built_ ? SUCCESS : fail(SCENE_NOT_PROCESSED, "the acceleration structure is missing");
  }

  ERROR_STATE setRenderBuffers(RenderBufferPtr b) override {
    if (!b) return INVALID_BUFFER_STATE;
    if (rendering_.load()) return fail(INVALID_ENGINE_STATE, "stop the render before replacing its buffers");
    buffers_ = std::move(b);
    return SUCCESS;
  }
  const RenderBuffer *getRenderBuffers() const override { return buffers_.get(); }
  RenderBuffer *getRenderBuffers() override { return buffers_.get(); }

  ERROR_STATE cleanup() override {
    rendering_.store(false);
    join();
    scene_built_ = accel_built_ = false;
    if (!buffers_ || !scene_) return INVALID_ENGINE_STATE;
    buffers_->resetBuffers();
    scene_->cleanup();
    return SUCCESS;
  }

  ERROR_STATE setRenderOptions(RenderOptionsPtr o) override {
    if (!o) return INVALID_ARGUMENT;
    if (rendering_.load()) return fail(INVALID_ENGINE_STATE, "stop the render before replacing its options");
    options_ = std::move(o);
    return SUCCESS;
  }
  const RenderOptions *getRenderOptions() const override { return options_.get(); }
  RenderOptions *getRenderOptions() override { return options_.get(); }

  /* api/engine.cpp:577-586: stops, waits for the frame in flight, frame index back to 1 */
  ERROR_STATE stopRender() override {
    rendering_.store(false);
    if (ctx_) nova_b200_cancel(ctx_); /* a frame in flight stops within a group of waves */
    join();
    frame_index_.store(1);
    return SUCCESS;
  }

  ERROR_STATE prepareRender() override {
    if (!options_) return RENDER_OPTIONS_NOT_INITIALIZED;
    if (!buffers_) return RENDER_BUFFER_NOT_INITIALIZED;
    return SUCCESS;
  }

  ERROR_STATE startRender() override {
    errors_ = exception::NovaException();
    if (!options_) return RENDER_OPTIONS_NOT_INITIALIZED;
    if (!buffers_) {
      errors_.addErrorType(exception::INVALID_RENDERBUFFER_STATE);
      return RENDER_BUFFER_NOT_INITIALIZED;
    }
    if (!scene_built_ || !accel_built_) return SCENE_NOT_PROCESSED; /* the device context comes with the scene */
    if (!ctx_) return RENDER_ENGINE_NOT_INITIALIZED;
    if (!options_->isUsingGpu())
      return fail(INVALID_ENGINE_STATE, "the B200 engine renders on the GPU only: call RenderOptions::useGpu(true)");
    const int flag = options_->getIntegratorFlag();
    if (!(flag & integrator::PATH)) {
      errors_.addErrorType(exception::INVALID_INTEGRATOR);
      return fail(RENDERER_EXCEPTION, "invalid integrator: the PATH bit is required");
    }
    if (!(flag & (integrator::COMBINED | integrator::NORMAL | integrator::DEPTH | integrator::EMISSIVE))) {
      errors_.addErrorType(exception::INVALID_RENDER_MODE);
      return fail(RENDERER_EXCEPTION, "invalid render mode: no COMBINED, NORMAL, DEPTH or EMISSIVE pass");
    }
    const int cam = scene_->getCurrentCameraId();
    if (cam < 0 || !scene_->getCamera((unsigned)cam)) return fail(INVALID_SCENE_TYPE, "the scene has no current camera");
    const unsigned bw = buffers_->getWidth(), bh = buffers_->getHeight();
    if (bw == 0 || bh == 0 || bw > 65536 || bh > 65536 || buffers_->getAccumulator().size() != (size_t)bw * bh * 4) {
      /* DrawEngine.cpp:44-50: zero or over 65536 pixels a side is a dimension error, else the state */
      const bool bad_dim = bw == 0 || bh == 0 || bw > 65536 || bh > 65536;
      errors_.addErrorType(bad_dim ? exception::INVALID_RENDERBUFFER_DIM : exception::INVALID_RENDERBUFFER_STATE);
      return fail(INVALID_BUFFER_STATE, "render buffers are not sized (RenderBuffer::resize)");
    }
    rendering_.store(false);
    join();
    frame_index_.store(0);
    buffers_->resetBuffers();
    rendering_.store(true);
    worker_ = std::thread([this] { render_loop(); });
    return SUCCESS;
  }

  void setUserCallback(EngineUserCallbackHandlerPtr cb) override { callback_ = std::move(cb); }
  bool isRendering() const override { return rendering_.load(); }
  void getRenderEngineError(char log[1024], size_t &size) override {
    std::lock_guard<std::mutex> g(err_mu_);
    size = std::min<size_t>(error_.size(), 1023);
    std::memcpy(log, error_.data(), size);
    log[size] = 0;
  }
  unsigned getFrameIndex() const override { return frame_index_.load(); }
  const exception::NovaException &errors() const { return errors_; }
};

/* ---- the device accelerator plug-in ------------------------------------------------------- */

/* The accelerator's device context, shared with the intersectors it hands out so that an
 * intersector stays valid after its accelerator is cleaned up or destroyed. */
using SharedCtx = std::shared_ptr<nova_b200_ctx>;

SharedCtx make_shared_ctx(int device) {
  nova_b200_ctx *c = nullptr;
  if (nova_b200_create(&c, device) != NOVA_B200_SUCCESS) return nullptr;
  return SharedCtx(c, [](nova_b200_ctx *p) { nova_b200_destroy(p); });
}

class B200IntersectorImpl final : public aggregate::DeviceIntersectorInterface {
  SharedCtx ctx_;

 public:
  explicit B200IntersectorImpl(SharedCtx c) : ctx_(std::move(c)) {}
  /* one renderGpu frame (api/engine.cpp:469-481): sample params.sample_index of params.sample_max
   * into render_buffers.partial_buffer */
  void traverse(const device_traversal_param_s &p) const override {
    nova_b200_frame f{};
    f.width = (int32_t)p.width, f.height = (int32_t)p.height;
    f.spp_total = (int32_t)p.sample_max;
    f.sample_begin = (int32_t)p.sample_index;
    f.sample_count = 1;
    f.max_depth = (int32_t)p.depth;
    f.rr_start = -1;
    f.reset = 1;
    std::memcpy(f.inv_P, p.camera.inv_P, 64);
    std::memcpy(f.inv_V, p.camera.inv_V, 64);
    if (ctx_) nova_b200_render(ctx_.get(), &f, p.render_buffers.partial_buffer, nullptr, nullptr);
  }
};

class B200AcceleratorImpl final : public aggregate::B200Accelerator {
  int device_;
  SharedCtx ctx_;
  ERROR_STATE status_ = RENDER_ENGINE_NOT_INITIALIZED;
  std::string err_;

 public:
  explicit B200AcceleratorImpl(int device) : device_(device), ctx_(make_shared_ctx(device)) {
    if (ctx_)
      status_ = SCENE_NOT_PROCESSED;
    else
      err_ = "no CUDA device " + std::to_string(device);
  }
  void build(aggregate::primitive_aggregate_data_s d) override {
    if (!ctx_) ctx_ = make_shared_ctx(device_); /* after cleanup() */
    if (!ctx_) return;
    status_ = upload_views(ctx_.get(), d, &err_);
  }
  /* releases this accelerator's hold on the device scene; intersectors already handed out keep
   * theirs until they are destroyed */
  void cleanup() override {
    ctx_.reset();
    status_ = RENDER_ENGINE_NOT_INITIALIZED;
  }
  /* the device traversal stack holds 64 entries; a path scatters up to 255 times */
  unsigned getMaxRecursiveDepth() const override { return 255; }
  void copyParamsToDevice(const device_traversal_param_s &) const override {}
  std::unique_ptr<aggregate::DeviceIntersectorInterface> getIntersectorObject() const override {
    return std::make_unique<B200IntersectorImpl>(ctx_);
  }
  ERROR_STATE lastStatus() const override { return status_; }
  void getError(char log[1024], size_t &size) const override {
    size = std::min<size_t>(err_.size(), 1023);
    std::memcpy(log, err_.data(), size);
    log[size] = 0;
  }
  ERROR_STATE closestHits(uint64_t n, const float *o, const float *d, int32_t *prim, float *t, float *u,
                          float *v) const override {
    if (status_ != SUCCESS) return status_;
    return (ERROR_STATE)nova_b200_trace_host(ctx_.get(), n, o, d, prim, t, u, v);
  }
};

}  // namespace

TransformPtr create_transform() { return std::make_unique<B200Transform>(); }
TrimeshPtr create_trimesh() { return std::make_unique<B200Trimesh>(); }
TexturePtr create_texture() { return std::make_unique<B200Texture>(); }
MaterialPtr create_material() { return std::make_unique<B200Material>(); }
CameraPtr create_camera() { return std::make_unique<B200Camera>(); }
RenderOptionsPtr create_renderoptions() { return std::make_unique<B200RenderOptions>(); }
RenderBufferPtr create_renderbuffer() { return std::make_unique<B200RenderBuffer>(); }
ScenePtr create_scene() { return std::make_unique<B200Scene>(); }
EnginePtr create_engine() { return std::make_unique<B200Engine>(0); }
EnginePtr create_engine(int device) { return std::make_unique<B200Engine>(device); }
ERROR_STATE init_threads(unsigned n) { return n == 0 ? THREADPOOL_CREATION_ERROR : SUCCESS; }

uint64_t get_error_status(const Engine &engine) {
  const auto *e = dynamic_cast<const B200Engine *>(&engine);
  return e ? e->errors().getErrorFlag() : (uint64_t)exception::GENERAL_ERROR;
}
std::vector<exception::ERROR> get_error_list(const Engine &engine) {
  const auto *e = dynamic_cast<const B200Engine *>(&engine);
  return e ? e->errors().getErrorList() : std::vector<exception::ERROR>{exception::GENERAL_ERROR};
}

std::unique_ptr<aggregate::DeviceAcceleratorInterface> aggregate::DeviceAcceleratorInterface::make() {
  return std::make_unique<B200AcceleratorImpl>(0);
}

}  // namespace nova
