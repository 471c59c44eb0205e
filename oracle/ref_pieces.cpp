/* ORACLE PIN — test infrastructure only; never linked into the product.
 *
 * Most of the reference's path cannot be compiled here (glm, boost and Embree are empty
 * submodules), but a few of its headers on this path need nothing else: the fast atan2 polynomial
 * of the environment lookup (corelib/internal/common/math/math_utils_approx.h:13-40), the texel
 * conversions (corelib/internal/common/math/math_texturing.h:8-21) and the frame's tile split
 * (corelib/nova/utils/nova_utils.h:34-53); and the mesh fixtures of the reference's unit tests
 * (tests/unit_test/utils/geometry_shapes.h: CUBE, QUAD, TRIANGLE), so the oracle's property tests
 * run on the reference's own inputs.  This file includes those
 * headers from the reference tree, unchanged, and wraps them in C entry points; `make -C oracle ref`
 * builds it into oracle/_ref/libref_pieces.so, and the tests hold the oracle's restatements to
 * them bit for bit.  No reference code is copied: it is compiled where it lies. */
#include <cstdint>
#include <cstring>
#include <vector>

#include <internal/common/math/math_texturing.h>
#include <internal/common/math/math_utils_approx.h>
#include <nova/utils/nova_utils.h>
#include <unit_test/utils/geometry_shapes.h>

extern "C" void ref_atan2_approx(uint64_t n, const float *y, const float *x, float *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = math::atan2_approx(y[i], x[i]);
}

/* rgb_uint2float as TexturePackSampler.h:34-88 calls it: on the float channels of a bilinear sample */
extern "C" void ref_rgb_uint2float(uint64_t n, const float *v, float *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = math::texture::rgb_uint2float(v[i]);
}

/* uvToPixel as TextureContext.h:56 calls it: a float coordinate and an unsigned dimension */
extern "C" void ref_uv_to_pixel(uint64_t n, const float *t, const uint32_t *dim, uint32_t *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = math::texture::uvToPixel(t[i], (unsigned)dim[i]);
}

/* divideByTiles(W, H, tiles_w, tiles_h): (x0, x1, y0, y1) per tile into rects (room for
 * tiles_w * tiles_h); returns the tile count */
extern "C" int32_t ref_divide_by_tiles(int32_t w, int32_t h, int32_t tiles_w, int32_t tiles_h, int32_t *rects) {
  const std::vector<nova::Tile> tiles = nova::divideByTiles(w, h, tiles_w, tiles_h);
  for (size_t k = 0; k < tiles.size(); k++) {
    rects[4 * k] = tiles[k].width_start, rects[4 * k + 1] = tiles[k].width_end;
    rects[4 * k + 2] = tiles[k].height_start, rects[4 * k + 3] = tiles[k].height_end;
  }
  return (int32_t)tiles.size();
}

namespace {
template<class T>
int64_t copy_out(const std::vector<T> &v, T *out, int64_t cap) {
  if (out && cap >= (int64_t)v.size()) std::memcpy(out, v.data(), v.size() * sizeof(T));
  return (int64_t)v.size();
}
const std::vector<float> *fixture_floats(const char *shape, const char *attr) {
  const bool cube = !std::strcmp(shape, "CUBE"), quad = !std::strcmp(shape, "QUAD"), tri = !std::strcmp(shape, "TRIANGLE");
  if (!cube && !quad && !tri) return nullptr;
  if (!std::strcmp(attr, "vertices")) return cube ? &CUBE::vertices : quad ? &QUAD::vertices : &TRIANGLE::vertices;
  if (!std::strcmp(attr, "normals")) return cube ? &CUBE::normals : quad ? &QUAD::normals : &TRIANGLE::normals;
  if (!std::strcmp(attr, "uv")) return cube ? &CUBE::uv : quad ? &QUAD::uv : &TRIANGLE::uv;
  if (!std::strcmp(attr, "tangents")) return cube ? &CUBE::tangents : quad ? &QUAD::tangents : &TRIANGLE::tangents;
  if (!std::strcmp(attr, "bitangents"))
    return cube ? &CUBE::bitangents : quad ? &QUAD::bitangents : &TRIANGLE::bitangents;
  return nullptr;
}
}  // namespace

/* A float attribute of a fixture mesh: its length, copied to out when cap allows; -1 if unknown. */
extern "C" int64_t ref_fixture_floats(const char *shape, const char *attr, float *out, int64_t cap) {
  const std::vector<float> *v = fixture_floats(shape, attr);
  return v ? copy_out(*v, out, cap) : -1;
}

/* A fixture mesh's triangle indices: their count, copied to out when cap allows; -1 if unknown. */
extern "C" int64_t ref_fixture_indices(const char *shape, uint32_t *out, int64_t cap) {
  if (!std::strcmp(shape, "CUBE")) return copy_out(CUBE::indices, out, cap);
  if (!std::strcmp(shape, "QUAD")) return copy_out(QUAD::indices, out, cap);
  if (!std::strcmp(shape, "TRIANGLE")) return copy_out(TRIANGLE::indices, out, cap);
  return -1;
}
