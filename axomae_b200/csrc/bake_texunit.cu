/* Diffuse irradiance bake with the semantics of the reference's CUDA kernel: the path its command line
 * takes with --gpu (sources/controller/cmd/API.cpp:29,52 -> TextureProcessing.cpp:19-45 ->
 * GPU_compute_irradiance, sources/processing/cuda/CubemapProcessing.cu:244-284, kernel :129-175).
 *
 * It differs from the CPU path (bake.cu) in three ways, all kept here:
 *   - the pgc3d hash is seeded with the output texel's own indices (i, j), not with the pixel of its
 *     approximate spherical coordinates;
 *   - directions map to uv with the exact acos / atan2f (the device's own functions), not the fast
 *     polynomial and the acos table;
 *   - the source is read through a float4 texture object with hardware bilinear filtering, wrap
 *     addressing and normalised coordinates (CubemapProcessing.cu:216-230), so the filter weights
 *     are the texture unit's 8-bit-fraction fixed point ones.
 * The output is RGBA with alpha 1 (gpgpu_device_write_buffer, :121-127).  Angles are evaluated as
 * the reference's expressions are written: products with PI (a double constant) in double, the
 * trigonometry in float.  This file is compiled with the default multiply-add contraction, like the
 * reference's CUDA sources (its CMake flags only add --expt-relaxed-constexpr -std=c++17).
 */
#include "context.cuh"

namespace {

constexpr double kPi = 3.14159265358979323846; /* PI, internal/common/math/math_spherical.h:8 (double) */

struct F3 {
  float x, y, z;
};

__device__ __forceinline__ F3 sph_to_cart(float phi, float theta) {
  return F3{sinf(theta) * cosf(phi), sinf(theta) * sinf(phi), cosf(theta)};
}

__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
  return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

__device__ __forceinline__ F3 normalize3(F3 a) {
  const float d = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
  return F3{a.x / d, a.y / d, a.z / d};
}

__device__ __forceinline__ F3 scale(float k, F3 v) { return F3{v.x * k, v.y * k, v.z * k}; }
__device__ __forceinline__ F3 add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }

/* The 3D hash of the kernel (integer arithmetic, then unsigned -> float times 1 / float(2^32 - 1)). */
__device__ __forceinline__ F3 pgc3d(unsigned x, unsigned y, unsigned z) {
  x = x * 1664525u + 1013904223u;
  y = y * 1664525u + 1013904223u;
  z = z * 1664525u + 1013904223u;
  x += y * z;
  y += z * x;
  z += x * y;
  x ^= x >> 16u;
  y ^= y >> 16u;
  z ^= z >> 16u;
  x += y * z;
  y += z * x;
  z += x * y;
  const float cste = 1.f / float(0xFFFFFFFFu);
  return F3{(float)x * cste, (float)y * cste, (float)z * cste};
}

/* One thread per output texel, 32 x 32 blocks as the reference launches them. */
__global__ void __launch_bounds__(1024) k_bake_texunit(float *out, cudaTextureObject_t tex, unsigned W, unsigned H,
                                                       unsigned samples) {
  const int i = blockDim.x * blockIdx.x + threadIdx.x;
  const int j = blockDim.y * blockIdx.y + threadIdx.y;
  if (i >= (int)W || j >= (int)H) return;
  const float u = (float)i / (float)W;
  const float v = (float)j / (float)H;
  const float phi0 = (float)(2 * kPi * u), theta0 = (float)(kPi * v); /* uvToSpherical */
  const F3 normal = sph_to_cart(phi0, theta0);
  const F3 some{1.f, 0.f, 0.f};
  const float dd = dot3(some, normal);
  F3 tangent{0.f, 1.f, 0.f};
  if (1.0 - fabsf(dd) > 1e-6) tangent = normalize3(cross3(some, normal));
  const F3 bitangent = cross3(normal, tangent);
  F3 irr{0.f, 0.f, 0.f};
  for (unsigned s = 0; s < samples; s++) {
    const F3 r = pgc3d((unsigned)i, (unsigned)j, s);
    const float phi = (float)(2 * kPi * r.x);
    const float theta = asinf(sqrtf(r.y));
    F3 c = sph_to_cart(phi, theta);
    c = add(add(scale(c.x, tangent), scale(c.y, bitangent)), scale(c.z, normal));
    const float th = acosf(c.z), ph = atan2f(c.y, c.x); /* cartesianToSpherical */
    const float tu = (float)(ph / (2 * kPi)), tv = (float)(th / kPi); /* sphericalToUv */
    const float4 t = tex2D<float4>(tex, tu, tv);
    irr.x += t.x;
    irr.y += t.y;
    irr.z += t.z;
  }
  irr.x /= samples;
  irr.y /= samples;
  irr.z /= samples;
  float *o = out + ((size_t)j * W + i) * 4;
  o[0] = irr.x;
  o[1] = irr.y;
  o[2] = irr.z;
  o[3] = 1.f;
}

/* RGB(A) source -> RGBA with alpha 1, as TextureProcessing.cpp:24-32 prepares it. */
__global__ void k_to_rgba(const float *src, size_t n, int ch, float4 *dst) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    dst[k] = make_float4(src[k * ch], src[k * ch + 1], src[k * ch + 2], 1.f);
}

}  // namespace

nova_b200_status nb_bake_texunit(nova_b200_ctx *c, const float *src, int32_t sw, int32_t sh, int32_t ch, int32_t ow,
                                 int32_t oh, int32_t samples, float *out) {
  using namespace nbctx;
  auto pow2 = [](int32_t v) { return v > 0 && (v & (v - 1)) == 0; };
  if (!src || !out) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  if (!pow2(ow) || !pow2(oh))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "irradiance size must be a power of two (TextureProcessing.cpp:11)%s");
  if (sw < 1 || sh < 1 || ch < 3 || ch > 4 || samples <= 0)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid source map or sample count%s");
  int max_w = 0, max_h = 0;
  cudaDeviceGetAttribute(&max_w, cudaDevAttrMaxTexture2DWidth, c->device);
  cudaDeviceGetAttribute(&max_h, cudaDevAttrMaxTexture2DHeight, c->device);
  if (sw > max_w || sh > max_h) return fail(c, NOVA_B200_INVALID_ARGUMENT, "source map larger than a 2D texture%s");
  cudaSetDevice(c->device);
  const size_t texels = (size_t)sw * sh;
  float4 *rgba = nullptr;
  const float *rows = src;
  if (ch == 3) {
    NB_CUDA(c, cudaMallocAsync(&rgba, texels * sizeof(float4), c->stream), "cudaMalloc(rgba source)");
    k_to_rgba<<<592, 256, 0, c->stream>>>(src, texels, ch, rgba);
    rows = reinterpret_cast<const float *>(rgba);
  }
  const cudaChannelFormatDesc fmt = cudaCreateChannelDesc(32, 32, 32, 32, cudaChannelFormatKindFloat);
  cudaArray_t array = nullptr;
  cudaTextureObject_t tex = 0;
  cudaError_t e = cudaMallocArray(&array, &fmt, (size_t)sw, (size_t)sh);
  if (e == cudaSuccess)
    e = cudaMemcpy2DToArrayAsync(array, 0, 0, rows, (size_t)sw * sizeof(float4), (size_t)sw * sizeof(float4),
                                 (size_t)sh, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) {
    cudaResourceDesc res{};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = array;
    cudaTextureDesc td{}; /* CubemapProcessing.cu:223-229 */
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    e = cudaCreateTextureObject(&tex, &res, &td, nullptr);
  }
  if (e == cudaSuccess) {
    const dim3 block(32, 32), grid((unsigned)ow / 32 + 1, (unsigned)oh / 32 + 1); /* :192-199 */
    cudaEventRecord(c->ev_begin, c->stream);
    k_bake_texunit<<<grid, block, 0, c->stream>>>(out, tex, (unsigned)ow, (unsigned)oh, (unsigned)samples);
    cudaEventRecord(c->ev_end, c->stream);
    e = cudaGetLastError();
  }
  const cudaError_t es = cudaStreamSynchronize(c->stream);
  if (tex) cudaDestroyTextureObject(tex);
  if (array) cudaFreeArray(array);
  if (rgba) cudaFreeAsync(rgba, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "bake (texture unit)");
  if (es != cudaSuccess) return cuda_fail(c, es, "bake (texture unit)");
  return NOVA_B200_SUCCESS;
}
