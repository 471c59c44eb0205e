/* Film outputs and the Radiance .hdr image format: the callers on either side of the render.
 *
 * Device kernels (one thread per pixel or per four floats; each reads its inputs once and writes
 * its outputs once, so they are bound by HBM bandwidth):
 *   k_accumulate     Engine::writeFramebuffer (corelib/nova/api/engine.cpp:351-363): the running
 *                    sum of one-sample frames and its mean, accumulated / (frame_index + 1).
 *   k_display_blend  NovaRenderer::copyBufferToPbo (sources/renderer/nova/NovaRenderer_draw.cpp:35-45):
 *                    the editor's display value old + 0.8 (new - old), old = accumulated / (frame + 1).
 *   k_snapshot       NovaRenderer::getSnapshotFloat (sources/renderer/nova/NovaRenderer.cpp:139-153)
 *                    through TextureOperations::processTexture / uvSample / bilinearInterpolate /
 *                    wrapAroundPixelCoords (sources/processing/TextureProcessing.h:157-250): a resample
 *                    of the film to another size with the reference's float / double conversions.
 *   k_rgbe_encode    float pixel -> shared-exponent RGBE bytes of the Radiance format (G. Ward,
 *   k_rgbe_decode    "Real Pixels", Graphics Gems II, 1991) and back, rounded the way the stb_image
 *                    routines the reference calls do it (stbi_write_hdr in IO::Loader::writeHdr,
 *                    stbi_loadf in IO::Loader::loadRadianceFile, sources/IO/Loader_image.cpp:50-62,
 *                    146-192; stb is an un-vendored submodule of the reference, github.com/nothings/stb).
 *
 * Host code: the file's text header and its run-length scanline packets, serial byte work on a
 * buffer of 4 bytes per pixel (the device encodes, the host only packs).
 */
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "context.cuh"

namespace {

/* ---- device kernels ---------------------------------------------------------------------- */

__global__ void k_accumulate(const float *partial, float *accum, float *final_buf, uint64_t n, float denom) {
  const uint64_t i4 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i4 + 4 <= n) {
    const float4 p = *reinterpret_cast<const float4 *>(partial + i4);
    float4 a = *reinterpret_cast<const float4 *>(accum + i4);
    a.x += p.x, a.y += p.y, a.z += p.z, a.w += p.w;
    *reinterpret_cast<float4 *>(accum + i4) = a;
    if (final_buf)
      *reinterpret_cast<float4 *>(final_buf + i4) = make_float4(a.x / denom, a.y / denom, a.z / denom, a.w / denom);
  } else {
    for (uint64_t i = i4; i < n; i++) {
      const float a = accum[i] + partial[i];
      accum[i] = a;
      if (final_buf) final_buf[i] = a / denom;
    }
  }
}

__device__ __forceinline__ float blend(float acc, float now, float denom) {
  const float old = acc / denom;
  return old + 0.8f * (now - old);
}

__global__ void k_display_blend(const float *partial, const float *accum, float *out, uint64_t n, float denom) {
  const uint64_t i4 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i4 + 4 <= n) {
    const float4 p = *reinterpret_cast<const float4 *>(partial + i4);
    const float4 a = *reinterpret_cast<const float4 *>(accum + i4);
    *reinterpret_cast<float4 *>(out + i4) =
        make_float4(blend(a.x, p.x, denom), blend(a.y, p.y, denom), blend(a.z, p.z, denom), blend(a.w, p.w, denom));
  } else {
    for (uint64_t i = i4; i < n; i++) out[i] = blend(accum[i], partial[i], denom);
  }
}

struct Film {
  const float *data;
  int w, h, ch;
  /* TextureOperations::discreteSample with wrapAroundPixelCoords (TextureProcessing.h:174-181, 233-250) */
  __device__ float3 texel(int x, int y) const {
    const int xc = x >= w ? x % w : (x < 0 ? w + (x % w) : x);
    const int yc = y >= h ? y % h : (y < 0 ? h + (y % h) : y);
    const float *p = data + ((size_t)yc * w + xc) * ch;
    return make_float3(p[0], p[1], p[2]);
  }
};

/* uvToPixel (math_texturing.h:19-21): float coordinate times the size, converted to unsigned the
 * way x86-64 code does it (64-bit truncation, low 32 bits). */
__device__ __forceinline__ unsigned uv_to_pixel(float coord, unsigned dim) {
  return (unsigned)(long long)__fmul_rn(coord, (float)dim);
}

__device__ __forceinline__ float wrap_uv(double c) {
  /* wrapAroundTexCoords<double> (TextureProcessing.h:214-230), returned as a float vec2 */
  const double ci = floor(c);
  return (float)((c > 1.0 || c < 0.0) ? c - ci : c);
}

__global__ void k_snapshot(Film src, float *dst, int dw, int dh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= dw || j >= dh) return;
  /* processTexture: u = i / dest_width, v = j / dest_height in double (math_texturing.h:14-17) */
  const float wu = wrap_uv((double)i / (double)dw), wv = wrap_uv((double)j / (double)dh);
  /* pixel coordinates: unsigned -> double -> float (glm::dvec2 into glm::vec2) */
  const float px = (float)(double)uv_to_pixel(wu, (unsigned)src.w);
  const float py = (float)(double)uv_to_pixel(wv, (unsigned)src.h);
  const float tlx = floorf(px), tly = floorf(py);
  const float trx = __fadd_rn(floorf(px), 1.f), bly = __fadd_rn(floorf(py), 1.f);
  /* bilinearInterpolate (TextureProcessing.h:183-199), literally: the weights come out 0 and 1 for
   * whole-pixel coordinates, and the arithmetic keeps the reference's signed zeros and NaN spread */
  const float u = __fdiv_rn(__fsub_rn(px, tlx), __fsub_rn(trx, tlx));
  const float v = __fdiv_rn(__fsub_rn(py, tly), __fsub_rn(bly, tly));
  const float hd = __fsub_rn(1.f, u);
  const float3 tl = src.texel((int)tlx, (int)tly), tr = src.texel((int)trx, (int)tly);
  const float3 bl = src.texel((int)tlx, (int)bly), br = src.texel((int)trx, (int)bly);
  const float vd = __fsub_rn(1.f, v);
  auto lerp2 = [&](float a, float b, float c, float d) {
    const float top = __fadd_rn(__fmul_rn(hd, a), __fmul_rn(u, b));
    const float bot = __fadd_rn(__fmul_rn(hd, c), __fmul_rn(u, d));
    return __fadd_rn(__fmul_rn(vd, top), __fmul_rn(v, bot));
  };
  /* dest index uses the source's channel stride; channel 3 is never written (:167-171) */
  float *o = dst + ((size_t)j * dw + i) * src.ch;
  o[0] = lerp2(tl.x, tr.x, bl.x, br.x);
  o[1] = lerp2(tl.y, tr.y, bl.y, br.y);
  o[2] = lerp2(tl.z, tr.z, bl.z, br.z);
}

/* Float RGB -> RGBE.  m = max(r, g, b) taken as max(r, max(g, b)) with "a > b ? a : b" (so a NaN
 * operand is passed over unless it is the first); m < 1e-32 -> all zero; else m = f 2^e with f in
 * [0.5, 1), scale = f * 256 / m, byte_c = low byte of the int32 truncation of c * scale, byte_e =
 * low byte of e + 128.  A non-finite m gives RGB 0 and exponent byte 128.  The truncations follow
 * x86-64 conversion (int32 truncation toward zero, NaN -> 0 in the low byte). */
__device__ __forceinline__ uchar4 rgbe_encode(float r, float g, float b) {
  const float gb = g > b ? g : b;
  const float m = r > gb ? r : gb;
  if (m < 1e-32f) return make_uchar4(0, 0, 0, 0);
  if (!isfinite(m)) return make_uchar4(0, 0, 0, 128);
  /* m is a normal float here (>= 1e-32): its exponent field gives e directly */
  const uint32_t bits = __float_as_uint(m);
  const int e = (int)((bits >> 23) & 0xffu) - 126;
  const float f = __uint_as_float((bits & 0x807fffffu) | (126u << 23));
  const float scale = __fdiv_rn(__fmul_rn(f, 256.f), m);
  auto byte = [](float x) -> unsigned char {
    return isnan(x) ? (unsigned char)0 : (unsigned char)((unsigned)(int)x & 0xffu);
  };
  return make_uchar4(byte(__fmul_rn(r, scale)), byte(__fmul_rn(g, scale)), byte(__fmul_rn(b, scale)),
                     (unsigned char)((unsigned)(e + 128) & 0xffu));
}

/* Encodes rows in file order (flip: bottom row first).  planar = 1 writes each row as four planes
 * of width bytes (R, G, B, E: the order of run-length scanlines), 0 as interleaved pixels. */
__global__ void k_rgbe_encode(const float *src, int w, int h, int ch, int flip, int planar, unsigned char *dst) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, row = blockIdx.y;
  if (x >= w || row >= h) return;
  const int srow = flip ? h - 1 - row : row;
  const float *p = src + ((size_t)srow * w + x) * ch;
  float r, g, b;
  if (ch >= 3) {
    r = p[0], g = p[1], b = p[2];
  } else {
    r = g = b = p[0];
  }
  const uchar4 q = rgbe_encode(r, g, b);
  if (planar) {
    unsigned char *o = dst + (size_t)row * w * 4;
    o[x] = q.x, o[w + x] = q.y, o[2 * w + x] = q.z, o[3 * w + x] = q.w;
  } else {
    reinterpret_cast<uchar4 *>(dst)[(size_t)row * w + x] = q;
  }
}

/* RGBE -> float: exponent byte 0 -> (0, 0, 0); else c = byte 2^(e - 136), exact; alpha 1 (the
 * loader widens 3-channel files to RGBA with alpha 1, Loader_image.cpp:161-170). */
__global__ void k_rgbe_decode(const uchar4 *src, uint64_t n, float4 *dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uchar4 q = src[i];
  if (q.w == 0) {
    dst[i] = make_float4(0.f, 0.f, 0.f, 1.f);
    return;
  }
  const double s = __longlong_as_double((long long)((int)q.w - 136 + 1023) << 52);
  dst[i] = make_float4((float)(q.x * s), (float)(q.y * s), (float)(q.z * s), 1.f);
}

/* ---- host: the file format ----------------------------------------------------------------- */

constexpr int kMaxDim = 1 << 24; /* the largest width / height the loader accepts */

bool rle_width(int w) { return w >= 8 && w < 32768; }

struct Reader {
  const std::vector<unsigned char> &b;
  size_t pos = 0;
  /* reading past the end yields zeros, as the reference's loader does */
  unsigned char get() { return pos < b.size() ? b[pos++] : (unsigned char)0; }
  std::string line() {
    std::string s;
    while (pos < b.size() && b[pos] != '\n' && s.size() < 1023) s.push_back((char)b[pos++]);
    while (pos < b.size() && b[pos] != '\n') pos++; /* an over-long line is cut, the rest skipped */
    if (pos < b.size()) pos++;
    return s;
  }
};

struct Header {
  int w = 0, h = 0;
  size_t data = 0; /* offset of the first scanline byte */
};

/* IO::Loader::loadHdrEnvmap's magic check (Loader_image.cpp:64-90) then the Radiance header as the
 * stb loader parses it: first line "#?RADIANCE" or "#?RGBE", lines up to an empty one with
 * "FORMAT=32-bit_rle_rgbe" among them, then "-Y <height> +X <width>". */
nova_b200_status parse_header(nova_b200_ctx *c, const std::vector<unsigned char> &bytes, Header &hd) {
  using namespace nbctx;
  char magic[32] = {0};
  std::memcpy(magic, bytes.data(), std::min<size_t>(31, bytes.size()));
  if (bytes.size() >= 4 && (unsigned char)magic[0] == 0x76 && (unsigned char)magic[1] == 0x2f &&
      (unsigned char)magic[2] == 0x31 && (unsigned char)magic[3] == 0x01)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "OpenEXR files are not supported by this library%s");
  if (!std::strstr(magic, "#?RADIANCE"))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "Must be an HDR/EXR format .%s");
  Reader r{bytes};
  const std::string first = r.line();
  if (first != "#?RADIANCE" && first != "#?RGBE") return fail(c, NOVA_B200_INVALID_ARGUMENT, "not an HDR file%s");
  bool format = false;
  for (;;) {
    if (r.pos >= bytes.size()) return fail(c, NOVA_B200_INVALID_ARGUMENT, "HDR header has no end%s");
    const std::string t = r.line();
    if (t.empty()) break;
    if (t == "FORMAT=32-bit_rle_rgbe") format = true;
  }
  if (!format) return fail(c, NOVA_B200_INVALID_ARGUMENT, "unsupported HDR format (not 32-bit_rle_rgbe)%s");
  const std::string res = r.line();
  const char *p = res.c_str();
  if (std::strncmp(p, "-Y ", 3)) return fail(c, NOVA_B200_INVALID_ARGUMENT, "unsupported HDR data layout%s");
  char *end = nullptr;
  const long h = std::strtol(p + 3, &end, 10);
  p = end;
  while (*p == ' ') p++;
  if (std::strncmp(p, "+X ", 3)) return fail(c, NOVA_B200_INVALID_ARGUMENT, "unsupported HDR data layout%s");
  const long w = std::strtol(p + 3, nullptr, 10);
  if (w <= 0 || h <= 0 || w > kMaxDim || h > kMaxDim)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "HDR image size out of range%s");
  hd.w = (int)w, hd.h = (int)h, hd.data = r.pos;
  return NOVA_B200_SUCCESS;
}

/* Scanlines -> interleaved RGBE bytes.  Rows of a width in [8, 32768) are run-length packets:
 * a row header (2, 2, width >> 8, width & 255), then for each of R, G, B, E packets that are
 * either a run (count + 128, value) or a dump (count, count bytes), count in 1..remaining.  A row
 * whose first bytes are not a run-length header means the file is flat from there: those 4 bytes
 * are pixel 0 of row 0 and the rest follow in order (the stb loader's rule, kept as is). */
nova_b200_status unpack(nova_b200_ctx *c, const std::vector<unsigned char> &bytes, const Header &hd,
                        std::vector<unsigned char> &rgbe) {
  using namespace nbctx;
  const size_t w = (size_t)hd.w, h = (size_t)hd.h;
  rgbe.assign(w * h * 4, 0);
  Reader r{bytes, hd.data};
  auto flat_from = [&](size_t first_pixel) {
    for (size_t i = first_pixel; i < w * h * 4; i++) rgbe[i] = r.get();
  };
  if (!rle_width(hd.w)) {
    flat_from(0);
    return NOVA_B200_SUCCESS;
  }
  std::vector<unsigned char> line(w * 4);
  for (size_t j = 0; j < h; j++) {
    const unsigned char c1 = r.get(), c2 = r.get(), c3 = r.get();
    if (c1 != 2 || c2 != 2 || (c3 & 0x80)) {
      rgbe[0] = c1, rgbe[1] = c2, rgbe[2] = c3, rgbe[3] = r.get();
      flat_from(4);
      return NOVA_B200_SUCCESS;
    }
    const size_t len = ((size_t)c3 << 8) | r.get();
    if (len != w) return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid decoded scanline length%s");
    for (int k = 0; k < 4; k++) {
      size_t i = 0;
      while (i < w) {
        unsigned count = r.get();
        const size_t left = w - i;
        if (count > 128) {
          const unsigned char value = r.get();
          count -= 128;
          if (count == 0 || count > left) return fail(c, NOVA_B200_INVALID_ARGUMENT, "bad RLE data in HDR%s");
          for (unsigned z = 0; z < count; z++) line[(i++) * 4 + k] = value;
        } else {
          if (count == 0 || count > left) return fail(c, NOVA_B200_INVALID_ARGUMENT, "bad RLE data in HDR%s");
          for (unsigned z = 0; z < count; z++) line[(i++) * 4 + k] = r.get();
        }
      }
    }
    std::memcpy(&rgbe[j * w * 4], line.data(), w * 4);
  }
  return NOVA_B200_SUCCESS;
}

/* One plane of a run-length row: runs of 3 or more equal bytes become run packets (at most 127),
 * everything else dump packets (at most 128). */
void pack_plane(const unsigned char *p, int w, std::string &out) {
  int x = 0;
  while (x < w) {
    int lit = x; /* start of the next run of >= 3, or w */
    while (lit < w) {
      if (lit + 2 < w && p[lit] == p[lit + 1] && p[lit] == p[lit + 2]) break;
      lit++;
    }
    while (x < lit) {
      const int n = std::min(lit - x, 128);
      out.push_back((char)n);
      out.append(reinterpret_cast<const char *>(p + x), (size_t)n);
      x += n;
    }
    if (lit < w) {
      int end = lit;
      while (end < w && p[end] == p[lit]) end++;
      while (x < end) {
        const int n = std::min(end - x, 127);
        out.push_back((char)(128 + n));
        out.push_back((char)p[lit]);
        x += n;
      }
    }
  }
}

nova_b200_status read_file(nova_b200_ctx *c, const char *path, std::vector<unsigned char> &bytes) {
  using namespace nbctx;
  if (!path) return fail(c, NOVA_B200_INVALID_ARGUMENT, "path is null%s");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(c, NOVA_B200_INVALID_ARGUMENT, "cannot open %s", path);
  bytes.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return NOVA_B200_SUCCESS;
}

nova_b200_status check_ctx(nova_b200_ctx *c) { return c ? NOVA_B200_SUCCESS : NOVA_B200_INVALID_ARGUMENT; }

}  // namespace

extern "C" nova_b200_status nova_b200_film_accumulate(nova_b200_ctx *c, const float *partial, float *accum,
                                                      float *final_buf, uint64_t n, uint32_t frame_index) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  if (!partial || !accum) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  if ((reinterpret_cast<uintptr_t>(partial) | reinterpret_cast<uintptr_t>(accum) |
       reinterpret_cast<uintptr_t>(final_buf)) & 15)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "film buffers must be 16-byte aligned%s");
  if (n == 0) return NOVA_B200_SUCCESS;
  cudaSetDevice(c->device);
  const uint64_t threads = (n + 3) / 4;
  cudaEventRecord(c->ev_begin, c->stream);
  k_accumulate<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(partial, accum, final_buf, n,
                                                                          (float)(frame_index + 1));
  NB_CUDA(c, cudaGetLastError(), "k_accumulate");
  cudaEventRecord(c->ev_end, c->stream);
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "film_accumulate");
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_display_blend(nova_b200_ctx *c, const float *partial, const float *accum,
                                                    float *out, uint64_t n, uint32_t current_frame) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  if (!partial || !accum || !out) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  if ((reinterpret_cast<uintptr_t>(partial) | reinterpret_cast<uintptr_t>(accum) | reinterpret_cast<uintptr_t>(out)) &
      15)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "film buffers must be 16-byte aligned%s");
  if (n == 0) return NOVA_B200_SUCCESS;
  cudaSetDevice(c->device);
  const uint64_t threads = (n + 3) / 4;
  cudaEventRecord(c->ev_begin, c->stream);
  k_display_blend<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(partial, accum, out, n,
                                                                             (float)(current_frame + 1));
  NB_CUDA(c, cudaGetLastError(), "k_display_blend");
  cudaEventRecord(c->ev_end, c->stream);
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "display_blend");
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_snapshot(nova_b200_ctx *c, const float *film, int32_t w, int32_t h,
                                               int32_t channels, float *dst, int32_t dw, int32_t dh) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  if (!film || !dst) return fail(c, NOVA_B200_INVALID_ARGUMENT, "null buffer%s");
  if (w <= 0 || h <= 0 || dw <= 0 || dh <= 0 || w > kMaxDim || h > kMaxDim || dw > kMaxDim || dh > 65535)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid snapshot size%s");
  if (channels < 3 || channels > 4) return fail(c, NOVA_B200_INVALID_ARGUMENT, "channels must be 3 or 4%s");
  cudaSetDevice(c->device);
  cudaEventRecord(c->ev_begin, c->stream);
  k_snapshot<<<dim3((unsigned)((dw + 127) / 128), (unsigned)dh), 128, 0, c->stream>>>(Film{film, w, h, channels}, dst,
                                                                                    dw, dh);
  NB_CUDA(c, cudaGetLastError(), "k_snapshot");
  cudaEventRecord(c->ev_end, c->stream);
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "snapshot");
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_hdr_info(nova_b200_ctx *c, const char *path, int32_t *width, int32_t *height) {
  std::vector<unsigned char> bytes;
  nova_b200_status st = read_file(c, path, bytes);
  if (st) return st;
  Header hd;
  if ((st = parse_header(c, bytes, hd))) return st;
  if (width) *width = hd.w;
  if (height) *height = hd.h;
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_hdr_read(nova_b200_ctx *c, const char *path, float *rgba_host,
                                               float *rgba_device, uint64_t capacity) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  std::vector<unsigned char> bytes, rgbe;
  nova_b200_status st = read_file(c, path, bytes);
  if (st) return st;
  Header hd;
  if ((st = parse_header(c, bytes, hd))) return st;
  const uint64_t npx = (uint64_t)hd.w * hd.h;
  if (npx > (1ull << 31)) return fail(c, NOVA_B200_INVALID_ARGUMENT, "HDR image larger than 2^31 pixels%s");
  if (capacity < npx * 4) return fail(c, NOVA_B200_INVALID_ARGUMENT, "output holds fewer than width * height * 4 floats%s");
  if (rgba_device && (reinterpret_cast<uintptr_t>(rgba_device) & 15))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "rgba_device must be 16-byte aligned%s");
  if ((st = unpack(c, bytes, hd, rgbe))) return st;
  cudaSetDevice(c->device);
  unsigned char *d_rgbe = nullptr;
  float4 *d_out = reinterpret_cast<float4 *>(rgba_device), *tmp = nullptr;
  NB_CUDA(c, cudaMallocAsync(&d_rgbe, npx * 4, c->stream), "cudaMalloc(hdr bytes)");
  cudaError_t e = cudaMemcpyAsync(d_rgbe, rgbe.data(), npx * 4, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && !d_out) {
    e = cudaMallocAsync(&tmp, npx * sizeof(float4), c->stream);
    d_out = tmp;
  }
  if (e == cudaSuccess) {
    cudaEventRecord(c->ev_begin, c->stream);
    k_rgbe_decode<<<(unsigned)((npx + 255) / 256), 256, 0, c->stream>>>(reinterpret_cast<const uchar4 *>(d_rgbe), npx,
                                                                         d_out);
    e = cudaGetLastError();
    cudaEventRecord(c->ev_end, c->stream);
  }
  if (e == cudaSuccess && rgba_host)
    e = cudaMemcpyAsync(rgba_host, d_out, npx * sizeof(float4), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFreeAsync(d_rgbe, c->stream);
  if (tmp) cudaFreeAsync(tmp, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "hdr_read");
  NB_CUDA(c, cudaStreamSynchronize(c->stream), "hdr_read");
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_hdr_write(nova_b200_ctx *c, const char *path, const float *pixels_host,
                                                const float *pixels_device, int32_t w, int32_t h, int32_t channels,
                                                int32_t flip) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  if (!path) return fail(c, NOVA_B200_INVALID_ARGUMENT, "path is null%s");
  if (!pixels_host && !pixels_device) return fail(c, NOVA_B200_INVALID_ARGUMENT, "no pixels%s");
  if (w <= 0 || h <= 0 || w > kMaxDim || h > 65535) return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid image size%s");
  if (channels < 1 || channels > 4) return fail(c, NOVA_B200_INVALID_ARGUMENT, "channels must be 1 to 4%s");
  const uint64_t npx = (uint64_t)w * h;
  const bool rle = rle_width(w);
  cudaSetDevice(c->device);
  std::vector<unsigned char> rgbe(npx * 4);
  unsigned char *d_rgbe = nullptr;
  float *d_src = const_cast<float *>(pixels_device), *tmp = nullptr;
  NB_CUDA(c, cudaMallocAsync(&d_rgbe, npx * 4, c->stream), "cudaMalloc(hdr bytes)");
  cudaError_t e = cudaSuccess;
  if (!d_src) {
    e = cudaMallocAsync(&tmp, npx * channels * sizeof(float), c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tmp, pixels_host, npx * channels * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    d_src = tmp;
  }
  if (e == cudaSuccess) {
    cudaEventRecord(c->ev_begin, c->stream);
    k_rgbe_encode<<<dim3((unsigned)((w + 127) / 128), (unsigned)h), 128, 0, c->stream>>>(d_src, w, h, channels, flip,
                                                                                         rle ? 1 : 0, d_rgbe);
    e = cudaGetLastError();
    cudaEventRecord(c->ev_end, c->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(rgbe.data(), d_rgbe, npx * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFreeAsync(d_rgbe, c->stream);
  if (tmp) cudaFreeAsync(tmp, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "hdr_write");
  std::string out = "#?RADIANCE\n# nova_b200\nFORMAT=32-bit_rle_rgbe\n\n-Y " + std::to_string(h) + " +X " +
                    std::to_string(w) + "\n";
  if (!rle) {
    out.append(reinterpret_cast<const char *>(rgbe.data()), rgbe.size());
  } else {
    out.reserve(out.size() + rgbe.size() + (size_t)h * 8);
    for (int row = 0; row < h; row++) {
      const char head[4] = {2, 2, (char)((w >> 8) & 0xff), (char)(w & 0xff)};
      out.append(head, 4);
      const unsigned char *p = rgbe.data() + (size_t)row * w * 4;
      for (int k = 0; k < 4; k++) pack_plane(p + (size_t)k * w, w, out);
    }
  }
  /* IO::Loader::writeHdr appends the extension (Loader_image.cpp:51-52) */
  const std::string file = std::string(path) + ".hdr";
  std::ofstream f(file, std::ios::binary);
  if (!f) return fail(c, NOVA_B200_INVALID_ARGUMENT, "cannot write %s", file.c_str());
  f.write(out.data(), (std::streamsize)out.size());
  if (!f) return fail(c, NOVA_B200_RENDERER_EXCEPTION, "write failed: %s", file.c_str());
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_bake_texture(nova_b200_ctx *c, const char *type, int32_t out_w, int32_t out_h,
                                                   int32_t samples, const char *path_in, const char *path_out) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  if (!type || std::strcmp(type, "irradiance") != 0)
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "bake type must be \"irradiance\"%s");
  auto pow2 = [](int32_t v) { return v > 0 && (v & (v - 1)) == 0; };
  if (!pow2(out_w) || !pow2(out_h))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "irradiance size must be a power of two (TextureProcessing.cpp:11)%s");
  if (samples <= 0) return fail(c, NOVA_B200_INVALID_ARGUMENT, "samples must be positive%s");
  if (!path_out) return fail(c, NOVA_B200_INVALID_ARGUMENT, "path_out is null%s");
  int32_t w = 0, h = 0;
  nova_b200_status st = nova_b200_hdr_info(c, path_in, &w, &h);
  if (st) return st;
  cudaSetDevice(c->device);
  const size_t src_n = (size_t)w * h * 4, out_n = (size_t)out_w * out_h * 4;
  float *src = nullptr, *out = nullptr;
  NB_CUDA(c, cudaMallocAsync(&src, src_n * sizeof(float), c->stream), "cudaMalloc(environment map)");
  cudaError_t e = cudaMallocAsync(&out, out_n * sizeof(float), c->stream);
  /* the reference's output starts as zeros and its alpha channel is never written */
  if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, out_n * sizeof(float), c->stream);
  if (e != cudaSuccess) {
    cudaFreeAsync(src, c->stream);
    return cuda_fail(c, e, "cudaMalloc(irradiance map)");
  }
  st = nova_b200_hdr_read(c, path_in, nullptr, src, src_n);
  if (!st) st = nb_bake(c, src, w, h, 4, out_w, out_h, samples, out);
  if (!st) st = nova_b200_hdr_write(c, path_out, nullptr, out, out_w, out_h, 4, 0);
  cudaFreeAsync(src, c->stream);
  cudaFreeAsync(out, c->stream);
  cudaStreamSynchronize(c->stream);
  return st;
}

extern "C" nova_b200_status nova_b200_last_call_ms(nova_b200_ctx *c, float *device_ms) {
  using namespace nbctx;
  if (check_ctx(c) || !device_ms) return NOVA_B200_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  NB_CUDA(c, cudaEventElapsedTime(device_ms, c->ev_begin, c->ev_end), "last_call_ms");
  return NOVA_B200_SUCCESS;
}
