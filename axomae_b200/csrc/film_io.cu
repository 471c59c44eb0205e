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
 * of width bytes (R, G, B, E: the order of run-length scanlines), 0 as interleaved pixels.  vec4:
 * 4-channel pixels at a 16-byte aligned address, read as one float4. */
__global__ void k_rgbe_encode(const float *src, int w, int h, int ch, int flip, int planar, int vec4,
                              unsigned char *dst) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, row = blockIdx.y;
  if (x >= w || row >= h) return;
  const int srow = flip ? h - 1 - row : row;
  const size_t px = (size_t)srow * w + x;
  float r, g, b;
  if (vec4) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(src) + px);
    r = v.x, g = v.y, b = v.z;
  } else if (ch >= 3) {
    const float *p = src + px * ch;
    r = p[0], g = p[1], b = p[2];
  } else {
    r = g = b = src[px * ch];
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
__device__ __forceinline__ float4 rgbe_decode(uint32_t word) {
  const uint32_t e = word >> 24;
  if (e == 0) return make_float4(0.f, 0.f, 0.f, 1.f);
  const double s = __longlong_as_double((long long)((int)e - 136 + 1023) << 52);
  return make_float4((float)((word & 0xffu) * s), (float)(((word >> 8) & 0xffu) * s),
                     (float)(((word >> 16) & 0xffu) * s), 1.f);
}

/* Four pixels per thread: one 16-byte load of RGBE words, four float4 stores (both buffers 16-byte
 * aligned); the last thread takes the ragged end pixel by pixel. */
__global__ void k_rgbe_decode(const uint32_t *src, uint64_t n, float4 *dst) {
  const uint64_t i4 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i4 + 4 <= n) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(src + i4));
    dst[i4] = rgbe_decode(q.x);
    dst[i4 + 1] = rgbe_decode(q.y);
    dst[i4 + 2] = rgbe_decode(q.z);
    dst[i4 + 3] = rgbe_decode(q.w);
  } else {
    for (uint64_t i = i4; i < n; i++) dst[i] = rgbe_decode(src[i]);
  }
}

/* Run-length packing, one warp per (row, plane) of the planar RGBE rows: runs of 3 or more equal
 * bytes become run packets (count + 128, value; count <= 127), the rest dump packets (count,
 * bytes; count <= 128).  The greedy scan is the serial one (next run start = first position whose
 * byte equals the next two; a run ends at the first different byte), with 32 positions tested per
 * step by a ballot; dump bytes are copied by all lanes.  Each warp writes its packets into its own
 * region of `cap` bytes (cap bounds the packets of any row: width + width / 128 + 2) and their size
 * into sizes; a region that would overflow sets *err and is cut. */
__global__ void k_rle_pack(const unsigned char *planar, int w, int n_planes, int cap, unsigned char *regions,
                           uint32_t *sizes, unsigned *err) {
  const int e = (int)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (e >= n_planes) return; /* whole warps leave together */
  const unsigned char *p = planar + (size_t)e * w; /* planes are consecutive: row-major (row, plane) */
  unsigned char *o = regions + (size_t)e * cap;
  int n = 0, x = 0;
  bool over = false;
  while (x < w) {
    int lit = w;
    for (int base = x; base < w; base += 32) {
      const int i = base + lane;
      const bool t = i + 2 < w && p[i] == p[i + 1] && p[i] == p[i + 2];
      const unsigned m = __ballot_sync(0xffffffffu, t);
      if (m) {
        lit = base + __ffs(m) - 1;
        break;
      }
    }
    while (x < lit) {
      const int cnt = min(lit - x, 128);
      if (n + 1 + cnt > cap) {
        over = true;
        break;
      }
      if (lane == 0) o[n] = (unsigned char)cnt;
      for (int k = lane; k < cnt; k += 32) o[n + 1 + k] = p[x + k];
      n += 1 + cnt;
      x += cnt;
    }
    if (over) break;
    if (lit < w) {
      const unsigned char v = p[lit];
      int end = w;
      for (int base = lit; base < w; base += 32) {
        const int i = base + lane;
        const unsigned m = __ballot_sync(0xffffffffu, i >= w || p[i] != v);
        if (m) {
          end = min(base + __ffs(m) - 1, w);
          break;
        }
      }
      while (x < end) {
        const int cnt = min(end - x, 127);
        if (n + 2 > cap) {
          over = true;
          break;
        }
        if (lane == 0) o[n] = (unsigned char)(128 + cnt), o[n + 1] = v;
        n += 2;
        x += cnt;
      }
      if (over) break;
    }
  }
  if (lane == 0) {
    if (over) atomicAdd(err, 1u);
    sizes[e] = (uint32_t)n;
  }
}

/* Exclusive scan of the packed sizes into file offsets, one block of 1024 threads: element
 * (row, plane 0) also carries the row's 4-byte header.  offsets[n] = total bytes. */
__global__ void __launch_bounds__(1024) k_rle_scan(const uint32_t *sizes, int n, uint64_t *offsets) {
  __shared__ uint64_t part[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const int b = min(t * chunk, n), e = min(b + chunk, n);
  uint64_t sum = 0;
  for (int i = b; i < e; i++) sum += sizes[i] + ((i & 3) == 0 ? 4u : 0u);
  part[t] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) { /* inclusive Hillis-Steele scan */
    const uint64_t v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint64_t run = part[t] - sum;
  for (int i = b; i < e; i++) {
    offsets[i] = run;
    run += sizes[i] + ((i & 3) == 0 ? 4u : 0u);
  }
  if (t == 1023) offsets[n] = part[1023];
}

/* One warp per (row, plane): its packets to their file offset; plane 0 writes the row header
 * (2, 2, width >> 8, width & 255) first. */
__global__ void k_rle_gather(const unsigned char *regions, const uint32_t *sizes, const uint64_t *offsets, int w,
                             int cap, int n_planes, unsigned char *out) {
  const int e = (int)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (e >= n_planes) return;
  uint64_t dst = offsets[e];
  if ((e & 3) == 0) {
    if (lane < 4) out[dst + lane] = lane < 2 ? 2 : (lane == 2 ? (unsigned char)(w >> 8) : (unsigned char)(w & 255));
    dst += 4;
  }
  const unsigned char *src = regions + (size_t)e * cap;
  const uint32_t n = sizes[e];
  for (uint32_t j = lane; j < n; j += 32) out[dst + j] = src[j];
}

/* Run-length expansion, one warp per (row, plane): the packets starting at file offset starts[e]
 * (found and checked on the host) into byte `plane` of each RGBE pixel of the row; lane 0 reads
 * each packet's count, all lanes copy or fill.  The body buffer is zero-padded past the file's end,
 * which the loader reads as zeros. */
__global__ void k_rle_unpack(const unsigned char *body, const uint64_t *starts, int w, int n_planes,
                             unsigned char *rgbe) {
  const int e = (int)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (e >= n_planes) return;
  const unsigned char *p = body + starts[e];
  unsigned char *o = rgbe + (size_t)(e >> 2) * w * 4 + (e & 3);
  int x = 0;
  while (x < w) {
    int cnt = __shfl_sync(0xffffffffu, lane == 0 ? (int)p[0] : 0, 0);
    if (cnt == 0) break; /* excluded by the host's check; never loops without progress */
    if (cnt > 128) {
      cnt = min(cnt - 128, w - x);
      const unsigned char v = p[1];
      for (int k = lane; k < cnt; k += 32) o[4 * (size_t)(x + k)] = v;
      p += 2;
    } else {
      cnt = min(cnt, w - x);
      for (int k = lane; k < cnt; k += 32) o[4 * (size_t)(x + k)] = p[1 + k];
      p += 1 + cnt;
    }
    x += cnt;
  }
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

/* Where the scanlines are.  Rows of a width in [8, 32768) are run-length packets: a row header
 * (2, 2, width >> 8, width & 255), then for each of R, G, B, E packets that are either a run
 * (count + 128, value) or a dump (count, count bytes), count in 1..remaining.  The host walks the
 * packet headers only (one byte per packet; dump data is skipped) to check them and to find where
 * each (row, plane) starts; the device expands them.  A row whose first bytes are not a run-length
 * header means the file is flat from there: those 4 bytes are pixel 0 of row 0 and the rest follow
 * in order (the stb loader's rule, kept as is).  Reading past the end yields zeros. */
struct Layout {
  bool flat = false;
  std::vector<unsigned char> flat_rgbe; /* flat files: the interleaved RGBE pixels */
  std::vector<uint64_t> starts;         /* run-length files: file offset of each (row, plane) */
};

nova_b200_status scan_rows(nova_b200_ctx *c, const std::vector<unsigned char> &bytes, const Header &hd,
                           Layout &L) {
  using namespace nbctx;
  const size_t w = (size_t)hd.w, h = (size_t)hd.h;
  Reader r{bytes, hd.data};
  auto flat_from = [&](size_t first_byte) {
    L.flat = true;
    L.flat_rgbe.assign(w * h * 4, 0);
    const size_t avail = r.pos < bytes.size() ? bytes.size() - r.pos : 0;
    const size_t n = std::min(avail, w * h * 4 - first_byte);
    if (n) std::memcpy(&L.flat_rgbe[first_byte], &bytes[r.pos], n);
  };
  if (!rle_width(hd.w)) {
    flat_from(0);
    return NOVA_B200_SUCCESS;
  }
  L.starts.resize(4 * h);
  for (size_t j = 0; j < h; j++) {
    const unsigned char c1 = r.get(), c2 = r.get(), c3 = r.get();
    if (c1 != 2 || c2 != 2 || (c3 & 0x80)) {
      const unsigned char c4 = r.get();
      flat_from(4);
      L.flat_rgbe[0] = c1, L.flat_rgbe[1] = c2, L.flat_rgbe[2] = c3, L.flat_rgbe[3] = c4;
      return NOVA_B200_SUCCESS;
    }
    const size_t len = ((size_t)c3 << 8) | r.get();
    if (len != w) return fail(c, NOVA_B200_INVALID_ARGUMENT, "invalid decoded scanline length%s");
    for (int k = 0; k < 4; k++) {
      L.starts[4 * j + k] = r.pos;
      size_t i = 0;
      while (i < w) {
        unsigned count = r.get();
        const size_t left = w - i;
        const bool run = count > 128;
        if (run) count -= 128;
        if (count == 0 || count > left) return fail(c, NOVA_B200_INVALID_ARGUMENT, "bad RLE data in HDR%s");
        if (run)
          r.get();
        else
          r.pos = std::min(r.pos + count, bytes.size() + 256); /* dump data: skipped, zeros past the end */
        i += count;
      }
    }
  }
  return NOVA_B200_SUCCESS;
}

/* The file, or its first `limit` bytes (limit 0: all); *whole tells whether all of it was read. */
nova_b200_status read_file(nova_b200_ctx *c, const char *path, std::vector<unsigned char> &bytes, size_t limit = 0,
                           bool *whole = nullptr) {
  using namespace nbctx;
  if (!path) return fail(c, NOVA_B200_INVALID_ARGUMENT, "path is null%s");
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return fail(c, NOVA_B200_INVALID_ARGUMENT, "cannot open %s", path);
  const std::streamoff size = f.tellg();
  if (size < 0) return fail(c, NOVA_B200_INVALID_ARGUMENT, "cannot read %s", path);
  const size_t n = limit ? std::min((size_t)size, limit) : (size_t)size;
  bytes.resize(n);
  f.seekg(0);
  if (n && !f.read(reinterpret_cast<char *>(bytes.data()), (std::streamsize)n))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "cannot read %s", path);
  if (whole) *whole = n == (size_t)size;
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
  /* the header from the first 64 KB; the whole file only when the header runs past them */
  std::vector<unsigned char> bytes;
  bool whole = false;
  nova_b200_status st = read_file(c, path, bytes, 65536, &whole);
  if (st) return st;
  Header hd;
  st = parse_header(c, bytes, hd);
  if (!whole && (st || hd.data >= bytes.size())) {
    if ((st = read_file(c, path, bytes))) return st;
    st = parse_header(c, bytes, hd);
  }
  if (st) return st;
  if (width) *width = hd.w;
  if (height) *height = hd.h;
  return NOVA_B200_SUCCESS;
}

extern "C" nova_b200_status nova_b200_hdr_read(nova_b200_ctx *c, const char *path, float *rgba_host,
                                               float *rgba_device, uint64_t capacity) {
  using namespace nbctx;
  if (check_ctx(c)) return NOVA_B200_INVALID_ARGUMENT;
  std::vector<unsigned char> bytes;
  nova_b200_status st = read_file(c, path, bytes);
  if (st) return st;
  Header hd;
  if ((st = parse_header(c, bytes, hd))) return st;
  const uint64_t npx = (uint64_t)hd.w * hd.h;
  if (npx > (1ull << 31)) return fail(c, NOVA_B200_INVALID_ARGUMENT, "HDR image larger than 2^31 pixels%s");
  if (capacity < npx * 4) return fail(c, NOVA_B200_INVALID_ARGUMENT, "output holds fewer than width * height * 4 floats%s");
  if (rgba_device && (reinterpret_cast<uintptr_t>(rgba_device) & 15))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "rgba_device must be 16-byte aligned%s");
  Layout L;
  if ((st = scan_rows(c, bytes, hd, L))) return st;
  cudaSetDevice(c->device);
  const int n_planes = 4 * hd.h;
  /* run-length files: the body (padded with zeros) and the plane offsets go to the device */
  const size_t body_n = L.flat ? 0 : bytes.size() - hd.data + 256;
  unsigned char *d_rgbe = nullptr, *d_body = nullptr;
  uint64_t *d_starts = nullptr;
  float4 *d_out = reinterpret_cast<float4 *>(rgba_device), *tmp = nullptr;
  NB_CUDA(c, cudaMallocAsync(&d_rgbe, npx * 4, c->stream), "cudaMalloc(hdr bytes)");
  cudaError_t e = cudaSuccess;
  if (L.flat) {
    e = cudaMemcpyAsync(d_rgbe, L.flat_rgbe.data(), npx * 4, cudaMemcpyHostToDevice, c->stream);
  } else {
    const size_t file_n = bytes.size() - hd.data;
    for (auto &o : L.starts) o -= hd.data;
    e = cudaMallocAsync(&d_body, body_n, c->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_starts, n_planes * sizeof(uint64_t), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_body + file_n, 0, body_n - file_n, c->stream);
    if (e == cudaSuccess && file_n)
      e = cudaMemcpyAsync(d_body, bytes.data() + hd.data, file_n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_starts, L.starts.data(), n_planes * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream);
  }
  if (e == cudaSuccess && !d_out) {
    e = cudaMallocAsync(&tmp, npx * sizeof(float4), c->stream);
    d_out = tmp;
  }
  if (e == cudaSuccess) {
    cudaEventRecord(c->ev_begin, c->stream);
    if (!L.flat)
      k_rle_unpack<<<(unsigned)(((uint64_t)n_planes * 32 + 127) / 128), 128, 0, c->stream>>>(d_body, d_starts, hd.w,
                                                                                               n_planes, d_rgbe);
    const uint64_t threads = (npx + 3) / 4;
    k_rgbe_decode<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(reinterpret_cast<const uint32_t *>(d_rgbe),
                                                                              npx, d_out);
    e = cudaGetLastError();
    cudaEventRecord(c->ev_end, c->stream);
  }
  if (e == cudaSuccess && rgba_host)
    e = cudaMemcpyAsync(rgba_host, d_out, npx * sizeof(float4), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFreeAsync(d_rgbe, c->stream);
  if (d_body) cudaFreeAsync(d_body, c->stream);
  if (d_starts) cudaFreeAsync(d_starts, c->stream);
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
  const bool vec4 = channels == 4 && !(reinterpret_cast<uintptr_t>(pixels_device) & 15);
  cudaSetDevice(c->device);
  const int n_planes = 4 * h;
  const int cap = w + w / 64 + 8; /* > width + width / 128 + 2, the most packets a row plane takes */
  const size_t regions_n = rle ? (size_t)n_planes * cap : 0, out_cap = rle ? regions_n + 4 * (size_t)h : npx * 4;
  unsigned char *d_rgbe = nullptr, *d_regions = nullptr, *d_out = nullptr;
  uint32_t *d_sizes = nullptr;
  uint64_t *d_offsets = nullptr;
  unsigned *d_err = nullptr;
  float *d_src = const_cast<float *>(pixels_device), *tmp = nullptr;
  NB_CUDA(c, cudaMallocAsync(&d_rgbe, npx * 4, c->stream), "cudaMalloc(hdr bytes)");
  cudaError_t e = cudaSuccess;
  if (!d_src) {
    e = cudaMallocAsync(&tmp, npx * channels * sizeof(float), c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tmp, pixels_host, npx * channels * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    d_src = tmp;
  }
  if (rle) {
    if (e == cudaSuccess) e = cudaMallocAsync(&d_regions, regions_n, c->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_out, out_cap, c->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_sizes, n_planes * sizeof(uint32_t), c->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_offsets, (n_planes + 1) * sizeof(uint64_t) + 16, c->stream);
    if (e == cudaSuccess) {
      d_err = reinterpret_cast<unsigned *>(d_offsets + n_planes + 1);
      e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), c->stream);
    }
  }
  if (e == cudaSuccess) {
    cudaEventRecord(c->ev_begin, c->stream);
    k_rgbe_encode<<<dim3((unsigned)((w + 127) / 128), (unsigned)h), 128, 0, c->stream>>>(
        d_src, w, h, channels, flip, rle ? 1 : 0, (vec4 || (tmp && channels == 4)) ? 1 : 0, d_rgbe);
    if (rle) {
      k_rle_pack<<<(unsigned)(((uint64_t)n_planes * 32 + 127) / 128), 128, 0, c->stream>>>(d_rgbe, w, n_planes, cap,
                                                                                             d_regions, d_sizes, d_err);
      k_rle_scan<<<1, 1024, 0, c->stream>>>(d_sizes, n_planes, d_offsets);
      k_rle_gather<<<(unsigned)(((uint64_t)n_planes * 32 + 255) / 256), 256, 0, c->stream>>>(
          d_regions, d_sizes, d_offsets, w, cap, n_planes, d_out);
    }
    e = cudaGetLastError();
    cudaEventRecord(c->ev_end, c->stream);
  }
  /* the packed size and the overflow flag, then exactly the packed bytes */
  uint64_t tail[2] = {npx * 4, 0};
  if (e == cudaSuccess && rle)
    e = cudaMemcpyAsync(tail, d_offsets + n_planes, sizeof(uint64_t) + sizeof(unsigned), cudaMemcpyDeviceToHost,
                        c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  std::string out = "#?RADIANCE\n# nova_b200\nFORMAT=32-bit_rle_rgbe\n\n-Y " + std::to_string(h) + " +X " +
                    std::to_string(w) + "\n";
  const size_t head_n = out.size(), body_n = (size_t)tail[0];
  const bool overflow = rle && (uint32_t)tail[1] != 0;
  if (e == cudaSuccess && !overflow && body_n <= out_cap) {
    out.resize(head_n + body_n);
    e = cudaMemcpyAsync(&out[head_n], rle ? d_out : d_rgbe, body_n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  }
  for (void *ptr : {(void *)d_rgbe, (void *)d_regions, (void *)d_out, (void *)d_sizes, (void *)d_offsets, (void *)tmp})
    if (ptr) cudaFreeAsync(ptr, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "hdr_write");
  if (overflow || body_n > out_cap) return fail(c, NOVA_B200_RENDERER_EXCEPTION, "run-length packing overflow%s");
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
  return nova_b200_bake_texture_flags(c, type, out_w, out_h, samples, path_in, path_out, 0u);
}

extern "C" nova_b200_status nova_b200_bake_texture_flags(nova_b200_ctx *c, const char *type, int32_t out_w,
                                                         int32_t out_h, int32_t samples, const char *path_in,
                                                         const char *path_out, uint32_t flags) {
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
  if (!st)
    st = (flags & NOVA_B200_BAKE_GPU_KERNEL) ? nb_bake_texunit(c, src, w, h, 4, out_w, out_h, samples, out)
                                             : nb_bake(c, src, w, h, 4, out_w, out_h, samples, out);
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
