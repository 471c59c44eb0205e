/* ORACLE — test infrastructure only (parity checker, never the shipped path).
 *
 * CPU restatement of the film outputs and the Radiance .hdr format around the Nova render:
 *   orc_film_accumulate   Engine::writeFramebuffer, corelib/nova/api/engine.cpp:351-363
 *   orc_display_blend     NovaRenderer::copyBufferToPbo, sources/renderer/nova/NovaRenderer_draw.cpp:35-45
 *   orc_snapshot          NovaRenderer::getSnapshotFloat, sources/renderer/nova/NovaRenderer.cpp:139-153, with
 *                         TextureOperations::processTexture / uvSample / bilinearInterpolate /
 *                         discreteSample / wrapAroundTexCoords / wrapAroundPixelCoords,
 *                         sources/processing/TextureProcessing.h:157-250, and math_texturing.h:14-21
 *   orc_rgbe_encode       the float -> RGBE pixel of stbi_write_hdr, called by IO::Loader::writeHdr
 *                         (sources/IO/Loader_image.cpp:50-62)
 *   orc_rgbe_decode       the RGBE -> float pixel of stbi_loadf, called by IO::Loader::loadRadianceFile
 *                         (Loader_image.cpp:146-192), widened to RGBA with alpha 1 (:161-170)
 *   orc_hdr_parse         the header and scanline rules of the same loader (with the magic check of
 *                         load_magic_header, Loader_image.cpp:64-78)
 *   orc_hdr_write         the whole file as IO::Loader::writeHdr writes it (Loader_image.cpp:50-62)
 *
 * stb (github.com/nothings/stb, stb_image.h / stb_image_write.h) is an un-vendored submodule of the
 * reference (vendor/stb is empty; the snapshot records no pinned commit).  What is restated here is
 * the published Radiance RGBE format (G. Ward, "Real Pixels", Graphics Gems II, 1991) with the
 * rounding stb documents for it: encode m = max component, f = frexp(m), scale = f * 256 / m,
 * bytes truncated; decode c = byte * 2^(e - 136); run-length scanlines as in Radiance's "new" RLE.
 * Written independently of the device code: scalar loops, libm frexp / ldexp, x86-64 conversions.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "oracle.h"

extern "C" void orc_film_accumulate(const float *partial, float *accum, float *final_buf, uint64_t n,
                                    uint32_t frame_index) {
  for (uint64_t i = 0; i < n; i++) {
    accum[i] += partial[i];
    const float mean = accum[i] / float(frame_index + 1);
    if (final_buf) final_buf[i] = mean;
  }
}

extern "C" void orc_display_blend(const float *partial, const float *accum, float *out, uint64_t n,
                                  uint32_t current_frame) {
  for (uint64_t i = 0; i < n; i++) {
    const float old = accum[i] / (float)(current_frame + 1);
    const float now = partial[i];
    out[i] = old + 0.8f * (now - old);
  }
}

namespace {

struct Tex {
  const float *data;
  int width, height, channels;
  void sample(int x, int y, float out[3]) const {
    int xc, yc;
    if (x >= width)
      xc = x % width;
    else if (x < 0)
      xc = width + (x % width);
    else
      xc = x;
    if (y >= height)
      yc = y % height;
    else if (y < 0)
      yc = height + (y % height);
    else
      yc = y;
    /* the wrapped coordinates travel as a float vec2 and come back through static_cast<int> */
    const float fx = (float)xc, fy = (float)yc;
    const int idx = ((int)fy * width + (int)fx) * channels;
    out[0] = data[idx], out[1] = data[idx + 1], out[2] = data[idx + 2];
  }
};

float wrap_tex_coord(double c) {
  double ci = std::floor(c);
  double w = (c > 1. || c < 0.) ? c - ci : c;
  return (float)w;
}

unsigned uv_to_pixel(float coord, unsigned dim) { return static_cast<unsigned>(coord * dim); }

}  // namespace

extern "C" void orc_snapshot(const float *film, int32_t width, int32_t height, int32_t channels, float *dst,
                             int32_t dst_width, int32_t dst_height) {
  const Tex t{film, width, height, channels};
  for (int j = 0; j < dst_height; j++)
    for (int i = 0; i < dst_width; i++) {
      const double u = static_cast<double>(i) / static_cast<double>(dst_width);
      const double v = static_cast<double>(j) / static_cast<double>(dst_height);
      const float wu = wrap_tex_coord(u), wv = wrap_tex_coord(v);
      const double pxd = (double)uv_to_pixel(wu, (unsigned)width), pyd = (double)uv_to_pixel(wv, (unsigned)height);
      const float px = (float)pxd, py = (float)pyd;
      const float tlx = std::floor(px), tly = std::floor(py);
      const float trx = std::floor(px) + 1, bly = std::floor(py) + 1;
      const float uu = (px - tlx) / (trx - tlx);
      const float vv = (py - tly) / (bly - tly);
      const float hdiff = (1 - uu);
      float tl[3], tr[3], bl[3], br[3];
      t.sample((int)tlx, (int)tly, tl);
      t.sample((int)trx, (int)tly, tr);
      t.sample((int)tlx, (int)bly, bl);
      t.sample((int)trx, (int)bly, br);
      float *o = dst + ((size_t)j * dst_width + i) * channels;
      for (int k = 0; k < 3; k++) {
        const float top = hdiff * tl[k] + uu * tr[k];
        const float bot = hdiff * bl[k] + uu * br[k];
        o[k] = (1 - vv) * top + vv * bot;
      }
    }
}

/* x86-64 float -> int32 conversion (cvttss2si): truncation, NaN and out-of-range -> INT32_MIN */
static int32_t cvt_i32(float x) {
  if (std::isnan(x) || x >= 2147483648.f || x < -2147483648.f) return INT32_MIN;
  return (int32_t)x;
}

extern "C" void orc_rgbe_encode(const float *px, uint64_t n, int32_t channels, uint8_t *out) {
  for (uint64_t i = 0; i < n; i++) {
    const float *p = px + i * channels;
    float lin[3];
    if (channels >= 3) {
      lin[0] = p[0], lin[1] = p[1], lin[2] = p[2];
    } else {
      lin[0] = lin[1] = lin[2] = p[0];
    }
    const float inner = lin[1] > lin[2] ? lin[1] : lin[2];
    const float maxcomp = lin[0] > inner ? lin[0] : inner;
    uint8_t *q = out + 4 * i;
    if (maxcomp < 1e-32f) {
      q[0] = q[1] = q[2] = q[3] = 0;
      continue;
    }
    int exponent = 0;
    const double mant = std::frexp((double)maxcomp, &exponent); /* glibc: exponent 0 for inf / NaN */
    const float normalize = (float)mant * 256.0f / maxcomp;
    for (int k = 0; k < 3; k++) q[k] = (uint8_t)(cvt_i32(lin[k] * normalize) & 0xff);
    q[3] = (uint8_t)((exponent + 128) & 0xff);
  }
}

extern "C" void orc_rgbe_decode(const uint8_t *in, uint64_t n, float *out_rgba) {
  for (uint64_t i = 0; i < n; i++) {
    const uint8_t *q = in + 4 * i;
    float *o = out_rgba + 4 * i;
    if (q[3] != 0) {
      const float f1 = (float)std::ldexp(1.0f, (int)q[3] - (128 + 8));
      o[0] = q[0] * f1, o[1] = q[1] * f1, o[2] = q[2] * f1;
    } else {
      o[0] = o[1] = o[2] = 0.f;
    }
    o[3] = 1.f;
  }
}

/* Parses a whole .hdr file held in memory.  Returns 0 and the size (and, with rgbe != NULL, the
 * width * height interleaved RGBE bytes) or a non-zero code: 1 not a Radiance file (magic or first
 * line), 2 format line missing, 3 bad resolution line, 4 bad scanline length, 5 bad run-length data,
 * 6 OpenEXR. */
extern "C" int32_t orc_hdr_parse(const uint8_t *bytes, uint64_t size, int32_t *width, int32_t *height,
                                 uint8_t *rgbe) {
  char head[32] = {0};
  for (uint64_t i = 0; i < 31 && i < size; i++) head[i] = (char)bytes[i];
  if (size >= 4 && bytes[0] == 0x76 && bytes[1] == 0x2f && bytes[2] == 0x31 && bytes[3] == 0x01) return 6;
  if (std::strstr(head, "#?RADIANCE") == nullptr) return 1;
  uint64_t pos = 0;
  auto next = [&]() -> uint8_t { return pos < size ? bytes[pos++] : 0; };
  auto text_line = [&]() {
    std::string s;
    for (;;) {
      if (pos >= size) break;
      const char ch = (char)bytes[pos++];
      if (ch == '\n') break;
      if (s.size() < 1023) s += ch;
    }
    return s;
  };
  const std::string first = text_line();
  if (first != "#?RADIANCE" && first != "#?RGBE") return 1;
  bool rle_format = false;
  for (;;) {
    if (pos >= size) return 2;
    const std::string line = text_line();
    if (line.empty()) break;
    if (line == "FORMAT=32-bit_rle_rgbe") rle_format = true;
  }
  if (!rle_format) return 2;
  const std::string res = text_line();
  long h = 0, w = 0;
  {
    const char *p = res.c_str();
    if (std::strncmp(p, "-Y ", 3) != 0) return 3;
    char *end;
    h = std::strtol(p + 3, &end, 10);
    p = end;
    while (*p == ' ') ++p;
    if (std::strncmp(p, "+X ", 3) != 0) return 3;
    w = std::strtol(p + 3, nullptr, 10);
  }
  if (w <= 0 || h <= 0 || w > (1 << 24) || h > (1 << 24)) return 3;
  *width = (int32_t)w, *height = (int32_t)h;
  if (!rgbe) return 0;
  const uint64_t npx = (uint64_t)w * (uint64_t)h;
  std::memset(rgbe, 0, npx * 4);
  auto read_flat = [&](uint64_t from_byte) {
    for (uint64_t b = from_byte; b < npx * 4; b++) rgbe[b] = next();
  };
  if (w < 8 || w >= 32768) {
    read_flat(0);
    return 0;
  }
  std::vector<uint8_t> planes(4 * (size_t)w);
  for (long row = 0; row < h; row++) {
    const uint8_t a = next(), b = next(), c = next();
    if (a != 2 || b != 2 || (c & 0x80) != 0) {
      rgbe[0] = a, rgbe[1] = b, rgbe[2] = c, rgbe[3] = next();
      read_flat(4);
      return 0;
    }
    const long len = ((long)c << 8) | next();
    if (len != w) return 4;
    for (int comp = 0; comp < 4; comp++) {
      uint8_t *plane = &planes[(size_t)comp * w];
      long x = 0;
      while (x < w) {
        int count = next();
        const bool run = count > 128;
        if (run) count -= 128;
        if (count == 0 || count > w - x) return 5;
        if (run) {
          const uint8_t value = next();
          std::memset(plane + x, value, (size_t)count);
          x += count;
        } else {
          for (int k = 0; k < count; k++) plane[x++] = next();
        }
      }
    }
    uint8_t *dst = rgbe + (uint64_t)row * w * 4;
    for (long x = 0; x < w; x++)
      for (int comp = 0; comp < 4; comp++) dst[4 * x + comp] = planes[(size_t)comp * w + x];
  }
  return 0;
}

/* A whole .hdr file as IO::Loader::writeHdr writes it (path + ".hdr"; stbi_write_hdr's layout):
 * the Radiance header, then per row either flat RGBE pixels (width < 8 or >= 32768) or a run-length
 * scanline: (2, 2, width >> 8, width & 255) and, per component, dumps of up to 128 bytes up to the
 * next run of 3 or more equal bytes, then that run in packets of up to 127.  flip: rows bottom-up.
 * Returns 0, or 1 if the file cannot be written. */
extern "C" int32_t orc_hdr_write(const char *path, const float *px, int32_t width, int32_t height, int32_t channels,
                                 int32_t flip) {
  std::string file = std::string(path) + ".hdr";
  FILE *f = std::fopen(file.c_str(), "wb");
  if (!f) return 1;
  std::fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n", height, width);
  std::vector<uint8_t> pix((size_t)width * 4), comp((size_t)width), buf;
  buf.reserve((size_t)width * 5 + 16);
  for (int i = 0; i < height; i++) {
    const int row = flip ? height - 1 - i : i;
    orc_rgbe_encode(px + (size_t)row * width * channels, (uint64_t)width, channels, pix.data());
    buf.clear();
    if (width < 8 || width >= 32768) {
      buf.insert(buf.end(), pix.begin(), pix.end());
    } else {
      buf.push_back(2), buf.push_back(2), buf.push_back((uint8_t)(width >> 8)), buf.push_back((uint8_t)(width & 255));
      for (int k = 0; k < 4; k++) {
        for (int x = 0; x < width; x++) comp[x] = pix[4 * (size_t)x + k];
        int x = 0;
        while (x < width) {
          int r = x;
          while (r + 2 < width && !(comp[r] == comp[r + 1] && comp[r] == comp[r + 2])) r++;
          if (r + 2 >= width) r = width;
          while (x < r) {
            const int len = std::min(r - x, 128);
            buf.push_back((uint8_t)len);
            buf.insert(buf.end(), comp.begin() + x, comp.begin() + x + len);
            x += len;
          }
          if (r + 2 < width) {
            const uint8_t v = comp[r];
            while (r < width && comp[r] == v) r++;
            while (x < r) {
              const int len = std::min(r - x, 127);
              buf.push_back((uint8_t)(128 + len));
              buf.push_back(v);
              x += len;
            }
          }
        }
      }
    }
    std::fwrite(buf.data(), 1, buf.size(), f);
  }
  return std::fclose(f) == 0 ? 0 : 1;
}
