/* nova_b200_bake: the irradiance bake command line on the B200 library.
 *
 *   nova_b200_bake --bake <type> <width> <height> <samples> <path_in> <path_out> [--gpu] [--device N]
 *
 * Mirrors the reference's `--bake` option (sources/controller/cmd/ProgramOptionsManager.cpp:76-79,
 * 116-137) and API::bakeTexture (sources/controller/cmd/API.cpp:44-62) without the Qt viewer it
 * opens afterwards: load the Radiance environment map (width * height RGBA, alpha 1), bake the
 * diffuse irradiance map of <width> x <height> texels (powers of two) with <samples> samples per
 * texel, write it to <path_out>.hdr.  Only the "irradiance" type is baked, as in the reference
 * (any other type leaves an empty image, which the reference's writer rejects).  The work is one
 * call, nova_b200_bake_texture_flags: the map is decoded, baked and encoded on the GPU.  --gpu / -g
 * selects the bake of the reference's CUDA kernel, as the reference's own --gpu option does
 * (ProgramOptionsManager.cpp:39-40,69); without it the bake follows the reference's CPU path.  Exit
 * status 0 on success, 1 on a usage or bake error.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/nova_b200.h"

namespace {

bool parse_int(const char *s, int &v) {
  char *end = nullptr;
  const long x = std::strtol(s, &end, 10);
  if (end == s || *end != 0 || x < 0 || x > (1 << 30)) return false;
  v = (int)x;
  return true;
}

int usage() {
  std::fprintf(stderr,
               "Usage: nova_b200_bake --bake [type] [width] [height] [samples] [path_in] [path_out] [--gpu] [--device N]\n"
               "Generates a texture of type [type] (irradiance) from the .hdr map [path_in] into [path_out].hdr\n");
  return 1;
}

int report(nova_b200_ctx *ctx, nova_b200_status st, const char *what) {
  char buf[1024] = {0};
  size_t n = 0;
  nova_b200_get_error(ctx, buf, &n);
  std::fprintf(stderr, "%s failed (status %d): %s\n", what, (int)st, buf);
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  const char *opts[6] = {};
  int device = 0, n_opts = -1;
  uint32_t flags = 0;
  for (int i = 1; i < argc; i++) {
    if (!std::strcmp(argv[i], "--bake") || !std::strcmp(argv[i], "-b")) {
      n_opts = 0;
      while (n_opts < 6 && i + 1 < argc && std::strncmp(argv[i + 1], "--", 2)) opts[n_opts++] = argv[++i];
    } else if (!std::strcmp(argv[i], "--gpu") || !std::strcmp(argv[i], "-g")) {
      flags |= NOVA_B200_BAKE_GPU_KERNEL;
    } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
      if (!parse_int(argv[++i], device)) return usage();
    } else {
      return usage();
    }
  }
  if (n_opts != 6) {
    std::fprintf(stderr, "Option \"--bake\" missing argument\n");
    return usage();
  }
  int out_w, out_h, samples;
  if (!parse_int(opts[1], out_w) || !parse_int(opts[2], out_h) || !parse_int(opts[3], samples)) {
    std::fprintf(stderr, "width, height and samples must be integers\n");
    return 1;
  }
  const std::string type = opts[0];
  if (type != "irradiance") {
    std::fprintf(stderr, "bake type \"%s\" produces no image (only \"irradiance\" is baked)\n", type.c_str());
    return 1;
  }

  nova_b200_ctx *ctx = nullptr;
  nova_b200_status st = nova_b200_create(&ctx, device);
  if (st) return report(ctx, st, "nova_b200_create");
  st = nova_b200_bake_texture_flags(ctx, type.c_str(), out_w, out_h, samples, opts[4], opts[5], flags);
  const int rc = st ? report(ctx, st, "irradiance bake") : 0;
  nova_b200_destroy(ctx);
  return rc;
}
