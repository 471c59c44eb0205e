/* Launch tuning and the autotuner (nova_b200_set_tuning / get_tuning / autotune).
 *
 * The reference has nothing to tune on its GPU path (one OptiX launch per frame) and only a tile
 * size on its CPU path (utils/nova_utils.h:34-53).  The wavefront's speed depends on the rays per
 * wave, the trace / shade block sizes, the pixel order in which paths start and the BVH layout;
 * none of them changes a result bit.  The autotuner times probe renders of the caller's own frames
 * (sample counts scaled down to about kProbePaths paths) and walks the parameters one at a time
 * (coordinate descent from the defaults), keeping a candidate only when it is faster by more than
 * kMinGain.  Results are cached in a text file, one line per workload key.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "context.cuh"

namespace {

constexpr uint64_t kProbePaths = 96ull << 20;
constexpr double kMinGain = 0.01;

bool valid_block(uint32_t b) { return b == 0 || b == 32 || b == 64 || b == 96 || b == 128; }

nova_b200_status check_tuning(nova_b200_ctx *c, const nova_b200_tuning &t) {
  using namespace nbctx;
  if (t.queue_capacity != 0 && (t.queue_capacity < 65536u || t.queue_capacity > (1u << 26)))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "queue_capacity must be 0 or 65536..67108864%s");
  if (!valid_block(t.trace_block) || !valid_block(t.shade_block))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "block sizes must be 0, 32, 64, 96 or 128%s");
  if ((t.tile_w == 0) != (t.tile_h == 0))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "tile_w and tile_h must both be 0 or both be set%s");
  if (t.trace_mode > 3) return fail(c, NOVA_B200_INVALID_ARGUMENT, "trace_mode must be 0, 1, 2 or 3%s");
  if (t.tile_w && !(t.tile_w == 1 && t.tile_h == 1) &&
      (t.tile_w > 64 || t.tile_h > 64 || (t.tile_w * t.tile_h) % 32 != 0))
    return fail(c, NOVA_B200_INVALID_ARGUMENT, "tiles must be 1 x 1 or at most 64 x 64 with a multiple of 32 pixels%s");
  return NOVA_B200_SUCCESS;
}

struct Probe {
  std::vector<nova_b200_ctx *> ctxs;
  std::vector<nova_b200_frame> frames;
};

/* Mrays/s of the probe under the tuning currently set on ctxs[0] (best of two renders). */
nova_b200_status measure(Probe &p, double &mrays) {
  double best = 0.0;
  for (int rep = 0; rep < 2; rep++) {
    nova_b200_render_stats st{};
    nova_b200_status s = nb_render_batch(p.ctxs.data(), p.frames.data(), (uint32_t)p.frames.size(), nullptr,
                                         nullptr, &st);
    if (s != NOVA_B200_SUCCESS) return s;
    if (st.device_ms > 0.0) best = std::max(best, (double)st.traced / st.device_ms / 1e3);
  }
  mrays = best;
  return NOVA_B200_SUCCESS;
}

std::string workload_key(const std::vector<nova_b200_ctx *> &ctxs, const nova_b200_frame *frames, uint32_t n,
                         uint32_t flags) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, ctxs[0]->device);
  uint64_t paths = 0;
  int depth = 0;
  for (uint32_t j = 0; j < n; j++) {
    paths += (uint64_t)frames[j].width * frames[j].height * (uint64_t)frames[j].sample_count;
    depth = std::max(depth, frames[j].max_depth);
  }
  const int lp = paths ? (int)std::lround(std::log2((double)paths)) : 0;
  std::ostringstream k;
  std::string name = prop.name;
  std::replace(name.begin(), name.end(), ' ', '_');
  /* with the width tuned, the key must not depend on the width the contexts happen to have */
  const int w = (flags & NOVA_B200_TUNE_BVH_WIDTH) ? 0 : ctxs[0]->bvh_width;
  k << name << "|sm" << prop.multiProcessorCount << "|n" << n << "|p2^" << lp << "|d" << depth << "|w" << w << "|f"
    << flags;
  return k.str();
}

bool read_cache(const char *path, const std::string &key, nova_b200_tuning &t) {
  if (!path) return false;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string k;
    nova_b200_tuning v{};
    if (ls >> k >> v.queue_capacity >> v.trace_block >> v.shade_block >> v.tile_w >> v.tile_h >> v.bvh_width >>
            v.trace_mode &&
        k == key) {
      t = v;
      return true;
    }
  }
  return false;
}

void write_cache(const char *path, const std::string &key, const nova_b200_tuning &t) {
  if (!path) return;
  std::vector<std::string> keep;
  {
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line))
      if (line.compare(0, key.size() + 1, key + " ") != 0 && !line.empty()) keep.push_back(line);
  }
  std::ofstream out(path, std::ios::trunc);
  for (const std::string &l : keep) out << l << "\n";
  out << key << " " << t.queue_capacity << " " << t.trace_block << " " << t.shade_block << " " << t.tile_w << " "
      << t.tile_h << " " << t.bvh_width << " " << t.trace_mode << "\n";
}

nova_b200_status rebuild_all(const std::vector<nova_b200_ctx *> &ctxs, int width) {
  nova_b200_bvh_options o{};
  o.width = width;
  for (nova_b200_ctx *c : ctxs) {
    if (c->bvh_width == width) continue;
    nova_b200_status s = nova_b200_build_bvh(c, &o);
    if (s != NOVA_B200_SUCCESS) return s;
  }
  return NOVA_B200_SUCCESS;
}

}  // namespace

extern "C" {

nova_b200_status nova_b200_set_tuning(nova_b200_ctx *c, const nova_b200_tuning *t) {
  if (!c) return NOVA_B200_INVALID_ARGUMENT;
  nova_b200_tuning v{};
  if (t) v = *t;
  nova_b200_status s = check_tuning(c, v);
  if (s != NOVA_B200_SUCCESS) return s;
  v.bvh_width = 0;
  c->tuning = v;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_get_tuning(nova_b200_ctx *c, nova_b200_tuning *t) {
  if (!c || !t) return NOVA_B200_INVALID_ARGUMENT;
  *t = c->tuning;
  t->bvh_width = c->bvh_width;
  return NOVA_B200_SUCCESS;
}

nova_b200_status nova_b200_autotune(nova_b200_ctx *const *ctxs, const nova_b200_frame *frames, uint32_t n,
                                    const char *cache_path, uint32_t flags, nova_b200_tuning *best) {
  using namespace nbctx;
  if (!ctxs || !ctxs[0]) return NOVA_B200_INVALID_ARGUMENT;
  nova_b200_ctx *x = ctxs[0];
  if (!frames || n == 0) return fail(x, NOVA_B200_INVALID_ARGUMENT, "empty batch%s");
  Probe p;
  p.ctxs.assign(ctxs, ctxs + n);
  for (nova_b200_ctx *c : p.ctxs) {
    if (!c) return fail(x, NOVA_B200_INVALID_ARGUMENT, "null context in batch%s");
    if (!c->bvh_ready) return fail(x, NOVA_B200_SCENE_NOT_PROCESSED, "build the acceleration structure first%s");
  }
  auto apply = [&](const nova_b200_tuning &t) {
    for (nova_b200_ctx *c : p.ctxs) {
      c->tuning = t;
      c->tuning.bvh_width = 0;
    }
  };
  const std::string key = workload_key(p.ctxs, frames, n, flags);
  nova_b200_tuning t{};
  if (read_cache(cache_path, key, t) && check_tuning(x, t) == NOVA_B200_SUCCESS) {
    if (t.bvh_width == 2 || t.bvh_width == 8) {
      nova_b200_status s = rebuild_all(p.ctxs, t.bvh_width);
      if (s != NOVA_B200_SUCCESS) return s;
    }
    apply(t);
    t.bvh_width = x->bvh_width;
    if (best) *best = t;
    return NOVA_B200_SUCCESS;
  }
  /* probe: the caller's frames with sample counts scaled to about kProbePaths paths in total */
  uint64_t total = 0;
  for (uint32_t j = 0; j < n; j++) total += (uint64_t)frames[j].width * frames[j].height * frames[j].sample_count;
  const double f = total > kProbePaths ? (double)kProbePaths / (double)total : 1.0;
  p.frames.assign(frames, frames + n);
  uint64_t probe_total = 0;
  for (nova_b200_frame &fr : p.frames) {
    fr.sample_count = std::max(1, (int32_t)std::floor(fr.sample_count * f));
    fr.reset = 1;
    probe_total += (uint64_t)fr.width * fr.height * fr.sample_count;
  }
  nova_b200_tuning cur{};
  apply(cur);
  double cur_rate = 0.0;
  nova_b200_status s = measure(p, cur_rate);
  if (s != NOVA_B200_SUCCESS) return s;
  auto consider = [&](const nova_b200_tuning &cand) -> nova_b200_status {
    apply(cand);
    double r = 0.0;
    nova_b200_status st = measure(p, r);
    if (st != NOVA_B200_SUCCESS) return st;
    if (r > cur_rate * (1.0 + kMinGain)) {
      cur = cand;
      cur_rate = r;
    }
    apply(cur);
    return NOVA_B200_SUCCESS;
  };
  /* rays per wave: up to the first power of two that holds the whole probe */
  for (uint32_t qc : {1u << 22, 1u << 24, 1u << 25}) {
    if ((uint64_t)qc > 2 * std::max<uint64_t>(probe_total, 1u << 22)) continue;
    nova_b200_tuning cand = cur;
    cand.queue_capacity = qc;
    if ((s = consider(cand)) != NOVA_B200_SUCCESS) return s;
  }
  for (uint32_t b : {64u, 96u}) {
    nova_b200_tuning cand = cur;
    cand.trace_block = b;
    if ((s = consider(cand)) != NOVA_B200_SUCCESS) return s;
  }
  for (uint32_t b : {64u, 96u}) {
    nova_b200_tuning cand = cur;
    cand.shade_block = b;
    if ((s = consider(cand)) != NOVA_B200_SUCCESS) return s;
  }
  if (x->bvh_width != 8) {
    nova_b200_tuning cand = cur;
    cand.trace_mode = 1;
    if ((s = consider(cand)) != NOVA_B200_SUCCESS) return s;
  }
  const uint32_t tiles[3][2] = {{1, 1}, {16, 2}, {8, 8}}; /* rows and two other tiles; 0 x 0 is 8 x 4 */
  for (const auto &tl : tiles) {
    nova_b200_tuning cand = cur;
    cand.tile_w = tl[0];
    cand.tile_h = tl[1];
    if ((s = consider(cand)) != NOVA_B200_SUCCESS) return s;
  }
  if (flags & NOVA_B200_TUNE_BVH_WIDTH) {
    const int w0 = x->bvh_width, w1 = w0 == 8 ? 2 : 8;
    if ((s = rebuild_all(p.ctxs, w1)) != NOVA_B200_SUCCESS) return s;
    double r = 0.0;
    if ((s = measure(p, r)) != NOVA_B200_SUCCESS) return s;
    if (r > cur_rate * (1.0 + kMinGain)) {
      cur_rate = r;
    } else if ((s = rebuild_all(p.ctxs, w0)) != NOVA_B200_SUCCESS) {
      return s;
    }
    cur.bvh_width = x->bvh_width;
  }
  apply(cur);
  cur.bvh_width = (flags & NOVA_B200_TUNE_BVH_WIDTH) ? x->bvh_width : 0;
  write_cache(cache_path, key, cur);
  cur.bvh_width = x->bvh_width;
  if (best) *best = cur;
  return NOVA_B200_SUCCESS;
}

}  // extern "C"
