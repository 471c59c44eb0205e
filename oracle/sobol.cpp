/* ORACLE — test infrastructure only (see oracle.h).
 *
 * Sobol sampler with hash-based Owen scrambling, restating
 *   corelib/internal/common/math/math_random.h:37-98 (SobolGenerator) and
 *   scripts/generate_luts_sobol.py:51-95 (direction vectors from Joe & Kuo data), and the acos
 *   lookup table of scripts/generate_luts_trigonometrics.py:11-18 / math_acos_lt.cpp:37-40.
 */
#include "oracle.h"
#include "oracle_internal.h"
#include <cmath>
#include <cstring>
#include <vector>

namespace orc {

struct jk_row {
  int d, s, a;
  int m[12];
};
static const jk_row kJoeKuo[255] = {
#include "../axomae_b200/csrc/joe_kuo_params.inc"
};

/* Joe & Kuo recurrence: m_k = 2a_1 m_{k-1} ^ 4a_2 m_{k-2} ^ ... ^ 2^{s-1} a_{s-1} m_{k-s+1}
 * ^ 2^s m_{k-s} ^ m_{k-s}; a_1 is the most significant of the s-1 coefficient bits.  V_i = m_i << (32-i). */
static void expand_row(const jk_row &r, uint32_t out[32]) {
  uint64_t m[40];
  for (int i = 0; i < r.s; i++) m[i] = (uint64_t)r.m[i];
  for (int k = r.s; k < 32; k++) {
    uint64_t v = (m[k - r.s] << r.s) ^ m[k - r.s];
    for (int j = 1; j < r.s; j++) {
      int bit = (r.a >> (r.s - 1 - j)) & 1; /* a_j */
      if (bit) v ^= m[k - j] << j;
    }
    m[k] = v;
  }
  for (int i = 0; i < 32; i++) out[i] = (uint32_t)(m[i] << (31 - i));
}

static std::vector<uint32_t> build_table() {
  std::vector<uint32_t> t(256 * 32, 0u); /* row 255 stays zero, as in the reference table */
  for (int d = 0; d < 255; d++) expand_row(kJoeKuo[d], &t[d * 32]);
  return t;
}

const uint32_t *sobol_table() {
  static const std::vector<uint32_t> table = build_table(); /* thread-safe one-time init */
  return table.data();
}

static inline uint32_t reverse_bits(uint32_t x) {
  x = (((x & 0xaaaaaaaau) >> 1) | ((x & 0x55555555u) << 1));
  x = (((x & 0xccccccccu) >> 2) | ((x & 0x33333333u) << 2));
  x = (((x & 0xf0f0f0f0u) >> 4) | ((x & 0x0f0f0f0fu) << 4));
  x = (((x & 0xff00ff00u) >> 8) | ((x & 0x00ff00ffu) << 8));
  return ((x >> 16) | (x << 16));
}

static inline uint32_t owen_hash(uint32_t x, uint32_t seed) {
  x ^= x * 0x3d20adeau;
  x += seed;
  x *= (seed >> 16) | 0x1u;
  x ^= x * 0x05526c56u;
  x ^= x * 0x53a22864u;
  return x;
}

/* math_random.h:73-86: XOR of the direction vectors selected by gray(index), Owen scramble, then
 * float(accum) * (1.f / float(0xFFFFFFFF)); float(0xFFFFFFFF) rounds to 2^32 so the factor is 2^-32. */
float sobol_sample(uint32_t index, unsigned dim, uint32_t seed) {
  const uint32_t *dv = sobol_table() + dim * 32;
  uint32_t accum = 0;
  uint32_t gc = index ^ (index >> 1);
  for (unsigned i = 0; i < 32; i++)
    if ((gc >> i) & 1u) accum ^= dv[i];
  accum = reverse_bits(owen_hash(reverse_bits(accum), seed));
  const float one_uint_max = 1.f / float(0xFFFFFFFFu);
  return float(accum) * one_uint_max;
}

std::vector<float> make_acos_lut(int precision) {
  std::vector<float> lut(precision);
  for (int i = 0; i < precision; i++) {
    double scaled = ((double)i / (double)precision) * 2.0 - 1.0;
    lut[i] = (float)std::acos(scaled);
  }
  return lut;
}

const float *acos_lut() {
  static const std::vector<float> lut = make_acos_lut(kAcosPrecision);
  return lut.data();
}

}  // namespace orc

extern "C" void orc_sobol_table(uint32_t out[256 * 32]) { std::memcpy(out, orc::sobol_table(), 256 * 32 * 4); }

extern "C" void orc_sobol_samples(const uint32_t *index, const uint32_t *dim, uint64_t n, uint32_t seed, float *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = orc::sobol_sample(index[i], dim[i], seed);
}

extern "C" void orc_acos_lut(float *out, int32_t precision) {
  std::vector<float> l = orc::make_acos_lut(precision);
  std::memcpy(out, l.data(), sizeof(float) * precision);
}
