/* Sobol sampler with hash-based Owen scrambling on the device.
 *
 * Same generator as the reference's SobolGenerator (corelib/internal/common/math/math_random.h:37-98):
 * the gray code of the sample index selects direction vectors of a 256 x 32 table (Joe & Kuo
 * dimensions 2..256, table row 255 zero), the XOR is Owen-scrambled by reverse -> hash(seed) ->
 * reverse, and the result is float(accum) * 2^-32.  Instead of the reference's 32-step loop over
 * every bit, the device table holds, per dimension, the XORs of the vectors of every byte value at
 * each of the four byte positions, so the XOR over the gray code's set bits is four lookups (the
 * same value: XOR is associative and commutative).
 * The per-path dimension counter of SobolSampler (sampler/Sampler.h:17-55) is the caller's `dim`.
 */
#pragma once
#include "dmath.cuh"

namespace nb {

constexpr int kSobolDims = 256;
constexpr int kSobolBits = 32;
constexpr int kSobolByteTable = 4 * 256; /* u32 entries per dimension in the device table */

NB_HD uint32_t reverse_bits32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __brev(x);
#else
  x = (((x & 0xaaaaaaaau) >> 1) | ((x & 0x55555555u) << 1));
  x = (((x & 0xccccccccu) >> 2) | ((x & 0x33333333u) << 2));
  x = (((x & 0xf0f0f0f0u) >> 4) | ((x & 0x0f0f0f0fu) << 4));
  x = (((x & 0xff00ff00u) >> 8) | ((x & 0x00ff00ffu) << 8));
  return ((x >> 16) | (x << 16));
#endif
}

NB_HD uint32_t owen_hash(uint32_t x, uint32_t seed) {
  x ^= x * 0x3d20adeau;
  x += seed;
  x *= (seed >> 16) | 0x1u;
  x ^= x * 0x05526c56u;
  x ^= x * 0x53a22864u;
  return x;
}

/* 2^-32 as a float: the reference's 1.f / float(0xFFFFFFFF) (float(0xFFFFFFFF) rounds to 2^32). */
constexpr float kOneOverUintMax = 2.3283064365386963e-10f;

/* tab: kSobolDims x kSobolByteTable byte-sliced direction vectors (context.cu, sobol_byte_tables). */
NB_D float sobol_sample(const uint32_t *__restrict__ tab, uint32_t index, unsigned dim, uint32_t seed) {
  const uint32_t *t = tab + (size_t)dim * kSobolByteTable;
  const uint32_t gc = index ^ (index >> 1);
  uint32_t accum = __ldg(t + (gc & 255u)) ^ __ldg(t + 256 + ((gc >> 8) & 255u));
  accum ^= __ldg(t + 512 + ((gc >> 16) & 255u)) ^ __ldg(t + 768 + (gc >> 24));
  accum = reverse_bits32(owen_hash(reverse_bits32(accum), seed));
  return __uint2float_rn(accum) * kOneOverUintMax;
}

}  // namespace nb
