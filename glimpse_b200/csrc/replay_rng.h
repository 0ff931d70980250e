// Counter-based random streams shared by the device kernels and the host.
//
// The reference draws every random number from one global std::mt19937
// (common/src/utils/random_number.h:35-60, global `rng` in
// common/src/utils/otools.h:122), in an order that depends on the data and,
// with --threads > 1, on thread scheduling. A batched GPU path cannot follow
// one sequential engine, so the library keys an independent stream on
// (seed, purpose, iteration, target) and generates it with Philox4x32-10
// (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3",
// SC'11). Word i of a stream is lane (i & 3) of Philox(counter = {i >> 2,
// target, iteration, purpose}, key = seed).
//
// The reference's distributions are kept as they are: the oracle swaps only
// the engine behind `random_number_generator`, and the device code restates
// the libstdc++ distributions the reference calls on top of it
// (uniform_int_distribution<unsigned>, generate_canonical<float,24>,
// selection sampling in std::sample), so both sides consume identical words.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GP_HD __host__ __device__ __forceinline__
#else
#define GP_HD inline
#endif

namespace gp {

// Stream purposes, one per draw site of the reference.
enum RngPurpose : uint32_t {
  RNG_PBWT = 1,       // haplotype_set.cpp:336-348 (pbwt_stored groups, pbwt_index starts)
  RNG_SAMPLE_H0 = 2,  // genotype.cpp:118-120
  RNG_SAMPLE_H1 = 3,  // genotype.cpp:123-125
  RNG_PHASE = 4,      // phasing_hmm.cpp:256,282,297 and phasing_hmm.h:409
  RNG_INIT_SEL = 5,   // haplotype_set.cpp:807,818,826 (std::sample)
};

GP_HD void philox_mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds.
GP_HD void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                         uint32_t k0, uint32_t k1, uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    philox_mulhilo(M0, c0, hi0, lo0);
    philox_mulhilo(M1, c2, hi1, lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n1 = lo1;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    const uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0; k1 += W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Word `index` of the stream (seed, purpose, iteration, target).
GP_HD uint32_t stream_word(uint64_t seed, uint32_t purpose, uint32_t iteration,
                           uint32_t target, uint64_t index) {
  uint32_t o[4];
  philox4x32_10((uint32_t)(index >> 2), target, iteration, purpose ^ ((uint32_t)(index >> 34) << 8),
                (uint32_t)seed, (uint32_t)(seed >> 32), o);
  return o[index & 3];
}

// std::uniform_real_distribution<float>(0,1) over a 32-bit engine, as
// libstdc++ computes it: generate_canonical<float, 24> takes one word, converts
// it to float (round to nearest), scales by 2^-32, and maps a result of 1.0 to
// the largest float below 1. random_number.h:71-73 (getFloat).
GP_HD float canonical_float(uint32_t w) {
  float r = (float)w * 2.3283064365386963e-10f;  // 2^-32, exact
  if (r >= 1.0f) r = 0.99999994039535522f;        // nextafter(1.0f, 0.0f)
  return r;
}

// Lemire's nearly-divisionless bounded draw (Lemire, "Fast Random Integer
// Generation in an Interval", ACM TOMACS 29(1), 2019), the method libstdc++'s
// uniform_int_distribution uses for a 32-bit engine. Draws from [0, range)
// with range in [1, 2^32). Consumes one word, or more on rejection; `pos` is
// advanced past every word used.
template <class NextWord>
GP_HD uint32_t bounded_u32(NextWord& next, uint32_t range) {
  uint64_t product = (uint64_t)next() * (uint64_t)range;
  uint32_t low = (uint32_t)product;
  if (low < range) {
    const uint32_t threshold = (uint32_t)(0u - range) % range;
    while (low < threshold) {
      product = (uint64_t)next() * (uint64_t)range;
      low = (uint32_t)product;
    }
  }
  return (uint32_t)(product >> 32);
}

// std::uniform_int_distribution<unsigned>{a, b} over a 32-bit engine
// (random_number.h:63-65, getInt): a full-range request returns the word.
template <class NextWord>
GP_HD uint32_t uniform_uint(NextWord& next, uint32_t a, uint32_t b) {
  const uint32_t urange = b - a;
  if (urange == 0xFFFFFFFFu) return next() + a;
  return bounded_u32(next, urange + 1u) + a;
}

// Sequential reader over one stream.
struct StreamCursor {
  uint64_t seed;
  uint32_t purpose, iteration, target;
  uint64_t pos;
  GP_HD StreamCursor(uint64_t s, uint32_t p, uint32_t it, uint32_t t, uint64_t start = 0)
      : seed(s), purpose(p), iteration(it), target(t), pos(start) {}
  GP_HD uint32_t operator()() { return stream_word(seed, purpose, iteration, target, pos++); }
};

}  // namespace gp
