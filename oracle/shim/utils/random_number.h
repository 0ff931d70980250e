/* Oracle shim (test infrastructure only) for common/src/utils/random_number.h.
 *
 * The class keeps the reference's name, members and distribution calls
 * (random_number.h:35-125): getInt, getFloat, getDouble, sample, and the public
 * `randomEngine` that std::sample is handed (haplotype_set.cpp:807,818,826).
 * Only the engine changes: instead of std::mt19937 it is a replay engine that
 * yields the words of one counter-based stream (glimpse_b200/csrc/replay_rng.h).
 * The oracle driver selects the stream (purpose, iteration, target) before each
 * reference call, so the reference code and the GPU kernels consume the same
 * words. `rng` is thread_local so that threaded oracle runs stay reproducible.
 *
 * With GP_NATIVE_RNG defined (the native-RNG oracle build) this header instead
 * includes the reference's own random_number.h, unmodified: std::mt19937 seeded
 * once, drawn in the reference's call order on one thread. */
#pragma once
#ifdef GP_NATIVE_RNG
#include <cmath>
#include_next <utils/random_number.h>
#else
#include <cfloat>
#include <cstdint>
#include <random>
#include <vector>
#include <istream>
#include <ostream>
#include "../../../glimpse_b200/csrc/replay_rng.h"

class replay_engine {
public:
  typedef uint32_t result_type;
  uint64_t seed = 15052011ull;
  uint32_t purpose = 0, iteration = 0, target = 0;
  uint64_t pos = 0;
  static constexpr result_type min() { return 0u; }
  static constexpr result_type max() { return 0xFFFFFFFFu; }
  result_type operator()() { return gp::stream_word(seed, purpose, iteration, target, pos++); }
  void select(uint32_t p, uint32_t it, uint32_t t) { purpose = p; iteration = it; target = t; pos = 0; }
  void seed_with(uint64_t s) { seed = s; pos = 0; }
  friend std::ostream& operator<<(std::ostream& o, const replay_engine& e) {
    return o << e.seed << ' ' << e.purpose << ' ' << e.iteration << ' ' << e.target << ' ' << e.pos;
  }
  friend std::istream& operator>>(std::istream& i, replay_engine& e) {
    return i >> e.seed >> e.purpose >> e.iteration >> e.target >> e.pos;
  }
};

class random_number_generator {
protected:
  unsigned int seed;
  std::uniform_int_distribution<unsigned int> uniformDistributionInt;
  std::uniform_real_distribution<double> uniformDistributionDouble;
  std::uniform_real_distribution<float> uniformDistributionFloat;
public:
  replay_engine randomEngine;

  random_number_generator(unsigned int _seed = 15052011)
      : seed(_seed), uniformDistributionInt(0, 32768), uniformDistributionDouble(0, 1.0),
        uniformDistributionFloat(0.0f, 1.0f) { randomEngine.seed_with(_seed); }

  void setSeed(unsigned int _seed) { seed = _seed; randomEngine.seed_with(_seed); }
  unsigned int getSeed() { return seed; }
  replay_engine& getEngine() { return randomEngine; }

  unsigned int getInt(unsigned int imin, unsigned int imax) {
    return uniformDistributionInt(randomEngine, std::uniform_int_distribution<unsigned int>{imin, imax}.param());
  }
  unsigned int getInt(unsigned int isize) { return getInt(0, isize - 1); }
  double getFloat(float fmin = 0.0f, float fmax = 1.0f) {
    return uniformDistributionFloat(randomEngine, std::uniform_real_distribution<float>{fmin, fmax}.param());
  }
  double getDouble(double fmin, double fmax) {
    return uniformDistributionDouble(randomEngine, std::uniform_real_distribution<double>{fmin, fmax}.param());
  }
  double getDouble() { return getDouble(0.0, 1.0); }
  bool flipCoin() { return (getDouble() < 0.5); }

  /* Categorical draw with a running float sum, as random_number.h:89-97. */
  int sample(std::vector<float>& vec, float sum) {
    float csum = vec[0];
    float u = getFloat() * sum;
    for (int i = 0; i < (int)vec.size() - 1; ++i) {
      if (u <= csum) return i;
      csum += vec[i + 1];
    }
    return vec.size() - 1;
  }
  int sample(std::vector<double>& vec, double sum) {
    double csum = vec[0];
    double u = getDouble() * sum;
    for (int i = 0; i < (int)vec.size() - 1; ++i) {
      if (u < csum) return i;
      csum += vec[i + 1];
    }
    return vec.size() - 1;
  }
};
#endif  // GP_NATIVE_RNG
