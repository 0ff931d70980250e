/* Oracle shim (test infrastructure only) for common/src/utils/otools.h.
 *
 * Supplies what the reference hot-path sources take from otools.h without
 * Boost/htslib: the STL includes, aligned_vector32, HAP_NUMBER / STAGE_*
 * constants (otools.h:78-86), the unphred table (otools.h:98; its 256 literals
 * are extracted from the reference source into _ref/unphred_table.inc by the
 * oracle Makefile), and logging/timer stand-ins. vrb.error throws instead of
 * calling exit(1) so a failed call surfaces as an error status in the harness. */
#pragma once
#include <vector>
#include <list>
#include <queue>
#include <stack>
#include <bitset>
#include <set>
#include <tuple>
#include <map>
#include <unordered_set>
#include <unordered_map>
#include <algorithm>
#include <numeric>
#include <array>
#include <cmath>
#include <string>
#include <exception>
#include <stdexcept>
#include <cassert>
#include <limits>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <fstream>
#include <iostream>
#include <boost/align/aligned_allocator.hpp>
#include <utils/random_number.h>
#include <utils/basic_stats.h>

template <typename T>
using aligned_vector32 = std::vector<T, boost::alignment::aligned_allocator<T, 32> >;

#define RARE_VARIANT_FREQ 0.001f
#define HAP_NUMBER 8
#define MAX_AMB 22
#define STAGE_INIT 0
#define STAGE_BURN 1
#define STAGE_MAIN 2
#define STAGE_RESTRICT 3
#define DIV2(v) ((v) >> 1)
#define MOD2(v) ((v) & 1)

const static float unphred[256] = {
#include "unphred_table.inc"
};

struct verbose {
  void bullet(const std::string&) {}
  void warning(const std::string&) {}
  void title(const std::string&) {}
  void wait(const std::string&) {}
  void progress(const std::string&, float) {}
  void error(const std::string& s) { throw std::runtime_error(s); }
};
struct string_utils {
  template <class T> std::string str(T v, int = 0) { std::ostringstream o; o << v; return o.str(); }
};
struct timer {
  void clock() {}
  long rel_time() { return 0; }
};
struct input_file : std::ifstream {
  explicit input_file(const std::string& f) : std::ifstream(f) {}
};

extern thread_local random_number_generator rng;
extern verbose vrb;
extern string_utils stb;
extern timer tac;
