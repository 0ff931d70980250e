/* Oracle shim (test infrastructure only). The reference includes simde's AVX2
 * header with SIMDE_ENABLE_NATIVE_ALIASES; on x86-64 built with -mavx2 -mfma,
 * simde forwards every _mm256_* name to the native intrinsic, so the native
 * header gives the same instructions and the same arithmetic. */
#pragma once
#include <immintrin.h>
