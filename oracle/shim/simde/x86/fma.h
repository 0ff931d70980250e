/* Oracle shim: simde FMA aliases resolve to the native intrinsics (see avx2.h). */
#pragma once
#include <immintrin.h>
