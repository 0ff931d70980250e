// Target genotype likelihoods from the FORMAT arrays of a target VCF/BCF, as
// genotype_reader::readTargetGenotypes reads them (phase/src/io/genotype_reader.cpp:427-500):
//   FORMAT/PL (int32):  phred = PL
//   FORMAT/GL (float):  phred = lroundf(-10 * GL)
// per sample and site, clamped to 255, into the uint8 phred layout that
// gp_targets_set takes (n x L x 3, ploidy + 1 bytes used) and the flat flags
// (n x L). The input is what htslib's bcf_get_format_int32 / _float return for
// each site, packed site after site: for site l, sample i, value c at
// src[(l * n + i) * P + c], with P = max ploidy + 1 over the targets.
//
// As in the reference:
//   * a site is read only when its value count divided by n equals P
//     (genotype_reader.cpp:433-435,473-475); otherwise it keeps the defaults;
//   * a sample whose values 0, 1 (and 2 when diploid) are not all present
//     (htslib's missing / vector-end markers) keeps the defaults;
//   * the defaults are phred 0 and flat (genotype.cpp:50-51);
//   * flat is cleared when the ploidy + 1 phred values are not all equal;
//   * a negative PL or a positive GL (a negative rounded phred) is an error.
//     The reference stops there; this returns GP_E_DATA naming the first such
//     entry in site-then-sample order, the order the reference reads.
//
// One CTA converts a tile of 32 sites x 32 samples: it reads each site's run of
// 32 samples (contiguous in the input), keeps the results in shared memory, and
// writes each sample's run of 32 sites (contiguous in the output).
#include <climits>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "context.h"
#include "internal.h"

namespace gp {
namespace {

constexpr int kTile = 32;
constexpr int kGlThreads = 256;

// htslib's markers: bcf_int32_missing / bcf_int32_vector_end, and the NaN
// payloads of bcf_float_missing / bcf_float_vector_end.
__device__ __forceinline__ bool absent(int32_t v) { return v == INT32_MIN || v == INT32_MIN + 1; }
__device__ __forceinline__ bool absent(float v) {
  const uint32_t b = __float_as_uint(v);
  return b == 0x7F800001u || b == 0x7F800002u;
}

// Rounded phred of one value; negative where the reference rejects it.
__device__ __forceinline__ long long phred_of(int32_t v) { return v; }
__device__ __forceinline__ long long phred_of(float v) {
  const float y = -10.0f * v;  // a float product, as in the reference
  // On the reference's x86-64 build, lroundf of NaN, of an infinity or of a
  // value outside the range of long returns LONG_MIN, which its check rejects.
  if (!(fabsf(y) < 9.2233720e18f)) return -1;
  return llroundf(y);
}

template <typename T>
__global__ void __launch_bounds__(kGlThreads) k_gl_input(const T* __restrict__ src, int n, int L, int P,
                                                         const int32_t* __restrict__ site_nval,
                                                         const int32_t* __restrict__ ploidy, uint8_t* __restrict__ gl,
                                                         uint8_t* __restrict__ flat,
                                                         unsigned long long* __restrict__ err) {
  // [site][sample]: phred 0 | phred 1 << 8 | phred 2 << 16 | flat << 24
  __shared__ uint32_t tile[kTile][kTile + 1];
  const int l0 = blockIdx.x * kTile, i0 = blockIdx.y * kTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kGlThreads / 32;
  for (int r = warp; r < kTile; r += kWarps) {
    const int l = l0 + r, i = i0 + lane;
    uint32_t out = 1u << 24;  // phred 0, flat
    if (l < L && i < n && (!site_nval || site_nval[l] / n == P)) {
      const int pl = ploidy[i];
      const T* v = src + ((size_t)l * n + i) * P;
      const T a = v[0], b = v[1];
      const T c = pl > 1 ? v[2] : a;
      if (!absent(a) && !absent(b) && !(pl > 1 && absent(c))) {
        const long long p0 = phred_of(a), p1 = phred_of(b), p2 = pl > 1 ? phred_of(c) : 0;
        if (p0 < 0 || p1 < 0 || p2 < 0) {
          atomicMin(err, (unsigned long long)l * (unsigned long long)n + (unsigned long long)i);
        } else {
          const uint32_t g0 = (uint32_t)(p0 < 255 ? p0 : 255), g1 = (uint32_t)(p1 < 255 ? p1 : 255);
          const uint32_t g2 = pl > 1 ? (uint32_t)(p2 < 255 ? p2 : 255) : 0u;
          const uint32_t glast = pl > 1 ? g2 : g1;  // gl[ploidy]
          const uint32_t fl = (g0 == g1 && g0 == glast) ? 1u : 0u;
          out = g0 | (g1 << 8) | (g2 << 16) | (fl << 24);
        }
      }
    }
    tile[r][lane] = out;
  }
  __syncthreads();
  for (int r = warp; r < kTile; r += kWarps) {
    const int i = i0 + r, l = l0 + lane;
    if (i < n && l < L) {
      const uint32_t o = tile[lane][r];
      uint8_t* g = gl + ((size_t)i * L + l) * 3;
      g[0] = (uint8_t)(o & 255u);
      g[1] = (uint8_t)((o >> 8) & 255u);
      g[2] = (uint8_t)((o >> 16) & 255u);
      flat[(size_t)i * L + l] = (uint8_t)(o >> 24);
    }
  }
}

template <typename T>
int gl_input(Context& c, int32_t n, int32_t L, const T* src, const int32_t* site_nval, const int32_t* ploidy,
             uint8_t* gl, uint8_t* flat, const char* fmt) {
  if (n <= 0 || L <= 0 || !src || !ploidy || !gl || !flat)
    return (c.fail(GP_E_ARG, std::string("gl from ") + fmt + ": bad argument"), GP_E_ARG);
  int P = 0;
  for (int i = 0; i < n; ++i) {
    if (ploidy[i] != 1 && ploidy[i] != 2)
      return (c.fail(GP_E_ARG, std::string("gl from ") + fmt + ": ploidy must be 1 or 2"), GP_E_ARG);
    P = ploidy[i] + 1 > P ? ploidy[i] + 1 : P;
  }
  if ((size_t)L * n > ((size_t)1 << 40) || (n + kTile - 1) / kTile > 65535)
    return (c.fail(GP_E_ARG, std::string("gl from ") + fmt + ": too many entries"), GP_E_ARG);
  const size_t nent = (size_t)L * n;
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) return c.cuda_fail(e, "gl input: current device");
  const int dev = c.cfg.device;
  if (prev != dev && (e = cudaSetDevice(dev)) != cudaSuccess) return c.cuda_fail(e, "gl input: set device");
  auto finish = [&](int rc) {
    if (prev != dev) cudaSetDevice(prev);
    return rc;
  };
  if ((e = c.glin_src.ensure(nent * P * sizeof(T))) != cudaSuccess ||
      (e = c.glin_ploidy.ensure((size_t)n * 4)) != cudaSuccess ||
      (e = c.glin_gl.ensure(nent * 3)) != cudaSuccess || (e = c.glin_flat.ensure(nent)) != cudaSuccess ||
      (e = c.glin_err.ensure(8)) != cudaSuccess ||
      (site_nval && (e = c.glin_nval.ensure((size_t)L * 4)) != cudaSuccess))
    return finish(c.cuda_fail(e, "gl input: alloc"));
  cudaStream_t s = c.stream;
  cudaMemcpyAsync(c.glin_src.ptr, src, nent * P * sizeof(T), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(c.glin_ploidy.ptr, ploidy, (size_t)n * 4, cudaMemcpyHostToDevice, s);
  if (site_nval) cudaMemcpyAsync(c.glin_nval.ptr, site_nval, (size_t)L * 4, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(c.glin_err.ptr, 0xff, 8, s);
  const dim3 grid((L + kTile - 1) / kTile, (n + kTile - 1) / kTile);
  k_gl_input<T><<<grid, kGlThreads, 0, s>>>(c.glin_src.as<T>(), n, L, P,
                                           site_nval ? c.glin_nval.as<int32_t>() : nullptr,
                                           c.glin_ploidy.as<int32_t>(), c.glin_gl.as<uint8_t>(),
                                           c.glin_flat.as<uint8_t>(), c.glin_err.as<unsigned long long>());
  c.prof.kernel_launches += 1;
  unsigned long long bad = 0;
  cudaMemcpyAsync(&bad, c.glin_err.ptr, 8, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return finish(c.cuda_fail(e, "gl input"));
  if (bad != ~0ull) {
    const unsigned long long site = bad / (unsigned long long)n, sample = bad % (unsigned long long)n;
    const std::string sign = std::string(fmt) == "PL" ? "negative" : "positive";
    return finish((c.fail(GP_E_DATA, "Found " + sign + " value in FORMAT/" + fmt + " for target [" +
                                         std::to_string(sample) + "] at site [" + std::to_string(site) + "]"),
                   GP_E_DATA));
  }
  cudaMemcpyAsync(gl, c.glin_gl.ptr, nent * 3, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(flat, c.glin_flat.ptr, nent, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return finish(c.cuda_fail(e, "gl input: copy out"));
  if ((e = cudaGetLastError()) != cudaSuccess) return finish(c.cuda_fail(e, "gl input: launch"));
  return finish(GP_OK);
}

}  // namespace
}  // namespace gp

extern "C" int gp_gl_from_pl(gp_ctx* ctx, int32_t n, int32_t L, const int32_t* pl, const int32_t* site_nval,
                             const int32_t* ploidy, uint8_t* gl, uint8_t* flat) {
  if (!ctx) return GP_E_ARG;
  return gp::gl_input<int32_t>(*reinterpret_cast<gp::Context*>(ctx), n, L, pl, site_nval, ploidy, gl, flat, "PL");
}

extern "C" int gp_gl_from_float(gp_ctx* ctx, int32_t n, int32_t L, const float* glf, const int32_t* site_nval,
                                const int32_t* ploidy, uint8_t* gl, uint8_t* flat) {
  if (!ctx) return GP_E_ARG;
  return gp::gl_input<float>(*reinterpret_cast<gp::Context*>(ctx), n, L, glf, site_nval, ploidy, gl, flat, "GL");
}
