// Ligation of consecutive phased chunks (GLIMPSE2_ligate,
// ligate/src/ligater/ligater_algorithm.cpp): the phase-flip counting over the
// overlap of two chunks and the allele swap of the records that follow.
//
// GT values are htslib's int32 encoding (2 per sample; bcf_gt_phased(a) =
// (a + 1) << 1 | 1, missing = allele field 0, bcf_int32_vector_end for the
// absent second allele of a haploid sample).
//
//   gp_ligate_overlap  ligater::update_distances (:108-127) over the overlap
//                      sites, then the decision of ligater::scan_overlap
//                      (:183-205): swap_next[i] = nmatch < nmism, and the
//                      entropy phase quality, computed on the host with the C
//                      library's logf as the reference computes it.
//   gp_ligate_swap     ligater::phase_update (:90-106) on a chunk's records.
//
// The counts are integers, so their order does not matter: one thread per
// sample walks the overlap sites (consecutive threads read consecutive samples
// of a site). The swap is one thread per (site, sample).
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "context.h"
#include "internal.h"

namespace gp {
namespace {

constexpr int32_t kGtVectorEnd = INT32_MIN + 1;  // bcf_int32_vector_end

__device__ __forceinline__ bool gt_missing(int32_t g) { return (g >> 1) == 0; }
__device__ __forceinline__ bool gt_phased(int32_t g) { return (g & 1) != 0; }
__device__ __forceinline__ int32_t gt_allele(int32_t g) { return (g >> 1) - 1; }
__device__ __forceinline__ int32_t gt_make_phased(int32_t a) { return ((a + 1) << 1) | 1; }

__global__ void k_ligate_counts(int n, int m, const int32_t* __restrict__ gta, const int32_t* __restrict__ gtb,
                                const uint8_t* __restrict__ swap_prev, int32_t* __restrict__ nmatch,
                                int32_t* __restrict__ nmism) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool sw = swap_prev[i] != 0;
  int32_t match = 0, mism = 0;
  for (int s = 0; s < m; ++s) {
    const size_t o = ((size_t)s * n + i) * 2;
    const int32_t a0 = gta[o], a1 = gta[o + 1], b0 = gtb[o], b1 = gtb[o + 1];
    if (a1 == kGtVectorEnd || b1 == kGtVectorEnd) continue;
    if (gt_missing(a0) || gt_missing(a1) || gt_missing(b0) || gt_missing(b1)) continue;
    if (!gt_phased(a1) || !gt_phased(b1)) continue;
    const int32_t x0 = gt_allele(a0), x1 = gt_allele(a1), y0 = gt_allele(b0), y1 = gt_allele(b1);
    if (x0 == x1 || y0 == y1) continue;
    if (x0 == y0 && x1 == y1) {
      if (sw) ++mism; else ++match;
    }
    if (x0 == y1 && x1 == y0) {
      if (sw) ++match; else ++mism;
    }
  }
  nmatch[i] = match;
  nmism[i] = mism;
}

__global__ void k_ligate_swap(int n, size_t nent, int32_t* __restrict__ gt, const uint8_t* __restrict__ swap) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nent; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % (size_t)n);
    if (!swap[i]) continue;
    int32_t* g = gt + e * 2;
    const int32_t g0 = g[0], g1 = g[1];
    if (gt_missing(g0) || g1 == kGtVectorEnd) continue;
    if (!gt_phased(g1)) continue;
    g[0] = gt_make_phased(gt_allele(g1) == 1 ? 1 : 0);
    g[1] = gt_make_phased(gt_allele(g0) == 1 ? 1 : 0);
  }
}

struct DeviceScope {
  int prev = -1, dev = 0;
  cudaError_t e = cudaSuccess;
  explicit DeviceScope(int d) : dev(d) {
    e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != dev) e = cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace gp

using gp::Context;

extern "C" int gp_ligate_overlap(gp_ctx* ctx, int32_t n, int32_t m, const int32_t* gta, const int32_t* gtb,
                                 const uint8_t* swap_prev, uint8_t* swap_next, int32_t* nmatch, int32_t* nmism,
                                 float* phaseq) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (n <= 0 || m < 0 || (m > 0 && (!gta || !gtb)) || !swap_prev || !swap_next || !nmatch || !nmism || !phaseq)
    return (c.fail(GP_E_ARG, "ligate_overlap: bad argument"), GP_E_ARG);
  if (m == 0) return (c.fail(GP_E_DATA, "Overlap is empty"), GP_E_DATA);  // ligater_algorithm.cpp:201
  gp::DeviceScope scope(c.cfg.device);
  if (scope.e != cudaSuccess) return c.cuda_fail(scope.e, "ligate_overlap: device");
  const size_t ngt = (size_t)m * n * 2;
  cudaError_t e;
  if ((e = c.lig_a.ensure(ngt * 4)) != cudaSuccess || (e = c.lig_b.ensure(ngt * 4)) != cudaSuccess ||
      (e = c.lig_s.ensure((size_t)n)) != cudaSuccess || (e = c.lig_cnt.ensure((size_t)n * 8)) != cudaSuccess)
    return c.cuda_fail(e, "ligate_overlap: alloc");
  cudaStream_t s = c.stream;
  cudaMemcpyAsync(c.lig_a.ptr, gta, ngt * 4, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(c.lig_b.ptr, gtb, ngt * 4, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(c.lig_s.ptr, swap_prev, (size_t)n, cudaMemcpyHostToDevice, s);
  int32_t* d_match = c.lig_cnt.as<int32_t>();
  int32_t* d_mism = d_match + n;
  gp::k_ligate_counts<<<(n + 127) / 128, 128, 0, s>>>(n, m, c.lig_a.as<int32_t>(), c.lig_b.as<int32_t>(),
                                                       c.lig_s.as<uint8_t>(), d_match, d_mism);
  c.prof.kernel_launches += 1;
  cudaMemcpyAsync(nmatch, d_match, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(nmism, d_mism, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return c.cuda_fail(e, "ligate_overlap");
  if ((e = cudaGetLastError()) != cudaSuccess) return c.cuda_fail(e, "ligate_overlap: launch");
  // ligater_algorithm.cpp:183-199
  for (int i = 0; i < n; ++i) {
    swap_next[i] = nmatch[i] < nmism[i] ? 1 : 0;
    float f = 99;
    if (nmatch[i] && nmism[i]) {
      const float f0 = (float)nmatch[i] / (nmatch[i] + nmism[i]);
      f = (99 * (0.7 + f0 * logf(f0) + (1 - f0) * logf(1 - f0)) / 0.7);
    }
    phaseq[i] = f;
  }
  return GP_OK;
}

extern "C" int gp_ligate_swap(gp_ctx* ctx, int32_t n, int32_t m, int32_t* gt, const uint8_t* swap) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (n <= 0 || m < 0 || (m > 0 && !gt) || !swap) return (c.fail(GP_E_ARG, "ligate_swap: bad argument"), GP_E_ARG);
  if (m == 0) return GP_OK;
  gp::DeviceScope scope(c.cfg.device);
  if (scope.e != cudaSuccess) return c.cuda_fail(scope.e, "ligate_swap: device");
  const size_t nent = (size_t)m * n;
  cudaError_t e;
  if ((e = c.lig_a.ensure(nent * 8)) != cudaSuccess || (e = c.lig_s.ensure((size_t)n)) != cudaSuccess)
    return c.cuda_fail(e, "ligate_swap: alloc");
  cudaStream_t s = c.stream;
  cudaMemcpyAsync(c.lig_a.ptr, gt, nent * 8, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(c.lig_s.ptr, swap, (size_t)n, cudaMemcpyHostToDevice, s);
  size_t blocks = (nent + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  gp::k_ligate_swap<<<(unsigned)blocks, 256, 0, s>>>(n, nent, c.lig_a.as<int32_t>(), c.lig_s.as<uint8_t>());
  c.prof.kernel_launches += 1;
  cudaMemcpyAsync(gt, c.lig_a.ptr, nent * 8, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return c.cuda_fail(e, "ligate_swap");
  if ((e = cudaGetLastError()) != cudaSuccess) return c.cuda_fail(e, "ligate_swap: launch");
  return GP_OK;
}
