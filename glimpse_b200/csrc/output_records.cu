// Output epilogue: the per-(site, target) GP values and the per-site INFO fields
// that genotype_writer::writeGenotypes puts in each record
// (phase/src/io/genotype_writer.cpp:98-201), computed on the device from the
// finalised genotype posteriors, so that the caller's writer only formats
// arrays. GT and DS come from gp_gp_get (k_gp_finalize applies the same rules).
//
// Per target i at site l (genotype_writer.cpp:115-182):
//   a target without stored posteriors at l is 0/0 with GP (1, 0, 0) and DS 0;
//   GP values are floored to 1e-3 (the third, for a diploid target, from the
//   floored first two), then raised by 1e-3 one at a time, in increasing order
//   of 1 - (gp - floored), until their sum reaches 0.9999. The order comes from
//   a std::map keyed by that float, so a value whose key equals an earlier
//   one's is never raised. A haploid target's third value (in a file with
//   diploid targets) is htslib's vector-end marker.
// Per site (genotype_writer.cpp:177-190), summed over targets in order in
// float as the reference sums them:
//   RAF  = calt / (calt + cref)
//   AF   = sum DS / number of target haplotypes
//   INFO = 1 - (sum (gp1 + 4 gp2) - sum DS^2) / (n_haps AF (1 - AF)), when every
//          target is diploid and 0 < AF < 1; otherwise 1; clamped at 0 and
//          rounded to 1e-3. (The writer omits INFO for mixed ploidy.)
// The reference is built with -mfma; its contractions are placed here
// explicitly (the library is built with --fmad=false): DS = fma(2, gp2, gp1)
// and sum DS^2 += DS * DS as fma(DS, DS, sum).
//
// One thread per site walks the targets in order (the sums are sequential in
// the reference); consecutive threads take consecutive sites, so every load and
// store of a step is contiguous across the warp.
#include <cstdint>

#include <cuda_runtime.h>

#include "context.h"
#include "internal.h"

namespace gp {
namespace {

__device__ __forceinline__ float floor_milli(float x) {
  return (float)((double)floorf((float)((double)x * 1000.0)) / 1000.0);
}

__global__ void k_output_records(int n, int L, int max_ploidy, int fploidy, int n_haps,
                                 const int32_t* __restrict__ ploidy, const uint8_t* __restrict__ flags,
                                 const float* __restrict__ gp0, const float* __restrict__ gp1,
                                 const uint32_t* __restrict__ cref, const uint32_t* __restrict__ calt,
                                 float* __restrict__ gp_out, float* __restrict__ raf, float* __restrict__ af,
                                 float* __restrict__ info) {
  const float vector_end = __uint_as_float(0x7F800002u);  // bcf_float_vector_end
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < L; l += gridDim.x * blockDim.x) {
    float ds_sum = 0.0f, ds2_sum = 0.0f, ds4_sum = 0.0f;
    for (int i = 0; i < n; ++i) {
      const size_t il = (size_t)i * L + l;
      const int pl = ploidy[i];
      float ds = 0.0f, g0 = 1.0f, g1 = 0.0f, g2 = 0.0f;
      if (flags[il] & 1u) {
        g0 = gp0[il];
        g1 = gp1[il];
        if (pl > 1) {
          g2 = fminf(fmaxf(__fsub_rn(__fsub_rn(1.0f, g1), g0), 0.0f), 1.0f);  // getGp2 (genotype.h:62-64)
          ds = fmaf(2.0f, g2, g1);
        } else {
          ds = g1;
        }
      }
      // GP floored, then raised in map order (genotype_writer.cpp:155-172)
      float p0 = floor_milli(g0), p1 = floor_milli(g1), p2 = 0.0f;
      const float k0 = __fsub_rn(1.0f, __fsub_rn(g0, p0));
      const float k1 = __fsub_rn(1.0f, __fsub_rn(g1, p1));
      float k2 = 0.0f;
      const bool has1 = k1 != k0;
      bool has2 = false;
      const bool third = max_ploidy > 1 && pl > 1;
      if (third) {
        p2 = floor_milli(fmaxf(__fsub_rn(1.0f, __fadd_rn(p0, p1)), 0.0f));
        k2 = __fsub_rn(1.0f, __fsub_rn(g2, p2));
        has2 = k2 != k0 && k2 != k1;
      }
      // kept entries in increasing key order (distinct keys)
      int ord[3];
      int m = 0;
      ord[m++] = 0;
      if (has1) {
        if (k1 < k0) { ord[1] = ord[0]; ord[0] = 1; } else { ord[1] = 1; }
        m = 2;
      }
      if (has2) {
        const float kk[3] = {k0, k1, k2};
        int pos = m;
        while (pos > 0 && k2 < kk[ord[pos - 1]]) {
          ord[pos] = ord[pos - 1];
          --pos;
        }
        ord[pos] = 2;
        ++m;
      }
      for (int q = 0; q < m; ++q) {
        float s = __fadd_rn(__fadd_rn(0.0f, p0), p1);
        if (pl > 1 && max_ploidy > 1) s = __fadd_rn(s, p2);
        if (!(s < 0.9999f)) break;
        const int e = ord[q];
        if (e == 0) p0 = __fadd_rn(p0, 0.001f);
        else if (e == 1) p1 = __fadd_rn(p1, 0.001f);
        else p2 = __fadd_rn(p2, 0.001f);
      }
      float* o = gp_out + il * 3;
      o[0] = p0;
      o[1] = p1;
      o[2] = third ? p2 : vector_end;
      // INFO sums (genotype_writer.cpp:175-180)
      ds_sum = __fadd_rn(ds_sum, ds);
      if (fploidy == 2) {
        ds2_sum = fmaf(ds, ds, ds2_sum);
        ds4_sum = (float)__dadd_rn((double)ds4_sum, __dadd_rn((double)g1, 4.0 * (double)g2));
      }
    }
    const uint32_t ca = calt[l], cr = cref[l];
    raf[l] = __fdiv_rn(__fmul_rn((float)ca, 1.0f), (float)(ca + cr));
    const float f = __fdiv_rn(ds_sum, (float)n_haps);
    af[l] = f;
    float inf = 1.0f;
    if (fploidy == 2 && f > 0.0f && f < 1.0f) {
      const double den = __dmul_rn((double)__fmul_rn((float)n_haps, f), __dsub_rn(1.0, (double)f));
      inf = (float)__dsub_rn(1.0, __ddiv_rn((double)__fsub_rn(ds4_sum, ds2_sum), den));
    }
    inf = inf < 0.0f ? 0.0f : inf;
    info[l] = (float)__ddiv_rn((double)roundf((float)((double)inf * 1000.0)), 1000.0);
  }
}

}  // namespace
}  // namespace gp

using gp::Context;

extern "C" int gp_output_records(gp_ctx* ctx, float* gp, float* raf, float* af, float* info) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  gp::TargetWork& T = c.tw;
  if (!T.finalized) return (c.fail(GP_E_STATE, "gp_finalize has not run"), GP_E_STATE);
  if (!gp || !raf || !af || !info) return (c.fail(GP_E_ARG, "output_records: bad argument"), GP_E_ARG);
  const int n = T.n, L = c.panel.L;
  int max_ploidy = 0, n_dip = 0, n_hap = 0, n_haps = 0;
  for (int i = 0; i < n; ++i) {
    const int p = T.ploidy_h[i];
    max_ploidy = p > max_ploidy ? p : max_ploidy;
    n_haps += p;
    (p > 1 ? n_dip : n_hap) += 1;
  }
  // genotype_reader.cpp:553-554: the maximum ploidy, negated when haploid and diploid targets mix
  const int fploidy = (n_dip > 0 && n_hap > 0) ? -max_ploidy : max_ploidy;
  const size_t nL = (size_t)n * L;
  cudaError_t e;
  if ((e = c.out_gp.ensure(nL * 3 * 4)) != cudaSuccess || (e = c.out_site.ensure((size_t)L * 3 * 4)) != cudaSuccess)
    return c.cuda_fail(e, "output_records: alloc");
  float* d_gp = c.out_gp.as<float>();
  float* d_raf = c.out_site.as<float>();
  float* d_af = d_raf + L;
  float* d_info = d_af + L;
  int blocks = (L + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  gp::k_output_records<<<blocks, 256, 0, c.stream>>>(n, L, max_ploidy, fploidy, n_haps, T.ploidy.as<int32_t>(),
                                                     T.gpflags.as<uint8_t>(), T.gp0.as<float>(), T.gp1.as<float>(),
                                                     c.panel.cref, c.panel.calt, d_gp, d_raf, d_af, d_info);
  c.prof.kernel_launches += 1;
  cudaMemcpyAsync(gp, d_gp, nL * 3 * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(raf, d_raf, (size_t)L * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(af, d_af, (size_t)L * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(info, d_info, (size_t)L * 4, cudaMemcpyDeviceToHost, c.stream);
  if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return c.cuda_fail(e, "output_records");
  if ((e = cudaGetLastError()) != cudaSuccess) return c.cuda_fail(e, "output_records: launch");
  return GP_OK;
}
