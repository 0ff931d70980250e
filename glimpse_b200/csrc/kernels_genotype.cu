// Per-site target kernels: haplotype likelihoods, haplotype sampling, genotype
// posterior accumulation, finalisation and dosages (common/src/objects/genotype.cpp,
// phase/src/io/genotype_writer.cpp:110-160).
#include "internal.h"
#include "genotype.h"

namespace gp {

__constant__ float c_unphred[256];

namespace {

// genotype::initHaplotypeLikelihoods (genotype.cpp:56-91).
__device__ __forceinline__ void init_hl(const uint8_t* g, bool fl, int ploidy, float min_gl, float& h0, float& h1) {
  if (!fl) {
    float t0 = c_unphred[g[0]], t1 = c_unphred[g[1]], t2 = ploidy > 1 ? c_unphred[g[2]] : 0.0f;
    const float sum = __fadd_rn(__fadd_rn(t0, t1), t2);
    t0 = t0 / sum;
    t1 = t1 / sum;
    t2 = t2 / sum;
    h0 = t0;
    h1 = t1;
    if (ploidy > 1) {
      h0 = (float)__fma_rn(0.5, (double)t1, (double)h0);
      h1 = (float)__fma_rn(0.5, (double)t1, (double)t2);
    }
  } else {
    h0 = 0.5f;
    h1 = 0.5f;
  }
  if (h0 < min_gl) { h0 = min_gl; h1 = __fsub_rn(1.0f, min_gl); }
  if (h1 < min_gl) { h0 = __fsub_rn(1.0f, min_gl); h1 = min_gl; }
}

// hap: 0 -> HL for H0 (conditioned on H1, `first` in the reference), 1 -> for H1.
__global__ void k_hl(const uint8_t* __restrict__ gl, const uint8_t* __restrict__ flat,
                     const int32_t* __restrict__ ploidy, const uint8_t* __restrict__ h0,
                     const uint8_t* __restrict__ h1, int L, int stage_init, int hap, float min_gl,
                     float* __restrict__ hl) {
  const int t = blockIdx.y;
  const int pl = ploidy[t];
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x) {
    const size_t ts = (size_t)t * L + s;
    const uint8_t* g = gl + ts * 3;
    const bool fl = flat[ts] != 0;
    float a, b;
    if (stage_init || pl < 2) {
      init_hl(g, fl, pl, min_gl, a, b);
    } else if (!fl) {
      // genotype::makeHaplotypeLikelihoods (genotype.cpp:94-116)
      float t0 = c_unphred[g[0]], t1 = c_unphred[g[1]], t2 = c_unphred[g[2]];
      const float sum = __fadd_rn(__fadd_rn(t0, t1), t2);
      t0 = t0 / sum;
      t1 = t1 / sum;
      t2 = t2 / sum;
      const int c = hap == 0 ? h1[ts] : h0[ts];
      const float x = c ? t1 : t0, y = c ? t2 : t1;
      a = x / __fadd_rn(x, y);
      b = y / __fadd_rn(x, y);
      if (a < min_gl) { a = min_gl; b = __fsub_rn(1.0f, min_gl); }
      if (b < min_gl) { a = __fsub_rn(1.0f, min_gl); b = min_gl; }
    } else {
      a = 0.5f;  // not read at flat sites (the reference leaves the buffer as it was)
      b = 0.5f;
    }
    hl[2 * ts] = a;
    hl[2 * ts + 1] = b;
  }
}

// genotype::sampleHaplotypeH0/H1 (genotype.cpp:118-125): H[l] = u_l > HP[2l].
__global__ void k_sample(const float* __restrict__ hp, const int32_t* __restrict__ ploidy, int L, uint64_t seed,
                         uint32_t purpose, int iteration, int only_diploid, uint8_t* __restrict__ h) {
  const int t = blockIdx.y;
  if (only_diploid && ploidy[t] < 2) return;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x) {
    const size_t ts = (size_t)t * L + s;
    const float u = canonical_float(stream_word(seed, purpose, (uint32_t)iteration, (uint32_t)t, (uint64_t)s));
    h[ts] = (uint8_t)(u > hp[2 * ts]);
  }
}

// genotype::storeGenotypePosteriorsAndHaplotypes (genotype.cpp:127-209), kept
// dense: flags bit0 = stored, bit1 = hds.
__global__ void k_gp_store(const float* __restrict__ hp0, const float* __restrict__ hp1,
                           const int32_t* __restrict__ ploidy, int L, int stored_cnt, float* __restrict__ gp0,
                           float* __restrict__ gp1, uint8_t* __restrict__ flags) {
  const int t = blockIdx.y;
  const int pl = ploidy[t];
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x) {
    const size_t ts = (size_t)t * L + s;
    const float a0 = hp0[2 * ts], a1 = hp0[2 * ts + 1];
    uint8_t f = flags[ts];
    if (pl > 1) {
      const float b0 = hp1[2 * ts], b1 = hp1[2 * ts + 1];
      const float p0 = fminf(fmaxf(__fmul_rn(a0, b0), 0.0f), 1.0f);
      const float p1 = fminf(fmaxf(fmaf(a0, b1, __fmul_rn(a1, b0)), 0.0f), 1.0f);
      const float p2 = fminf(fmaxf(__fmul_rn(a1, b1), 0.0f), 1.0f);
      const float den = __fadd_rn(__fadd_rn(p0, p1), p2);
      const bool hds = a1 < b1;
      if (f & 1) {
        gp0[ts] = __fadd_rn(gp0[ts], p0 / den);
        gp1[ts] = __fadd_rn(gp1[ts], p1 / den);
        flags[ts] = (uint8_t)(1 | (hds ? 2 : 0));
      } else if (p0 / den < 0.99999f) {
        gp0[ts] = __fadd_rn(p0 / den, (float)stored_cnt);
        gp1[ts] = p1 / den;
        flags[ts] = (uint8_t)(1 | (hds ? 2 : 0));
      }
    } else {
      const float sc = 1.0f / __fadd_rn(a0, a1);
      if (f & 1) {
        gp0[ts] = __fadd_rn(gp0[ts], __fmul_rn(a0, sc));
        gp1[ts] = __fadd_rn(gp1[ts], __fmul_rn(a1, sc));
        flags[ts] = 1;
      } else if (__fmul_rn(a0, sc) < 0.99999f) {
        gp0[ts] = __fadd_rn(__fmul_rn(a0, sc), (float)(stored_cnt % 16));
        gp1[ts] = __fmul_rn(a1, sc);
        flags[ts] = 1;
      }
    }
  }
}

// genotype::sortAndNormAndInferGenotype (genotype.cpp:211-244) and the DS/GT
// of genotype_writer.cpp:110-160.
__global__ void k_gp_finalize(const int32_t* __restrict__ ploidy, int L, int stored_cnt,
                              const uint8_t* __restrict__ flags, float* __restrict__ gp0, float* __restrict__ gp1,
                              float* __restrict__ ds, uint8_t* __restrict__ gt0, uint8_t* __restrict__ gt1,
                              uint8_t* __restrict__ h0, uint8_t* __restrict__ h1) {
  const int t = blockIdx.y;
  const int pl = ploidy[t];
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x) {
    const size_t ts = (size_t)t * L + s;
    const uint8_t f = flags[ts];
    if (!(f & 1)) {
      gp0[ts] = 1.0f;
      gp1[ts] = 0.0f;
      ds[ts] = 0.0f;
      gt0[ts] = gt1[ts] = 0;
      h0[ts] = 0;
      h1[ts] = 0;
      continue;
    }
    const float g0 = gp0[ts] / (float)stored_cnt;
    const float g1 = gp1[ts] / (float)stored_cnt;
    gp0[ts] = g0;
    gp1[ts] = g1;
    const float g2 = __fsub_rn(__fsub_rn(1.0f, g1), g0);
    if (pl > 1) {
      int call = 0;
      if (g0 > g1 && g0 > g2) call = 0;
      else if (g1 > g0 && g1 > g2) call = 1;
      else if (g2 > g0 && g2 > g1) call = 2;
      h0[ts] = call == 2;
      h1[ts] = call >= 1;
      const float g2c = fminf(fmaxf(g2, 0.0f), 1.0f);
      const float d = fmaf(2.0f, g2c, g1);
      ds[ts] = (float)((double)roundf((float)((double)d * 1000.0)) / 1000.0);
      if (g1 > g0 && g1 > g2c) {
        const int hds = (f >> 1) & 1;
        gt0[ts] = hds == 0;
        gt1[ts] = hds == 1;
      } else {
        gt0[ts] = gt1[ts] = (uint8_t)(g0 < g2c);
      }
    } else {
      h0[ts] = g1 > g0;
      h1[ts] = 0;
      ds[ts] = (float)((double)roundf((float)((double)g1 * 1000.0)) / 1000.0);
      gt0[ts] = (uint8_t)(g0 < g1);
      gt1[ts] = 0;
    }
  }
}

dim3 site_grid(int L, int n) {
  int g = (L + 255) / 256;
  if (g > 512) g = 512;
  return dim3(g, n);
}

}  // namespace

cudaError_t upload_unphred(const float* table) { return cudaMemcpyToSymbol(c_unphred, table, 256 * sizeof(float)); }

void launch_hl(const uint8_t* gl, const uint8_t* flat, const int32_t* ploidy, const uint8_t* h0, const uint8_t* h1,
               int n, int L, int stage_init, int hap, float min_gl, float* hl, cudaStream_t s) {
  k_hl<<<site_grid(L, n), 256, 0, s>>>(gl, flat, ploidy, h0, h1, L, stage_init, hap, min_gl, hl);
}

void launch_sample(const float* hp, const int32_t* ploidy, int n, int L, uint64_t seed, uint32_t purpose,
                   int iteration, int only_diploid, uint8_t* h, cudaStream_t s) {
  k_sample<<<site_grid(L, n), 256, 0, s>>>(hp, ploidy, L, seed, purpose, iteration, only_diploid, h);
}

void launch_gp_store(const float* hp0, const float* hp1, const int32_t* ploidy, int n, int L, int stored_cnt,
                     float* gp0, float* gp1, uint8_t* flags, cudaStream_t s) {
  k_gp_store<<<site_grid(L, n), 256, 0, s>>>(hp0, hp1, ploidy, L, stored_cnt, gp0, gp1, flags);
}

void launch_gp_finalize(const int32_t* ploidy, int n, int L, int stored_cnt, const uint8_t* flags, float* gp0,
                        float* gp1, float* ds, uint8_t* gt0, uint8_t* gt1, uint8_t* h0, uint8_t* h1,
                        cudaStream_t s) {
  k_gp_finalize<<<site_grid(L, n), 256, 0, s>>>(ploidy, L, stored_cnt, flags, gp0, gp1, ds, gt0, gt1, h0, h1);
}

}  // namespace gp
