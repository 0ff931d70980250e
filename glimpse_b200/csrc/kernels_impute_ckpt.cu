// The precision variant of the imputation forward-backward: checkpointed
// forward messages with recompute, and an FP64 chunk log-likelihood.
//
// Same HMM and same per-site arithmetic as the full-store chains
// (kernels_impute_warp.cu, after imputation_hmm.cpp:80-353): forward
// alpha_l = (alpha_{l-1} (1 - t) / AlphaSum_{l-1} + t / K) e_l, backward
// beta likewise with betaSum, prob_hid of each allele = sum over states of
// alpha_l x (backward message before the emission at l). What differs is what
// is kept between the passes:
//   * the forward pass keeps only the row after the last site of every block of
//     32 polymorphic sites (FP32, or BF16 for the lower-memory variant), with
//     that site's AlphaSum in FP32;
//   * the backward pass walks the blocks from the last to the first; for each
//     it recomputes the block's 32 forward rows in FP32 from the previous
//     block's checkpoint into a per-haplotype scratch of 32 rows (it stays in
//     L2), then runs the backward steps over the block reading them;
//   * the log of every AlphaSum is accumulated in FP64: the chunk
//     log-likelihood sum_l log AlphaSum_l (the reference keeps no such value).
// With FP32 checkpoints the recomputed rows equal the first pass's bit for bit.
#include <cuda_bf16.h>

#include "internal.h"

namespace gp {
namespace {

struct CkptArgs {
  const int32_t* poly;
  const int32_t* npoly;
  const int32_t* nstates;
  const uint32_t* hvar;
  const float4* em;
  const float2* tr;
  const uint8_t* fl;
  int L, WB, Kp;
  void* ckpt;       // [t][WB][Kp] rows after each block's last site (float or BF16)
  float* csum;      // [t][WB] AlphaSum at those sites
  float* scratch;   // [t][32][Kp] the recomputed rows of one block
  float* hp;        // [t][2L]: (prob_hid 0, prob_hid 1) at each polymorphic site
  double* loglik;   // [t] sum of log AlphaSum over the polymorphic sites
};

__device__ __forceinline__ float& comp4(float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ uint32_t comp4u(const uint4& v, int c) {
  return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}
// Two floats rounded to BF16 (the first in the low half, the lower address).
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t u) { return __bfloat162float(__ushort_as_bfloat16((unsigned short)(u & 0xFFFFu))); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __bfloat162float(__ushort_as_bfloat16((unsigned short)(u >> 16))); }

// One warp per haplotype, no block barriers: lane l owns the 4 J states
// 128 j + 4 l + c (c = 0..3; states from K up are masked), so its entries of a
// row are one aligned 16-byte vector; the per-site sums are warp butterflies in
// a fixed order (over the lane's quads and components, then the lanes).
constexpr int kCkWarps = 2;  // haplotypes (warps) per CTA

__device__ __forceinline__ float warp_sum_ck(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}

template <int J, bool BF16>
__global__ void __launch_bounds__(32 * kCkWarps) k_impute_ckpt_warp(CkptArgs a, int n) {
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.x * kCkWarps + (threadIdx.x >> 5);
  if (t >= n) return;
  const int np = a.npoly[t], K = a.nstates[t];
  if (np <= 0 || K <= 0) return;
  const int Kp = a.Kp;
  const uint32_t* hv = a.hvar + (size_t)t * a.WB * Kp;
  const float4* E = a.em + (size_t)t * a.L;
  const float2* TR = a.tr + (size_t)t * a.L;
  const uint8_t* F = a.fl + (size_t)t * a.L;
  const int32_t* PL = a.poly + (size_t)t * a.L;
  float* HP = a.hp + (size_t)t * 2 * a.L;
  float* scr = a.scratch + (size_t)t * 32 * Kp;
  float* cs = a.csum + (size_t)t * a.WB;
  const float invK = 1.0f / (float)K;
  const int kb = 4 * lane;
  // state k of (j, c) is kb + 128 j + c; quad j is held when kb + 128 j < Kp
  auto held = [&](int j) { return kb + 128 * j < Kp; };
  auto valid = [&](int j, int c) { return kb + 128 * j + c < K; };
  uint4 w[J];
  auto load_words = [&](int blk) {
#pragma unroll
    for (int j = 0; j < J; ++j)
      w[j] = held(j) ? *reinterpret_cast<const uint4*>(hv + (size_t)blk * Kp + kb + 128 * j) : make_uint4(0, 0, 0, 0);
  };
  auto ckpt_off = [&](int blk, int j) { return ((size_t)t * a.WB + blk) * Kp + kb + 128 * j; };
  // one forward step at site l from (x, acc) of site l - 1
  auto fwd_step = [&](int l, float4 (&x)[J], float& acc) {
    const uint8_t f = F[l];
    const float4 e = E[l];
    const float ex = f ? 1.0f : e.x, ey = f ? 1.0f : e.y;
    float f1, f2 = 0.f;
    if (l == 0) {
      f1 = invK;
    } else {
      const float2 tp = TR[l - 1];
      f1 = tp.x;
      f2 = tp.y / acc;
    }
    const uint32_t m = 1u << (l & 31);
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < J; ++j) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float xo = comp4(x[j], c);
        const float pc = l == 0 ? f1 : fmaf(xo, f2, f1);
        const float xn = valid(j, c) ? __fmul_rn(pc, (comp4u(w[j], c) & m) ? ey : ex) : 0.f;
        comp4(x[j], c) = xn;
        s = __fadd_rn(s, xn);
      }
    }
    s = warp_sum_ck(s);
    acc = (l == 0 && f) ? 1.0f : s;  // AlphaSum = 1 at a flat first site (imputation_hmm.cpp:156)
  };

  // ---- forward: checkpoints and the FP64 log-likelihood ----
  float4 x[J];
#pragma unroll
  for (int j = 0; j < J; ++j) x[j] = make_float4(0.f, 0.f, 0.f, 0.f);
  float acc = 0.f;
  double ll = 0.0;
  for (int l = 0; l < np; ++l) {
    if ((l & 31) == 0) load_words(l >> 5);
    fwd_step(l, x, acc);
    if (lane == 0) ll += log((double)acc);
    if ((l & 31) == 31 && l + 1 < np) {
      const int blk = l >> 5;
#pragma unroll
      for (int j = 0; j < J; ++j) {
        if (!held(j)) continue;
        if (BF16) {
          const uint32_t lo = pack_bf16x2(x[j].x, x[j].y), hi = pack_bf16x2(x[j].z, x[j].w);
          *reinterpret_cast<uint2*>(reinterpret_cast<__nv_bfloat16*>(a.ckpt) + ckpt_off(blk, j)) = make_uint2(lo, hi);
        } else {
          *reinterpret_cast<float4*>(reinterpret_cast<float*>(a.ckpt) + ckpt_off(blk, j)) = x[j];
        }
      }
      if (lane == 0) cs[blk] = acc;
    }
  }
  if (lane == 0) a.loglik[t] = ll;

  // ---- backward, block by block with the forward rows recomputed ----
  float4 xb[J];
#pragma unroll
  for (int j = 0; j < J; ++j) xb[j] = make_float4(0.f, 0.f, 0.f, 0.f);
  float bacc = 0.f;
  const int nblk = (np + 31) >> 5;
  for (int b = nblk - 1; b >= 0; --b) {
    const int s0 = b << 5, s1 = min(np, s0 + 32) - 1;
    load_words(b);
    float aacc = 0.f;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      x[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (b > 0 && held(j)) {
        if (BF16) {
          const uint2 u = *reinterpret_cast<const uint2*>(reinterpret_cast<const __nv_bfloat16*>(a.ckpt) +
                                                         ckpt_off(b - 1, j));
          x[j] = make_float4(bf16_lo(u.x), bf16_hi(u.x), bf16_lo(u.y), bf16_hi(u.y));
        } else {
          x[j] = *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(a.ckpt) + ckpt_off(b - 1, j));
        }
      }
    }
    if (b > 0) aacc = cs[b - 1];
    for (int l = s0; l <= s1; ++l) {
      fwd_step(l, x, aacc);
#pragma unroll
      for (int j = 0; j < J; ++j)
        if (held(j)) *reinterpret_cast<float4*>(scr + (size_t)(l - s0) * Kp + kb + 128 * j) = x[j];
    }
    for (int l = s1; l >= s0; --l) {
      const uint8_t f = F[l];
      const float4 e = E[l];
      const float ex = f ? 1.0f : e.x, ey = f ? 1.0f : e.y;
      const bool last = l == np - 1;
      float f1 = invK, f2 = 0.f;
      if (!last) {
        const float2 tt = TR[l];
        f1 = tt.x;
        f2 = tt.y / bacc;
      }
      const uint32_t m = 1u << (l & 31);
      float v0 = 0.f, v1 = 0.f, v2 = 0.f;  // betaSum, prob_hid 0, prob_hid 1
#pragma unroll
      for (int j = 0; j < J; ++j) {
        float4 al = make_float4(0.f, 0.f, 0.f, 0.f);
        if (held(j)) al = *reinterpret_cast<const float4*>(scr + (size_t)(l - s0) * Kp + kb + 128 * j);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (!valid(j, c)) continue;
          const bool bit = (comp4u(w[j], c) & m) != 0u;
          const float pc = last ? f1 : fmaf(comp4(xb[j], c), f2, f1);
          const float ac = comp4(al, c);
          const float d = last ? ac : __fmul_rn(ac, pc);  // alpha alone at the last site
          if (bit) v2 = __fadd_rn(v2, d);
          else v1 = __fadd_rn(v1, d);
          const float xn = __fmul_rn(pc, bit ? ey : ex);
          comp4(xb[j], c) = xn;
          v0 = __fadd_rn(v0, xn);
        }
      }
      v0 = warp_sum_ck(v0);
      v1 = warp_sum_ck(v1);
      v2 = warp_sum_ck(v2);
      bacc = (last && f) ? 1.0f : v0;  // betaSum = 1 at a flat last site (imputation_hmm.cpp:285)
      if (lane == 0) *reinterpret_cast<float2*>(HP + 2 * PL[l]) = make_float2(v1, v2);
    }
  }
}

}  // namespace

int launch_impute_ckpt(ImputeWork& w, bool bf16, void* ckpt, float* csum, float* scratch, double* loglik, float* hp,
                       cudaStream_t s) {
  CkptArgs a;
  a.poly = w.poly.as<int32_t>();
  a.npoly = w.npoly.as<int32_t>();
  a.nstates = w.nstates.as<int32_t>();
  a.hvar = w.hvar.as<uint32_t>();
  a.em = w.em.as<float4>();
  a.tr = w.tr.as<float2>();
  a.fl = w.fl.as<uint8_t>();
  a.L = w.L;
  a.WB = w.WB;
  a.Kp = w.Kp;
  a.ckpt = ckpt;
  a.csum = csum;
  a.scratch = scratch;
  a.hp = hp;
  a.loglik = loglik;
  if (w.Kp > kMaxStates) return GP_E_ARG;
  // quads per lane: the smallest instantiated J with 128 J >= Kp
  const int jn = (w.Kp + 127) / 128;
  const int grid = (w.n + kCkWarps - 1) / kCkWarps;
#define GP_CK_LAUNCH(JJ)                                                                     \
  if (jn <= JJ) {                                                                            \
    if (bf16) k_impute_ckpt_warp<JJ, true><<<grid, 32 * kCkWarps, 0, s>>>(a, w.n);            \
    else k_impute_ckpt_warp<JJ, false><<<grid, 32 * kCkWarps, 0, s>>>(a, w.n);                \
    return GP_OK;                                                                            \
  }
  GP_CK_LAUNCH(2)
  GP_CK_LAUNCH(4)
  GP_CK_LAUNCH(6)
  GP_CK_LAUNCH(8)
  GP_CK_LAUNCH(10)
  GP_CK_LAUNCH(12)
  GP_CK_LAUNCH(16)
#undef GP_CK_LAUNCH
  return GP_OK;
}

}  // namespace gp
