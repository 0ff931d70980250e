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
// One CTA of 256 threads runs one haplotype; thread x owns states x + 256 j.
// The per-site sums are block reductions in one fixed tree.
#include <cuda_bf16.h>

#include "internal.h"

namespace gp {
namespace {

constexpr int kCT = 256, kCJ = kMaxStates / kCT, kCW = kCT / 32;

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

// Sums of N values over the CTA: warp butterflies, then the warps in one tree.
// The partials alternate between two buffers, so one barrier per reduction
// suffices: a reduction's writes go to the buffer that the previous one did
// not read, and the one before that was read before the previous barrier.
template <int N>
__device__ __forceinline__ void cta_sum(float (&v)[N], float (*red)[3][kCW], int& buf) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] = __fadd_rn(v[i], __shfl_xor_sync(0xFFFFFFFFu, v[i], o));
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int i = 0; i < N; ++i) red[buf][i][threadIdx.x >> 5] = v[i];
  __syncthreads();
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const float* r = red[buf][i];
    v[i] = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                     __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
  }
  buf ^= 1;
}

template <bool BF16>
__global__ void __launch_bounds__(kCT) k_impute_ckpt(CkptArgs a) {
  static_assert(kCW == 8, "eight warps");
  __shared__ float red[2][3][kCW];
  int buf = 0;
  const int t = blockIdx.x, tid = threadIdx.x;
  const int np = a.npoly[t], K = a.nstates[t];
  if (np <= 0 || K <= 0) return;
  const uint32_t* hv = a.hvar + (size_t)t * a.WB * a.Kp;
  const float4* E = a.em + (size_t)t * a.L;
  const float2* TR = a.tr + (size_t)t * a.L;
  const uint8_t* F = a.fl + (size_t)t * a.L;
  const int32_t* PL = a.poly + (size_t)t * a.L;
  float* HP = a.hp + (size_t)t * 2 * a.L;
  float* scr = a.scratch + (size_t)t * 32 * a.Kp;
  float* cs = a.csum + (size_t)t * a.WB;
  const float invK = 1.0f / (float)K;
  bool valid[kCJ];
#pragma unroll
  for (int j = 0; j < kCJ; ++j) valid[j] = tid + kCT * j < K;
  uint32_t w[kCJ];
  auto load_words = [&](int blk) {
#pragma unroll
    for (int j = 0; j < kCJ; ++j) w[j] = valid[j] ? hv[(size_t)blk * a.Kp + tid + kCT * j] : 0u;
  };
  auto store_ckpt = [&](int blk, const float (&x)[kCJ]) {
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {
      if (!valid[j]) continue;
      const size_t o = ((size_t)t * a.WB + blk) * a.Kp + tid + kCT * j;
      if (BF16) reinterpret_cast<__nv_bfloat16*>(a.ckpt)[o] = __float2bfloat16_rn(x[j]);
      else reinterpret_cast<float*>(a.ckpt)[o] = x[j];
    }
  };
  auto load_ckpt = [&](int blk, float (&x)[kCJ]) {
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {
      if (!valid[j]) {
        x[j] = 0.f;
        continue;
      }
      const size_t o = ((size_t)t * a.WB + blk) * a.Kp + tid + kCT * j;
      x[j] = BF16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(a.ckpt)[o])
                  : reinterpret_cast<const float*>(a.ckpt)[o];
    }
  };
  // one forward step at site l from (x, acc) of site l - 1
  auto fwd_step = [&](int l, float (&x)[kCJ], float& acc) {
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
    float s[1] = {0.f};
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {
      const float pc = l == 0 ? f1 : fmaf(x[j], f2, f1);
      x[j] = valid[j] ? __fmul_rn(pc, (w[j] & m) ? ey : ex) : 0.f;
      s[0] = __fadd_rn(s[0], x[j]);
    }
    cta_sum<1>(s, red, buf);
    acc = (l == 0 && f) ? 1.0f : s[0];  // AlphaSum = 1 at a flat first site (imputation_hmm.cpp:156)
  };

  // ---- forward: checkpoints and the FP64 log-likelihood ----
  float x[kCJ];
  float acc = 0.f;
  double ll = 0.0;
#pragma unroll
  for (int j = 0; j < kCJ; ++j) x[j] = 0.f;
  for (int l = 0; l < np; ++l) {
    if ((l & 31) == 0) load_words(l >> 5);
    fwd_step(l, x, acc);
    ll += log((double)acc);
    if ((l & 31) == 31 && l + 1 < np) {
      store_ckpt(l >> 5, x);
      if (tid == 0) cs[l >> 5] = acc;
    }
  }
  if (tid == 0) a.loglik[t] = ll;

  // ---- backward, block by block with the forward rows recomputed ----
  float xb[kCJ];
  float bacc = 0.f;
#pragma unroll
  for (int j = 0; j < kCJ; ++j) xb[j] = 0.f;
  const int nblk = (np + 31) >> 5;
  for (int b = nblk - 1; b >= 0; --b) {
    const int s0 = b << 5, s1 = min(np, s0 + 32) - 1;
    load_words(b);
    float xa[kCJ];
    float aacc = 0.f;
    if (b > 0) {
      load_ckpt(b - 1, xa);
      aacc = cs[b - 1];
    } else {
#pragma unroll
      for (int j = 0; j < kCJ; ++j) xa[j] = 0.f;
    }
    for (int l = s0; l <= s1; ++l) {
      fwd_step(l, xa, aacc);
#pragma unroll
      for (int j = 0; j < kCJ; ++j)
        if (valid[j]) scr[(size_t)(l - s0) * a.Kp + tid + kCT * j] = xa[j];
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
      float v[3] = {0.f, 0.f, 0.f};  // betaSum, prob_hid 0, prob_hid 1
#pragma unroll
      for (int j = 0; j < kCJ; ++j) {
        if (!valid[j]) continue;
        const bool bit = (w[j] & m) != 0u;
        const float al = scr[(size_t)(l - s0) * a.Kp + tid + kCT * j];
        const float pc = last ? f1 : fmaf(xb[j], f2, f1);
        const float d = last ? al : __fmul_rn(al, pc);  // alpha alone at the last site
        if (bit) v[2] = __fadd_rn(v[2], d);
        else v[1] = __fadd_rn(v[1], d);
        xb[j] = __fmul_rn(pc, bit ? ey : ex);
        v[0] = __fadd_rn(v[0], xb[j]);
      }
      cta_sum<3>(v, red, buf);
      bacc = (last && f) ? 1.0f : v[0];  // betaSum = 1 at a flat last site (imputation_hmm.cpp:285)
      if (tid == 0) *reinterpret_cast<float2*>(HP + 2 * PL[l]) = make_float2(v[1], v[2]);
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
  if (bf16) k_impute_ckpt<true><<<w.n, kCT, 0, s>>>(a);
  else k_impute_ckpt<false><<<w.n, kCT, 0, s>>>(a);
  return GP_OK;
}

}  // namespace gp
