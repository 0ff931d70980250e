// The precision variant of the imputation forward-backward: checkpointed
// messages with recompute, and an FP64 chunk log-likelihood.
//
// Same HMM and same per-site arithmetic as the full-store chains
// (kernels_impute_warp.cu, after imputation_hmm.cpp:80-353): forward
// alpha_l = (alpha_{l-1} (1 - t) / AlphaSum_{l-1} + t / K) e_l, backward
// beta likewise with betaSum, prob_hid of each allele = sum over states of
// alpha_l x (backward message before the emission at l, 1 at the last site).
// What differs is what is kept between the passes. As in the full-store
// chains, each haplotype is split at M (a multiple of 32, about np / 2) into a
// forward and a backward chain that run concurrently, one CTA each:
//   phase A  forward  [0, M)      keeps the alpha row after the last site of
//                                 every block of 32 polymorphic sites, and its
//                                 AlphaSum
//            backward [np-1, M]   keeps the beta row after the first site of
//                                 every block, and its betaSum
//   phase B  forward  [M, np)     per block: the block's backward messages are
//                                 recomputed from the next block's checkpoint
//                                 into a 32-row scratch, then the forward steps
//                                 form the posteriors from them
//            backward [M-1, 0]    per block: the block's alpha rows are
//                                 recomputed from the previous block's
//                                 checkpoint into the scratch, then the
//                                 backward steps form the posteriors
// Checkpoints are FP32, or BF16 for the lower-memory variant; recomputed rows
// are FP32 (with FP32 checkpoints they equal the first pass's bit for bit).
// The log of every AlphaSum is accumulated in FP64: the chunk log-likelihood
// sum_l log AlphaSum_l (the reference keeps no such value).
// One CTA of 256 threads runs one chain; thread x owns states x + 256 j. The
// per-site sums are block reductions in one fixed tree.
#include <cuda_bf16.h>

#include "internal.h"

namespace gp {
namespace {

constexpr int kCT = 256, kCW = kCT / 32;

struct CkptArgs {
  const int32_t* poly;
  const int32_t* npoly;
  const int32_t* nstates;
  const uint32_t* hvar;
  const float4* em;
  const float2* tr;
  const uint8_t* fl;
  int n, L, WB, Kp;
  void* ckpt;       // [2][t][WB][Kp]: alpha after each block's last site, beta after its first (float or BF16)
  float* csum;      // [2][t][WB]: AlphaSum / betaSum at those sites
  float* scratch;   // [t][2][32][Kp]: the recomputed rows of one block, per chain
  float* hp;        // [t][2L]: (prob_hid 0, prob_hid 1) at each polymorphic site
  double* llpart;   // [t]: sum of log AlphaSum over [0, M)
  double* loglik;   // [t]: sum of log AlphaSum over the polymorphic sites
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
    const float4 p = reinterpret_cast<const float4*>(red[buf][i])[0], q = reinterpret_cast<const float4*>(red[buf][i])[1];
    v[i] = __fadd_rn(__fadd_rn(__fadd_rn(p.x, p.y), __fadd_rn(p.z, p.w)),
                     __fadd_rn(__fadd_rn(q.x, q.y), __fadd_rn(q.z, q.w)));
  }
  buf ^= 1;
}

// M of the meet-in-the-middle split (as the full-store chains take it).
__device__ __forceinline__ int ckpt_split(int np) { return (np / 2) & ~31; }

// Phase A (PB = false) or phase B (PB = true) of one chain: CTA 2 t + role runs
// haplotype t's forward (role 0) or backward (role 1) chain. J: states per
// thread, from the launch's largest K.
template <int J, bool BF16, bool PB>
__global__ void __launch_bounds__(kCT) k_impute_ckpt(CkptArgs a) {
  constexpr int kCJ = J;
  static_assert(kCW == 8, "eight warps");
  __shared__ __align__(16) float red[2][3][kCW];  // rows of 8 partials read as two float4
  int buf = 0;
  const int t = blockIdx.x >> 1, role = blockIdx.x & 1, tid = threadIdx.x;
  const int np = a.npoly[t], K = a.nstates[t];
  if (np <= 0 || K <= 0) return;
  const int M = ckpt_split(np);
  const int Kp = a.Kp;
  const uint32_t* hv = a.hvar + (size_t)t * a.WB * Kp;
  const float4* E = a.em + (size_t)t * a.L;
  const float2* TR = a.tr + (size_t)t * a.L;
  const uint8_t* F = a.fl + (size_t)t * a.L;
  const int32_t* PL = a.poly + (size_t)t * a.L;
  float* HP = a.hp + (size_t)t * 2 * a.L;
  float* scr = a.scratch + ((size_t)t * 2 + role) * 32 * Kp;
  const float invK = 1.0f / (float)K;
  bool valid[kCJ];
#pragma unroll
  for (int j = 0; j < kCJ; ++j) valid[j] = tid + kCT * j < K;
  uint32_t w[kCJ];
  auto load_words = [&](int blk) {
#pragma unroll
    for (int j = 0; j < kCJ; ++j) w[j] = valid[j] ? hv[(size_t)blk * Kp + tid + kCT * j] : 0u;
  };
  // checkpoint d (0 alpha, 1 beta) of block blk
  auto row_off = [&](int d, int blk, int j) {
    return (((size_t)d * a.n + t) * a.WB + blk) * Kp + tid + kCT * j;
  };
  auto sum_off = [&](int d, int blk) { return ((size_t)d * a.n + t) * a.WB + blk; };
  auto store_row = [&](int d, int blk, const float (&x)[kCJ]) {
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {
      if (!valid[j]) continue;
      if (BF16) reinterpret_cast<__nv_bfloat16*>(a.ckpt)[row_off(d, blk, j)] = __float2bfloat16_rn(x[j]);
      else reinterpret_cast<float*>(a.ckpt)[row_off(d, blk, j)] = x[j];
    }
  };
  auto load_row = [&](int d, int blk, float (&x)[kCJ]) {
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {
      x[j] = 0.f;
      if (!valid[j]) continue;
      x[j] = BF16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(a.ckpt)[row_off(d, blk, j)])
                  : reinterpret_cast<const float*>(a.ckpt)[row_off(d, blk, j)];
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
  // one backward step at site l from (xb, bacc) of site l + 1; pc gets the
  // message before the emission at l (1 at the last site), as the full store keeps it
  auto bwd_step = [&](int l, float (&xb)[kCJ], float& bacc, float (&pc)[kCJ]) {
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
    float s[1] = {0.f};
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {
      pc[j] = 0.f;
      if (!valid[j]) continue;
      const float p = last ? f1 : fmaf(xb[j], f2, f1);
      pc[j] = last ? 1.0f : p;
      xb[j] = __fmul_rn(p, (w[j] & m) ? ey : ex);
      s[0] = __fadd_rn(s[0], xb[j]);
    }
    cta_sum<1>(s, red, buf);
    bacc = (last && f) ? 1.0f : s[0];  // betaSum = 1 at a flat last site (imputation_hmm.cpp:285)
  };

  float x[kCJ], pc[kCJ];
  if (!PB) {
    if (role == 0) {
      // ---- phase A forward over [0, M): alpha checkpoints, log-likelihood ----
      if (M == 0) return;
      float acc = 0.f;
      double ll = 0.0;
#pragma unroll
      for (int j = 0; j < kCJ; ++j) x[j] = 0.f;
      for (int l = 0; l < M; ++l) {
        if ((l & 31) == 0) load_words(l >> 5);
        fwd_step(l, x, acc);
        if (tid == 0) ll += log((double)acc);  // thread 0 alone keeps the FP64 sum
        if ((l & 31) == 31) {
          store_row(0, l >> 5, x);
          if (tid == 0) a.csum[sum_off(0, l >> 5)] = acc;
        }
      }
      if (tid == 0) a.llpart[t] = ll;
    } else {
      // ---- phase A backward over [np-1, M]: beta checkpoints ----
      float bacc = 0.f;
#pragma unroll
      for (int j = 0; j < kCJ; ++j) x[j] = 0.f;
      for (int l = np - 1; l >= M; --l) {
        if (l == np - 1 || (l & 31) == 31) load_words(l >> 5);
        bwd_step(l, x, bacc, pc);
        if ((l & 31) == 0) {
          store_row(1, l >> 5, x);
          if (tid == 0) a.csum[sum_off(1, l >> 5)] = bacc;
        }
      }
    }
    return;
  }

  const int nblk = (np + 31) >> 5;
  if (role == 0) {
    // ---- phase B forward over [M, np): per block, the backward messages
    // recomputed from the next block's checkpoint, then alpha and the posteriors ----
    float acc = 0.f;
    double ll = 0.0;
    if (M > 0) {
      load_row(0, (M >> 5) - 1, x);
      acc = a.csum[sum_off(0, (M >> 5) - 1)];
      ll = a.llpart[t];
    } else {
#pragma unroll
      for (int j = 0; j < kCJ; ++j) x[j] = 0.f;
    }
    for (int b = M >> 5; b < nblk; ++b) {
      const int s0 = b << 5, s1 = min(np, s0 + 32) - 1;
      load_words(b);
      float xb[kCJ];
      float bacc = 0.f;
      if (b + 1 < nblk) {
        load_row(1, b + 1, xb);
        bacc = a.csum[sum_off(1, b + 1)];
      } else {
#pragma unroll
        for (int j = 0; j < kCJ; ++j) xb[j] = 0.f;
      }
      for (int l = s1; l >= s0; --l) {
        bwd_step(l, xb, bacc, pc);
#pragma unroll
        for (int j = 0; j < kCJ; ++j)
          if (valid[j]) scr[(size_t)(l - s0) * Kp + tid + kCT * j] = pc[j];
      }
      for (int l = s0; l <= s1; ++l) {
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
        float v[3] = {0.f, 0.f, 0.f};  // AlphaSum, prob_hid 0, prob_hid 1
#pragma unroll
        for (int j = 0; j < kCJ; ++j) {
          const float p = l == 0 ? f1 : fmaf(x[j], f2, f1);
          const bool bit = (w[j] & m) != 0u;
          x[j] = valid[j] ? __fmul_rn(p, bit ? ey : ex) : 0.f;
          v[0] = __fadd_rn(v[0], x[j]);
          if (!valid[j]) continue;
          const float d = __fmul_rn(x[j], scr[(size_t)(l - s0) * Kp + tid + kCT * j]);  // alpha x message (1 at the last site)
          if (bit) v[2] = __fadd_rn(v[2], d);
          else v[1] = __fadd_rn(v[1], d);
        }
        cta_sum<3>(v, red, buf);
        acc = (l == 0 && f) ? 1.0f : v[0];  // AlphaSum = 1 at a flat first site (imputation_hmm.cpp:156)
        if (tid == 0) ll += log((double)acc);  // thread 0 alone keeps the FP64 sum
        if (tid == 0) *reinterpret_cast<float2*>(HP + 2 * PL[l]) = make_float2(v[1], v[2]);
      }
    }
    if (tid == 0) a.loglik[t] = ll;
  } else {
    // ---- phase B backward over [M-1, 0]: per block, the alpha rows recomputed
    // from the previous block's checkpoint, then beta and the posteriors ----
    if (M == 0) return;
    float xb[kCJ];
    load_row(1, M >> 5, xb);
    float bacc = a.csum[sum_off(1, M >> 5)];
    for (int b = (M >> 5) - 1; b >= 0; --b) {
      const int s0 = b << 5, s1 = s0 + 31;
      load_words(b);
      float aacc = 0.f;
      if (b > 0) {
        load_row(0, b - 1, x);
        aacc = a.csum[sum_off(0, b - 1)];
      } else {
#pragma unroll
        for (int j = 0; j < kCJ; ++j) x[j] = 0.f;
      }
      for (int l = s0; l <= s1; ++l) {
        fwd_step(l, x, aacc);
#pragma unroll
        for (int j = 0; j < kCJ; ++j)
          if (valid[j]) scr[(size_t)(l - s0) * Kp + tid + kCT * j] = x[j];
      }
      for (int l = s1; l >= s0; --l) {  // l < M <= np - 1: never the last site
        const uint8_t f = F[l];
        const float4 e = E[l];
        const float ex = f ? 1.0f : e.x, ey = f ? 1.0f : e.y;
        const float2 tt = TR[l];
        const float f1 = tt.x, f2 = tt.y / bacc;
        const uint32_t m = 1u << (l & 31);
        float v[3] = {0.f, 0.f, 0.f};  // betaSum, prob_hid 0, prob_hid 1
#pragma unroll
        for (int j = 0; j < kCJ; ++j) {
          if (!valid[j]) continue;
          const bool bit = (w[j] & m) != 0u;
          const float al = scr[(size_t)(l - s0) * Kp + tid + kCT * j];
          const float p = fmaf(xb[j], f2, f1);
          const float d = __fmul_rn(al, p);
          if (bit) v[2] = __fadd_rn(v[2], d);
          else v[1] = __fadd_rn(v[1], d);
          xb[j] = __fmul_rn(p, bit ? ey : ex);
          v[0] = __fadd_rn(v[0], xb[j]);
        }
        cta_sum<3>(v, red, buf);
        bacc = v[0];
        if (tid == 0) *reinterpret_cast<float2*>(HP + 2 * PL[l]) = make_float2(v[1], v[2]);
      }
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
  a.n = w.n;
  a.L = w.L;
  a.WB = w.WB;
  a.Kp = w.Kp;
  a.ckpt = ckpt;
  a.csum = csum;
  a.scratch = scratch;
  a.hp = hp;
  a.loglik = loglik;
  a.llpart = loglik + w.n;
  if (w.Kp > kMaxStates) return GP_E_ARG;
  const int grid = 2 * w.n;
  const int jn = (w.Kp + kCT - 1) / kCT;  // states per thread; the smallest instantiated J >= jn
#define GP_CK_LAUNCH(JJ)                                         \
  if (jn <= JJ) {                                                \
    if (bf16) {                                                  \
      k_impute_ckpt<JJ, true, false><<<grid, kCT, 0, s>>>(a);    \
      k_impute_ckpt<JJ, true, true><<<grid, kCT, 0, s>>>(a);     \
    } else {                                                     \
      k_impute_ckpt<JJ, false, false><<<grid, kCT, 0, s>>>(a);   \
      k_impute_ckpt<JJ, false, true><<<grid, kCT, 0, s>>>(a);    \
    }                                                            \
    return GP_OK;                                                \
  }
  GP_CK_LAUNCH(2)
  GP_CK_LAUNCH(3)
  GP_CK_LAUNCH(4)
  GP_CK_LAUNCH(5)
  GP_CK_LAUNCH(6)
  GP_CK_LAUNCH(8)
#undef GP_CK_LAUNCH
  return GP_OK;
}

}  // namespace gp
