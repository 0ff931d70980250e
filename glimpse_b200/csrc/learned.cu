// The learned state-selection proposal (learned.h): features, the label HMM,
// training-set construction, scoring and the rank union, and the C-ABI.
//
// There is no counterpart in the reference, which selects conditioning states
// by PBWT alone (haplotype_set.cpp:682-728; union conditioning_set.cpp:96-104).
// The proposal sits in that place: its candidates are the PBWT selection at a
// larger K, and its output replaces the union of compactSelection.
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <cmath>
#include <random>

#include "context.h"
#include "genotype.h"
#include "learned.h"
#include "mlp.h"
#include "tc.h"

namespace gp {

int mlp_forward_device(Context& c, const __nv_bfloat16* x, int n, float* score, __nv_bfloat16* h1, __nv_bfloat16* h2);
int mlp_train_device(Context& c, int n, int rows, float lr, bool want_grad);

namespace {

// Target bit planes over the common rows (bit i of word w = common row 32 w + i):
// the two current haplotypes, and from the genotype likelihoods the sites with
// a confident call (the best genotype ahead of the next by at least 10 phred),
// whether that call carries an alternative allele, and whether it carries a
// reference allele.
__global__ void k_pack_targets(const uint8_t* __restrict__ h0, const uint8_t* __restrict__ h1,
                               const uint8_t* __restrict__ gl, const uint8_t* __restrict__ flat,
                               const int32_t* __restrict__ ploidy, const int32_t* __restrict__ common2tot, int n_com,
                               int W, int L, uint32_t* __restrict__ planes) {
  const int t = blockIdx.y;
  const int wi = blockIdx.x * blockDim.x + threadIdx.x;
  if (wi >= W) return;
  const int pl = ploidy[t];
  uint32_t b0 = 0, b1 = 0, cf = 0, ga = 0, gr = 0;
  for (int i = 0; i < 32; ++i) {
    const int r = wi * 32 + i;
    if (r >= n_com) break;
    const size_t ts = (size_t)t * L + common2tot[r];
    const uint32_t bit = 1u << i;
    if (h0[ts]) b0 |= bit;
    if (h1[ts]) b1 |= bit;
    if (flat[ts]) continue;
    const uint8_t* g = gl + ts * 3;
    int best, margin;
    if (pl > 1) {
      const int p0 = g[0], p1 = g[1], p2 = g[2];
      best = p0 <= p1 && p0 <= p2 ? 0 : (p1 <= p2 ? 1 : 2);
      const int lo = min(p0, min(p1, p2));
      const int nx = best == 0 ? min(p1, p2) : (best == 1 ? min(p0, p2) : min(p0, p1));
      margin = nx - lo;
      if (best >= 1) ga |= bit;
      if (best <= 1) gr |= bit;
    } else {
      best = g[1] < g[0] ? 1 : 0;
      margin = abs((int)g[0] - (int)g[1]);
      if (best == 1) ga |= bit;
      else gr |= bit;
    }
    if (margin >= 10) cf |= bit;
  }
  uint32_t* p = planes + (size_t)t * kPlanes * W + wi;
  p[0] = b0;
  p[W] = b1;
  p[2 * W] = cf;
  p[3 * W] = ga;
  p[4 * W] = gr;
}

struct FeatArgs {
  const uint32_t* refT;
  int W, n_com, nwin, Kpc;
  const uint32_t* planes;
  const uint32_t* cand;
  const int32_t* ncand;
  const int32_t* kfinal;
  const int32_t* urank;  // [n][N]: PBWT level << 16 | insertion index of the candidate in the union
  int N, depth;
  int t0;            // first target of the launch (blockIdx.z = t - t0)
  __nv_bfloat16* x;  // rows (((t - t0) * nwin + w) * Kpc + k), kMlpInP columns
};

__device__ __forceinline__ uint32_t valid_mask(int wi, int n_com) {
  const int r0 = wi * 32;
  return n_com - r0 >= 32 ? 0xFFFFFFFFu : (n_com > r0 ? (1u << (n_com - r0)) - 1u : 0u);
}

// Matching common sites of x (= candidate XOR target haplotype) going down from
// row pos (inclusive), at most 64 words.
__device__ int run_down(const uint32_t* cr, const uint32_t* th, int pos) {
  int wi = pos >> 5, b = pos & 31;
  uint32_t v = (cr[wi] ^ th[wi]) & (b == 31 ? 0xFFFFFFFFu : ((2u << b) - 1u));
  if (v) return b - (31 - __clz(v));
  int run = b + 1;
  for (int k = 1; k < 64 && wi - k >= 0; ++k) {
    const uint32_t x = cr[wi - k] ^ th[wi - k];
    if (x) return run + __clz(x);
    run += 32;
  }
  return run;
}

// Matching common sites going up from row pos (inclusive), within n_com.
__device__ int run_up(const uint32_t* cr, const uint32_t* th, int pos, int W, int n_com) {
  int wi = pos >> 5, b = pos & 31;
  uint32_t v = ((cr[wi] ^ th[wi]) | ~valid_mask(wi, n_com)) >> b;
  if (v) return __ffs(v) - 1;
  int run = 32 - b;
  for (int k = 1; k < 64 && wi + k < W; ++k) {
    const uint32_t x = (cr[wi + k] ^ th[wi + k]) | ~valid_mask(wi + k, n_com);
    if (x) return run + __ffs(x) - 1;
    run += 32;
  }
  return run;
}

// One thread per (target, window, candidate): the kMlpIn features, as BF16.
__global__ void __launch_bounds__(128) k_features(FeatArgs a) {
  const int t = a.t0 + blockIdx.z, w = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.Kpc) return;
  __nv_bfloat16* row = a.x + (((size_t)blockIdx.z * a.nwin + w) * a.Kpc + k) * kMlpInP;
  float f[kMlpInP];
#pragma unroll
  for (int i = 0; i < kMlpInP; ++i) f[i] = 0.f;
  if (k < a.ncand[t]) {
    const uint32_t c = a.cand[(size_t)t * a.Kpc + k];
    const uint32_t* cr = a.refT + (size_t)c * a.W;
    const uint32_t* P = a.planes + (size_t)t * kPlanes * a.W;
    const uint32_t *T0 = P, *T1 = P + a.W, *CF = P + 2 * a.W, *GA = P + 3 * a.W, *GR = P + 4 * a.W;
    // per-window counts for w-4 .. w+4
    float m0[9], m1[9], ag[9], dg[9], ncf[9];
    int present = 0;
    float mm0 = 0.f, mm1 = 0.f, cdens = 0.f, t0d = 0.f, t1d = 0.f, hom_mm = 0.f, het = 0.f, het_m = 0.f,
          hom_mm3 = 0.f;
#pragma unroll
    for (int o = 0; o < 9; ++o) {
      const int wx = w + o - 4;
      m0[o] = m1[o] = ag[o] = dg[o] = ncf[o] = 0.f;
      if (wx < 0 || wx >= a.nwin) continue;
      if (o >= 2 && o <= 6) ++present;
      int c0 = 0, c1 = 0, ca = 0, cd = 0, cc = 0, nv = 0;
      for (int q = 0; q < kWinWords; ++q) {
        const int wi = wx * kWinWords + q;
        if (wi >= a.W) break;
        const uint32_t vm = valid_mask(wi, a.n_com);
        const uint32_t cw = cr[wi], t0 = T0[wi], t1 = T1[wi], cf = CF[wi];
        const uint32_t agree = (cw & GA[wi]) | (~cw & GR[wi]);
        nv += __popc(vm);
        c0 += __popc(~(cw ^ t0) & vm);
        c1 += __popc(~(cw ^ t1) & vm);
        ca += __popc(cf & agree & vm);
        cd += __popc(cf & ~agree & vm);
        cc += __popc(cf & vm);
        if (o == 4) {
          cdens += __popc(cw & vm);
          t0d += __popc(t0 & vm);
          t1d += __popc(t1 & vm);
          const uint32_t hom = ~(t0 ^ t1) & vm, hets = (t0 ^ t1) & vm;
          hom_mm += __popc((cw ^ t0) & hom);
          het += __popc(hets);
          het_m += __popc(~(cw ^ t0) & hets);
        }
        if (o >= 3 && o <= 5) hom_mm3 += __popc((cw ^ t0) & ~(t0 ^ t1) & vm);
      }
      const float inv = nv > 0 ? 1.f / nv : 0.f;
      m0[o] = c0 * inv;
      m1[o] = c1 * inv;
      ag[o] = (float)ca;
      dg[o] = (float)cd;
      ncf[o] = (float)cc;
      if (o == 4) {
        mm0 = (float)(nv - c0);
        mm1 = (float)(nv - c1);
        cdens *= inv;
        t0d *= inv;
        t1d *= inv;
        het_m = het > 0.f ? het_m / het : 0.f;
        het *= inv;
      }
    }
#pragma unroll
    for (int o = 0; o < 5; ++o) {
      f[o] = m0[o + 2];
      f[5 + o] = m1[o + 2];
      f[10 + o] = ag[o + 2] / fmaxf(1.f, ncf[o + 2]);
      f[15 + o] = dg[o + 2] / fmaxf(1.f, ncf[o + 2]);
    }
    const int first = w * kWinSites, last = min(a.n_com, (w + 1) * kWinSites) - 1;
    const float lr = 1.f / 11.f;
    f[20] = log2f(1.f + run_down(cr, T0, last)) * lr;
    f[21] = log2f(1.f + run_up(cr, T0, first, a.W, a.n_com)) * lr;
    f[22] = log2f(1.f + run_down(cr, T1, last)) * lr;
    f[23] = log2f(1.f + run_up(cr, T1, first, a.W, a.n_com)) * lr;
    f[24] = expf(-mm0);
    f[25] = expf(-mm1);
    f[26] = fmaxf(m0[4], m1[4]);
    f[27] = fminf(m0[4], m1[4]);
    float s0 = 0.f, s1 = 0.f;
    for (int o = 2; o <= 6; ++o) {
      s0 += m0[o];
      s1 += m1[o];
    }
    f[28] = present ? s0 / present : 0.f;
    f[29] = present ? s1 / present : 0.f;
    f[30] = m0[0];
    f[31] = m1[0];
    f[32] = m0[8];
    f[33] = m1[8];
    float sa = 0.f, sd = 0.f, sc = 0.f;
    for (int o = 0; o < 9; ++o) {
      sa += ag[o];
      sd += dg[o];
      sc += ncf[o];
    }
    f[34] = sa / fmaxf(1.f, sc);
    f[35] = sd / fmaxf(1.f, sc);
    f[36] = cdens;
    f[37] = t0d;
    f[38] = t1d;
    f[39] = ncf[4] / (float)kWinSites;
    f[40] = (float)w / (float)a.nwin;
    f[41] = log2f((float)max(1, a.kfinal[t])) / 11.f;
    const int ur = a.urank[(size_t)t * a.N + c];
    f[42] = (float)(ur >> 16) / (float)a.depth;  // PBWT level of the candidate's first push
    f[43] = expf(-hom_mm);
    f[44] = expf(-hom_mm3);
    f[45] = het;
    f[46] = het_m;
    f[47] = (float)(ur & 0xFFFF) / (float)a.Kpc;  // its rank in the PBWT union order
  }
  uint4* dst = reinterpret_cast<uint4*>(row);
#pragma unroll
  for (int q = 0; q < kMlpInP / 8; ++q)
    dst[q] = make_uint4(tc::pack_bf16(f[8 * q], f[8 * q + 1]), tc::pack_bf16(f[8 * q + 2], f[8 * q + 3]),
                        tc::pack_bf16(f[8 * q + 4], f[8 * q + 5]), tc::pack_bf16(f[8 * q + 6], f[8 * q + 7]));
}

template <int T>
__device__ __forceinline__ float block_sum(float v, float* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < T / 32; ++i) s += red[i];
  return s;
}

// Label HMM: the haploid Li-Stephens forward-backward over every candidate of a
// target (states k = threadIdx.x + 256 j), on the site records of the
// imputation path (em, tr, fl, hvar of the candidate conditioning set), with
// per-site normalisation. Accumulates the state posteriors of each window:
// mass[t][w][k] = sum over the window's polymorphic sites of
// alpha(k) beta(k) / sum_k' alpha(k') beta(k'); nsites[t][w] counts those sites.
constexpr int kPostThreads = 256, kPostJ = kMaxCand / kPostThreads;

struct PostArgs {
  const int32_t* poly;
  const int32_t* npoly;
  const int32_t* nstates;
  const uint32_t* hvar;
  const float4* em;
  const float2* tr;
  const uint8_t* fl;
  const int32_t* site_win;
  float* astore;
  const int64_t* aoff;
  int L, WB, Kp, Kpc, nwin;
  float* mass;
  int32_t* nsites;  // written when not null
};

__global__ void __launch_bounds__(kPostThreads) k_state_post(PostArgs a) {
  __shared__ float red[kPostThreads / 32];
  const int t = blockIdx.x, tid = threadIdx.x;
  const int np = a.npoly[t], K = a.nstates[t];
  if (np <= 0 || K <= 0) return;
  const uint32_t* hv = a.hvar + (size_t)t * a.WB * a.Kp;
  const float4* E = a.em + (size_t)t * a.L;
  const float2* TR = a.tr + (size_t)t * a.L;
  const uint8_t* F = a.fl + (size_t)t * a.L;
  const int32_t* PL = a.poly + (size_t)t * a.L;
  float* A = a.astore + a.aoff[t];
  const float invK = 1.f / (float)K;
  auto emit = [&](int l, int j, uint32_t word) {
    const int k = tid + kPostThreads * j;
    if (k >= K) return 0.f;
    if (F[l]) return 1.f;
    const float4 e = E[l];
    return ((word >> (l & 31)) & 1u) ? e.y : e.x;
  };
  uint32_t wd[kPostJ];
  float x[kPostJ];
  // forward, normalised alpha stored per site
  for (int l = 0; l < np; ++l) {
    if ((l & 31) == 0)
#pragma unroll
      for (int j = 0; j < kPostJ; ++j) {
        const int k = tid + kPostThreads * j;
        wd[j] = k < K ? hv[(size_t)(l >> 5) * a.Kp + k] : 0u;
      }
    float s = 0.f;
    const float2 tp = l > 0 ? TR[l - 1] : make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kPostJ; ++j) {
      const float e = emit(l, j, wd[j]);
      x[j] = (l == 0 ? invK : fmaf(x[j], tp.y, tp.x)) * e;
      s += x[j];
    }
    const float inv = 1.f / block_sum<kPostThreads>(s, red);
    float* row = A + (size_t)l * a.Kp;
#pragma unroll
    for (int j = 0; j < kPostJ; ++j) {
      x[j] *= inv;
      const int k = tid + kPostThreads * j;
      if (k < K) row[k] = x[j];
    }
  }
  // backward with the window accumulation
  float acc[kPostJ];
  float eb[kPostJ];
  float seb = 0.f;
  int wcur = -1, nsw = 0;
#pragma unroll
  for (int j = 0; j < kPostJ; ++j) acc[j] = 0.f;
  auto flush = [&]() {
    if (wcur < 0) return;
    float* m = a.mass + ((size_t)t * a.nwin + wcur) * a.Kpc;
#pragma unroll
    for (int j = 0; j < kPostJ; ++j) {
      const int k = tid + kPostThreads * j;
      if (k < K) m[k] = acc[j];
      acc[j] = 0.f;
    }
    if (a.nsites && tid == 0) a.nsites[(size_t)t * a.nwin + wcur] = nsw;
    nsw = 0;
  };
  for (int l = np - 1; l >= 0; --l) {
    if (l == np - 1 || (l & 31) == 31)
#pragma unroll
      for (int j = 0; j < kPostJ; ++j) {
        const int k = tid + kPostThreads * j;
        wd[j] = k < K ? hv[(size_t)(l >> 5) * a.Kp + k] : 0u;
      }
    const float2 tp = l < np - 1 ? TR[l] : make_float2(0.f, 0.f);
    const float* row = A + (size_t)l * a.Kp;
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kPostJ; ++j) {
      const int k = tid + kPostThreads * j;
      // beta normalised by the previous site's sum of emission-weighted betas
      x[j] = l == np - 1 ? (k < K ? 1.f : 0.f) : (k < K ? fmaf(eb[j] / seb, tp.y, tp.x) : 0.f);
      s += k < K ? row[k] * x[j] : 0.f;
    }
    const float inv = 1.f / block_sum<kPostThreads>(s, red);
    const int wn = a.site_win[PL[l]];
    if (wn != wcur) {
      flush();
      wcur = wn;
    }
    ++nsw;
    float se = 0.f;
#pragma unroll
    for (int j = 0; j < kPostJ; ++j) {
      const int k = tid + kPostThreads * j;
      if (k < K) acc[j] = fmaf(row[k] * x[j], inv, acc[j]);
      eb[j] = emit(l, j, wd[j]) * x[j];
      se += eb[j];
    }
    seb = block_sum<kPostThreads>(se, red);
  }
  flush();
}

// Training labels: y = min(1, kpos * q), q the larger of the two haplotypes'
// share of the window's posterior mass held by the candidate; weight 1 + 10 y.
// Rows past a target's candidate count get weight 0.
__global__ void k_labels(const float* __restrict__ mass0, const float* __restrict__ mass1,
                         const int32_t* __restrict__ nsites, const int32_t* __restrict__ ncand, int nwin, int Kpc,
                         float kpos, float* __restrict__ y, float* __restrict__ wt) {
  const int t = blockIdx.z, w = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Kpc) return;
  const size_t r = ((size_t)t * nwin + w) * Kpc + k;
  const int ns = nsites[(size_t)t * nwin + w];
  float yy = 0.f, ww = 0.f;
  if (k < ncand[t]) {
    const float q = ns > 0 ? fmaxf(mass0[r], mass1 ? mass1[r] : 0.f) / (float)ns : 0.f;
    yy = fminf(1.f, kpos * q);
    ww = ns > 0 ? 1.f + 10.f * yy : 0.f;
  }
  y[r] = yy;
  wt[r] = ww;
}

__global__ void k_gather_rows(const __nv_bfloat16* __restrict__ xall, const float* __restrict__ yall,
                              const float* __restrict__ wall, const int64_t* __restrict__ idx, int n,
                              __nv_bfloat16* __restrict__ x, float* __restrict__ y, float* __restrict__ wt) {
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (i >= n) return;
  const int64_t r = idx[i];
  const uint4* src = reinterpret_cast<const uint4*>(xall + r * kMlpInP);
  uint4* dst = reinterpret_cast<uint4*>(x + (size_t)i * kMlpInP);
  if (threadIdx.x < kMlpInP / 8) dst[threadIdx.x] = src[threadIdx.x];
  if (threadIdx.x == 0) {
    y[i] = yall[r];
    wt[i] = wall[r];
  }
}

// Per (target, window): the top kTopR candidates by score, one block argmax per
// rank; best[t][k] keeps a candidate's best rank over windows, cnt[t][k] the
// number of windows that ranked it.
// Order-preserving map of a float to an int (for atomicMax over scores).
__device__ __forceinline__ int fkey(float v) {
  const int b = __float_as_int(v);
  return b >= 0 ? b : b ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float fval(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

__global__ void __launch_bounds__(256) k_window_topr(const float* __restrict__ score, const int32_t* __restrict__ ncand,
                                                     int nwin, int Kpc, int32_t* __restrict__ best,
                                                     int32_t* __restrict__ cnt, int32_t* __restrict__ maxs) {
  __shared__ float sc[kMaxCand];
  __shared__ float rv[8];
  __shared__ int rk[8];
  const int t = blockIdx.y, w = blockIdx.x, tid = threadIdx.x;
  const int nc = ncand[t];
  const float* s = score + ((size_t)t * nwin + w) * Kpc;
  for (int k = tid; k < kMaxCand; k += blockDim.x) sc[k] = k < nc ? s[k] : -INFINITY;
  __syncthreads();
  for (int r = 0; r < kTopR && r < nc; ++r) {
    float bv = -INFINITY;
    int bk = 0x7FFFFFFF;
    for (int k = tid; k < kMaxCand; k += blockDim.x)
      if (sc[k] > bv || (sc[k] == bv && k < bk)) {
        bv = sc[k];
        bk = k;
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
      const int ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
      if (ov > bv || (ov == bv && ok < bk)) {
        bv = ov;
        bk = ok;
      }
    }
    if ((tid & 31) == 0) {
      rv[tid >> 5] = bv;
      rk[tid >> 5] = bk;
    }
    __syncthreads();
    if (tid == 0) {
      float v = rv[0];
      int kk = rk[0];
      for (int i = 1; i < 8; ++i)
        if (rv[i] > v || (rv[i] == v && rk[i] < kk)) {
          v = rv[i];
          kk = rk[i];
        }
      if (v > -INFINITY && kk < nc) {
        atomicMin(&best[(size_t)t * Kpc + kk], r);
        atomicAdd(&cnt[(size_t)t * Kpc + kk], 1);
        atomicMax(&maxs[(size_t)t * Kpc + kk], fkey(v));
        sc[kk] = -INFINITY;
      }
    }
    __syncthreads();
  }
}

// Per target: the union in rank order (best rank, then more windows, then
// candidate order), cut at the target's K; states written in increasing id order.
__global__ void __launch_bounds__(256) k_union_select(const uint32_t* __restrict__ cand,
                                                      const int32_t* __restrict__ ncand,
                                                      const int32_t* __restrict__ kfinal,
                                                      const int32_t* __restrict__ best, const int32_t* __restrict__ cnt,
                                                      const int32_t* __restrict__ maxs, float min_logit, int kmin,
                                                      int Kpc, int Kp, uint32_t* __restrict__ states,
                                                      int32_t* __restrict__ nstates) {
  __shared__ uint32_t key[kMaxCand];
  __shared__ uint8_t sel[kMaxCand];
  typedef cub::BlockScan<int, 256> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int base;
  const int t = blockIdx.x, tid = threadIdx.x;
  const int nc = ncand[t];
  int npow = 1;
  while (npow < nc) npow <<= 1;
  for (int k = tid; k < npow; k += blockDim.x) {
    const int b = k < nc ? best[(size_t)t * Kpc + k] : kTopR;
    key[k] = b < kTopR ? ((uint32_t)b << 22) | ((uint32_t)(1023 - min(1023, cnt[(size_t)t * Kpc + k])) << 12) |
                             (uint32_t)k
                       : 0xFFFFFFFFu;
  }
  for (int k = tid; k < kMaxCand; k += blockDim.x) sel[k] = 0;
  __syncthreads();
  for (int size = 2; size <= npow; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < npow / 2; i += blockDim.x) {
        const int pos = 2 * i - (i & (stride - 1));
        const int pr = pos + stride;
        const bool up = (pos & size) == 0;
        const uint32_t x = key[pos], y = key[pr];
        if ((x > y) == up) {
          key[pos] = y;
          key[pr] = x;
        }
      }
      __syncthreads();
    }
  int m = min(kfinal[t], nc);
  if (kmin > 0) {
    // adaptive size: the candidates some window scores at least min_logit, at
    // least kmin, at most the target's K
    __shared__ int n_ok;
    if (tid == 0) n_ok = 0;
    __syncthreads();
    int mine = 0;
    for (int k = tid; k < nc; k += blockDim.x)
      if (best[(size_t)t * Kpc + k] < kTopR && fval(maxs[(size_t)t * Kpc + k]) >= min_logit) ++mine;
    atomicAdd(&n_ok, mine);
    __syncthreads();
    m = min(m, max(kmin, n_ok));
  }
  for (int i = tid; i < m; i += blockDim.x)
    if (key[i] != 0xFFFFFFFFu) sel[key[i] & 0xFFFu] = 1;
  if (tid == 0) base = 0;
  __syncthreads();
  for (int k0 = 0; k0 < nc; k0 += 256) {
    const int k = k0 + tid;
    const int f = k < nc ? sel[k] : 0;
    int pos, tot;
    Scan(tmp).ExclusiveSum(f, pos, tot);
    if (f) states[(size_t)t * Kp + base + pos] = cand[(size_t)t * Kpc + k];
    __syncthreads();
    if (tid == 0) base += tot;
    __syncthreads();
  }
  if (tid == 0) nstates[t] = base;
}

}  // namespace

// Window of every panel site: that of the last common site at or before it.
int Context::learned_prepare_panel() {
  LearnedWork& lw = learned;
  if (lw.nwin > 0) return GP_OK;
  const int L = host.L;
  std::vector<int32_t> sw(L);
  int r = -1;
  for (int s = 0; s < L; ++s) {
    if (host.common[s]) ++r;
    sw[s] = std::max(0, r) / kWinSites;
  }
  lw.nwin = std::max(1, (host.n_com + kWinSites - 1) / kWinSites);
  cudaError_t e = lw.site_win.ensure((size_t)L * 4);
  if (e != cudaSuccess) return cuda_fail(e, "learned alloc");
  cudaMemcpy(lw.site_win.ptr, sw.data(), (size_t)L * 4, cudaMemcpyHostToDevice);
  return GP_OK;
}

// The candidates of the last PBWT selection (impute.states, stride Kpc) into
// learned.cand, and features for every (target, window, candidate) into x.
int Context::learned_features(int Kpc, DevBuf& xout) {
  int rc = learned_prepare_features(Kpc);
  if (rc != GP_OK) return rc;
  cudaError_t e;
  if ((e = xout.ensure((size_t)tw.n * learned.nwin * Kpc * kMlpInP * 2)) != cudaSuccess)
    return cuda_fail(e, "learned features alloc");
  return learned_feature_rows(Kpc, xout, 0, tw.n);
}

// What the feature rows of every target read: the candidates (the PBWT
// selection's states), the targets' bit planes and the candidates' PBWT ranks.
int Context::learned_prepare_features(int Kpc) {
  LearnedWork& lw = learned;
  TargetWork& T = tw;
  ImputeWork& w = impute;
  const int n = T.n, W = panel.W;
  cudaError_t e;
  if ((e = lw.cand.ensure((size_t)n * Kpc * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = lw.ncand.ensure((size_t)n * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = lw.planes.ensure((size_t)n * kPlanes * W * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = lw.urank.ensure((size_t)n * host.N * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if (!pbwt_active) cudaMemsetAsync(lw.urank.ptr, 0, (size_t)n * host.N * 4, stream);  // whole panel: no union
  cudaMemcpyAsync(lw.cand.ptr, w.states.ptr, (size_t)n * Kpc * 4, cudaMemcpyDeviceToDevice, stream);
  cudaMemcpyAsync(lw.ncand.ptr, w.nstates.ptr, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream);
  k_pack_targets<<<dim3((W + 127) / 128, n), 128, 0, stream>>>(T.h0.as<uint8_t>(), T.h1.as<uint8_t>(),
                                                               T.gl.as<uint8_t>(), T.flat.as<uint8_t>(),
                                                               T.ploidy.as<int32_t>(), pbwt.common2tot, host.n_com, W,
                                                               host.L, lw.planes.as<uint32_t>());
  prof.kernel_launches += 1;
  return cudaGetLastError() == cudaSuccess ? GP_OK : cuda_fail(cudaGetLastError(), "learned planes launch");
}

// Feature rows of targets [t0, t0 + nc) into xout from its first row.
int Context::learned_feature_rows(int Kpc, DevBuf& xout, int t0, int nc) {
  LearnedWork& lw = learned;
  FeatArgs fa;
  fa.refT = panel.refT;
  fa.W = panel.W;
  fa.n_com = host.n_com;
  fa.nwin = lw.nwin;
  fa.Kpc = Kpc;
  fa.planes = lw.planes.as<uint32_t>();
  fa.cand = lw.cand.as<uint32_t>();
  fa.ncand = lw.ncand.as<int32_t>();
  fa.kfinal = lw.d_kfinal.as<int32_t>();
  fa.urank = lw.urank.as<int32_t>();
  fa.N = host.N;
  fa.depth = cfg.pbwt_depth;
  fa.t0 = t0;
  fa.x = xout.as<__nv_bfloat16>();
  k_features<<<dim3((Kpc + 127) / 128, lw.nwin, nc), 128, 0, stream>>>(fa);
  prof.kernel_launches += 1;
  return cudaGetLastError() == cudaSuccess ? GP_OK : cuda_fail(cudaGetLastError(), "learned features launch");
}

// Burn-in / main selection with the learned proposal: PBWT candidates (the
// targets' PBWT K is the candidate count), features, scores, then the union of
// per-window ranks cut at each target's own K. Leaves the states in
// impute.states with stride Kp.
int Context::learned_select_states(int stage, int iteration, int& Kp) {
  LearnedWork& lw = learned;
  TargetWork& T = tw;
  ImputeWork& w = impute;
  const int n = T.n;
  const int Kpc = (std::min(lw.kcand, host.N) + 31) / 32 * 32;
  cudaError_t e0;
  if ((e0 = w.states.ensure((size_t)n * Kpc * 4)) != cudaSuccess) return cuda_fail(e0, "alloc states");
  if ((e0 = w.nstates.ensure((size_t)n * 4)) != cudaSuccess) return cuda_fail(e0, "alloc nstates");
  int rc = pbwt_select_states(stage, iteration, Kpc);
  if (rc != GP_OK) return rc;
  rc = learned_prepare_features(Kpc);
  if (rc != GP_OK) return rc;
  const size_t per_t = (size_t)lw.nwin * Kpc;  // feature rows of one target
  const size_t rows = (size_t)n * per_t;
  cudaError_t e;
  if ((e = lw.score.ensure(rows * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = lw.best.ensure((size_t)n * Kpc * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = lw.cnt.ensure((size_t)n * Kpc * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  // Feature rows and their scores in chunks of targets whose rows fit the
  // memory budget (the rows are 128 B each; the scores are kept for all).
  const size_t row_bytes = (size_t)kMlpInP * 2;
  // at most 8 GiB of rows at a time (64M rows), so that the rows do not take
  // the stores' memory; the device is asked only when the buffer must grow
  const size_t want = std::min<size_t>(rows * row_bytes, size_t(8) << 30);
  const size_t budget = store_budget(lw.x.cap, want);
  const int nc = (int)std::max<size_t>(1, std::min<size_t>(n, budget / (per_t * row_bytes)));
  if ((e = lw.x.ensure((size_t)nc * per_t * row_bytes)) != cudaSuccess) return cuda_fail(e, "learned features alloc");
  for (int t0 = 0; t0 < n; t0 += nc) {
    const int m = std::min(nc, n - t0);
    rc = learned_feature_rows(Kpc, lw.x, t0, m);
    if (rc != GP_OK) return rc;
    rc = mlp_forward_device(*this, lw.x.as<__nv_bfloat16>(), (int)((size_t)m * per_t),
                            lw.score.as<float>() + (size_t)t0 * per_t, nullptr, nullptr);
    if (rc != GP_OK) return rc;
  }
  if ((e = lw.maxs.ensure((size_t)n * Kpc * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  cudaMemsetAsync(lw.maxs.ptr, 0x80, (size_t)n * Kpc * 4, stream);  // below every score's key
  cudaMemsetAsync(lw.best.ptr, 0x7F, (size_t)n * Kpc * 4, stream);
  cudaMemsetAsync(lw.cnt.ptr, 0, (size_t)n * Kpc * 4, stream);
  k_window_topr<<<dim3(lw.nwin, n), 256, 0, stream>>>(lw.score.as<float>(), lw.ncand.as<int32_t>(), lw.nwin, Kpc,
                                                       lw.best.as<int32_t>(), lw.cnt.as<int32_t>(),
                                                       lw.maxs.as<int32_t>());
  int kmax = 1;
  for (int i = 0; i < n; ++i) kmax = std::max(kmax, std::min(lw.kfinal[i], host.N));
  Kp = (kmax + 31) / 32 * 32;
  if ((e = w.states.ensure((size_t)n * Kp * 4)) != cudaSuccess) return cuda_fail(e, "alloc states");
  k_union_select<<<n, 256, 0, stream>>>(lw.cand.as<uint32_t>(), lw.ncand.as<int32_t>(), lw.d_kfinal.as<int32_t>(),
                                        lw.best.as<int32_t>(), lw.cnt.as<int32_t>(), lw.maxs.as<int32_t>(),
                                        lw.min_logit, lw.kmin, Kpc, Kp,
                                        w.states.as<uint32_t>(), w.nstates.as<int32_t>());
  prof.kernel_launches += 2;
  return cudaGetLastError() == cudaSuccess ? GP_OK : cuda_fail(cudaGetLastError(), "learned selection launch");
}

// Per-window state posteriors of both haplotypes of every target over its PBWT
// candidates (the label HMM), from the current haplotypes.
int Context::learned_labels(int Kpc, float kpos, DevBuf& yout, DevBuf& wout) {
  LearnedWork& lw = learned;
  TargetWork& T = tw;
  ImputeWork& w = impute;
  const int n = T.n, L = panel.L;
  int rc = build_condsets_device(n, Kpc);
  if (rc != GP_OK) return rc;
  std::vector<int64_t> aoff(n);
  int64_t tot = 0;
  for (int i = 0; i < n; ++i) {
    aoff[i] = tot;
    tot += (int64_t)impute_np[i] * Kpc;
  }
  const size_t mrows = (size_t)n * lw.nwin * Kpc;
  cudaError_t e;
  if ((e = lw.astore.ensure((size_t)std::max<int64_t>(tot, 1) * 4)) != cudaSuccess)
    return cuda_fail(e, "label HMM store");
  if ((e = lw.aoff.ensure((size_t)n * 8)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  for (DevBuf* b : {&lw.mass0, &lw.mass1})
    if ((e = b->ensure(mrows * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = lw.nsites.ensure((size_t)n * lw.nwin * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = yout.ensure(mrows * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = wout.ensure(mrows * 4)) != cudaSuccess) return cuda_fail(e, "learned alloc");
  if ((e = w.em.ensure((size_t)n * L * 16)) != cudaSuccess) return cuda_fail(e, "alloc em");
  if ((e = w.tr.ensure((size_t)n * L * 8)) != cudaSuccess) return cuda_fail(e, "alloc tr");
  if ((e = w.fl.ensure((size_t)n * L)) != cudaSuccess) return cuda_fail(e, "alloc fl");
  cudaMemcpyAsync(lw.aoff.ptr, aoff.data(), (size_t)n * 8, cudaMemcpyHostToDevice, stream);
  cudaMemsetAsync(lw.mass0.ptr, 0, mrows * 4, stream);
  cudaMemsetAsync(lw.mass1.ptr, 0, mrows * 4, stream);
  cudaMemsetAsync(lw.nsites.ptr, 0, (size_t)n * lw.nwin * 4, stream);
  PostArgs pa;
  pa.poly = w.poly.as<int32_t>();
  pa.npoly = w.npoly.as<int32_t>();
  pa.nstates = w.nstates.as<int32_t>();
  pa.hvar = w.hvar.as<uint32_t>();
  pa.em = w.em.as<float4>();
  pa.tr = w.tr.as<float2>();
  pa.fl = w.fl.as<uint8_t>();
  pa.site_win = lw.site_win.as<int32_t>();
  pa.astore = lw.astore.as<float>();
  pa.aoff = lw.aoff.as<int64_t>();
  pa.L = L;
  pa.WB = w.WB;
  pa.Kp = Kpc;
  pa.Kpc = Kpc;
  pa.nwin = lw.nwin;
  for (int h = 0; h < 2; ++h) {
    // haplotype likelihoods as a burn-in iteration forms them (caller_algorithm.cpp:58-70)
    launch_hl(T.gl.as<uint8_t>(), T.flat.as<uint8_t>(), T.ploidy.as<int32_t>(), T.h0.as<uint8_t>(),
              T.h1.as<uint8_t>(), n, L, 0, h, mc.min_gl, T.hl.as<float>(), stream);
    launch_site_records(panel, mc, w, T.hl.as<float>(), T.flat.as<uint8_t>(), stream);
    pa.mass = (h ? lw.mass1 : lw.mass0).as<float>();
    pa.nsites = h ? nullptr : lw.nsites.as<int32_t>();
    k_state_post<<<n, kPostThreads, 0, stream>>>(pa);
    prof.kernel_launches += 3;
  }
  k_labels<<<dim3((Kpc + 255) / 256, lw.nwin, n), 256, 0, stream>>>(
      lw.mass0.as<float>(), lw.mass1.as<float>(), lw.nsites.as<int32_t>(), lw.ncand.as<int32_t>(), lw.nwin, Kpc,
      kpos, yout.as<float>(), wout.as<float>());
  prof.kernel_launches += 1;
  return cudaGetLastError() == cudaSuccess ? GP_OK : cuda_fail(cudaGetLastError(), "label HMM launch");
}

// Per-target K arrays for the learned mode: PBWT at the candidate count, the
// caller's K for the conditioning set.
int Context::learned_apply_k(bool reset_state) {
  TargetWork& T = tw;
  LearnedWork& lw = learned;
  if (T.n <= 0) return GP_OK;
  if (lw.on) {
    if (lw.kfinal.size() != (size_t)T.n) lw.kfinal = T.kpbwt_h;
    for (int i = 0; i < T.n; ++i) T.kpbwt_h[i] = std::max(lw.kcand, lw.kfinal[i]);
  } else if (lw.kfinal.size() == (size_t)T.n) {
    T.kpbwt_h = lw.kfinal;
    lw.kfinal.clear();
  }
  if (lw.on) {
    cudaError_t e = lw.d_kfinal.ensure((size_t)T.n * 4);
    if (e != cudaSuccess) return cuda_fail(e, "learned alloc");
    std::vector<int32_t> kf(T.n);
    for (int i = 0; i < T.n; ++i) kf[i] = std::min(lw.kfinal[i], host.N);
    cudaMemcpyAsync(lw.d_kfinal.ptr, kf.data(), (size_t)T.n * 4, cudaMemcpyHostToDevice, stream);
  }
  return pbwt_prepare_targets(reset_state);
}

}  // namespace gp

using gp::Context;

extern "C" {

int gp_learned_enable(gp_ctx* ctx, int32_t enable, int32_t kcand) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (enable && (kcand <= 0 || kcand > gp::kMaxCand))
    return (c.fail(GP_E_ARG, "learned: candidates per target must be in 1..2048"), GP_E_ARG);
  if (enable && !c.mlp.ready) return (c.fail(GP_E_STATE, "learned: the network has no parameters"), GP_E_STATE);
  int rc = c.learned_prepare_panel();
  if (rc != GP_OK) return rc;
  c.learned.on = enable != 0;
  c.learned.kcand = kcand;
  return c.learned_apply_k();
}

int gp_learned_size(gp_ctx* ctx, float min_prob, int32_t kmin) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (kmin < 0 || (kmin > 0 && !(min_prob > 0.f && min_prob < 1.f)))
    return (c.fail(GP_E_ARG, "learned size: kmin >= 0 and 0 < min_prob < 1"), GP_E_ARG);
  c.learned.kmin = kmin;
  c.learned.min_logit = kmin > 0 ? std::log(min_prob / (1.f - min_prob)) : 0.f;
  return GP_OK;
}

int32_t gp_learned_windows(gp_ctx* ctx) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  const int rc = c.learned_prepare_panel();
  return rc != GP_OK ? rc : c.learned.nwin;
}

int gp_state_posteriors(gp_ctx* ctx, int32_t n, const int64_t* states_off, const uint32_t* states, const float* hl,
                        const uint8_t* flat, float* mass, int32_t* nsites) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (n <= 0 || n > GP_MAX_BATCH || !states_off || !states || !hl || !flat || !mass || !nsites)
    return (c.fail(GP_E_ARG, "state posteriors: bad argument"), GP_E_ARG);
  int rc = c.learned_prepare_panel();
  if (rc != GP_OK) return rc;
  const int L = c.panel.L, nwin = c.learned.nwin;
  std::vector<int64_t> off(states_off, states_off + n + 1);
  std::vector<uint32_t> st(states, states + off[n]);
  gp::ImputeWork& w = c.impute;
  cudaError_t e;
  if ((e = w.hl.ensure((size_t)n * 2 * L * 4)) != cudaSuccess) return c.cuda_fail(e, "alloc hl");
  if ((e = w.flat.ensure((size_t)n * L)) != cudaSuccess) return c.cuda_fail(e, "alloc flat");
  cudaMemcpyAsync(w.hl.ptr, hl, (size_t)n * 2 * L * 4, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(w.flat.ptr, flat, (size_t)n * L, cudaMemcpyHostToDevice, c.stream);
  rc = c.build_condsets(n, off, st);
  if (rc != GP_OK) return rc;
  const int Kp = w.Kp;
  std::vector<int64_t> aoff(n);
  int64_t tot = 0;
  for (int i = 0; i < n; ++i) {
    aoff[i] = tot;
    tot += (int64_t)c.impute_np[i] * Kp;
  }
  gp::LearnedWork& lw = c.learned;
  if ((e = w.em.ensure((size_t)n * L * 16)) != cudaSuccess) return c.cuda_fail(e, "alloc em");
  if ((e = w.tr.ensure((size_t)n * L * 8)) != cudaSuccess) return c.cuda_fail(e, "alloc tr");
  if ((e = w.fl.ensure((size_t)n * L)) != cudaSuccess) return c.cuda_fail(e, "alloc fl");
  if ((e = lw.astore.ensure((size_t)std::max<int64_t>(tot, 1) * 4)) != cudaSuccess)
    return c.cuda_fail(e, "label HMM store");
  if ((e = lw.aoff.ensure((size_t)n * 8)) != cudaSuccess) return c.cuda_fail(e, "alloc");
  if ((e = lw.mass0.ensure((size_t)n * nwin * Kp * 4)) != cudaSuccess) return c.cuda_fail(e, "alloc");
  if ((e = lw.nsites.ensure((size_t)n * nwin * 4)) != cudaSuccess) return c.cuda_fail(e, "alloc");
  cudaMemcpyAsync(lw.aoff.ptr, aoff.data(), (size_t)n * 8, cudaMemcpyHostToDevice, c.stream);
  cudaMemsetAsync(lw.mass0.ptr, 0, (size_t)n * nwin * Kp * 4, c.stream);
  cudaMemsetAsync(lw.nsites.ptr, 0, (size_t)n * nwin * 4, c.stream);
  gp::launch_site_records(c.panel, c.mc, w, w.hl.as<float>(), w.flat.as<uint8_t>(), c.stream);
  gp::PostArgs pa;
  pa.poly = w.poly.as<int32_t>();
  pa.npoly = w.npoly.as<int32_t>();
  pa.nstates = w.nstates.as<int32_t>();
  pa.hvar = w.hvar.as<uint32_t>();
  pa.em = w.em.as<float4>();
  pa.tr = w.tr.as<float2>();
  pa.fl = w.fl.as<uint8_t>();
  pa.site_win = lw.site_win.as<int32_t>();
  pa.astore = lw.astore.as<float>();
  pa.aoff = lw.aoff.as<int64_t>();
  pa.L = L;
  pa.WB = w.WB;
  pa.Kp = Kp;
  pa.Kpc = Kp;
  pa.nwin = nwin;
  pa.mass = lw.mass0.as<float>();
  pa.nsites = lw.nsites.as<int32_t>();
  gp::k_state_post<<<n, gp::kPostThreads, 0, c.stream>>>(pa);
  c.prof.kernel_launches += 2;
  std::vector<float> m((size_t)n * nwin * Kp);
  cudaMemcpyAsync(m.data(), lw.mass0.ptr, m.size() * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(nsites, lw.nsites.ptr, (size_t)n * nwin * 4, cudaMemcpyDeviceToHost, c.stream);
  if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return c.cuda_fail(e, "state posteriors");
  for (int i = 0; i < n; ++i) {
    const int K = (int)(off[i + 1] - off[i]);
    for (int ww = 0; ww < nwin; ++ww)
      std::copy(m.begin() + ((size_t)i * nwin + ww) * Kp, m.begin() + ((size_t)i * nwin + ww) * Kp + K,
                mass + (size_t)nwin * off[i] + (size_t)ww * K);
  }
  return GP_OK;
}

int gp_learned_train(gp_ctx* ctx, int32_t kcand, float kpos, int32_t steps, int32_t batch, float lr, uint64_t seed,
                     float* losses) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (c.tw.n <= 0) return (c.fail(GP_E_STATE, "learned: no targets"), GP_E_STATE);
  if (kcand <= 0 || kcand > gp::kMaxCand || steps < 0 || batch <= 0 || batch % 128 || !(kpos > 0.f))
    return (c.fail(GP_E_ARG, "learned train: bad argument"), GP_E_ARG);
  if (!c.mlp.ready) {
    int rc = gp_mlp_init(ctx, seed);
    if (rc != GP_OK) return rc;
  }
  int rc = c.learned_prepare_panel();
  if (rc != GP_OK) return rc;
  // candidates: the PBWT selection at kcand for every target, from the current haplotypes
  const bool was_on = c.learned.on;
  const int was_kcand = c.learned.kcand;
  c.learned.on = true;
  c.learned.kcand = kcand;
  rc = c.learned_apply_k();
  if (rc != GP_OK) return rc;
  const int Kpc = (std::min(kcand, c.host.N) + 31) / 32 * 32;
  gp::LearnedWork& lw = c.learned;
  cudaError_t e = c.impute.states.ensure((size_t)c.tw.n * Kpc * 4);
  if (e == cudaSuccess) e = c.impute.nstates.ensure((size_t)c.tw.n * 4);
  if (e != cudaSuccess) return c.cuda_fail(e, "alloc states");
  // the sweep advances the targets' PBWT state (tar_hap); training leaves it as it was
  const size_t nh = c.tw.hap_target.size();
  if ((e = lw.tarhap_save.ensure(std::max<size_t>(nh, 1))) != cudaSuccess) return c.cuda_fail(e, "learned alloc");
  cudaMemcpyAsync(lw.tarhap_save.ptr, c.tw.tar_hap.ptr, nh, cudaMemcpyDeviceToDevice, c.stream);
  rc = c.pbwt_select_states(GP_STAGE_BURN, 1 << 20, Kpc);
  cudaMemcpyAsync(c.tw.tar_hap.ptr, lw.tarhap_save.ptr, nh, cudaMemcpyDeviceToDevice, c.stream);
  if (rc == GP_OK) rc = c.learned_features(Kpc, lw.xall);
  if (rc == GP_OK) rc = c.learned_labels(Kpc, kpos, lw.yall, lw.wall);
  c.learned.on = was_on;
  c.learned.kcand = was_kcand;
  int rc2 = c.learned_apply_k();
  if (rc != GP_OK) return rc;
  if (rc2 != GP_OK) return rc2;
  // rows with weight: the candidates of windows with polymorphic sites
  const size_t rows = (size_t)c.tw.n * lw.nwin * Kpc;
  std::vector<float> wt(rows);
  // on the context's stream: the labels were written there, and that stream does
  // not synchronise with the legacy default stream
  cudaMemcpyAsync(wt.data(), lw.wall.ptr, rows * 4, cudaMemcpyDeviceToHost, c.stream);
  if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return c.cuda_fail(e, "learned labels");
  std::vector<int64_t> pool;
  pool.reserve(rows);
  for (size_t r = 0; r < rows; ++r)
    if (wt[r] > 0.f) pool.push_back((int64_t)r);
  if (pool.empty()) return (c.fail(GP_E_DATA, "learned train: no labelled rows"), GP_E_DATA);
  rc = gp::mlp_rows(c, batch);
  if (rc != GP_OK) return rc;
  e = lw.idx.ensure((size_t)batch * 8);
  if (e != cudaSuccess) return c.cuda_fail(e, "learned alloc");
  std::mt19937_64 g(seed ^ 0x5DEECE66Dull);
  std::shuffle(pool.begin(), pool.end(), g);
  size_t at = 0;
  std::vector<int64_t> idx(batch);
  gp::MlpState& M = c.mlp;
  for (int s = 0; s < steps; ++s) {
    for (int i = 0; i < batch; ++i) {
      if (at == pool.size()) {
        std::shuffle(pool.begin(), pool.end(), g);
        at = 0;
      }
      idx[i] = pool[at++];
    }
    cudaMemcpyAsync(lw.idx.ptr, idx.data(), (size_t)batch * 8, cudaMemcpyHostToDevice, c.stream);
    gp::k_gather_rows<<<batch / 8, dim3(32, 8), 0, c.stream>>>(lw.xall.as<__nv_bfloat16>(), lw.yall.as<float>(),
                                                               lw.wall.as<float>(), lw.idx.as<int64_t>(), batch,
                                                               M.x.as<__nv_bfloat16>(), M.y.as<float>(),
                                                               M.wt.as<float>());
    c.prof.kernel_launches += 1;
    rc = gp::mlp_train_device(c, batch, batch, lr, false);
    if (rc != GP_OK) return rc;
    if (losses) {
      cudaMemcpyAsync(&losses[s], M.loss.ptr, 4, cudaMemcpyDeviceToHost, c.stream);
    }
    if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return c.cuda_fail(e, "learned train");
  }
  // the label HMM's store and the training rows are not needed by selection:
  // give their memory back to the iteration's stores
  for (gp::DevBuf* b : {&lw.astore, &lw.aoff, &lw.mass0, &lw.mass1, &lw.xall, &lw.yall, &lw.wall, &lw.idx})
    b->release();
  return gp::check_mlp_err(c, "learned train");
}

}  // extern "C"
