// Conditioning-set construction and the haploid Li-Stephens forward-backward
// (the imputation HMM) for a batch of target haplotypes.
//
// Reference: phase/src/containers/conditioning_set.cpp:123-196 (polymorphic
// sites, Hvar bit gather, transitions) and phase/src/models/imputation_hmm.cpp
// (init :124-134, forward :143-235, backward :237-430).
//
// Layouts (per batch entry t):
//   poly[t][l]        site of the l-th polymorphic site (common, or rare with a
//                     selected carrier), polyidx[t][site] the inverse (-1: mono)
//   hvar[t][b][k]     32-bit word: bit i = allele of state k at poly site 32b+i
//   em[t][l]          (emission0, emission1, HL0, HL1) at poly site l
//   tr[t][l]          (t, nt) between poly sites l and l+1
//   alpha[off_t + l*Kp + k]  forward messages, stored for every poly site
//
// The kernels are compiled with --fmad=false: every fused multiply-add below is
// written as fmaf() exactly where the reference's compiled arithmetic has one
// (explicit _mm256_fmadd_ps, and GCC's contraction of a*b+c in -O3 -mfma builds).
#include <cub/block/block_scan.cuh>

#include "internal.h"

namespace gp {

namespace {

__global__ void k_mark_common(const uint8_t* __restrict__ common, uint8_t* __restrict__ mark, int L) {
  const int t = blockIdx.y;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x)
    mark[(size_t)t * L + s] = common[s];
}

// Rare sites are polymorphic when a selected state carries the non-major allele
// (conditioning_set.cpp:127-143: Svar built from ShapRef of the states).
__global__ void k_mark_rare(const int64_t* __restrict__ shap_off, const int32_t* __restrict__ shap_sites,
                            const uint32_t* __restrict__ states, const int32_t* __restrict__ nstates, int Kp,
                            uint8_t* __restrict__ mark, int L) {
  const int t = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nstates[t]) return;
  const uint32_t h = states[(size_t)t * Kp + k];
  for (int64_t j = shap_off[h]; j < shap_off[h + 1]; ++j) mark[(size_t)t * L + shap_sites[j]] = 1;
}

// Ordered compaction of marked sites: poly list and site -> poly index.
template <int THREADS, int ITEMS>
__global__ void k_compact_poly(const uint8_t* __restrict__ mark, int L, int32_t* __restrict__ poly,
                               int32_t* __restrict__ polyidx, int32_t* __restrict__ npoly) {
  typedef cub::BlockScan<int, THREADS> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int carry;
  const int t = blockIdx.x;
  const uint8_t* m = mark + (size_t)t * L;
  int32_t* pl = poly + (size_t)t * L;
  int32_t* pi = polyidx + (size_t)t * L;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < L; base += THREADS * ITEMS) {
    int v[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int s = base + threadIdx.x * ITEMS + i;
      v[i] = (s < L) ? (int)m[s] : 0;
    }
    int ex[ITEMS];
    int total;
    Scan(tmp).ExclusiveSum(v, ex, total);
    const int c = carry;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int s = base + threadIdx.x * ITEMS + i;
      if (s < L) {
        if (v[i]) {
          pl[c + ex[i]] = s;
          pi[s] = c + ex[i];
        } else {
          pi[s] = -1;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) carry = c + total;
    __syncthreads();
  }
  if (threadIdx.x == 0) npoly[t] = carry;
}

// Hvar words: common sites gather the state's bit from the panel, rare sites
// start at the major allele (conditioning_set.cpp:145-176; Hvar.set(lrel, major)).
__global__ void k_build_hvar(const int32_t* __restrict__ poly, const int32_t* __restrict__ npoly,
                             const int32_t* __restrict__ comrow, const uint8_t* __restrict__ major,
                             const uint32_t* __restrict__ refT, int W, const uint32_t* __restrict__ states,
                             const int32_t* __restrict__ nstates, int Kp, int L, int WB,
                             uint32_t* __restrict__ hvar) {
  const int t = blockIdx.z;
  const int b = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int np = npoly[t];
  if (b * 32 >= np || k >= Kp) return;
  uint32_t word = 0;
  if (k < nstates[t]) {
    const uint32_t* row = refT + (size_t)states[(size_t)t * Kp + k] * W;
    const int32_t* pl = poly + (size_t)t * L;
    int cached = -1;
    uint32_t cw = 0;
    const int n = min(32, np - b * 32);
    for (int i = 0; i < n; ++i) {
      const int s = pl[b * 32 + i];
      const int r = comrow[s];
      uint32_t bit;
      if (r >= 0) {
        if ((r >> 5) != cached) {
          cached = r >> 5;
          cw = row[cached];
        }
        bit = (cw >> (r & 31)) & 1u;
      } else {
        bit = major[s];
      }
      word |= bit << i;
    }
  }
  hvar[((size_t)t * WB + b) * Kp + k] = word;
}

// Rare carriers among the states flip their bit to the non-major allele
// (conditioning_set.cpp:171-172). One thread owns every word of its state.
__global__ void k_flip_rare(const int64_t* __restrict__ shap_off, const int32_t* __restrict__ shap_sites,
                            const int32_t* __restrict__ polyidx, const uint32_t* __restrict__ states,
                            const int32_t* __restrict__ nstates, int Kp, int L, int WB,
                            uint32_t* __restrict__ hvar) {
  const int t = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nstates[t]) return;
  const uint32_t h = states[(size_t)t * Kp + k];
  for (int64_t j = shap_off[h]; j < shap_off[h + 1]; ++j) {
    const int l = polyidx[(size_t)t * L + shap_sites[j]];
    if (l < 0) continue;
    hvar[((size_t)t * WB + (l >> 5)) * Kp + k] ^= 1u << (l & 31);
  }
}

// Emissions (imputation_hmm.cpp:124-134), transitions (conditioning_set.cpp:184-196)
// and site flags per poly site.
__global__ void k_site_records(const int32_t* __restrict__ poly, const int32_t* __restrict__ npoly,
                               const double* __restrict__ cm, const uint8_t* __restrict__ lq,
                               const float* __restrict__ hl, const uint8_t* __restrict__ flat, int L,
                               ModelConst mc, float4* __restrict__ em, float2* __restrict__ tr,
                               uint8_t* __restrict__ fl) {
  const int t = blockIdx.y;
  const int np = npoly[t];
  const int32_t* pl = poly + (size_t)t * L;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < np; l += gridDim.x * blockDim.x) {
    const int s = pl[l];
    const float h0 = hl[(size_t)t * 2 * L + 2 * s];
    const float h1 = hl[(size_t)t * 2 * L + 2 * s + 1];
    const float p0 = fmaf(h0, mc.ee_imp, h1 * mc.ed_imp);
    const float p1 = fmaf(h0, mc.ed_imp, h1 * mc.ee_imp);
    em[(size_t)t * L + l] = make_float4(p0 / (p0 + p1), p1 / (p0 + p1), h0, h1);
    fl[(size_t)t * L + l] = (uint8_t)((flat[(size_t)t * L + s] ? 1 : 0) | (lq[s] ? 2 : 0));
    if (l + 1 < np) {
      const double d = mc.nrho * (cm[pl[l + 1]] - cm[s]);
      double x = -expm1(d);
      x = x < 1e-7 ? 1e-7 : (x > mc.one_l ? mc.one_l : x);
      const float tt = (float)x;
      tr[(size_t)t * L + l] = make_float2(tt, 1.0f - tt);
    }
  }
}

// Sum of up to three values over the block; every thread receives the totals.
// Partial sums are combined lane-butterfly first, then warp by warp in order,
// so all threads (and all launches) see bit-identical results.
template <int NV>
__device__ __forceinline__ void block_sum(float (&v)[NV], float (*red)[kImputeThreads / kWarp][4], int& buf) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = __fadd_rn(v[i], __shfl_xor_sync(0xffffffffu, v[i], o));
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) red[buf][warp][i] = v[i];
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    float s = red[buf][0][i];
#pragma unroll
    for (int w = 1; w < kImputeThreads / kWarp; ++w) s = __fadd_rn(s, red[buf][w][i]);
    v[i] = s;
  }
  buf ^= 1;
}

// One block per haplotype. Thread `tid` owns states k = tid + 256*j. The
// forward pass stores every alpha row; the backward pass keeps beta in
// registers, reads alpha back and forms the allele posteriors.
//
// Latency hiding: the per-site records (emissions, transitions, flags) of the
// next 32-site block and the Hvar words of the next block are fetched while the
// current block is processed (records go through a double-buffered shared-memory
// stage), and the backward pass fetches the alpha row of site l-1 while it
// works on site l. Only the per-site reduction stays on the critical path.
struct SiteStage {
  float4 em[2][32];
  float2 tr[2][32];
  uint8_t fl[2][32];
};

__device__ __forceinline__ void stage_records(SiteStage& st, int buf, int lane, int l, int np, const float4* E,
                                              const float2* T, const uint8_t* F) {
  if (l < np) {
    st.em[buf][lane] = E[l];
    st.tr[buf][lane] = T[l];
    st.fl[buf][lane] = F[l];
  }
}

__global__ void __launch_bounds__(kImputeThreads) k_impute_fb(
    const int32_t* __restrict__ poly, const int32_t* __restrict__ npoly, const int32_t* __restrict__ nstates,
    const uint32_t* __restrict__ hvar, const float4* __restrict__ em, const float2* __restrict__ tr,
    const uint8_t* __restrict__ fl, const int64_t* __restrict__ alpha_off, float* __restrict__ alpha_pool,
    int L, int WB, int Kp, ModelConst mc, float* __restrict__ hp) {
  __shared__ float red[2][kImputeThreads / kWarp][4];
  __shared__ SiteStage st;
  int buf = 0;
  const int t = blockIdx.x;
  const int np = npoly[t];
  const int K = nstates[t];
  if (np == 0 || K == 0) return;
  const float Kf = (float)K;
  float* alpha = alpha_pool + alpha_off[t];
  const uint32_t* hv = hvar + (size_t)t * WB * Kp;
  const float4* E = em + (size_t)t * L;
  const float2* T = tr + (size_t)t * L;
  const uint8_t* F = fl + (size_t)t * L;
  const int tid = threadIdx.x;
  const bool loader = tid < 32;
  constexpr int J = kImputeStatesPerThread;
  const int nblk = (np + 31) >> 5;

  float a[J];
  uint32_t w[J], wn[J];
  float asum = 0.f;  // AlphaSum of the previous site

  // ---------------- forward (imputation_hmm.cpp:143-235) ----------------
  if (loader) stage_records(st, 0, tid, tid, np, E, T, F);
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int k = tid + j * kImputeThreads;
    w[j] = (k < K) ? hv[k] : 0u;
  }
  // T[l-1] of the first site of each block lives in the previous stage; keep it.
  float2 t_prev_block = make_float2(0.f, 0.f);
  __syncthreads();
  for (int b = 0; b < nblk; ++b) {
    const int cur = b & 1;
    // prefetch block b+1
    float4 pe; float2 pt; uint8_t pf = 0;
    const int ln = ((b + 1) << 5) + tid;
    const bool have_next = (b + 1 < nblk);
    if (loader && have_next && ln < np) { pe = E[ln]; pt = T[ln]; pf = F[ln]; }
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k = tid + j * kImputeThreads;
      wn[j] = (have_next && k < K) ? hv[(size_t)(b + 1) * Kp + k] : 0u;
    }
    const int n_in = min(32, np - (b << 5));
    for (int i = 0; i < n_in; ++i) {
      const int l = (b << 5) + i;
      const uint8_t f = st.fl[cur][i];
      const float2 tt = (i == 0) ? t_prev_block : st.tr[cur][i - 1];
      float part[1] = {0.f};
      if (f) {  // flat or low-quality: no emission
        if (l == 0) {
          const float v = 1.0f / Kf;
#pragma unroll
          for (int j = 0; j < J; ++j) a[j] = v;
        } else {
          const float fact1 = tt.x / Kf;
          const float fact2 = tt.y / asum;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              a[j] = fmaf(a[j], fact2, fact1);
              part[0] = __fadd_rn(part[0], a[j]);
            }
          }
        }
      } else {
        const float4 e = st.em[cur][i];
        if (l == 0) {
          const float fact1 = 1.0f / Kf;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              a[j] = __fmul_rn(((w[j] >> i) & 1u) ? e.y : e.x, fact1);
              part[0] = __fadd_rn(part[0], a[j]);
            }
          }
        } else {
          const float fact1 = tt.x / Kf;
          const float fact2 = tt.y / asum;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              a[j] = __fmul_rn(fmaf(a[j], fact2, fact1), ((w[j] >> i) & 1u) ? e.y : e.x);
              part[0] = __fadd_rn(part[0], a[j]);
            }
          }
        }
      }
      float* row = alpha + (size_t)l * Kp;
#pragma unroll
      for (int j = 0; j < J; ++j) {
        const int k = tid + j * kImputeThreads;
        if (k < K) row[k] = a[j];
      }
      if (f && l == 0) {
        asum = 1.0f;  // AlphaSum[0] = 1 at a flat first site (imputation_hmm.cpp:156)
      } else {
        block_sum<1>(part, red, buf);
        asum = part[0];
      }
    }
    t_prev_block = st.tr[cur][31 < n_in - 1 ? 31 : n_in - 1];
    if (loader && have_next && ln < np) {
      st.em[cur ^ 1][tid] = pe;
      st.tr[cur ^ 1][tid] = pt;
      st.fl[cur ^ 1][tid] = pf;
    }
#pragma unroll
    for (int j = 0; j < J; ++j) w[j] = wn[j];
    __syncthreads();
  }

  // ---------------- backward (imputation_hmm.cpp:237-416) ----------------
  float bv[J];
  float bsum_next = 0.f;
  const int lastb = nblk - 1;
  if (loader) stage_records(st, lastb & 1, tid, (lastb << 5) + tid, np, E, T, F);
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int k = tid + j * kImputeThreads;
    w[j] = (k < K) ? hv[(size_t)lastb * Kp + k] : 0u;
  }
  float an[J];  // alpha row of the next site to process
  {
    const float* row = alpha + (size_t)(np - 1) * Kp;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k = tid + j * kImputeThreads;
      an[j] = (k < K) ? row[k] : 0.f;
    }
  }
  __syncthreads();
  for (int b = lastb; b >= 0; --b) {
    const int cur = b & 1;
    float4 pe; float2 pt; uint8_t pf = 0;
    const bool have_next = b > 0;
    const int ln = ((b - 1) << 5) + tid;
    if (loader && have_next) { pe = E[ln]; pt = T[ln]; pf = F[ln]; }
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k = tid + j * kImputeThreads;
      wn[j] = (have_next && k < K) ? hv[(size_t)(b - 1) * Kp + k] : 0u;
    }
    const int n_in = min(32, np - (b << 5));
    for (int i = n_in - 1; i >= 0; --i) {
      const int l = (b << 5) + i;
      float av[J];
#pragma unroll
      for (int j = 0; j < J; ++j) av[j] = an[j];
      if (l > 0) {
        const float* row = alpha + (size_t)(l - 1) * Kp;
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const int k = tid + j * kImputeThreads;
          an[j] = (k < K) ? row[k] : 0.f;
        }
      }
      const uint8_t f = st.fl[cur][i];
      float v[3] = {0.f, 0.f, 0.f};  // prob_hid[0], prob_hid[1], betaSum
      const float4 e = st.em[cur][i];
      const bool last = (l == np - 1);
      if (f) {
        if (last) {
          const float fact1 = 1.0f / Kf;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              if ((w[j] >> i) & 1u) v[1] = __fadd_rn(v[1], av[j]); else v[0] = __fadd_rn(v[0], av[j]);
              bv[j] = fact1;
            }
          }
        } else {
          const float2 tt = st.tr[cur][i];
          const float fact1 = tt.x / Kf;
          const float fact2 = tt.y / bsum_next;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              const float pc = fmaf(bv[j], fact2, fact1);
              const float dot = __fmul_rn(av[j], pc);
              if ((w[j] >> i) & 1u) v[1] = __fadd_rn(v[1], dot); else v[0] = __fadd_rn(v[0], dot);
              v[2] = __fadd_rn(v[2], pc);
              bv[j] = pc;
            }
          }
        }
      } else {
        if (last) {
          const float fact1 = 1.0f / Kf;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              const bool bit = (w[j] >> i) & 1u;
              if (bit) v[1] = __fadd_rn(v[1], av[j]); else v[0] = __fadd_rn(v[0], av[j]);
              const float pn = __fmul_rn(bit ? e.y : e.x, fact1);
              v[2] = __fadd_rn(v[2], pn);
              bv[j] = pn;
            }
          }
        } else {
          const float2 tt = st.tr[cur][i];
          const float fact1 = tt.x / Kf;
          const float fact2 = tt.y / bsum_next;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * kImputeThreads;
            if (k < K) {
              const bool bit = (w[j] >> i) & 1u;
              const float pc = fmaf(bv[j], fact2, fact1);
              const float dot = __fmul_rn(av[j], pc);
              const float pn = __fmul_rn(pc, bit ? e.y : e.x);
              if (bit) v[1] = __fadd_rn(v[1], dot); else v[0] = __fadd_rn(v[0], dot);
              v[2] = __fadd_rn(v[2], pn);
              bv[j] = pn;
            }
          }
        }
      }
      block_sum<3>(v, red, buf);
      float bsum = v[2];
      float po0, po1;
      if (f) {
        if (last) bsum = 1.0f;
        po0 = fmaf(v[0], mc.ee_imp, __fmul_rn(v[1], mc.ed_imp));
        po1 = fmaf(v[0], mc.ed_imp, __fmul_rn(v[1], mc.ee_imp));
        if (!(f & 1)) {
          po0 = __fmul_rn(po0, e.z);
          po1 = __fmul_rn(po1, e.w);
        }
      } else {
        const float ph0 = v[0] / e.x;
        const float ph1 = v[1] / e.y;
        po0 = __fmul_rn(fmaf(ph0, mc.ee_imp, __fmul_rn(ph1, mc.ed_imp)), e.z);
        po1 = __fmul_rn(fmaf(ph0, mc.ed_imp, __fmul_rn(ph1, mc.ee_imp)), e.w);
      }
      if (tid == 0) {
        const int s = poly[(size_t)t * L + l];
        const float den = __fadd_rn(po0, po1);
        hp[(size_t)t * 2 * L + 2 * s] = po0 / den;
        hp[(size_t)t * 2 * L + 2 * s + 1] = po1 / den;
      }
      bsum_next = bsum;
    }
    if (loader && have_next) {
      st.em[cur ^ 1][tid] = pe;
      st.tr[cur ^ 1][tid] = pt;
      st.fl[cur ^ 1][tid] = pf;
    }
#pragma unroll
    for (int j = 0; j < J; ++j) w[j] = wn[j];
    __syncthreads();
  }
}

// Monomorphic sites take the major allele directly (imputation_hmm.cpp:417-429).
__global__ void k_impute_mono(const int32_t* __restrict__ polyidx, const uint8_t* __restrict__ major,
                              const float* __restrict__ hl, const uint8_t* __restrict__ flat, int L, ModelConst mc,
                              float* __restrict__ hp) {
  const int t = blockIdx.y;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x) {
    if (polyidx[(size_t)t * L + s] >= 0) continue;
    float p0 = major[s] ? mc.ed_imp : mc.ee_imp;
    float p1 = major[s] ? mc.ee_imp : mc.ed_imp;
    if (!flat[(size_t)t * L + s]) {
      p0 = __fmul_rn(p0, hl[(size_t)t * 2 * L + 2 * s]);
      p1 = __fmul_rn(p1, hl[(size_t)t * 2 * L + 2 * s + 1]);
    }
    const float den = __fadd_rn(p0, p1);
    hp[(size_t)t * 2 * L + 2 * s] = p0 / den;
    hp[(size_t)t * 2 * L + 2 * s + 1] = p1 / den;
  }
}

int grid_for(int n, int threads, int cap = 4096) {
  int g = (n + threads - 1) / threads;
  return g < 1 ? 1 : (g > cap ? cap : g);
}

}  // namespace

void launch_mark_poly(const DevPanel& P, ImputeWork& w, cudaStream_t s) {
  dim3 g1(grid_for(P.L, 256, 512), w.n);
  k_mark_common<<<g1, 256, 0, s>>>(P.common, w.mark.as<uint8_t>(), P.L);
  dim3 g2((w.Kp + 127) / 128, w.n);
  k_mark_rare<<<g2, 128, 0, s>>>(P.shap_off, P.shap_sites, w.states.as<uint32_t>(), w.nstates.as<int32_t>(), w.Kp,
                                  w.mark.as<uint8_t>(), P.L);
}

void launch_compact_poly(const DevPanel& P, ImputeWork& w, cudaStream_t s) {
  k_compact_poly<512, 8><<<w.n, 512, 0, s>>>(w.mark.as<uint8_t>(), P.L, w.poly.as<int32_t>(),
                                               w.polyidx.as<int32_t>(), w.npoly.as<int32_t>());
}

void launch_build_hvar(const DevPanel& P, ImputeWork& w, cudaStream_t s) {
  dim3 g((w.Kp + 127) / 128, w.WB, w.n);
  k_build_hvar<<<g, 128, 0, s>>>(w.poly.as<int32_t>(), w.npoly.as<int32_t>(), P.comrow, P.major, P.refT, P.W,
                                 w.states.as<uint32_t>(), w.nstates.as<int32_t>(), w.Kp, P.L, w.WB,
                                 w.hvar.as<uint32_t>());
  dim3 g2((w.Kp + 127) / 128, w.n);
  k_flip_rare<<<g2, 128, 0, s>>>(P.shap_off, P.shap_sites, w.polyidx.as<int32_t>(), w.states.as<uint32_t>(),
                                  w.nstates.as<int32_t>(), w.Kp, P.L, w.WB, w.hvar.as<uint32_t>());
}

void launch_site_records(const DevPanel& P, const ModelConst& mc, ImputeWork& w, const float* hl,
                         const uint8_t* flat, cudaStream_t s) {
  dim3 g(grid_for(P.L, 256, 256), w.n);
  k_site_records<<<g, 256, 0, s>>>(w.poly.as<int32_t>(), w.npoly.as<int32_t>(), P.cm, P.lq, hl, flat, P.L, mc,
                                   w.em.as<float4>(), w.tr.as<float2>(), w.fl.as<uint8_t>());
}

void launch_impute_fb(const ModelConst& mc, ImputeWork& w, float* hp, cudaStream_t s) {
  k_impute_fb<<<w.n, kImputeThreads, 0, s>>>(w.poly.as<int32_t>(), w.npoly.as<int32_t>(), w.nstates.as<int32_t>(),
                                             w.hvar.as<uint32_t>(), w.em.as<float4>(), w.tr.as<float2>(),
                                             w.fl.as<uint8_t>(), w.alpha_off.as<int64_t>(), w.alpha.as<float>(),
                                             w.L, w.WB, w.Kp, mc, hp);
}

void launch_impute_mono(const DevPanel& P, const ModelConst& mc, ImputeWork& w, const float* hl,
                        const uint8_t* flat, float* hp, cudaStream_t s) {
  dim3 g(grid_for(P.L, 256, 512), w.n);
  k_impute_mono<<<g, 256, 0, s>>>(w.polyidx.as<int32_t>(), P.major, hl, flat, P.L, mc, hp);
}

}  // namespace gp
