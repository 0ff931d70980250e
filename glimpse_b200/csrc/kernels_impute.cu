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
// One CTA per (32-site block, haplotype). The common sites of a block are
// consecutive common rows, so they span at most two 32-bit words of a panel
// haplotype's row (refT); the CTA first describes every site of the block by the
// position of its bit in that 64-bit pair (or marks it rare), then each thread
// builds the words of its states from two gathered words and register shifts.
__global__ void k_build_hvar(const int32_t* __restrict__ poly, const int32_t* __restrict__ npoly,
                             const int32_t* __restrict__ comrow, const uint8_t* __restrict__ major,
                             const uint32_t* __restrict__ refT, int W, const uint32_t* __restrict__ states,
                             const int32_t* __restrict__ nstates, int Kp, int L, int WB,
                             uint32_t* __restrict__ hvar) {
  __shared__ int s_row[32];
  __shared__ uint32_t s_rmaj;
  const int t = blockIdx.y;
  const int b = blockIdx.x;
  const int np = npoly[t];
  if (b * 32 >= np) return;
  const int n = min(32, np - b * 32);
  if (threadIdx.x < 32) {
    const int i = threadIdx.x;
    int r = -1;
    uint32_t maj = 0u;
    if (i < n) {
      const int site = poly[(size_t)t * L + b * 32 + i];
      r = comrow[site];
      if (r < 0) maj = major[site] ? 1u : 0u;
    }
    s_row[i] = r;
    const uint32_t mb = __ballot_sync(0xffffffffu, maj != 0u);
    if (i == 0) s_rmaj = mb;
  }
  __syncthreads();
  // first common row of the block (rows increase with the site)
  int r0 = -1;
  for (int i = 0; i < n && r0 < 0; ++i) r0 = s_row[i];
  const uint32_t rmaj = s_rmaj;
  const int K = nstates[t];
  uint32_t* out = hvar + ((size_t)t * WB + b) * Kp;
  if (r0 < 0) {  // no common site: the major alleles only
    for (int k = threadIdx.x; k < Kp; k += blockDim.x) out[k] = k < K ? rmaj : 0u;
    return;
  }
  const int w0 = r0 >> 5;
  const bool two = w0 + 1 < W;
  // Runs of consecutive common sites of the block: their rows are consecutive
  // too, so each run is one shifted bit field of the (word w0, word w0 + 1)
  // pair (src: its first bit there, dst: its first site, len: its sites).
  __shared__ uint32_t s_run[32];
  __shared__ int s_nrun;
  if (threadIdx.x == 0) {
    int nr = 0;
    for (int i = 0; i < n;) {
      if (s_row[i] < 0) {
        ++i;
        continue;
      }
      int j = i;
      while (j + 1 < n && s_row[j + 1] >= 0) ++j;
      s_run[nr++] = (uint32_t)(s_row[i] - (w0 << 5)) | ((uint32_t)i << 8) | ((uint32_t)(j - i + 1) << 16);
      i = j + 1;
    }
    s_nrun = nr;
  }
  __syncthreads();
  const int nrun = s_nrun;
  for (int k = threadIdx.x; k < Kp; k += blockDim.x) {
    uint32_t word = 0u;
    if (k < K) {
      const uint32_t* row = refT + (size_t)states[(size_t)t * Kp + k] * W + w0;
      const uint64_t pair = (uint64_t)row[0] | (two ? (uint64_t)row[1] << 32 : 0ull);
      word = rmaj;
      for (int q = 0; q < nrun; ++q) {
        const uint32_t rq = s_run[q];
        const int src = rq & 0xff, dst = (rq >> 8) & 0xff, len = (int)(rq >> 16);
        word |= (uint32_t)((pair >> src) & ((1ull << len) - 1ull)) << dst;
      }
    }
    out[k] = word;
  }
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
// tr[l] = (t / K, 1 - t): the forward/backward recursions divide the
// transition by the number of states at every site (imputation_hmm.cpp:160,209,289,371);
// the quotient is taken here once per site, with the same float division.
__global__ void k_site_records(const int32_t* __restrict__ poly, const int32_t* __restrict__ npoly,
                               const int32_t* __restrict__ nstates, const double* __restrict__ cm,
                               const uint8_t* __restrict__ lq,
                               const float* __restrict__ hl, const uint8_t* __restrict__ flat, int L,
                               ModelConst mc, float4* __restrict__ em, float2* __restrict__ tr,
                               uint8_t* __restrict__ fl) {
  const int t = blockIdx.y;
  const int np = npoly[t];
  const float Kf = (float)nstates[t];
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
      tr[(size_t)t * L + l] = make_float2(tt / Kf, 1.0f - tt);
    }
  }
}

// Posteriors of every site of a haplotype (imputation_hmm.cpp:337-368 and 417-429).
// Poly sites: hp holds (prob_hid[0], prob_hid[1]) as the forward-backward left
// it; the division by the emission, the mixing with the error rates and the HL
// factor are applied here, off the sequential chain. Monomorphic sites take the
// major allele directly.
__global__ void k_impute_finish(const int32_t* __restrict__ polyidx, const uint8_t* __restrict__ major,
                                const float4* __restrict__ em, const uint8_t* __restrict__ fl,
                                const float* __restrict__ hl, const uint8_t* __restrict__ flat, int L, ModelConst mc,
                                float* __restrict__ hp) {
  const int t = blockIdx.y;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L; s += gridDim.x * blockDim.x) {
    const int pi = polyidx[(size_t)t * L + s];
    float2* out = reinterpret_cast<float2*>(hp + (size_t)t * 2 * L + 2 * s);
    if (pi >= 0) {
      const float2 p = *out;
      const float4 e = em[(size_t)t * L + pi];
      const uint8_t f = fl[(size_t)t * L + pi];
      float po0, po1;
      if (f) {
        po0 = fmaf(p.x, mc.ee_imp, __fmul_rn(p.y, mc.ed_imp));
        po1 = fmaf(p.x, mc.ed_imp, __fmul_rn(p.y, mc.ee_imp));
        if (!(f & 1)) {
          po0 = __fmul_rn(po0, e.z);
          po1 = __fmul_rn(po1, e.w);
        }
      } else {
        const float ph0 = p.x / e.x;
        const float ph1 = p.y / e.y;
        po0 = __fmul_rn(fmaf(ph0, mc.ee_imp, __fmul_rn(ph1, mc.ed_imp)), e.z);
        po1 = __fmul_rn(fmaf(ph0, mc.ed_imp, __fmul_rn(ph1, mc.ee_imp)), e.w);
      }
      const float den = __fadd_rn(po0, po1);
      *out = make_float2(po0 / den, po1 / den);
      continue;
    }
    float p0 = major[s] ? mc.ed_imp : mc.ee_imp;
    float p1 = major[s] ? mc.ee_imp : mc.ed_imp;
    if (!flat[(size_t)t * L + s]) {
      p0 = __fmul_rn(p0, hl[(size_t)t * 2 * L + 2 * s]);
      p1 = __fmul_rn(p1, hl[(size_t)t * 2 * L + 2 * s + 1]);
    }
    const float den = __fadd_rn(p0, p1);
    *out = make_float2(p0 / den, p1 / den);
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
  dim3 g(w.WB, w.n);
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
  k_site_records<<<g, 256, 0, s>>>(w.poly.as<int32_t>(), w.npoly.as<int32_t>(), w.nstates.as<int32_t>(), P.cm, P.lq,
                                   hl, flat, P.L, mc,
                                   w.em.as<float4>(), w.tr.as<float2>(), w.fl.as<uint8_t>());
}

void launch_impute_finish(const DevPanel& P, const ModelConst& mc, ImputeWork& w, const float* hl,
                          const uint8_t* flat, float* hp, cudaStream_t s) {
  dim3 g(grid_for(P.L, 256, 512), w.n);
  k_impute_finish<<<g, 256, 0, s>>>(w.polyidx.as<int32_t>(), P.major, w.em.as<float4>(), w.fl.as<uint8_t>(), hl, flat,
                                    P.L, mc, hp);
}

}  // namespace gp
