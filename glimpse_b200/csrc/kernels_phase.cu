// The 8-hypothesis phasing HMM with Gibbs phase resampling
// (phase/src/models/phasing_hmm.{h,cpp}, rephaseHaplotypes :247-302).
//
// One block per diploid target. Thread `tid` owns states k = tid + 256*j and,
// for each, the 8 hypothesis messages prob[k][0..7] in registers. Per-site
// hypothesis sums (probSumH) are block reductions; SUMK is per state.
// Segment-start messages (phasingProb) and flat-het messages (imputeProb) from
// the backward pass are stored in global memory as [seg][k][8] rows.
#include <cstddef>

#include <cub/block/block_scan.cuh>

#include "internal.h"
#include "phase.h"

namespace gp {

namespace {

constexpr int PT = kPhaseThreads;
constexpr int NW = PT / kWarp;

// ---------------------------------------------------------------------------
// VAR list and segmentation (phasing_hmm.cpp:65-140)
// ---------------------------------------------------------------------------
template <int THREADS, int ITEMS>
__global__ void k_build_vars(const int32_t* __restrict__ poly, const int32_t* __restrict__ npoly,
                             const uint8_t* __restrict__ h0, const uint8_t* __restrict__ h1,
                             const uint8_t* __restrict__ flat, const uint8_t* __restrict__ lq, int L,
                             const int32_t* __restrict__ tsel, PhaseVars V) {
  typedef cub::BlockScan<int, THREADS> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int carry[3];
  const int b = blockIdx.x;
  const int t = tsel ? tsel[b] : b;
  const int np = npoly[t];
  const int32_t* pl = poly + (size_t)t * L;
  const uint8_t* H0 = h0 + (size_t)t * L;
  const uint8_t* H1 = h1 + (size_t)t * L;
  const uint8_t* FL = flat + (size_t)t * L;
  int32_t* vrel = V.rel + (size_t)b * V.lv;
  uint8_t* vcode = V.code + (size_t)b * V.lv;
  int32_t* vseg = V.seg + (size_t)b * V.lv;
  int32_t* vmiss = V.miss + (size_t)b * V.lv;
  int32_t* sstart = V.seg_start + (size_t)b * (V.lv + 2);
  if (threadIdx.x < 3) carry[threadIdx.x] = 0;
  __syncthreads();
  for (int base = 0; base < np; base += THREADS * ITEMS) {
    int isv[ITEMS], isph[ITEMS], isfh[ITEMS], code[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int l = base + threadIdx.x * ITEMS + i;
      isv[i] = isph[i] = isfh[i] = 0;
      code[i] = 0;
      if (l < np) {
        const int s = pl[l];
        const int a0 = H0[s], a1 = H1[s];
        const bool nf = !FL[s] && !lq[s];
        if (nf) {
          isv[i] = 1;
          if (a0 != a1) { isph[i] = 1; code[i] = 0; }
          else code[i] = VT_HOM | (a0 << 3);
        } else if (a0 != a1) {
          isv[i] = 1;
          isfh[i] = 1;
          code[i] = VT_FLAT | (a0 << 3);
        }
      }
    }
    int exv[ITEMS], exh[ITEMS], exm[ITEMS];
    int tv, th, tm;
    Scan(tmp).ExclusiveSum(isv, exv, tv);
    __syncthreads();
    Scan(tmp).ExclusiveSum(isph, exh, th);
    __syncthreads();
    Scan(tmp).ExclusiveSum(isfh, exm, tm);
    const int cv = carry[0], ch = carry[1], cmm = carry[2];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int l = base + threadIdx.x * ITEMS + i;
      if (l < np && isv[i]) {
        const int vi = cv + exv[i];
        const int hc = ch + exh[i];  // peak hets before this entry
        int c = code[i];
        int seg;
        if (isph[i]) {
          c = hc % 3;  // VAR_TYP = n_het % 3
          seg = hc / 3;
          if (hc > 0 && hc % 3 == 0) sstart[seg] = vi;
        } else {
          seg = (hc > 0 ? hc - 1 : 0) / 3;
        }
        vrel[vi] = l;
        vcode[vi] = (uint8_t)c;
        vseg[vi] = seg;
        vmiss[vi] = isfh[i] ? cmm + exm[i] : -1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      carry[0] = cv + tv;
      carry[1] = ch + th;
      carry[2] = cmm + tm;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int nv = carry[0], nh = carry[1], nm = carry[2];
    const int nseg = (nh > 0 ? nh - 1 : 0) / 3 + 1;
    sstart[0] = 0;
    sstart[nseg] = nv;
    V.nvar[b] = nv;
    V.nseg[b] = nseg;
    V.nmiss[b] = nm;
  }
}

// Per-entry transitions (conditioning_set.h:101-105, as getTransition is called
// in phasing_hmm.cpp:152,201 and phasing_hmm.h:381) and segment flags.
__device__ __forceinline__ float transition(const double* __restrict__ cm, int prev, int next, const ModelConst& mc);

__global__ void k_var_records(const int32_t* __restrict__ tsel, const int32_t* __restrict__ poly, int L,
                              const double* __restrict__ cm, ModelConst mc, PhaseVars V) {
  const int b = blockIdx.y;
  const int t = tsel ? tsel[b] : b;
  const int nv = V.nvar[b];
  const int32_t* pl = poly + (size_t)t * L;
  const int32_t* vrel = V.rel + (size_t)b * V.lv;
  const int32_t* vseg = V.seg + (size_t)b * V.lv;
  const int32_t* sstart = V.seg_start + (size_t)b * (V.lv + 2);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const int s = pl[vrel[i]];
    float yn = 0.f;
    if (i + 1 < nv) yn = transition(cm, s, pl[vrel[i + 1]], mc);
    V.yt_next[(size_t)b * V.lv + i] = yn;
    float yp = 0.f;
    if (i > 0) yp = transition(cm, pl[vrel[i - 1]], s, mc);
    V.yt_prev[(size_t)b * V.lv + i] = yp;
    const int seg = vseg[i];
    const int locus = i - sstart[seg];
    const int seglen = sstart[seg + 1] - sstart[seg];
    const int fl = (locus == 0 ? 1 : 0) | (locus == seglen - 1 ? 2 : 0);
    V.flags[(size_t)b * V.lv + i] = (uint8_t)fl;
    const int x = vrel[i] | ((int)V.code[(size_t)b * V.lv + i] << 24) | (fl << 28);
    const int miss = V.miss[(size_t)b * V.lv + i];
    V.recb[(size_t)b * V.lv + i] = make_int4(x, seg, miss, __float_as_int(yn));
    V.recf[(size_t)b * V.lv + i] = make_int4(x, seg, miss, __float_as_int(yp));
  }
}

// ---------------------------------------------------------------------------
// Block reduction of 8 values (one per hypothesis).
// Within a warp a reduce-scatter leaves lane L with the warp sum of value
// ((L>>4)&1)*4 + ((L>>3)&1)*2 + ((L>>2)&1); warps are then combined in order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_sum8(float (&v)[8], float (*red)[NW][8], int& buf, float (&out)[8]) {
  const int lane = threadIdx.x & 31;
  float a[4], bb[2], c;
  {
    const bool up = lane & 16;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float send = up ? v[i] : v[i + 4];
      const float keep = up ? v[i + 4] : v[i];
      a[i] = __fadd_rn(keep, __shfl_xor_sync(0xffffffffu, send, 16));
    }
  }
  {
    const bool up = lane & 8;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float send = up ? a[i] : a[i + 2];
      const float keep = up ? a[i + 2] : a[i];
      bb[i] = __fadd_rn(keep, __shfl_xor_sync(0xffffffffu, send, 8));
    }
  }
  {
    const bool up = lane & 4;
    const float send = up ? bb[0] : bb[1];
    const float keep = up ? bb[1] : bb[0];
    c = __fadd_rn(keep, __shfl_xor_sync(0xffffffffu, send, 4));
  }
  c = __fadd_rn(c, __shfl_xor_sync(0xffffffffu, c, 2));
  c = __fadd_rn(c, __shfl_xor_sync(0xffffffffu, c, 1));
  const int warp = threadIdx.x >> 5;
  if ((lane & 3) == 0) red[buf][warp][((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1)] = c;
  __syncthreads();
  // lane l combines warps for hypotheses (l >> 3) and (l >> 3) + 4; butterflies
  // over the warp index (l & 7) give the lanes of a group identical totals
  static_assert(NW == 8, "one lane per warp partial");
  float x0 = red[buf][lane & 7][lane >> 3];
  float x1 = red[buf][lane & 7][(lane >> 3) + 4];
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    x0 = __fadd_rn(x0, __shfl_xor_sync(0xffffffffu, x0, o));
    x1 = __fadd_rn(x1, __shfl_xor_sync(0xffffffffu, x1, o));
  }
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    out[h] = __shfl_sync(0xffffffffu, x0, 8 * h);
    out[h + 4] = __shfl_sync(0xffffffffu, x1, 8 * h);
  }
  buf ^= 1;
}

// horizontal_add of 8 lanes as the reference's AVX reduction orders it
// (phasing_hmm.h:47-57): ((v0+v4)+(v1+v5)) + ((v2+v6)+(v3+v7)).
__device__ __forceinline__ float hadd8(const float (&v)[8]) {
  const float l0 = __fadd_rn(v[0], v[4]), l1 = __fadd_rn(v[1], v[5]);
  const float l2 = __fadd_rn(v[2], v[6]), l3 = __fadd_rn(v[3], v[7]);
  return __fadd_rn(__fadd_rn(l0, l1), __fadd_rn(l2, l3));
}

// Hypothesis allele at a het of type `typ` (ALLELE(HAP_NUMBER-h-1, 2-typ), phasing_hmm.h:45).
__device__ __forceinline__ int hyp_allele(int h, int typ) { return ((7 - h) >> (2 - typ)) & 1; }

__device__ __forceinline__ float transition(const double* __restrict__ cm, int prev, int next, const ModelConst& mc) {
  const double d = mc.nrho * (cm[next] - cm[prev]);
  double x = -expm1(d);
  x = x < 1e-7 ? 1e-7 : (x > mc.one_l ? mc.one_l : x);
  return (float)x;  // conditioning_set.h:101-105
}

struct PhaseShared {
  // per VAR code: emissions of the 8 hypotheses for a state allele of 0 ([0..7]) and 1 ([8..15]); read as float4
  __align__(16) float etab[16][16];
  float red[2][NW][8];
  float sumH[8];
  float sumT;
  float hprobs[64];
  float of1[8];
  int dip;
  int err;
};
static_assert(alignof(PhaseShared) >= 16 && offsetof(PhaseShared, etab) % 16 == 0, "etab rows are read as float4");

// Emission table of the VAR codes (phasing_hmm.h:140-366): a peak het of type
// typ emits ee where the state allele equals the hypothesis allele and ed
// elsewhere; a peak hom emits 1 for the observed allele and ed/ee for the other;
// a flat het emits nothing (1). Entries of unused codes are 1.
__device__ __forceinline__ void fill_emission_table(float (*etab)[16], const ModelConst& mc, int tid) {
  if (tid < 16 * 16) {
    const int code = tid >> 4, a = (tid >> 3) & 1, h = tid & 7;
    const int typ = code & 7, alt = (code >> 3) & 1;
    const float mism = mc.ed_phs / mc.ee_phs;
    float e = 1.0f;
    if (typ < 3) e = (a == hyp_allele(h, typ)) ? mc.ee_phs : mc.ed_phs;
    else if (typ == VT_HOM) e = (a != alt) ? mism : 1.0f;
    etab[code][a * 8 + h] = e;
  }
}

// One site update: INIT / RUN / COLLAPSE (phasing_hmm.h:140-366) for every VAR
// type at once: the type enters only through the emission vectors e0 / e1 (state
// allele 0 / 1), and a factor of exactly 1 leaves a product unchanged, so peak
// hets, peak homs and flat hets share one loop. m selects the site's bit in the
// Hvar words. Ends with the hypothesis sums.
template <int J, int MODE>
__device__ __forceinline__ void site_update(float (&prob)[J][8], const float (&sumk)[J], const uint32_t (&w)[J],
                                            uint32_t m, int K, int tid, const float (&e0)[8], const float (&e1)[8],
                                            float yt, float nt, float (&sumH)[8], float& sumT, float (*red)[NW][8],
                                            int& buf) {
  float tF[8];
  float ntp = 0.f;
  if (MODE != 0) {
    const float sc = yt / __fmul_rn((float)K, sumT);
#pragma unroll
    for (int h = 0; h < 8; ++h) tF[h] = __fmul_rn(sumH[h], sc);
    ntp = nt / sumT;
  }
  float part[8];
#pragma unroll
  for (int h = 0; h < 8; ++h) part[h] = 0.f;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int k = tid + j * PT;
    if (k >= K) continue;
    const bool bit = (w[j] & m) != 0u;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      const float e = bit ? e1[h] : e0[h];
      float v;
      if (MODE == 0) v = e;
      else if (MODE == 1) v = __fmul_rn(fmaf(prob[j][h], ntp, tF[h]), e);
      else v = __fmul_rn(fmaf(sumk[j], ntp, tF[h]), e);
      prob[j][h] = v;
      part[h] = __fadd_rn(part[h], v);
    }
  }
  block_sum8(part, red, buf, sumH);
  sumT = hadd8(sumH);
}

// INIT at a flat het: every message is 1 / (8 K) (phasing_hmm.h:140-366).
template <int J>
__device__ __forceinline__ void site_init_flat(float (&prob)[J][8], int K, float (&sumH)[8], float& sumT) {
  const float v = 1.0f / (float)(8u * (unsigned)K);
#pragma unroll
  for (int j = 0; j < J; ++j)
#pragma unroll
    for (int h = 0; h < 8; ++h) prob[j][h] = v;
#pragma unroll
  for (int h = 0; h < 8; ++h) sumH[h] = 0.125f;
  sumT = 1.0f;
}

// Emission vectors of a VAR code from the shared table.
__device__ __forceinline__ void load_emissions(const float (*etab)[16], int code, float (&e0)[8], float (&e1)[8]) {
  const float4* r = reinterpret_cast<const float4*>(etab[code]);
  const float4 a = r[0], b = r[1], c = r[2], d = r[3];
  e0[0] = a.x; e0[1] = a.y; e0[2] = a.z; e0[3] = a.w; e0[4] = b.x; e0[5] = b.y; e0[6] = b.z; e0[7] = b.w;
  e1[0] = c.x; e1[1] = c.y; e1[2] = c.z; e1[3] = c.w; e1[4] = d.x; e1[5] = d.y; e1[6] = d.z; e1[7] = d.w;
}

// One VAR site with the mode chosen at run time (warp-uniform).
template <int J>
__device__ __forceinline__ void site_step(int mode, int code, float (&prob)[J][8], const float (&sumk)[J],
                                          const uint32_t (&w)[J], uint32_t m, int K, int tid,
                                          const float (*etab)[16], float yt, float nt, float (&sumH)[8],
                                          float& sumT, float (*red)[NW][8], int& buf) {
  if (mode == 0 && (code & 7) == VT_FLAT) {
    site_init_flat<J>(prob, K, sumH, sumT);
    return;
  }
  float e0[8], e1[8];
  load_emissions(etab, code, e0, e1);
  if (mode == 1) site_update<J, 1>(prob, sumk, w, m, K, tid, e0, e1, yt, nt, sumH, sumT, red, buf);
  else if (mode == 2) site_update<J, 2>(prob, sumk, w, m, K, tid, e0, e1, yt, nt, sumH, sumT, red, buf);
  else site_update<J, 0>(prob, sumk, w, m, K, tid, e0, e1, yt, nt, sumH, sumT, red, buf);
}

// Packed VAR records (PhaseVars::recb / recf) of 32 consecutive entries,
// double-buffered in shared memory.
struct VarStage {
  int4 rec[2][32];
};

struct VarRec {
  int l, code, fl, seg, miss;
  float yt;
};

__device__ __forceinline__ VarRec unpack_rec(int4 r) {
  VarRec v;
  v.l = r.x & 0xffffff;
  v.code = (r.x >> 24) & 15;
  v.fl = (r.x >> 28) & 3;
  v.seg = r.y;
  v.miss = r.z;
  v.yt = __int_as_float(r.w);
  return v;
}

// Hvar words of the poly block holding the current site, with the adjacent
// block (in sweep direction) fetched ahead.
template <int J>
struct WordCache {
  uint32_t w[J], wn[J];
  int cur = -1, nxt = -1;
  __device__ __forceinline__ void fetch(uint32_t (&dst)[J], const uint32_t* hv, int blk, int nblk, int Kp, int K,
                                        int tid) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k = tid + j * PT;
      dst[j] = (blk >= 0 && blk < nblk && k < K) ? hv[(size_t)blk * Kp + k] : 0u;
    }
  }
  __device__ __forceinline__ void need(int blk, int dir, const uint32_t* hv, int nblk, int Kp, int K, int tid) {
    if (blk == cur) return;
    if (blk == nxt) {
#pragma unroll
      for (int j = 0; j < J; ++j) w[j] = wn[j];
    } else {
      fetch(w, hv, blk, nblk, Kp, K, tid);
    }
    cur = blk;
    nxt = blk + dir;
    fetch(wn, hv, nxt, nblk, Kp, K, tid);
  }
};

template <int J>
__global__ void __launch_bounds__(PT, 2) k_phase(const int32_t* __restrict__ tsel, const int32_t* __restrict__ nstates,
                                              const int32_t* __restrict__ npoly, const uint32_t* __restrict__ hvar,
                                              int WB, int Kp, int L, PhaseVars V, PhaseStore S, ModelConst mc,
                                              uint64_t seed, int iteration, const int32_t* __restrict__ target_ids) {
  __shared__ PhaseShared sm;
  __shared__ VarStage vs;
  int buf = 0;
  const int b = S.order ? S.order[blockIdx.x] : blockIdx.x;
  const int t = tsel ? tsel[b] : b;
  const int K = nstates[t];
  const int nv = V.nvar[b];
  const int tid = threadIdx.x;
  const bool loader = tid < 32;
  if (tid == 0) sm.err = 0;
  fill_emission_table(sm.etab, mc, tid);  // read after the first barrier below
  const uint32_t* hv = hvar + (size_t)t * WB * Kp;
  const int nblk_poly = (npoly[t] + 31) >> 5;
  const size_t vbase = (size_t)b * V.lv;
  float* PP = S.pprob + S.pprob_off[b];            // [nseg][K][8]
  float* PPS = S.pprob_sum + (size_t)b * (V.lv + 2) * 8;  // [nseg][8]
  float* PPSS = S.pprob_sumsum + (size_t)b * (V.lv + 2);  // [nseg]
  float* IP = S.iprob + S.iprob_off[b];            // [nmiss][K][8]
  float* IPS = S.iprob_sum + (size_t)b * V.lv * 8;  // [nmiss][8]
  float* OF1 = S.of1 + (size_t)b * V.lv * 8;        // [nmiss][8]
  int32_t* dip = S.dip + (size_t)b * (V.lv + 2);
  const uint32_t rng_target = target_ids ? (uint32_t)target_ids[b] : (uint32_t)t;
  const int nvb = (nv + 31) >> 5;

  float prob[J][8];
  float sumk[J];
  float sumH[8];
  float sumT = 0.f;
#pragma unroll
  for (int j = 0; j < J; ++j) sumk[j] = 0.f;
  WordCache<J> wc;

  auto do_sumk = [&]() {
#pragma unroll
    for (int j = 0; j < J; ++j) sumk[j] = hadd8(prob[j]);
  };
  auto store_rows = [&](float* dst) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k = tid + j * PT;
      if (k < K) {
        float4* d4 = reinterpret_cast<float4*>(dst + (size_t)k * 8);
        d4[0] = make_float4(prob[j][0], prob[j][1], prob[j][2], prob[j][3]);
        d4[1] = make_float4(prob[j][4], prob[j][5], prob[j][6], prob[j][7]);
      }
    }
  };

  // ---------------- backward (phasing_hmm.cpp:193-245) ----------------
  if (nvb > 0) {
    const int lb = nvb - 1;
    if (loader && (lb << 5) + tid < nv) vs.rec[lb & 1][tid] = V.recb[vbase + (lb << 5) + tid];
  }
  __syncthreads();
  for (int vb = nvb - 1; vb >= 0; --vb) {
    const int cur = vb & 1;
    int4 pre;
    const bool have_next = vb > 0;
    if (loader && have_next) pre = V.recb[vbase + ((vb - 1) << 5) + tid];
    const int n_in = min(32, nv - (vb << 5));
    for (int ii = n_in - 1; ii >= 0; --ii) {
      const int i = (vb << 5) + ii;
      const VarRec r = unpack_rec(vs.rec[cur][ii]);
      const int l = r.l;
      wc.need(l >> 5, -1, hv, nblk_poly, Kp, K, tid);
      const int code = r.code;
      const int typ = code & 7;
      const int seg = r.seg;
      const int fl = r.fl;
      const float yt = r.yt;
      const float nt = 1.0f - yt;
      const int mode = (i == nv - 1) ? 0 : ((fl & 2) ? 2 : 1);
      site_step<J>(mode, code, prob, sumk, wc.w, 1u << (l & 31), K, tid, sm.etab, yt, nt, sumH, sumT, sm.red, buf);
      if (fl & 1) {
        do_sumk();
        store_rows(PP + (size_t)seg * K * 8);
        if (tid < 8) PPS[seg * 8 + tid] = sumH[tid];
        if (tid == 0) PPSS[seg] = sumT;
      }
      if (typ == VT_FLAT) {
        const int m = r.miss;
        store_rows(IP + (size_t)m * K * 8);
        if (tid < 8) IPS[m * 8 + tid] = sumH[tid];
      }
    }
    if (loader && have_next) vs.rec[cur ^ 1][tid] = pre;
    __syncthreads();
  }
  __syncthreads();

  // ---------------- first diplotype draw (phasing_hmm.cpp:249-256) ----------------
  if (tid == 0) {
    int d0 = 7;
    if (nv > 0) {
      float dp[8];
      float sd = 0.f;
      for (int d = 0; d < 8; ++d) {
        dp[d] = __fmul_rn(PPS[d] / PPSS[0], PPS[7 - d] / PPSS[0]);
        sd = __fadd_rn(sd, dp[d]);
      }
      const float u = __fmul_rn(canonical_float(stream_word(seed, RNG_PHASE, iteration, rng_target, 0)), sd);
      float cs = dp[0];
      d0 = 7;
      for (int d = 0; d < 7; ++d) {
        if (u <= cs) { d0 = d; break; }
        cs = __fadd_rn(cs, dp[d + 1]);
      }
    }
    dip[0] = d0;
    sm.dip = d0;
  }
  __syncthreads();

  // ---------------- forward (phasing_hmm.cpp:142-191) ----------------
  wc.cur = wc.nxt = -1;
  if (nvb > 0 && loader && tid < nv) vs.rec[0][tid] = V.recf[vbase + tid];
  __syncthreads();
  for (int vb = 0; vb < nvb; ++vb) {
    const int cur = vb & 1;
    int4 pre;
    const bool have_next = vb + 1 < nvb;
    if (loader && have_next && ((vb + 1) << 5) + tid < nv) pre = V.recf[vbase + ((vb + 1) << 5) + tid];
    const int n_in = min(32, nv - (vb << 5));
    for (int ii = 0; ii < n_in; ++ii) {
      const int i = (vb << 5) + ii;
      const VarRec r = unpack_rec(vs.rec[cur][ii]);
      const int l = r.l;
      wc.need(l >> 5, 1, hv, nblk_poly, Kp, K, tid);
      const int code = r.code;
      const int typ = code & 7;
      const int seg = r.seg;
      const int fl = r.fl;
      const float yt = r.yt;
      const float nt = 1.0f - yt;
      const int mode = (i == 0) ? 0 : ((fl & 1) ? 2 : 1);
      site_step<J>(mode, code, prob, sumk, wc.w, 1u << (l & 31), K, tid, sm.etab, yt, nt, sumH, sumT, sm.red, buf);
      const bool seg_end = (fl & 2) != 0;
      if (seg_end) do_sumk();
      if (seg_end && i != nv - 1) {
        // TRANS_HAP (phasing_hmm.h:376-397)
        const float yt2 = V.yt_next[vbase + i];
        const float nt2 = 1.0f - yt2;
        const float fact2 = nt2 / sumT;
        const float* nxt = PP + (size_t)(seg + 1) * K * 8;
        float sumHP = 0.f;
#pragma unroll
        for (int h1 = 0; h1 < 8; ++h1) {
          const float fact1 = __fmul_rn(sumH[h1] / sumT, yt2) / (float)K;
          float acc[8];
#pragma unroll
          for (int h2 = 0; h2 < 8; ++h2) acc[h2] = 0.f;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            const int k = tid + j * PT;
            if (k < K) {
              const float p0 = fmaf(prob[j][h1], fact2, fact1);
              const float4* s4 = reinterpret_cast<const float4*>(nxt + (size_t)k * 8);
              const float4 x = s4[0], y = s4[1];
              acc[0] = fmaf(p0, x.x, acc[0]); acc[1] = fmaf(p0, x.y, acc[1]);
              acc[2] = fmaf(p0, x.z, acc[2]); acc[3] = fmaf(p0, x.w, acc[3]);
              acc[4] = fmaf(p0, y.x, acc[4]); acc[5] = fmaf(p0, y.y, acc[5]);
              acc[6] = fmaf(p0, y.z, acc[6]); acc[7] = fmaf(p0, y.w, acc[7]);
            }
          }
          float tot[8];
          block_sum8(acc, sm.red, buf, tot);
          if (tid == 0)
#pragma unroll
            for (int h2 = 0; h2 < 8; ++h2) sm.hprobs[h1 * 8 + h2] = tot[h2];
          sumHP = __fadd_rn(sumHP, hadd8(tot));
        }
        // SAMPLE_DIP (phasing_hmm.h:400-411)
        if (tid == 0) {
          const bool bad1 = isnan(sumHP) || isinf(sumHP) || sumHP < 1.17549435e-38f;
          const int prev = sm.dip;
          float dp[8];
          float sd = 0.f;
          for (int d = 0; d < 8; ++d) {
            dp[d] = __fmul_rn(sm.hprobs[prev * 8 + d] / sumHP, sm.hprobs[(7 - prev) * 8 + (7 - d)] / sumHP);
            sd = __fadd_rn(sd, dp[d]);
          }
          const bool bad2 = isnan(sd) || isinf(sd) || sd < 1.17549435e-38f;
          int nd = prev;
          if (bad1 || bad2) {
            sm.err = 1;
          } else {
            const float u = __fmul_rn(canonical_float(stream_word(seed, RNG_PHASE, iteration, rng_target,
                                                                  (uint64_t)(seg + 1))), sd);
            float cs = dp[0];
            nd = 7;
            for (int d = 0; d < 7; ++d) {
              if (u <= cs) { nd = d; break; }
              cs = __fadd_rn(cs, dp[d + 1]);
            }
          }
          dip[seg + 1] = nd;
          sm.dip = nd;
        }
        __syncthreads();
      }
      if (typ == VT_FLAT) {
        // IMPUTE_FLAT_HET (phasing_hmm.h:414-447)
        const int m = r.miss;
        const float* src = IP + (size_t)m * K * 8;
        float sR[8], sL[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          sR[h] = 1.0f / IPS[m * 8 + h];
          sL[h] = 1.0f / sumH[h];
        }
        float s0[8], s1[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) s0[h] = s1[h] = 0.f;
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const int k = tid + j * PT;
          if (k < K) {
            const int bit = (wc.w[j] >> (l & 31)) & 1u;
            const float4* s4 = reinterpret_cast<const float4*>(src + (size_t)k * 8);
            const float4 x = s4[0], y = s4[1];
            const float ip[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
#pragma unroll
            for (int h = 0; h < 8; ++h) {
              const float p1 = __fmul_rn(ip[h], sR[h]);
              const float p2 = __fmul_rn(prob[j][h], sL[h]);
              if (bit) s1[h] = fmaf(p1, p2, s1[h]); else s0[h] = fmaf(p1, p2, s0[h]);
            }
          }
        }
        float t0[8], t1[8];
        block_sum8(s0, sm.red, buf, t0);
        block_sum8(s1, sm.red, buf, t1);
        if (tid < 8) {
          const float r = t1[tid] / __fadd_rn(t0[tid], t1[tid]);
          OF1[m * 8 + tid] = fmaxf(0.0f, fminf(1.0f, r));
        }
      }
    }
    if (loader && have_next && ((vb + 1) << 5) + tid < nv) vs.rec[cur ^ 1][tid] = pre;
    __syncthreads();
  }
  if (tid == 0) S.err[b] = sm.err;
}

// Allele write-back for peak and flat hets (phasing_hmm.cpp:260-292).
__global__ void k_phase_writeback(const int32_t* __restrict__ tsel, const int32_t* __restrict__ poly, int L,
                                  PhaseVars V, PhaseStore S, ModelConst mc, uint64_t seed, int iteration,
                                  const int32_t* __restrict__ target_ids, uint8_t* __restrict__ h0,
                                  uint8_t* __restrict__ h1) {
  const int b = blockIdx.y;
  const int t = tsel ? tsel[b] : b;
  const int nv = V.nvar[b];
  const int nseg = V.nseg[b];
  const uint32_t rng_target = target_ids ? (uint32_t)target_ids[b] : (uint32_t)t;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const int code = V.code[(size_t)b * V.lv + i];
    const int typ = code & 7;
    if (typ == VT_HOM) continue;
    const int l = V.rel[(size_t)b * V.lv + i];
    const int s = poly[(size_t)t * L + l];
    const int seg = V.seg[(size_t)b * V.lv + i];
    const int i0 = S.dip[(size_t)b * (V.lv + 2) + seg];
    const int i1 = 7 - i0;
    if (typ < 3) {
      h0[(size_t)t * L + s] = (uint8_t)hyp_allele(i0, typ);
      h1[(size_t)t * L + s] = (uint8_t)hyp_allele(i1, typ);
    } else {
      const int m = V.miss[(size_t)b * V.lv + i];
      const float* of = S.of1 + ((size_t)b * V.lv + m) * 8;
      const float h0a0 = 1.0f - of[i0], h0a1 = of[i0];
      const float h1a0 = 1.0f - of[i1], h1a1 = of[i1];
      float p01 = __fmul_rn(fmaf(h0a0, mc.ee_phs, __fmul_rn(h0a1, mc.ed_phs)),
                            fmaf(h1a1, mc.ee_phs, __fmul_rn(h1a0, mc.ed_phs)));
      float p10 = __fmul_rn(fmaf(h0a1, mc.ee_phs, __fmul_rn(h0a0, mc.ed_phs)),
                            fmaf(h1a0, mc.ee_phs, __fmul_rn(h1a1, mc.ed_phs)));
      float sum = __fadd_rn(p01, p10);
      p01 = fminf(fmaxf(p01 / sum, 0.0f), 1.0f);
      p10 = fminf(fmaxf(p10 / sum, 0.0f), 1.0f);
      sum = __fadd_rn(p01, p10);
      const float u = canonical_float(stream_word(seed, RNG_PHASE, iteration, rng_target, (uint64_t)(nseg + m)));
      const bool rf = __dmul_rn((double)u, (double)sum) < (double)p01;
      h0[(size_t)t * L + s] = (uint8_t)(!rf);  // H0 written twice, H1 untouched (phasing_hmm.cpp:283-284)
    }
  }
}

// Shuffle of hets at monomorphic sites (phasing_hmm.cpp:293-301): the m-th such
// het draws word nseg + nmiss + m of the target's phasing stream.
template <int THREADS, int ITEMS>
__global__ void k_mono_shuffle(const int32_t* __restrict__ tsel, const int32_t* __restrict__ polyidx, int L,
                               PhaseVars V, uint64_t seed, int iteration, const int32_t* __restrict__ target_ids,
                               uint8_t* __restrict__ h0, uint8_t* __restrict__ h1) {
  typedef cub::BlockScan<int, THREADS> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int carry;
  const int b = blockIdx.x;
  const int t = tsel ? tsel[b] : b;
  const uint32_t rng_target = target_ids ? (uint32_t)target_ids[b] : (uint32_t)t;
  const uint64_t base_word = (uint64_t)V.nseg[b] + (uint64_t)V.nmiss[b];
  uint8_t* H0 = h0 + (size_t)t * L;
  uint8_t* H1 = h1 + (size_t)t * L;
  const int32_t* pi = polyidx + (size_t)t * L;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < L; base += THREADS * ITEMS) {
    int v[ITEMS], ex[ITEMS], tot;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int s = base + threadIdx.x * ITEMS + i;
      v[i] = (s < L && pi[s] < 0 && H0[s] != H1[s]) ? 1 : 0;
    }
    Scan(tmp).ExclusiveSum(v, ex, tot);
    const int c = carry;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (!v[i]) continue;
      const int s = base + threadIdx.x * ITEMS + i;
      const float u = canonical_float(stream_word(seed, RNG_PHASE, iteration, rng_target, base_word + c + ex[i]));
      const bool rf = u < 0.5f;
      H0[s] = (uint8_t)rf;
      H1[s] = (uint8_t)!rf;
    }
    __syncthreads();
    if (threadIdx.x == 0) carry = c + tot;
    __syncthreads();
  }
}

}  // namespace

void launch_build_vars(const int32_t* tsel, int nb, const int32_t* poly, const int32_t* npoly, const uint8_t* h0,
                       const uint8_t* h1, const uint8_t* flat, const uint8_t* lq, int L, PhaseVars V,
                       cudaStream_t s) {
  k_build_vars<512, 8><<<nb, 512, 0, s>>>(poly, npoly, h0, h1, flat, lq, L, tsel, V);
}

void launch_var_records(const int32_t* tsel, int nb, const int32_t* poly, int L, const double* cm,
                        const ModelConst& mc, PhaseVars V, cudaStream_t s) {
  k_var_records<<<dim3(32, nb), 256, 0, s>>>(tsel, poly, L, cm, mc, V);
}

int launch_phase(int J, const int32_t* tsel, int nb, const int32_t* nstates, const uint32_t* hvar, int WB, int Kp,
                 const int32_t* poly, const int32_t* npoly, int L, const double* cm, PhaseVars V, PhaseStore S,
                 const ModelConst& mc, uint64_t seed, int iteration, const int32_t* target_ids, cudaStream_t s) {
  (void)cm;
  switch (J) {
    case 1: k_phase<1><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 2: k_phase<2><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 3: k_phase<3><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 4: k_phase<4><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 5: k_phase<5><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 6: k_phase<6><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 7: k_phase<7><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    case 8: k_phase<8><<<nb, PT, 0, s>>>(tsel, nstates, npoly, hvar, WB, Kp, L, V, S, mc, seed, iteration, target_ids); break;
    default: return GP_E_ARG;
  }
  return GP_OK;
}

void launch_phase_writeback(const int32_t* tsel, int nb, const int32_t* poly, const int32_t* polyidx, int L,
                            PhaseVars V, PhaseStore S, const ModelConst& mc, uint64_t seed, int iteration,
                            const int32_t* target_ids, uint8_t* h0, uint8_t* h1, cudaStream_t s) {
  dim3 g(64, nb);
  k_phase_writeback<<<g, 256, 0, s>>>(tsel, poly, L, V, S, mc, seed, iteration, target_ids, h0, h1);
  k_mono_shuffle<512, 8><<<nb, 512, 0, s>>>(tsel, polyidx, L, V, seed, iteration, target_ids, h0, h1);
}

}  // namespace gp
