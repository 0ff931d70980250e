// Imputation HMM forward-backward with W warps per chain and 4 states per lane
// per quad.
//
// The haploid Li-Stephens recursion (phase/src/models/imputation_hmm.cpp:143-416)
// is sequential over sites with a sum over all K states at every site. A chain
// (one haplotype in one direction) is run by W warps of one CTA. The states are
// padded in front to the launch's 128 W J states (J quads per warp, from the
// largest K of the call) and warp w, lane `lane`, local quad j owns the 4
// consecutive padded states 128 (W j + w) + 4 lane + c, c = 0..3 (state k =
// padded index - pad). Every chain runs all J quads, so a site is one
// straight-line block for the scheduler; padded states are held at 0, and quads
// without a state are neither stored nor fetched. Rows of
// the store are kept in padded coordinates with stride Ks, so a lane's 4 values
// of a row are one aligned 16-byte vector: phase 1 writes a row with one 16-byte
// store per lane and quad, phase 2 stages rows with 16-byte cp.async. The
// per-site sums are warp butterflies followed, for W > 1, by an exchange of the
// W partial sums through shared memory behind a named barrier of the chain.
// Hvar words of the next 32-site block and the stored rows of the next D sites
// go through a per-warp shared-memory ring filled by cp.async; per-site records
// (emissions, transitions, flags) of the next block are loaded one block ahead.
//
// Each haplotype is split at M (a multiple of 32) into two chains that run
// concurrently and meet in the middle (no waiting between them):
//   phase 1  forward  [0, M)       stores alpha rows
//            backward [np-1, M]    stores the pre-emission backward rows (prob_curr,
//                                  1 at the last site) and leaves Beta at M
//   phase 2  forward  [M, np)      alpha from row M-1; posteriors from alpha x prob_curr
//            backward [M-1, 0]     Beta from site M; posteriors from stored alpha x prob_curr
// Rows [0, M) of the store hold alpha and rows [M, np) prob_curr: one 4-byte
// write and one read per (site, state), plus 1/8 byte of Hvar per pass.
//
// Sums follow a fixed order (per lane over quads and components, then a lane
// butterfly, then the warps in order), so results are deterministic. Every fused
// multiply-add is an explicit fmaf where the reference's compiled arithmetic has
// one (build with --fmad=false).
#include <algorithm>
#include <type_traits>

#include "internal.h"

namespace gp {

namespace {

constexpr int kMaxChainsPerCta = 4;     // chains per CTA: 1, 2 or 4 (the autotuner's choice)
constexpr int kWarpsPerChain = 1;       // W
constexpr int kRowDepth = 3;         // stored rows fetched this many sites ahead
constexpr int kRing = kRowDepth + 1;      // ring slots

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

struct WarpScratch {
  float* asum;          // [n] AlphaSum at site M-1
  float* bsum;          // [n] betaSum at site M
  float* brow;          // [n][Ks] Beta at site M, padded coordinates
  const int32_t* split; // [n] M
};

// Per-warp shared memory: records (2 blocks), Hvar words (2 blocks) and a row
// ring, both holding the warp's own states: [buffer][quad j][lane] x 16 bytes.
struct WarpSmem {
  float4* em;       // [2][32]
  float2* tr;       // [2][32]
  int32_t* pl;      // [2][32] site of the poly index
  uint4* words;     // [2][J][32]
  float4* ring;     // [kRing][J][32]
  uint8_t* fl;      // [2][32]
};

__host__ __device__ __forceinline__ size_t warp_smem_bytes(int J) {
  return 2 * 32 * 16 + 2 * 32 * 8 + 2 * 32 * 4 + (size_t)(2 + kRing) * J * 32 * 16 + 2 * 32;
}

__device__ __forceinline__ WarpSmem carve(char* base, int J) {
  WarpSmem m;
  size_t o = 0;
  m.em = reinterpret_cast<float4*>(base + o);
  o += 2 * 32 * 16;
  m.tr = reinterpret_cast<float2*>(base + o);
  o += 2 * 32 * 8;
  m.pl = reinterpret_cast<int32_t*>(base + o);
  o += 2 * 32 * 4;
  m.words = reinterpret_cast<uint4*>(base + o);
  o += (size_t)2 * J * 32 * 16;
  m.ring = reinterpret_cast<float4*>(base + o);
  o += (size_t)kRing * J * 32 * 16;
  m.fl = reinterpret_cast<uint8_t*>(base + o);
  return m;
}

// Sum over the W warps of a chain of each warp's partial sums (x, y, z), in
// warp order, through a double-buffered exchange slot and a named barrier of
// the chain's 32 W threads.
template <int W>
__device__ __forceinline__ float3 chain_sum(float x, float y, float z, float4* xch, int parity, int wi, int lane,
                                            int bar_id) {
  if (W == 1) return make_float3(x, y, z);
  float4* slot = xch + parity * W;
  if (lane == 0) slot[wi] = make_float4(x, y, z, 0.f);
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(32 * W) : "memory");
  float4 s = slot[0];
#pragma unroll
  for (int i = 1; i < W; ++i) {
    const float4 v = slot[i];
    s.x = __fadd_rn(s.x, v.x);
    s.y = __fadd_rn(s.y, v.y);
    s.z = __fadd_rn(s.z, v.z);
  }
  return make_float3(s.x, s.y, s.z);
}

__device__ __forceinline__ float& comp(float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ uint32_t compu(const uint4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ float compf(const float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }

// One site of a chain for the owned states, specialised at compile time:
//   FWD   forward (alpha) or backward (Beta) recursion
//   POST  phase 2: form prob_hid from the stored row instead of storing a row
//   INIT  first forward / last backward site: the pre-emission value is 1/K
// Flat or low-quality sites pass emissions (1, 1): the product by 1.0 is exact,
// so the same loop serves both kinds of site.
// At the last site the forward posterior uses alpha alone and the stored
// prob_curr is 1 there, so alpha x 1 is used unchanged (imputation_hmm.cpp:337-368).
// m selects the current site's bit in the Hvar words; rowl points at this lane's
// staged row vector of local quad 0 (shared, quad j at offset 32 j) and srowl at
// its stored row vector (global, quad j at offset 32 W j). Every chain of a
// launch runs the launch's J quads, so a site is one straight-line block; the
// padded states (vf = 0) are kept at 0, and the vectors are written whole.
template <int J, int W, bool FWD, bool POST, bool INIT>
__device__ __forceinline__ void chain_step(float4 (&x)[J], const uint4 (&w)[J], uint32_t m, float (&q0)[4],
                                           float (&q1)[4], float (&q2)[4], const float4 (&vf)[J], uint32_t qmask,
                                           float fact1,
                                           float fact2, float ex, float ey, const float4* rowl, float4* srowl) {
  // components (0, 1) and (2, 3) of a quad are processed as packed pairs
  const f2 fact1p = f2_pack(fact1, fact1), fact2p = f2_pack(fact2, fact2);
  f2 q0p[2] = {f2_pack(q0[0], q0[1]), f2_pack(q0[2], q0[3])};
#pragma unroll
  for (int j = 0; j < J; ++j) {
    float4 r4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (POST) r4 = rowl[32 * j];
    float4 st;
    bool bit[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) bit[c] = (compu(w[j], c) & m) != 0u;
    const f2 xp[2] = {f2_pack(x[j].x, x[j].y), f2_pack(x[j].z, x[j].w)};
    const f2 vp[2] = {f2_pack(vf[j].x, vf[j].y), f2_pack(vf[j].z, vf[j].w)};
    float pcv[4], nx[4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const f2 pc = INIT ? fact1p : f2_fma(xp[h], fact2p, fact1p);
      const f2 e = f2_pack(bit[2 * h] ? ey : ex, bit[2 * h + 1] ? ey : ex);
      // padded states are multiplied by 0, valid ones by 1 (exact)
      const f2 n2 = f2_mul(f2_mul(pc, e), vp[h]);
      q0p[h] = f2_add(q0p[h], n2);
      f2_unpack(pc, pcv[2 * h], pcv[2 * h + 1]);
      f2_unpack(n2, nx[2 * h], nx[2 * h + 1]);
    }
    x[j] = make_float4(nx[0], nx[1], nx[2], nx[3]);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (POST) {
        const float r = compf(r4, c);
        float d;
        if (FWD) d = __fmul_rn(nx[c], r);           // alpha x stored prob_curr (1 at the last site)
        else d = INIT ? r : __fmul_rn(r, pcv[c]);  // stored alpha x prob_curr; alpha alone at the last site
        if (bit[c]) q2[c] = __fadd_rn(q2[c], d);
        else q1[c] = __fadd_rn(q1[c], d);
      } else {
        comp(st, c) = FWD ? nx[c] : (INIT ? 1.0f : pcv[c]);
      }
    }
    if (!POST && ((qmask >> j) & 1u)) srowl[32 * W * j] = st;
  }
  f2_unpack(q0p[0], q0[0], q0[1]);
  f2_unpack(q0p[1], q0[2], q0[3]);
}

// Arguments of one launch, shared by the forward and backward chains.
struct ChainArgs {
  int nchains;
  const int32_t* __restrict__ poly;
  const int32_t* __restrict__ npoly;
  const int32_t* __restrict__ nstates;
  const uint32_t* __restrict__ hvar;
  const float4* __restrict__ em;
  const float2* __restrict__ tr;
  const uint8_t* __restrict__ fl;
  const int64_t* __restrict__ store_off;
  float* __restrict__ store_pool;
  WarpScratch sc;
  int L, WB, Kp, Ks;
  ModelConst mc;
  float* __restrict__ hp;
  const int32_t* __restrict__ order;  // [n] haplotype of chain pair c (longest first), or null for the identity
};

// Hvar words of this lane's states (state index kb + 128 W j + c) of one block
// row, into dst[32 j] (dst already offset by the lane); padded states skipped.
template <int J, int W>
__device__ __forceinline__ void fetch_words(uint4* dst, const uint32_t* row, int kb) {
#pragma unroll
  for (int j = 0; j < J; ++j) {
    uint32_t* d = reinterpret_cast<uint32_t*>(dst + 32 * j);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int k = kb + 128 * W * j + c;
      if (k >= 0) cp_async4(d + c, row + k);
    }
  }
}

// This lane's vectors of a stored row (padded coordinates; quad j at vector
// offset 32 W j from the lane's quad 0) into dst[32 j].
template <int J, int W>
__device__ __forceinline__ void fetch_row(float4* dst, const float4* rowl, uint32_t qmask) {
#pragma unroll
  for (int j = 0; j < J; ++j)
    if ((qmask >> j) & 1u) cp_async16(dst + 32 * j, rowl + 32 * W * j);
}

template <int J, int W, bool FWD, bool POST>
__device__ __forceinline__ void run_chain(const ChainArgs& A, char* smem, float4* xch, int t, int wi, int lane,
                                          int bar_id) {
  const int np = A.npoly[t];
  const int K = A.nstates[t];
  const int M = A.sc.split[t];
  if (np == 0 || K == 0) return;
  const int lo = (FWD == POST) ? M : 0;   // phase 1: forward [0, M), backward [M, np)
  const int hi = (FWD == POST) ? np : M;  // phase 2: forward [M, np), backward [0, M)
  if (lo >= hi) return;
  const int Kp = A.Kp, Ks = A.Ks;
  const int pad = 128 * W * J - K;    // every chain is padded in front to the launch's 128 W J states
  const int pb = 128 * wi + 4 * lane;  // padded index of this lane's quad 0
  const int kb = pb - pad;             // its state index
  float4 vf[J];                        // 1 for a state, 0 for padding
  uint32_t qmask = 0u;                 // bit j: quad j holds at least one state (is stored and fetched)
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int q = pb + 128 * W * j;
    vf[j] = make_float4(q >= pad ? 1.f : 0.f, q + 1 >= pad ? 1.f : 0.f, q + 2 >= pad ? 1.f : 0.f,
                        q + 3 >= pad ? 1.f : 0.f);
    if (q + 3 >= pad) qmask |= 1u << j;
  }
  WarpSmem S = carve(smem, J);
  float* store = A.store_pool + A.store_off[t];
  const uint32_t* hv = A.hvar + (size_t)t * A.WB * Kp;
  const float4* E = A.em + (size_t)t * A.L;
  const float2* T = A.tr + (size_t)t * A.L;
  const uint8_t* F = A.fl + (size_t)t * A.L;
  float* HP = A.hp + (size_t)t * 2 * A.L;
  const int32_t* PL = A.poly + (size_t)t * A.L;
  const int n = hi - lo;
  const float Kf = (float)K;
  auto site_of = [&](int s) { return FWD ? lo + s : hi - 1 - s; };
  auto row_vec = [&](int l) { return reinterpret_cast<float4*>(store + (size_t)l * Ks + pb); };
  constexpr int dir = FWD ? 1 : -1;
  uint4* wl = S.words + lane;   // this lane's words; block buffer (b & 1) at offset 32 J (b & 1)
  float4* rl = S.ring + lane;   // this lane's staged row vectors; slot s at offset 32 J s

  // Ring entries of fully padded quads are never fetched; they hold 0.
  if (POST) {
#pragma unroll
    for (int d = 0; d < kRing; ++d)
#pragma unroll
      for (int j = 0; j < J; ++j)
        if (!((qmask >> j) & 1u)) rl[(d * J + j) * 32] = make_float4(0.f, 0.f, 0.f, 0.f);
  }

  // ---- prologue: records and Hvar words of the first two blocks, first rows ----
  const int b_first = site_of(0) >> 5;
  const int b_last = site_of(n - 1) >> 5;
  {
    const int l = (b_first << 5) + lane;
    if (l < np) {
      S.em[(b_first & 1) * 32 + lane] = E[l];
      S.tr[(b_first & 1) * 32 + lane] = T[l];
      S.fl[(b_first & 1) * 32 + lane] = F[l];
      S.pl[(b_first & 1) * 32 + lane] = PL[l];
    }
    fetch_words<J, W>(wl + (b_first & 1) * 32 * J, hv + (size_t)b_first * Kp, kb);
    if (b_first != b_last) {
      const int b2 = b_first + dir;
      fetch_words<J, W>(wl + (b2 & 1) * 32 * J, hv + (size_t)b2 * Kp, kb);
    }
  }
  cp_commit();
  if (POST) {
#pragma unroll
    for (int d = 0; d < kRowDepth; ++d) {
      if (d < n) fetch_row<J, W>(rl + (d % kRing) * 32 * J, row_vec(site_of(d)), qmask);
      cp_commit();
    }
  }

  float4 x[J];  // alpha (forward) or Beta (backward)
  uint4 w[J];   // Hvar words of the current block
#pragma unroll
  for (int j = 0; j < J; ++j) {
    x[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    w[j] = make_uint4(0u, 0u, 0u, 0u);
  }
  float acc = 0.f;  // AlphaSum / betaSum of the previous step
  float2 t_prev = make_float2(0.f, 0.f);
  if (FWD && lo > 0) {
    const float4* r = row_vec(lo - 1);
#pragma unroll
    for (int j = 0; j < J; ++j)
      if ((qmask >> j) & 1u) x[j] = r[32 * W * j];
    acc = A.sc.asum[t];
    t_prev = T[lo - 1];
  }
  if (!FWD && hi < np) {
    const float4* r = reinterpret_cast<const float4*>(A.sc.brow + (size_t)t * Ks + pb);
#pragma unroll
    for (int j = 0; j < J; ++j)
      x[j] = r[32 * W * j];
    acc = A.sc.bsum[t];
  }
  float4 pe = make_float4(0.f, 0.f, 0.f, 0.f);
  float2 pt = make_float2(0.f, 0.f);
  uint8_t pf = 0;
  int32_t pp = 0;
  if (b_first != b_last) {
    const int ln = ((b_first + dir) << 5) + lane;
    if (ln < np) { pe = E[ln]; pt = T[ln]; pf = F[ln]; pp = PL[ln]; }
  }
  int cur_block = b_first;
  if (!POST) cp_wait<0>();  // words of the first block (phase 2 waits per site below)

  auto step = [&](int s, auto init_tag) {
    constexpr bool INIT = decltype(init_tag)::value;
    const int l = site_of(s);
    const int b = l >> 5;
    const int i = l & 31;
    const bool new_block = INIT || (s == 0) || (b != cur_block);
    if (b != cur_block) {
      S.em[(b & 1) * 32 + lane] = pe;
      S.tr[(b & 1) * 32 + lane] = pt;
      S.fl[(b & 1) * 32 + lane] = pf;
      S.pl[(b & 1) * 32 + lane] = pp;
      cur_block = b;
      if (b != b_last) {
        const int bn = b + dir;
        const int ln = (bn << 5) + lane;
        if (ln < np) { pe = E[ln]; pt = T[ln]; pf = F[ln]; pp = PL[ln]; }
        fetch_words<J, W>(wl + (bn & 1) * 32 * J, hv + (size_t)bn * Kp, kb);
      }
      if (!POST) {
        cp_commit();
        cp_wait<1>();  // this block's words; the next block's may still be in flight
      }
    }
    if (POST) {
      if (s + kRowDepth < n)
        fetch_row<J, W>(rl + ((s + kRowDepth) % kRing) * 32 * J, row_vec(site_of(s + kRowDepth)), qmask);
      cp_commit();
      cp_wait<kRowDepth>();
    }
    __syncwarp();
    if (new_block) {
      const uint4* wb = wl + (b & 1) * 32 * J;
#pragma unroll
      for (int j = 0; j < J; ++j)
        w[j] = wb[32 * j];
    }
    const uint32_t m = 1u << i;
    const uint8_t f = S.fl[(b & 1) * 32 + i];
    const float4 e = S.em[(b & 1) * 32 + i];
    const float4* rowl = rl + (s % kRing) * 32 * J;
    float4* srowl = row_vec(l);
    float q0[4] = {0.f, 0.f, 0.f, 0.f}, q1[4] = {0.f, 0.f, 0.f, 0.f}, q2[4] = {0.f, 0.f, 0.f, 0.f};
    float fact1, fact2;
    if (INIT) {
      fact1 = 1.0f / Kf;
      fact2 = 0.f;
    } else if (FWD) {
      fact1 = t_prev.x;  // t / K of the previous site
      fact2 = t_prev.y / acc;
    } else {
      const float2 tt = S.tr[(b & 1) * 32 + i];
      fact1 = tt.x;
      fact2 = tt.y / acc;
    }
    const float ex = f ? 1.0f : e.x, ey = f ? 1.0f : e.y;
    chain_step<J, W, FWD, POST, INIT>(x, w, m, q0, q1, q2, vf, qmask, fact1, fact2, ex, ey, rowl, srowl);
    const float v0 = warp_sum(__fadd_rn(__fadd_rn(q0[0], q0[1]), __fadd_rn(q0[2], q0[3])));
    float v1 = 0.f, v2 = 0.f;
    if (POST) {
      v1 = warp_sum(__fadd_rn(__fadd_rn(q1[0], q1[1]), __fadd_rn(q1[2], q1[3])));
      v2 = warp_sum(__fadd_rn(__fadd_rn(q2[0], q2[1]), __fadd_rn(q2[2], q2[3])));
    }
    const float3 tot = chain_sum<W>(v0, v1, v2, xch, s & 1, wi, lane, bar_id);
    // AlphaSum = 1 at a flat first site, betaSum = 1 at a flat last site (imputation_hmm.cpp:156,285)
    acc = (INIT && f) ? 1.0f : tot.x;
    if (FWD) t_prev = S.tr[(b & 1) * 32 + i];
    // prob_hid of the two alleles; k_impute_finish turns them into HP
    if (POST && wi == 0 && lane == 0)
      *reinterpret_cast<float2*>(HP + 2 * S.pl[(b & 1) * 32 + i]) = make_float2(tot.y, tot.z);
    __syncwarp();
  };

  // The recursion starts at site 0 (forward) or np - 1 (backward) with 1/K.
  const bool starts = FWD ? (lo == 0) : (hi == np);
  int s0 = 0;
  if (starts) {
    step(0, std::integral_constant<bool, true>());
    s0 = 1;
  }
  for (int s = s0; s < n; ++s) step(s, std::integral_constant<bool, false>());

  cp_wait<0>();
  if (!POST) {
    if (FWD) {
      if (wi == 0 && lane == 0) A.sc.asum[t] = acc;
    } else {
      float4* r = reinterpret_cast<float4*>(A.sc.brow + (size_t)t * Ks + pb);
#pragma unroll
      for (int j = 0; j < J; ++j)
        r[32 * W * j] = x[j];
      if (wi == 0 && lane == 0) A.sc.bsum[t] = acc;
    }
  }
}

// Chain c = blockIdx.x * (chains per CTA) + (warp / W) is run by the W warps
// (warp % W = 0..W-1) of its slot: haplotype order[c / 2] (c / 2 without an
// order), forward for even chains and backward for odd ones. Every warp of a chain takes the same branches, so the
// chain's named barrier (id 1 + slot) always sees all 32 W threads.
template <int J, int W, bool POST>
__global__ void __launch_bounds__(32 * W * kMaxChainsPerCta) k_impute_warp(ChainArgs A) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ float4 xch[kMaxChainsPerCta][2 * W];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int slot = warp / W, wi = warp % W;
  const int chain = blockIdx.x * (int)(blockDim.x / (32 * W)) + slot;
  if (chain >= A.nchains) return;
  char* smem = smem_raw + (size_t)warp * warp_smem_bytes(J);
  const int t = A.order ? A.order[chain >> 1] : chain >> 1;
  if ((chain & 1) == 0) run_chain<J, W, true, POST>(A, smem, xch[slot], t, wi, lane, 1 + slot);
  else run_chain<J, W, false, POST>(A, smem, xch[slot], t, wi, lane, 1 + slot);
}

}  // namespace

size_t impute_warp_smem(int J, int cpc) { return (size_t)kWarpsPerChain * cpc * warp_smem_bytes(J); }

// Local quads per warp for at most Kmax states (the J of launch_impute_warp).
int impute_groups(int Kmax) {
  const int W = kWarpsPerChain;
  return std::max(1, ((Kmax + 127) / 128 + W - 1) / W);
}

// Row stride of the store in padded coordinates for at most Kmax states.
int impute_store_stride(int Kmax) { return 128 * kWarpsPerChain * impute_groups(Kmax); }

template <int J, bool POST>
static int launch_chains(const ChainArgs& a, int cpc, cudaStream_t s) {
  constexpr int W = kWarpsPerChain;
  if (cpc < 1 || cpc > kMaxChainsPerCta) return GP_E_ARG;
  const size_t sm = impute_warp_smem(J, cpc);
  if (sm > 200 * 1024) return GP_E_ARG;
  if (set_smem_limit_once<k_impute_warp<J, W, POST>>(200 * 1024) != cudaSuccess)
    return GP_E_CUDA;
  const dim3 g((a.nchains + cpc - 1) / cpc);
  k_impute_warp<J, W, POST><<<g, 32 * W * cpc, sm, s>>>(a);
  return GP_OK;
}

int launch_impute_warp(int phase, int J, const ModelConst& mc, ImputeWork& w, float* hp, cudaStream_t s, int first,
                       int count, int cpc) {
  ChainArgs a;
  a.sc.asum = w.split_scr.as<float>();
  a.sc.bsum = a.sc.asum + w.n;
  a.sc.brow = a.sc.asum + ((2 * w.n + 3) & ~3);  // 16-byte aligned rows of Ks floats
  a.sc.split = w.split.as<int32_t>();
  if (count < 0) count = w.n;
  if (first < 0 || first + count > w.n || (first > 0 && !w.order.ptr)) return GP_E_ARG;
  if (count == 0) return GP_OK;
  a.nchains = 2 * count;
  a.poly = w.poly.as<int32_t>();
  a.npoly = w.npoly.as<int32_t>();
  a.nstates = w.nstates.as<int32_t>();
  a.hvar = w.hvar.as<uint32_t>();
  a.em = w.em.as<float4>();
  a.tr = w.tr.as<float2>();
  a.fl = w.fl.as<uint8_t>();
  a.store_off = w.alpha_off.as<int64_t>();
  a.store_pool = w.alpha.as<float>();
  a.L = w.L;
  a.WB = w.WB;
  a.Kp = w.Kp;
  a.Ks = w.Ks;
  a.mc = mc;
  a.hp = hp;
  a.order = w.order.ptr ? w.order.as<int32_t>() + first : nullptr;
#define GP_WARP(JJ) \
  case JJ: return phase == 2 ? launch_chains<JJ, true>(a, cpc, s) : launch_chains<JJ, false>(a, cpc, s);
  switch (J) {
    GP_WARP(1) GP_WARP(2) GP_WARP(3) GP_WARP(4) GP_WARP(5) GP_WARP(6) GP_WARP(7) GP_WARP(8)
    GP_WARP(9) GP_WARP(10) GP_WARP(11) GP_WARP(12) GP_WARP(13) GP_WARP(14) GP_WARP(15) GP_WARP(16)
    default: return GP_E_ARG;
  }
#undef GP_WARP
}

}  // namespace gp
