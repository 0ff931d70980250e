// Imputation HMM forward-backward with one warp per chain.
//
// The haploid Li-Stephens recursion (phase/src/models/imputation_hmm.cpp:143-416)
// is sequential over sites with a sum over all K states at every site. Here a
// single warp runs one chain: lane `lane` owns states k = lane + 32 j (j < J),
// the per-site sums are warp butterflies (no block barrier), and all memory
// traffic is streamed ahead of the chain:
//   * Hvar words of the next 32-site block and the stored rows of the next D
//     sites go through a per-warp shared-memory ring filled by cp.async;
//   * per-site records (emissions, transitions, flags) of the next block are
//     loaded by the lanes one block ahead.
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
// Sums follow a fixed order (lane-sequential over j, then a lane butterfly), so
// results are deterministic. Every fused multiply-add is an explicit fmaf where
// the reference's compiled arithmetic has one (build with --fmad=false).
#include <type_traits>

#include "internal.h"

namespace gp {

namespace {

constexpr int kWarpsPerCta = 2;
constexpr int kRowDepth = 3;              // stored rows fetched this many sites ahead
constexpr int kRing = kRowDepth + 1;      // ring slots

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Copy Kp 4-byte values (Kp a multiple of 32, at most 32 * J, 16-byte aligned)
// into shared memory: 16-byte chunk lane + 32 c for c < J / 4.
template <int J>
__device__ __forceinline__ void copy_row_async(void* dst, const void* src, int Kp, int lane) {
  const int chunks = Kp >> 2;
  const char* s = static_cast<const char*>(src) + 16 * lane;
  char* d = static_cast<char*>(dst) + 16 * lane;
#pragma unroll
  for (int c = 0; c < J / 4; ++c)
    if (lane + 32 * c < chunks) cp_async16(d + 512 * c, s + 512 * c);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

struct WarpScratch {
  float* asum;          // [n] AlphaSum at site M-1
  float* bsum;          // [n] betaSum at site M
  float* brow;          // [n][Kp] Beta at site M
  const int32_t* split; // [n] M
};

// Per-warp shared memory: records (2 blocks), Hvar words (2 blocks), row ring.
struct WarpSmem {
  float4* em;     // [2][32]
  float2* tr;     // [2][32]
  int32_t* pl;    // [2][32] site of the poly index
  uint8_t* fl;    // [2][32]
  uint32_t* words;  // [2][Kp]
  float* ring;    // [kRing][Kp]
};

__device__ __forceinline__ WarpSmem carve(char* base, int Kp) {
  WarpSmem m;
  m.em = reinterpret_cast<float4*>(base);
  m.tr = reinterpret_cast<float2*>(base + 2 * 32 * 16);
  m.words = reinterpret_cast<uint32_t*>(base + 2 * 32 * 16 + 2 * 32 * 8);
  m.ring = reinterpret_cast<float*>(base + 2 * 32 * 16 + 2 * 32 * 8 + 2 * (size_t)Kp * 4);
  m.pl = reinterpret_cast<int32_t*>(base + 2 * 32 * 16 + 2 * 32 * 8 + 2 * (size_t)Kp * 4 +
                                    (size_t)kRing * Kp * 4);
  m.fl = reinterpret_cast<uint8_t*>(base + 2 * 32 * 16 + 2 * 32 * 8 + 2 * (size_t)Kp * 4 +
                                    (size_t)kRing * Kp * 4 + 2 * 32 * 4);
  return m;
}

__host__ __device__ __forceinline__ size_t warp_smem_bytes(int Kp) {
  return 2 * 32 * 16 + 2 * 32 * 8 + 2 * (size_t)Kp * 4 + (size_t)kRing * Kp * 4 + 2 * 32 * 4 + 2 * 32 + 64;
}

// One site of a chain for the owned states, specialised at compile time:
//   FWD   forward (alpha) or backward (Beta) recursion
//   POST  phase 2: form prob_hid from the stored row instead of storing a row
//   INIT  first forward / last backward site: the pre-emission value is 1/K
// Flat or low-quality sites pass emissions (1, 1): the product by 1.0 is exact,
// so the same loop serves both kinds of site.
// At the last site the forward posterior uses alpha alone and the stored
// prob_curr is 1 there, so alpha x 1 is used unchanged (imputation_hmm.cpp:337-368).
// m selects the current site's bit in the Hvar words; rowl / srowl point at this
// lane's state of group 0 in the staged row (shared) and in the stored row
// (global), so group j is at offset 32 j. Padded lanes of groups 0..3 never
// dereference them.
template <int J, bool FWD, bool POST, bool INIT>
__device__ __forceinline__ void chain_step(float (&x)[J], const uint32_t (&w)[J], uint32_t m, float (&q0)[4],
                                           float (&q1)[4], float (&q2)[4], const bool (&vg)[4], int jn, float fact1,
                                           float fact2, float ex, float ey, const float* rowl, float* srowl) {
#pragma unroll
  for (int j0 = 0; j0 < J; j0 += 4) {
    if (j0 >= jn) break;  // jn is the same on every lane
    {
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int j = j0 + jj;
        const bool valid = j >= 4 || vg[jj];
        const bool bit = (w[j] & m) != 0u;
        const float pcv = INIT ? fact1 : fmaf(x[j], fact2, fact1);
        float nx = __fmul_rn(pcv, bit ? ey : ex);
        if (j < 4) nx = valid ? nx : 0.f;
        x[j] = nx;
        q0[jj] = __fadd_rn(q0[jj], nx);
        if (POST) {
          float r = 0.f;
          if (valid) r = rowl[32 * j];
          float d;
          if (FWD) d = __fmul_rn(nx, r);           // alpha x stored prob_curr (1 at the last site)
          else d = INIT ? r : __fmul_rn(r, pcv);  // stored alpha x prob_curr; alpha alone at the last site
          if (bit) q2[jj] = __fadd_rn(q2[jj], d);
          else q1[jj] = __fadd_rn(q1[jj], d);
        } else if (valid) {
          srowl[32 * j] = FWD ? nx : (INIT ? 1.0f : pcv);
        }
      }
    }
  }
}

// State layout inside a chain: the K states are padded to 32 * jn states with
// jn a multiple of 4, and the padding is put in front: lane `lane` of group j
// holds state k = 32 j + lane - pad (pad = 32 jn - K < 128). Only groups 0..3
// contain padding, so only they carry validity masks; padded states are kept at
// exactly 0 and therefore add nothing to any sum. Groups are processed in
// chunks of 4 behind one warp-uniform branch, so a chain's work follows its own K.
//
// Site bits: the 32-bit Hvar word of a state covers a 32-site block; it is kept
// shifted so that the current site's bit is the sign bit (bit-reversed for the
// forward direction), which turns the emission choice into a sign test.
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
  int L, WB, Kp;
  ModelConst mc;
  float* __restrict__ hp;
};

// One chain (a haplotype in one direction) over its sites [lo, hi), with the
// direction FWD and the phase (POST = phase 2) fixed at compile time, so the
// per-site loop carries no dispatch. The first site of a chain is peeled when it
// starts the recursion (INIT).
template <int J, bool FWD, bool POST>
__device__ __forceinline__ void run_chain(const ChainArgs& A, char* smem, int t, int lane) {
  const int np = A.npoly[t];
  const int K = A.nstates[t];
  const int M = A.sc.split[t];
  if (np == 0 || K == 0) return;
  const int lo = (FWD == POST) ? M : 0;   // phase 1: forward [0, M), backward [M, np)
  const int hi = (FWD == POST) ? np : M;  // phase 2: forward [M, np), backward [0, M)
  if (lo >= hi) return;
  const int Kp = A.Kp;
  const int jn = (((K + 31) >> 5) + 3) & ~3;  // groups in use, a multiple of 4
  const int pad = 32 * jn - K;
  bool vg[4];                                 // validity of this lane in groups 0..3
#pragma unroll
  for (int j = 0; j < 4; ++j) vg[j] = (32 * j + lane) >= pad;
  const int kb = lane - pad;                  // state index of group 0 for this lane
  WarpSmem S = carve(smem, Kp);
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
  // index of the value owned by (j, lane) in a K-long row; padding reads entry 0
  auto idx = [&](int j) { return max(32 * j + kb, 0); };
  constexpr int dir = FWD ? 1 : -1;

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
    copy_row_async<J>(S.words + (size_t)(b_first & 1) * Kp, hv + (size_t)b_first * Kp, Kp, lane);
    if (b_first != b_last) {
      const int b2 = b_first + dir;
      copy_row_async<J>(S.words + (size_t)(b2 & 1) * Kp, hv + (size_t)b2 * Kp, Kp, lane);
    }
  }
  cp_commit();
  if (POST) {
#pragma unroll
    for (int d = 0; d < kRowDepth; ++d) {
      if (d < n) copy_row_async<J>(S.ring + (size_t)(d % kRing) * Kp, store + (size_t)site_of(d) * Kp, Kp, lane);
      cp_commit();
    }
  }

  float x[J];      // alpha (forward) or Beta (backward)
  uint32_t w[J];   // Hvar words of the current block
#pragma unroll
  for (int j = 0; j < J; ++j) {
    x[j] = 0.f;
    w[j] = 0u;
  }
  float acc = 0.f;  // AlphaSum / betaSum of the previous step
  float2 t_prev = make_float2(0.f, 0.f);
  if (FWD && lo > 0) {
#pragma unroll
    for (int j = 0; j < J; ++j)
      if (j < jn) x[j] = (j >= 4 || vg[j & 3]) ? store[(size_t)(lo - 1) * Kp + idx(j)] : 0.f;
    acc = A.sc.asum[t];
    t_prev = T[lo - 1];
  }
  if (!FWD && hi < np) {
#pragma unroll
    for (int j = 0; j < J; ++j)
      if (j < jn) x[j] = (j >= 4 || vg[j & 3]) ? A.sc.brow[(size_t)t * Kp + idx(j)] : 0.f;
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
        copy_row_async<J>(S.words + (size_t)(bn & 1) * Kp, hv + (size_t)bn * Kp, Kp, lane);
      }
      if (!POST) {
        cp_commit();
        cp_wait<1>();  // this block's words; the next block's may still be in flight
      }
    }
    if (POST) {
      if (s + kRowDepth < n)
        copy_row_async<J>(S.ring + (size_t)((s + kRowDepth) % kRing) * Kp,
                          store + (size_t)site_of(s + kRowDepth) * Kp, Kp, lane);
      cp_commit();
      cp_wait<kRowDepth>();
    }
    __syncwarp();
    if (new_block) {
      const uint32_t* wbl = S.words + (size_t)(b & 1) * Kp + kb;
#pragma unroll
      for (int j = 0; j < J; ++j)
        if (j < jn) w[j] = (j >= 4 || vg[j & 3]) ? wbl[32 * j] : 0u;
    }
    const uint32_t m = 1u << i;
    const uint8_t f = S.fl[(b & 1) * 32 + i];
    const float4 e = S.em[(b & 1) * 32 + i];
    const float* rowl = S.ring + (size_t)(s % kRing) * Kp + kb;
    float* srowl = store + (size_t)l * Kp + kb;
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
    chain_step<J, FWD, POST, INIT>(x, w, m, q0, q1, q2, vg, jn, fact1, fact2, ex, ey, rowl, srowl);
    const float v0 = warp_sum(__fadd_rn(__fadd_rn(q0[0], q0[1]), __fadd_rn(q0[2], q0[3])));
    // AlphaSum = 1 at a flat first site, betaSum = 1 at a flat last site (imputation_hmm.cpp:156,285)
    acc = (INIT && f) ? 1.0f : v0;
    if (FWD) t_prev = S.tr[(b & 1) * 32 + i];
    if (POST) {
      const float v1 = warp_sum(__fadd_rn(__fadd_rn(q1[0], q1[1]), __fadd_rn(q1[2], q1[3])));
      const float v2 = warp_sum(__fadd_rn(__fadd_rn(q2[0], q2[1]), __fadd_rn(q2[2], q2[3])));
      // prob_hid of the two alleles; k_impute_finish turns them into HP
      if (lane == 0) *reinterpret_cast<float2*>(HP + 2 * S.pl[(b & 1) * 32 + i]) = make_float2(v1, v2);
    }
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
      if (lane == 0) A.sc.asum[t] = acc;
    } else {
#pragma unroll
      for (int j = 0; j < J; ++j)
        if (j < jn && (j >= 4 || vg[j & 3])) A.sc.brow[(size_t)t * Kp + idx(j)] = x[j];
      if (lane == 0) A.sc.bsum[t] = acc;
    }
  }
}

// Warp `warp` of the CTA runs chain blockIdx.x * kWarpsPerCta + warp: target
// chain / 2, forward for even chains and backward for odd ones.
template <int J, bool POST>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_impute_warp(ChainArgs A) {
  static_assert(J % 4 == 0, "groups are processed in chunks of 4");
  extern __shared__ __align__(16) char smem_raw[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int chain = blockIdx.x * kWarpsPerCta + warp;
  if (chain >= A.nchains) return;
  char* smem = smem_raw + (size_t)warp * warp_smem_bytes(A.Kp);
  if ((chain & 1) == 0) run_chain<J, true, POST>(A, smem, chain >> 1, lane);
  else run_chain<J, false, POST>(A, smem, chain >> 1, lane);
}

}  // namespace

size_t impute_warp_smem(int Kp) { return (size_t)kWarpsPerCta * warp_smem_bytes(Kp); }

template <int J, bool POST>
static void launch_chains(const ChainArgs& a, dim3 g, size_t sm, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_impute_warp<J, POST>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  k_impute_warp<J, POST><<<g, 32 * kWarpsPerCta, sm, s>>>(a);
}

int launch_impute_warp(int phase, int J, const ModelConst& mc, ImputeWork& w, float* hp, cudaStream_t s) {
  ChainArgs a;
  a.sc.asum = w.split_scr.as<float>();
  a.sc.bsum = a.sc.asum + w.n;
  a.sc.brow = a.sc.bsum + w.n;
  a.sc.split = w.split.as<int32_t>();
  a.nchains = 2 * w.n;
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
  a.mc = mc;
  a.hp = hp;
  const dim3 g((a.nchains + kWarpsPerCta - 1) / kWarpsPerCta);
  const size_t sm = impute_warp_smem(w.Kp);
#define GP_WARP(JJ)                                                           \
  case JJ:                                                                    \
    if (phase == 2) launch_chains<JJ, true>(a, g, sm, s);                     \
    else launch_chains<JJ, false>(a, g, sm, s);                               \
    break;
  switch (J) {
    GP_WARP(8) GP_WARP(16) GP_WARP(24) GP_WARP(32) GP_WARP(40) GP_WARP(48) GP_WARP(56) GP_WARP(64)
    default: return GP_E_ARG;
  }
#undef GP_WARP
  return GP_OK;
}

}  // namespace gp
