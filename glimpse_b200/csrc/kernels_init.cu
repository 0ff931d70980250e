// Init-stage state selection: haplotype_set::initRareTar (haplotype_set.cpp:108-169)
// and haplotype_set::performSelection_RARE_INIT_GL (haplotype_set.cpp:775-833).
//
// The reference draws with std::sample over its engine. libstdc++ implements
// std::sample for forward iterators as selection sampling (Knuth, TAOCP vol. 2,
// Algorithm S), drawing two positions per engine call when the population is
// small enough (population^2 <= 2^32 - 1), and bounds each draw with Lemire's
// method; k_init_select restates that procedure on the target's stream
// (RNG_INIT_SEL, iteration, target) so that both sides pick the same states.
#include <cub/block/block_scan.cuh>

#include "genotype.h"

namespace gp {

__constant__ float c_unphred_init[256];

namespace {

// Rare non-reference calls from the GLs, in site order.
template <int THREADS, int ITEMS>
__global__ void k_init_rare_tar(InitSelArgs a) {
  typedef cub::BlockScan<int, THREADS> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int carry;
  const int t = blockIdx.x;
  const int L = a.L;
  const int pl = a.ploidy[t];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < L; base += THREADS * ITEMS) {
    int v[ITEMS], ex[ITEMS], tot;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int s = base + threadIdx.x * ITEMS + i;
      v[i] = 0;
      if (s >= L) continue;
      const size_t ts = (size_t)t * L + s;
      if (a.flat[ts] || a.common[s] || a.lq[s]) continue;
      const uint8_t* g = a.gl + ts * 3;
      const int mg = 2 * a.major[s];
      if (!(g[1] <= g[mg] || g[2 - mg] <= g[mg])) continue;
      float t0 = c_unphred_init[g[0]], t1 = c_unphred_init[g[1]], t2 = pl > 1 ? c_unphred_init[g[2]] : 0.0f;
      float sum = __fadd_rn(__fadd_rn(t0, t1), t2);
      t0 = t0 / sum; t1 = t1 / sum; t2 = t2 / sum;
      const float af = (float)((double)a.calt[s] * 1.0 / (double)a.N);
      const float q = __fsub_rn(1.0f, af);
      t0 = __fmul_rn(t0, __fmul_rn(q, q));
      t1 = __fmul_rn(t1, __fmul_rn(__fmul_rn(2.0f, af), q));
      t2 = __fmul_rn(t2, __fmul_rn(af, af));
      sum = __fadd_rn(__fadd_rn(t0, t1), t2);
      t0 = t0 / sum; t1 = t1 / sum; t2 = t2 / sum;
      const float tt[3] = {t0, t1, t2};
      if (__fadd_rn(tt[1], tt[2 - mg]) > tt[mg]) v[i] = 1;
    }
    Scan(tmp).ExclusiveSum(v, ex, tot);
    const int c = carry;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
      if (v[i]) a.sind[(size_t)t * L + c + ex[i]] = base + threadIdx.x * ITEMS + i;
    __syncthreads();
    if (threadIdx.x == 0) carry = c + tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.nsind[t] = carry;
}

struct SetBits {
  uint32_t* bm;
  int count;
  __device__ bool insert(uint32_t h) {
    const uint32_t m = 1u << (h & 31);
    uint32_t& w = bm[h >> 5];
    if (w & m) return false;
    w |= m;
    ++count;
    return true;
  }
};

// uniform_int_distribution<long>{0, b} over a 32-bit engine (b < 2^32 - 1 here).
__device__ __forceinline__ uint64_t uniform_upto(StreamCursor& g, uint64_t b) {
  if (b == 0xFFFFFFFFull) return g();
  return bounded_u32(g, (uint32_t)(b + 1));
}

// std::sample(first, first + P, out, n, g) for a forward range: calls emit(i)
// for each selected position i in increasing order.
template <class Emit>
__device__ void std_sample(StreamCursor& g, int64_t P, int64_t n, Emit&& emit) {
  if (P <= 0) return;
  int64_t unsampled = P;
  if (n > unsampled) n = unsampled;
  int64_t idx = 0;
  if ((0xFFFFFFFFull / (uint64_t)unsampled) >= (uint64_t)unsampled) {
    while (n != 0 && unsampled >= 2) {
      const uint64_t b0 = (uint64_t)unsampled, b1 = (uint64_t)unsampled - 1;
      const uint64_t x = uniform_upto(g, b0 * b1 - 1);
      const uint64_t p1 = x / b1, p2 = x % b1;
      --unsampled;
      if ((int64_t)p1 < n) { emit(idx); --n; }
      ++idx;
      if (n == 0) break;
      --unsampled;
      if ((int64_t)p2 < n) { emit(idx); --n; }
      ++idx;
    }
  }
  for (; n != 0; ++idx) {
    --unsampled;
    if ((int64_t)uniform_upto(g, (uint64_t)unsampled) < n) { emit(idx); --n; }
  }
}

// One thread per target.
__global__ void k_init_select(InitSelArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const int W = (a.N + 31) / 32;
  SetBits set{a.bitmap + (size_t)t * W, 0};
  for (int i = 0; i < W; ++i) set.bm[i] = 0u;
  StreamCursor g(a.seed, RNG_INIT_SEL, (uint32_t)a.iteration, (uint32_t)t);
  const int k_init = a.kinit;
  const int k_init8 = (int)floorf(__fmul_rn((float)k_init, 0.8f));
  const int ns = a.nsind[t];
  const int32_t* S = a.sind + (size_t)t * a.L;
  if (ns > 0) {
    if (ns > k_init8) {
      // ascending (MAC, site) order, MAC = min(cref, calt) (variant.cpp:45-47)
      bool done = false;
      for (int mac = 0; mac <= a.max_mac && !done; ++mac) {
        for (int r = 0; r < ns; ++r) {
          if (set.count >= k_init8) { done = true; break; }
          const int v = S[r];
          const int m = (int)min(a.cref[v], a.calt[v]);
          if (m != mac) continue;
          const int64_t o = a.svar_off[v], sz = a.svar_off[v + 1] - o;
          int picked[5];
          int np = 0;
          std_sample(g, sz, 5, [&](int64_t i) { picked[np++] = (int)i; });
          for (int i = 0; i < np && set.count < k_init8; ++i) set.insert((uint32_t)a.svar_haps[o + picked[i]]);
        }
      }
    } else {
      const int size_max = max((int)floor((double)k_init8 * 1.0 / (double)ns), 1);
      for (int r = 0; r < ns; ++r) {
        const int v = S[r];
        const int64_t o = a.svar_off[v], sz = a.svar_off[v + 1] - o;
        std_sample(g, sz, size_max, [&](int64_t i) {
          if (set.count < k_init8) set.insert((uint32_t)a.svar_haps[o + i]);
        });
      }
    }
  }
  if (set.count < k_init) {
    std_sample(g, a.N, k_init, [&](int64_t i) {
      if (set.count < k_init) set.insert((uint32_t)i);
    });
  }
  // std::set iteration order: ascending haplotype ids
  int k = 0;
  for (int i = 0; i < W; ++i) {
    uint32_t w = set.bm[i];
    while (w) {
      const int b = __ffs(w) - 1;
      w &= w - 1;
      if (k < a.Kp) a.states[(size_t)t * a.Kp + k] = (uint32_t)(i * 32 + b);
      ++k;
    }
  }
  a.nstates[t] = k;
}

}  // namespace

cudaError_t upload_unphred_init(const float* table) {
  return cudaMemcpyToSymbol(c_unphred_init, table, 256 * sizeof(float));
}

void launch_init_select(const InitSelArgs& a, cudaStream_t s) {
  k_init_rare_tar<512, 8><<<a.n, 512, 0, s>>>(a);
  k_init_select<<<(a.n + 31) / 32, 32, 0, s>>>(a);
}

}  // namespace gp
