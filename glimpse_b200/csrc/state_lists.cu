// Conditioning states given by the caller (the reference's --state-list):
// per target haplotype, reference haplotypes that every conditioning set of
// its target holds whatever the selection picks.
//
// conditioning_set::compactSelection (conditioning_set.cpp:114-121) appends the
// list rows of the target's haplotypes to the selected states and sorts them
// without duplicates, for every set but the whole panel's (Kpbwt >=
// n_ref_haps, conditioning_set.cpp:105-113). Here the rows of each target are
// merged once on the host into one sorted list without duplicates (the union
// the reference forms per call); after each stage's selection, k_merge_lists
// forms selection ∪ list per target in one CTA: both into shared memory, a
// bitonic sort, and a ballot compaction of the first of every run of equal ids.
#include <algorithm>
#include <string>

#include "context.h"

namespace gp {
namespace {

constexpr int kMergeThreads = 256;

__global__ void __launch_bounds__(kMergeThreads)
    k_merge_lists(const uint32_t* __restrict__ in, int Kin, const int32_t* nin,
                  const int64_t* __restrict__ loff, const int32_t* __restrict__ lids, uint32_t* __restrict__ out,
                  int Kout, int32_t* nout) {
  __shared__ uint32_t v[kMaxStates];
  __shared__ int wsum[kMergeThreads / 32];
  const int t = blockIdx.x, tid = threadIdx.x;
  const int na = nin[t];
  const int64_t l0 = loff[t];
  const int nb = (int)(loff[t + 1] - l0);
  const int m = na + nb;  // <= Kout <= kMaxStates (checked on the host)
  int S = 32;
  while (S < m) S <<= 1;
  for (int i = tid; i < S; i += kMergeThreads)
    v[i] = i < na ? in[(size_t)t * Kin + i] : i < m ? (uint32_t)lids[l0 + (i - na)] : 0xFFFFFFFFu;
  __syncthreads();
  for (int k = 2; k <= S; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < S; i += kMergeThreads) {
        const int p = i ^ j;
        if (p > i) {
          const uint32_t a = v[i], b = v[p];
          if ((a > b) == ((i & k) == 0)) {
            v[i] = b;
            v[p] = a;
          }
        }
      }
      __syncthreads();
    }
  const int lane = tid & 31, wid = tid >> 5;
  int base = 0;
  for (int c = 0; c < m; c += kMergeThreads) {
    const int i = c + tid;
    const uint32_t x = i < m ? v[i] : 0u;
    const bool keep = i < m && (i == 0 || v[i - 1] != x);
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < kMergeThreads / 32; ++q) {
      off += q < wid ? wsum[q] : 0;
      tot += wsum[q];
    }
    if (keep) out[(size_t)t * Kout + base + off + __popc(bal & ((1u << lane) - 1u))] = x;
    base += tot;
    __syncthreads();
  }
  if (tid == 0) nout[t] = base;
}

}  // namespace

// haplotype_set::read_list_states (haplotype_set.cpp:835-857), then the union of
// each target's rows (conditioning_set.cpp:116-119) formed once.
int Context::set_state_lists(int n_haps, const int64_t* off, const int32_t* ids) {
  TargetWork& T = tw;
  if (n_haps == 0) {
    list_len.clear();
    return GP_OK;
  }
  if (T.n <= 0) return (fail(GP_E_STATE, "state lists: no targets"), GP_E_STATE);
  int nh = 0;
  for (int i = 0; i < T.n; ++i) nh += T.ploidy_h[i];
  if (n_haps != nh || !off || !ids || off[0] != 0)
    return (fail(GP_E_ARG, "state lists: expected " + std::to_string(nh) + " rows, one per target haplotype"),
            GP_E_ARG);
  const int N = panel.N;
  for (int h = 0; h < n_haps; ++h) {
    if (off[h + 1] <= off[h])
      return (fail(GP_E_ARG, "List of states for haplotype " + std::to_string(h) + " is empty."), GP_E_ARG);
    for (int64_t j = off[h]; j < off[h + 1]; ++j)
      if (ids[j] < 0 || ids[j] >= N)
        return (fail(GP_E_ARG, "State given for haplotype " + std::to_string(h) +
                                   " has an impossible value: " + std::to_string(ids[j])),
                GP_E_ARG);
  }
  std::vector<int64_t> loff(T.n + 1, 0);
  std::vector<int32_t> lids;
  std::vector<int32_t> len(T.n);
  int h = 0;
  for (int i = 0; i < T.n; ++i) {
    const size_t s0 = lids.size();
    for (int j = 0; j < T.ploidy_h[i]; ++j, ++h) lids.insert(lids.end(), ids + off[h], ids + off[h + 1]);
    std::sort(lids.begin() + s0, lids.end());
    lids.erase(std::unique(lids.begin() + s0, lids.end()), lids.end());
    len[i] = (int32_t)(lids.size() - s0);
    loff[i + 1] = (int64_t)lids.size();
  }
  cudaError_t e;
  if ((e = list_off.ensure(loff.size() * 8)) != cudaSuccess) return cuda_fail(e, "alloc state lists");
  if ((e = list_ids.ensure(lids.size() * 4)) != cudaSuccess) return cuda_fail(e, "alloc state lists");
  cudaMemcpyAsync(list_off.ptr, loff.data(), loff.size() * 8, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(list_ids.ptr, lids.data(), lids.size() * 4, cudaMemcpyHostToDevice, stream);
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "state lists upload");
  list_len = std::move(len);
  return GP_OK;
}

// Selected states (stride Kp) ∪ each target's list into a stride of Kp plus
// the longest list; the states buffer and Kp are replaced by the merged ones.
int Context::merge_state_lists(int& Kp) {
  ImputeWork& w = impute;
  const int n = tw.n;
  const int lmax = *std::max_element(list_len.begin(), list_len.end());
  const int Kout = (Kp + lmax + 31) / 32 * 32;
  if (Kout > kMaxStates)
    return (fail(GP_E_ARG, "conditioning states plus state list exceed " + std::to_string(kMaxStates) +
                               " per target"),
            GP_E_ARG);
  cudaError_t e;
  if ((e = merged_states.ensure((size_t)n * Kout * 4)) != cudaSuccess) return cuda_fail(e, "alloc states");
  k_merge_lists<<<n, kMergeThreads, 0, stream>>>(w.states.as<uint32_t>(), Kp, w.nstates.as<int32_t>(),
                                                 list_off.as<int64_t>(), list_ids.as<int32_t>(),
                                                 merged_states.as<uint32_t>(), Kout, w.nstates.as<int32_t>());
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "state list merge launch");
  prof.kernel_launches += 1;
  std::swap(w.states, merged_states);
  Kp = Kout;
  return GP_OK;
}

}  // namespace gp

extern "C" int gp_state_lists_set(gp_ctx* ctx, int32_t n_haps, const int64_t* offsets, const int32_t* ids) {
  if (!ctx) return GP_E_ARG;
  gp::Context& c = *reinterpret_cast<gp::Context*>(ctx);
  if (n_haps < 0) return (c.fail(GP_E_ARG, "state lists: negative row count"), GP_E_ARG);
  return c.set_state_lists(n_haps, offsets, ids);
}
