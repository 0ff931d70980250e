// Internal declarations shared by the CUDA translation units of libglimpse_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/glimpse_b200.h"
#include "replay_rng.h"

namespace gp {

constexpr int kWarp = 32;

#ifdef __CUDACC__
// Two floats in one 64-bit register pair (lo = first); the packed mul / add /
// fma (sm_100a) round each element exactly as the scalar instructions do.
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2_pack(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
#endif
constexpr int kImputeThreads = 256;           // threads per haplotype in the imputation HMM
constexpr int kImputeStatesPerThread = 8;     // registers per thread for owned states
constexpr int kMaxStates = kImputeThreads * kImputeStatesPerThread;  // 2048
constexpr int kHaps = 8;                      // HAP_NUMBER (phasing_hmm.h:38)

// Status carried out of host helpers.
struct Status {
  int code = GP_OK;
  std::string msg;
};

// A kernel's dynamic shared-memory limit, set once per device (the attribute is
// per device; contexts may sit on different devices). F is the kernel.
template <auto F>
cudaError_t set_smem_limit_once(int bytes) {
  static std::atomic<uint64_t> done{0};  // bit d: set on device d
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (dev < 64 && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(F, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && dev < 64) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

// Host-side fault injection for tests: true when GLIMPSE_B200_FAIL_ALLOC=n is
// set and this is the n-th buffer growth since it was read (the variable is
// re-read whenever its value changes). The growth then reports
// cudaErrorMemoryAllocation without calling cudaMalloc.
bool inject_alloc_failure();

// Growable device buffer (bytes); contents are not preserved on growth.
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    if (inject_alloc_failure()) return cudaErrorMemoryAllocation;
    size_t want = bytes + bytes / 8 + 256;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Panel resident in device memory.
struct DevPanel {
  int N = 0, L = 0, n_com = 0, n_com_hq = 0, W = 0;  // W: 32-bit words per haplotype over common rows
  double* cm = nullptr;
  uint8_t* lq = nullptr;
  uint8_t* common = nullptr;
  uint8_t* major = nullptr;
  uint32_t* cref = nullptr;
  uint32_t* calt = nullptr;
  int32_t* comrow = nullptr;       // site -> common row, -1 for rare
  uint32_t* refT = nullptr;        // [N][W] haplotype-major bits over common rows (bit r%32 of word r/32)
  int64_t* shap_off = nullptr;     // [N+1]
  int32_t* shap_sites = nullptr;   // rare sites carrying the non-major allele, per haplotype
  int64_t shap_nnz = 0;
  int64_t* svar_off = nullptr;     // [L+1] SvarRef CSR
  int32_t* svar_haps = nullptr;
};

// Per-batch scratch for the imputation path (sized for n haplotypes).
struct ImputeWork {
  int n = 0, L = 0, Kp = 0, WB = 0;  // WB: 32-site blocks per haplotype (upper bound)
  int Ks = 0;                         // row stride of the forward-backward store (padded state coordinates)
  DevBuf states, nstates, states_off;
  DevBuf mark, polyidx, poly, npoly;
  DevBuf hvar, em, tr, fl;
  DevBuf alpha, alpha_off, split, split_scr;
  DevBuf order;  // [n] haplotypes in decreasing order of poly sites (chain launch order); ptr null: identity
  DevBuf hl, hp, flat;
};

// Scratch of the phasing HMM.
struct PhaseWork {
  DevBuf rel, code, seg, miss, seg_start, counts, ytp, ytn, vflags, recb, recf;
  DevBuf pool;  // the stored segment-start and flat-het messages of one chunk of entries
  DevBuf offs, pprob_sum, pprob_sumsum, iprob_sum, of1, dip, err, order;
  std::vector<DevBuf*> all() {
    return {&rel, &code, &seg, &miss, &seg_start, &counts, &ytp, &ytn, &vflags, &recb, &recf, &pool, &offs,
            &pprob_sum, &pprob_sumsum, &iprob_sum, &of1, &dip, &err, &order};
  }
};

// Model constants derived from gp_config the way the reference derives them
// (conditioning_set.cpp:27-37, caller_initialise.cpp:150-153).
struct ModelConst {
  float ed_imp, ee_imp, ed_phs, ee_phs, min_gl;
  double nrho, one_l;
};

// Kernel launchers (kernels_impute.cu).
void launch_mark_poly(const DevPanel& P, ImputeWork& w, cudaStream_t s);
void launch_compact_poly(const DevPanel& P, ImputeWork& w, cudaStream_t s);
void launch_build_hvar(const DevPanel& P, ImputeWork& w, cudaStream_t s);
void launch_site_records(const DevPanel& P, const ModelConst& mc, ImputeWork& w, const float* hl,
                         const uint8_t* flat, cudaStream_t s);
// Chains of the haplotypes order[first .. first + count) (count < 0: all n),
// cpc chains per CTA (1, 2 or 4; GP_E_ARG when their shared memory does not fit).
int launch_impute_warp(int phase, int J, const ModelConst& mc, ImputeWork& w, float* hp, cudaStream_t s,
                       int first = 0, int count = -1, int cpc = 2);
// Register groups per lane of the imputation chain kernel for at most Kmax
// states (the J of launch_impute_warp).
int impute_groups(int Kmax);
// Row stride (floats) of the forward-backward store for at most Kmax states; the
// scratch split_scr holds round_up(2 n, 4) + n * stride floats.
int impute_store_stride(int Kmax);
// The checkpointed forward-backward (kernels_impute_ckpt.cu) over the batch's
// conditioning sets: leaves prob_hid pairs in hp for k_impute_finish.
int launch_impute_ckpt(ImputeWork& w, bool bf16, void* ckpt, float* csum, float* scratch, double* loglik, float* hp,
                       cudaStream_t s);
void launch_impute_finish(const DevPanel& P, const ModelConst& mc, ImputeWork& w, const float* hl,
                        const uint8_t* flat, float* hp, cudaStream_t s);

}  // namespace gp
