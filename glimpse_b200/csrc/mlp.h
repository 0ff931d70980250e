// The learned state-selection proposal's network: an MLP that scores candidate
// reference haplotypes for a (target, window) from kMlpIn features,
// kMlpIn -> 256 -> 256 -> 1 with ReLU, BF16 weights and activations, FP32
// accumulation. Forward and backward GEMMs run on the tensor cores
// (tcgen05.mma, accumulators in tensor memory; mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "internal.h"

namespace gp {

constexpr int kMlpIn = 48;    // features per candidate
constexpr int kMlpInP = 64;   // padded to the MMA's K granularity (zero columns)
constexpr int kMlpHid = 256;  // hidden units per layer

// Device-resident network, optimiser state and training scratch.
struct MlpState {
  bool ready = false;
  // parameters: the packed FP32 master vector and the BF16 copies the GEMMs read
  DevBuf param;                       // kMlpParams floats (layout below)
  DevBuf w1, w2, w2t;                 // BF16: w1 [256][64], w2 [256][256], w2t [256][256] (transposed)
  DevBuf m, v;                        // Adam moments over the packed parameter vector
  DevBuf grad;                        // packed FP32 gradient
  DevBuf partial;                     // split-K partial sums of the weight gradients
  DevBuf hpart;                       // per-block partial sums of the small gradients and the loss
  int64_t step = 0;
  // per-batch scratch (rows padded to 128)
  DevBuf x, xt, y, wt, score, h1, h1t, h2, dz2, dz2t, dz1, dz1t, loss, err;
  DevBuf xf;                          // FP32 staging of host feature rows
  int cap_rows = 0;
  std::vector<DevBuf*> all() {
    return {&param, &w1, &w2, &w2t, &m, &v, &grad, &partial, &hpart, &x, &xt, &y, &wt, &score,
            &h1, &h1t, &h2, &dz2, &dz2t, &dz1, &dz1t, &loss, &err, &xf};
  }
};

// Packed parameter vector: w1 | b1 | w2 | b2 | w3 | b3.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHid * kMlpInP;
constexpr int kOffW2 = kOffB1 + kMlpHid;
constexpr int kOffB2 = kOffW2 + kMlpHid * kMlpHid;
constexpr int kOffW3 = kOffB2 + kMlpHid;
constexpr int kOffB3 = kOffW3 + kMlpHid;
constexpr int kMlpParams = kOffB3 + 1;

struct MlpFwdArgs {
  const __nv_bfloat16* x;   // [n][64] features (BF16, zero-padded columns 48..63)
  const __nv_bfloat16* w1;  // [256][64]
  const __nv_bfloat16* w2;  // [256][256]
  const float* b1;
  const float* b2;
  const float* w3;
  const float* b3;
  float* score;             // [n]
  __nv_bfloat16* h1;        // [n][256] ReLU outputs of layer 1, or null
  __nv_bfloat16* h2;        // [n][256] ReLU outputs of layer 2, or null
  int n;
  int* err;                 // set to 1 when a wait on the tensor core timed out
};

// Shared memory of the fused forward kernel.
size_t mlp_fwd_smem();
cudaError_t launch_mlp_fwd(const MlpFwdArgs& a, int grid, cudaStream_t s);

// D = A * B^T over a K range per grid.z slice: A [M][lda], B [N][ldb] (BF16,
// K contiguous). epi 0: FP32 partial sums out_f[z][M][N]; epi 1: BF16
// out_b[M][N] = D * (mask[M][N] > 0).
struct GemmArgs {
  const __nv_bfloat16* a;
  const __nv_bfloat16* b;
  int M, N, K, lda, ldb, kchunk;
  float* out_f;
  __nv_bfloat16* out_b;
  const __nv_bfloat16* mask;
  int* err;
};
cudaError_t launch_gemm_tn(const GemmArgs& g, int NT, int epi, int splits, cudaStream_t s);

struct Context;
// Training scratch for at least rows rows (a multiple of 128).
int mlp_rows(Context& c, int rows);
// GP_E_CUDA when a tensor-core wait of the last launches timed out (synchronises).
int check_mlp_err(Context& c, const char* what);

}  // namespace gp
