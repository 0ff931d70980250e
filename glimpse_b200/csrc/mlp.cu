// Tensor-core kernels of the learned state-selection proposal's MLP
// (kMlpIn -> 256 -> 256 -> 1, ReLU; BF16 weights and activations, FP32
// accumulation in tensor memory).
//
// k_mlp_fwd: the whole forward pass of 128-row tiles in one persistent kernel.
//   W1 (32 KB) and W2 (128 KB) stay in shared memory for the CTA's lifetime in
//   the canonical K-major layout (tc.h). Per tile: the feature rows are staged
//   by cp.async; one thread issues the layer-1 MMAs (M 128, N 256, K 64) into
//   tensor-memory columns 0-255; the four warps read their 32 rows back
//   (tcgen05.ld), add the bias, apply ReLU, round to BF16 and write the hidden
//   tile to shared memory in two K halves of 128, each followed by its 8
//   layer-2 MMAs into columns 256-511; the layer-2 epilogue adds the bias,
//   applies ReLU and takes the dot product with w3 in FP32: the score. Thread t
//   of the CTA owns row t of the tile (tensor-memory lane t).
// k_gemm_tn: D = A * B^T for the weight gradients (split over K) and for the
//   layer-1 input gradient (masked by the ReLU of layer 1), two cp.async stages
//   feeding tcgen05.mma.
// Every wait on the tensor core is bounded (tc::mbar_wait); a time-out sets
// the error flag, the CTA stops, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "context.h"
#include "mlp.h"
#include "tc.h"

namespace gp {
namespace {

constexpr int kTileM = 128;
constexpr uint32_t kSmemW1 = 0;
constexpr uint32_t kSmemW2 = kSmemW1 + kMlpHid * kMlpInP * 2;   // 32 KB
constexpr uint32_t kSmemX = kSmemW2 + kMlpHid * kMlpHid * 2;    // +128 KB
constexpr uint32_t kSmemH = kSmemX + kTileM * kMlpInP * 2;      // +16 KB
constexpr uint32_t kSmemB1 = kSmemH + kTileM * 128 * 2;         // +32 KB (one K half of the hidden tile)
constexpr uint32_t kSmemB2 = kSmemB1 + kMlpHid * 4;
constexpr uint32_t kSmemW3 = kSmemB2 + kMlpHid * 4;
constexpr uint32_t kSmemPart = kSmemW3 + kMlpHid * 4;  // the two halves' partial dot products
constexpr uint32_t kSmemBar = kSmemPart + 256 * 4;
constexpr uint32_t kSmemFwd = kSmemBar + 64;

// cp.async of a row-major BF16 matrix [rows][kext] (K contiguous, row stride ld
// elements) into a canonical K-major tile; rows at or beyond nvalid read zeros.
__device__ __forceinline__ void stage_kmajor(uint8_t* tile, const __nv_bfloat16* src, int rows, int kext, int ld,
                                             int nvalid, int k0, int kvalid) {
  const int chunks = rows * (kext >> 3);
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int r = c / (kext >> 3), kc = c % (kext >> 3);
    const int k = k0 + kc * 8;
    const bool ok = r < nvalid && k < kvalid;
    const __nv_bfloat16* g = ok ? src + (size_t)r * ld + k : src;
    tc::cp_async16(tile + tc::kmajor_off(r, kc * 8, kext), g, ok ? 16u : 0u);
  }
}

constexpr int kFwdThreads = 256;  // warps w and w + 4 share tensor-memory lanes 32 (w % 4) .. + 31 (the tile's
                                  // rows) and split the columns of every epilogue step between them

__global__ void __launch_bounds__(kFwdThreads, 1) k_mlp_fwd(MlpFwdArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmemBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmemBar + 8);
  int* abort_flag = reinterpret_cast<int*>(sm + kSmemBar + 12);
  float* b1s = reinterpret_cast<float*>(sm + kSmemB1);
  float* b2s = reinterpret_cast<float*>(sm + kSmemB2);
  float* w3s = reinterpret_cast<float*>(sm + kSmemW3);
  float* part = reinterpret_cast<float*>(sm + kSmemPart);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int trow = tid & (kTileM - 1);  // the tile row (tensor-memory lane) this thread reads
  const int chalf = tid >> 7;           // which half of each epilogue step's columns it takes
  const int ntiles = (a.n + kTileM - 1) / kTileM;
  if ((int)blockIdx.x >= ntiles) return;

  if (warp == 0) tc::tmem_alloc(tslot, 512);
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::fence_mbar_init();
    *abort_flag = 0;
  }
  stage_kmajor(sm + kSmemW1, a.w1, kMlpHid, kMlpInP, kMlpInP, kMlpHid, 0, kMlpInP);
  stage_kmajor(sm + kSmemW2, a.w2, kMlpHid, kMlpHid, kMlpHid, kMlpHid, 0, kMlpHid);
  tc::cp_async_commit();
  for (int j = tid; j < kMlpHid; j += blockDim.x) {
    b1s[j] = a.b1[j];
    b2s[j] = a.b2[j];
    w3s[j] = a.w3[j];
  }
  const float b3 = a.b3[0];
  tc::cp_async_wait<0>();
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t sW1 = tc::smem_u32(sm + kSmemW1), sW2 = tc::smem_u32(sm + kSmemW2);
  const uint32_t sX = tc::smem_u32(sm + kSmemX), sH = tc::smem_u32(sm + kSmemH);
  constexpr uint32_t idesc = tc::idesc_bf16(kTileM, kMlpHid);
  uint32_t phase = 0;

  auto wait_mma = [&]() {
    if (!tc::mbar_wait(bar, phase)) *abort_flag = 1;
    phase ^= 1u;
    __syncthreads();
    tc::fence_after_sync();
    return *abort_flag == 0;
  };

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * kTileM;
    const int row = r0 + trow;
    stage_kmajor(sm + kSmemX, a.x + (size_t)r0 * kMlpInP, kTileM, kMlpInP, kMlpInP, a.n - r0, 0, kMlpInP);
    tc::cp_async_commit();
    tc::cp_async_wait<0>();
    tc::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < kMlpInP / 16; ++s)
        tc::mma_bf16(tbase, tc::smem_desc(sX + s * 256, 128, (kMlpInP / 8) * 128),
                     tc::smem_desc(sW1 + s * 256, 128, (kMlpInP / 8) * 128), idesc, s > 0);
      tc::commit(bar);
    }
    if (!wait_mma()) break;
    bool ok = true;
    for (int h = 0; h < 2 && ok; ++h) {
      // layer-1 epilogue for hidden units [128 h, 128 h + 128): bias, ReLU, BF16;
      // this thread takes 64 of them
#pragma unroll 1
      for (int c = 0; c < 2; ++c) {
        const int c0 = chalf * 64 + c * 32;  // column within the half
        float v[32];
        tc::tmem_ld32(tbase + lane_off + h * 128 + c0, v);
        uint32_t p[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int j = h * 128 + c0 + 2 * i;
          p[i] = tc::pack_bf16(fmaxf(v[2 * i] + b1s[j], 0.f), fmaxf(v[2 * i + 1] + b1s[j + 1], 0.f));
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint4 u = make_uint4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
          *reinterpret_cast<uint4*>(sm + kSmemH + tc::kmajor_off(trow, c0 + q * 8, 128)) = u;
          if (a.h1 && row < a.n)
            *reinterpret_cast<uint4*>(a.h1 + (size_t)row * kMlpHid + h * 128 + c0 + q * 8) = u;
        }
      }
      tc::fence_proxy_async();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after_sync();
#pragma unroll
        for (int s = 0; s < 8; ++s)
          tc::mma_bf16(tbase + 256, tc::smem_desc(sH + s * 256, 128, 16 * 128),
                       tc::smem_desc(sW2 + (h * 8 + s) * 256, 128, (kMlpHid / 8) * 128), idesc, h > 0 || s > 0);
        tc::commit(bar);
      }
      ok = wait_mma();
    }
    if (!ok) break;
    // layer-2 epilogue: bias, ReLU, dot with w3 in FP32 (this thread: 128 of the
    // 256 columns in order; the two halves are added below)
    float acc = 0.f;
#pragma unroll 1
    for (int c = chalf * 4; c < chalf * 4 + 4; ++c) {
      float v[32];
      tc::tmem_ld32(tbase + lane_off + 256 + c * 32, v);
      uint32_t p[16];
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int j = c * 32 + i;
        v[i] = fmaxf(v[i] + b2s[j], 0.f);
        acc = fmaf(v[i], w3s[j], acc);
      }
      if (a.h2 && row < a.n) {
#pragma unroll
        for (int i = 0; i < 16; ++i) p[i] = tc::pack_bf16(v[2 * i], v[2 * i + 1]);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4*>(a.h2 + (size_t)row * kMlpHid + c * 32 + q * 8) =
              make_uint4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
      }
    }
    part[tid] = acc;
    tc::fence_before_sync();
    __syncthreads();
    if (chalf == 0 && row < a.n) a.score[row] = (part[trow] + part[trow + kTileM]) + b3;
  }
  if (*abort_flag && tid == 0) atomicExch(a.err, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tbase, 512);
}

// D = A * B^T, M tile 128, N tile NT, K blocks of 64 in two cp.async stages.
template <int NT, int EPI>
__global__ void __launch_bounds__(128) k_gemm_tn(GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t sm[];
  constexpr uint32_t kA = kTileM * 64 * 2, kB = NT * 64 * 2, kStage = kA + kB;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * kStage);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 2 * kStage + 16);
  int* abort_flag = reinterpret_cast<int*>(sm + 2 * kStage + 20);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * NT;
  const int kbeg = blockIdx.z * g.kchunk, kend = min(g.K, kbeg + g.kchunk);
  const int nkb = kend > kbeg ? (kend - kbeg + 63) / 64 : 0;
  constexpr uint32_t ncols = NT < 32 ? 32 : NT;
  if (warp == 0) tc::tmem_alloc(tslot, ncols);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    tc::fence_mbar_init();
    *abort_flag = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  constexpr uint32_t idesc = tc::idesc_bf16(kTileM, NT);
  uint32_t uses[2] = {0u, 0u};  // completed MMA batches per stage
  auto load = [&](int kb) {
    uint8_t* st = sm + (kb & 1) * kStage;
    const int k0 = kbeg + kb * 64;
    stage_kmajor(st, g.a + (size_t)m0 * g.lda, kTileM, 64, g.lda, g.M - m0, k0, kend);
    stage_kmajor(st + kA, g.b + (size_t)n0 * g.ldb, NT, 64, g.ldb, g.N - n0, k0, kend);
    tc::cp_async_commit();
  };
  if (nkb > 0) load(0);
  for (int kb = 0; kb < nkb; ++kb) {
    if (kb + 1 < nkb) {
      if (kb >= 1) {  // the stage about to be refilled was read by the MMAs of block kb - 1
        const int s = (kb + 1) & 1;
        if (!tc::mbar_wait(&bar[s], uses[s] & 1u)) *abort_flag = 1;
        uses[s]++;
      }
      load(kb + 1);
      tc::cp_async_wait<1>();
    } else {
      tc::cp_async_wait<0>();
    }
    tc::fence_proxy_async();
    __syncthreads();
    if (*abort_flag) break;
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t sa = tc::smem_u32(sm + (kb & 1) * kStage), sb = sa + kA;
#pragma unroll
      for (int s = 0; s < 4; ++s)
        tc::mma_bf16(tbase, tc::smem_desc(sa + s * 256, 128, 1024), tc::smem_desc(sb + s * 256, 128, 1024), idesc,
                     kb > 0 || s > 0);
      tc::commit(&bar[kb & 1]);
    }
  }
  // the last commit covers every MMA issued before it
  if (nkb > 0 && !*abort_flag) {
    const int s = (nkb - 1) & 1;
    if (!tc::mbar_wait(&bar[s], uses[s] & 1u)) *abort_flag = 1;
  }
  __syncthreads();
  tc::fence_after_sync();
  const int row = m0 + tid;
  if (!*abort_flag) {
    // every thread takes part in the warp-wide tensor-memory loads; only rows
    // below M store
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
    for (int c = 0; c < NT / 32; ++c) {
      float v[32];
      if (nkb > 0) {
        tc::tmem_ld32(tbase + lane_off + c * 32, v);
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 0.f;
      }
      const int nb = n0 + c * 32;
      if (row >= g.M) continue;
      if (EPI == 0) {
        float* o = g.out_f + ((size_t)blockIdx.z * g.M + row) * g.N;
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (nb + i < g.N) o[nb + i] = v[i];
      } else {
        const __nv_bfloat16* mk = g.mask + (size_t)row * g.N;
        __nv_bfloat16* o = g.out_b + (size_t)row * g.N;
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (nb + i < g.N) o[nb + i] = __float2bfloat16_rn(__bfloat162float(mk[nb + i]) > 0.f ? v[i] : 0.f);
      }
    }
  }
  if (*abort_flag && tid == 0) atomicExch(g.err, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tbase, ncols);
}

// FP32 feature rows [n][kMlpIn] to zero-padded BF16 rows [rows][kMlpInP].
__global__ void k_feat_bf16(const float* __restrict__ x, int n, int rows, __nv_bfloat16* __restrict__ out) {
  const int64_t tot = (int64_t)rows * kMlpInP;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / kMlpInP), c = (int)(i % kMlpInP);
    out[i] = __float2bfloat16_rn(r < n && c < kMlpIn ? x[(size_t)r * kMlpIn + c] : 0.f);
  }
}

// out[c][r] = in[r][c] for a [R][C] BF16 matrix, 32 x 32 tiles through shared memory.
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int R, int C, __nv_bfloat16* __restrict__ out) {
  __shared__ __nv_bfloat16 t[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    t[i][threadIdx.x] = (r < R && c < C) ? in[(size_t)r * C + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(size_t)c * R + r] = t[threadIdx.x][i];
  }
}

// Columns of the per-block partial sums (hpart rows): dL/dw3 | dL/db2 | dL/db3,
// loss | dL/db1. They are added over the blocks in block order (k_sum_head), so
// a training step gives the same parameters on every run.
constexpr int kHpW3 = 0, kHpB2 = kMlpHid, kHpB3 = 2 * kMlpHid, kHpLoss = 2 * kMlpHid + 1,
              kHpB1 = 2 * kMlpHid + 2, kHpCols = 3 * kMlpHid + 2;

// Loss head and the gradients it feeds, for rows [blockIdx.x * rpb, ...):
// p = sigmoid(score), loss = wt * BCE(p, y) / n, ds = (p - y) * wt / n;
// dz2[r][j] = ds * w3[j] where h2[r][j] > 0; the block's sums of dL/dw3, dL/db2,
// dL/db3 and the loss go to its row of hpart. Thread j owns hidden unit j.
__global__ void k_bwd_head(const float* __restrict__ score, const float* __restrict__ y, const float* __restrict__ wt,
                           const __nv_bfloat16* __restrict__ h2, const float* __restrict__ w3, int rows, int rpb,
                           float inv_n, __nv_bfloat16* __restrict__ dz2, float* __restrict__ hpart) {
  const int j = threadIdx.x;
  const int rb = blockIdx.x * rpb, re = min(rows, rb + rpb);
  const float w3j = w3[j];
  float gw3 = 0.f, gb2 = 0.f, gb3 = 0.f, ls = 0.f;
  for (int r = rb; r < re; ++r) {
    const float s = score[r], yy = y[r], ww = wt[r];
    const float p = 1.f / (1.f + expf(-s));
    const float ds = (p - yy) * ww * inv_n;
    const float h = __bfloat162float(h2[(size_t)r * kMlpHid + j]);
    const float dz = h > 0.f ? ds * w3j : 0.f;
    dz2[(size_t)r * kMlpHid + j] = __float2bfloat16_rn(dz);
    gw3 = fmaf(ds, h, gw3);
    gb2 += dz;
    if (j == 0) {
      gb3 += ds;
      ls += ww * inv_n * (fmaxf(s, 0.f) - s * yy + log1pf(expf(-fabsf(s))));
    }
  }
  float* row = hpart + (size_t)blockIdx.x * kHpCols;
  row[kHpW3 + j] = gw3;
  row[kHpB2 + j] = gb2;
  if (j == 0) {
    row[kHpB3] = gb3;
    row[kHpLoss] = ls;
  }
}

// The block's sums over rows of m[r][j] (m: [rows][256] BF16) into its row of
// hpart (dL/db1 columns), thread j per column.
__global__ void k_colsum(const __nv_bfloat16* __restrict__ m, int rows, int rpb, float* __restrict__ hpart) {
  const int j = threadIdx.x;
  const int rb = blockIdx.x * rpb, re = min(rows, rb + rpb);
  float acc = 0.f;
  for (int r = rb; r < re; ++r) acc += __bfloat162float(m[(size_t)r * kMlpHid + j]);
  hpart[(size_t)blockIdx.x * kHpCols + kHpB1 + j] = acc;
}

// The hpart columns added over the blocks in block order, into the gradient
// vector and the loss.
__global__ void k_sum_head(const float* __restrict__ hpart, int blocks, float* __restrict__ grad,
                           float* __restrict__ loss) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kHpCols; c += gridDim.x * blockDim.x) {
    float v = 0.f;
    for (int b = 0; b < blocks; ++b) v += hpart[(size_t)b * kHpCols + c];
    if (c < kHpB2) grad[kOffW3 + c] = v;
    else if (c < kHpB3) grad[kOffB2 + c - kHpB2] = v;
    else if (c == kHpB3) grad[kOffB3] = v;
    else if (c == kHpLoss) *loss = v;
    else grad[kOffB1 + c - kHpB1] = v;
  }
}

// dst[i] = sum over splits of part[z][i].
__global__ void k_sum_splits(const float* __restrict__ part, int n, int splits, float* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int z = 0; z < splits; ++z) acc += part[(size_t)z * n + i];
    dst[i] = acc;
  }
}

// Adam over the packed parameters (FP32 master copies), then the BF16 copies the GEMMs read.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_pack_weights(const float* __restrict__ p, __nv_bfloat16* __restrict__ w1,
                               __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w2t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpHid * kMlpHid; i += gridDim.x * blockDim.x) {
    if (i < kMlpHid * kMlpInP) w1[i] = __float2bfloat16_rn(p[kOffW1 + i]);
    const int r = i / kMlpHid, c = i % kMlpHid;
    const __nv_bfloat16 b = __float2bfloat16_rn(p[kOffW2 + i]);
    w2[i] = b;
    w2t[(size_t)c * kMlpHid + r] = b;
  }
}

}  // namespace

size_t mlp_fwd_smem() { return kSmemFwd; }

cudaError_t launch_mlp_fwd(const MlpFwdArgs& a, int grid, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const int ntiles = (a.n + kTileM - 1) / kTileM;
  grid = std::max(1, std::min(grid, ntiles));
  cudaError_t e = set_smem_limit_once<k_mlp_fwd>((int)kSmemFwd);
  if (e != cudaSuccess) return e;
  k_mlp_fwd<<<grid, kFwdThreads, kSmemFwd, s>>>(a);
  return cudaGetLastError();
}

template <int NT, int EPI>
static cudaError_t gemm_launch(const GemmArgs& g, int splits, cudaStream_t s) {
  constexpr size_t smem = 2 * (kTileM * 64 * 2 + NT * 64 * 2) + 64;
  cudaError_t e = set_smem_limit_once<k_gemm_tn<NT, EPI>>((int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((g.M + kTileM - 1) / kTileM, (g.N + NT - 1) / NT, splits);
  k_gemm_tn<NT, EPI><<<grid, 128, smem, s>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_gemm_tn(const GemmArgs& g, int NT, int epi, int splits, cudaStream_t s) {
  if ((g.K & 7) || (g.lda & 7) || (g.ldb & 7)) return cudaErrorInvalidValue;  // 16-byte rows of K chunks
  if (NT == 256 && epi == 0) return gemm_launch<256, 0>(g, splits, s);
  if (NT == 256 && epi == 1) return gemm_launch<256, 1>(g, splits, s);
  if (NT == 64 && epi == 0) return gemm_launch<64, 0>(g, splits, s);
  return cudaErrorInvalidValue;
}

}  // namespace gp

// ---- host side: parameters, forward and one training step ----
namespace gp {
namespace {

int mlp_ensure(Context& c) {
  MlpState& M = c.mlp;
  if (M.ready) return GP_OK;
  cudaError_t e;
  for (DevBuf* b : {&M.param, &M.m, &M.v, &M.grad})
    if ((e = b->ensure((size_t)kMlpParams * 4)) != cudaSuccess) return c.cuda_fail(e, "mlp alloc");
  if ((e = M.w1.ensure((size_t)kMlpHid * kMlpInP * 2)) != cudaSuccess) return c.cuda_fail(e, "mlp alloc");
  if ((e = M.w2.ensure((size_t)kMlpHid * kMlpHid * 2)) != cudaSuccess) return c.cuda_fail(e, "mlp alloc");
  if ((e = M.w2t.ensure((size_t)kMlpHid * kMlpHid * 2)) != cudaSuccess) return c.cuda_fail(e, "mlp alloc");
  if ((e = M.err.ensure(8)) != cudaSuccess) return c.cuda_fail(e, "mlp alloc");
  if ((e = M.loss.ensure(8)) != cudaSuccess) return c.cuda_fail(e, "mlp alloc");
  cudaMemsetAsync(M.m.ptr, 0, (size_t)kMlpParams * 4, c.stream);
  cudaMemsetAsync(M.v.ptr, 0, (size_t)kMlpParams * 4, c.stream);
  cudaMemsetAsync(M.err.ptr, 0, 8, c.stream);
  M.step = 0;
  M.ready = true;
  return GP_OK;
}

float* params(MlpState& M) { return M.param.as<float>(); }

void pack(Context& c) {
  MlpState& M = c.mlp;
  k_pack_weights<<<256, 256, 0, c.stream>>>(params(M), M.w1.as<__nv_bfloat16>(), M.w2.as<__nv_bfloat16>(),
                                            M.w2t.as<__nv_bfloat16>());
  c.prof.kernel_launches += 1;
}

}  // namespace

int mlp_rows(Context& c, int rows) {
  MlpState& M = c.mlp;
  if (rows <= M.cap_rows) return GP_OK;
  const size_t R = (size_t)rows;
  cudaError_t e;
  if ((e = M.x.ensure(R * kMlpInP * 2)) != cudaSuccess) return c.cuda_fail(e, "mlp rows");
  if ((e = M.xt.ensure(R * kMlpInP * 2)) != cudaSuccess) return c.cuda_fail(e, "mlp rows");
  for (DevBuf* b : {&M.y, &M.wt, &M.score})
    if ((e = b->ensure(R * 4)) != cudaSuccess) return c.cuda_fail(e, "mlp rows");
  for (DevBuf* b : {&M.h1, &M.h1t, &M.h2, &M.dz2, &M.dz2t, &M.dz1, &M.dz1t})
    if ((e = b->ensure(R * kMlpHid * 2)) != cudaSuccess) return c.cuda_fail(e, "mlp rows");
  M.cap_rows = rows;
  return GP_OK;
}

int check_mlp_err(Context& c, const char* what) {
  int32_t err = 0;
  cudaMemcpyAsync(&err, c.mlp.err.ptr, 4, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return c.cuda_fail(e, what);
  if (err) {
    cudaMemsetAsync(c.mlp.err.ptr, 0, 4, c.stream);
    return (c.fail(GP_E_CUDA, std::string(what) + ": a tensor-core wait timed out"), GP_E_CUDA);
  }
  return GP_OK;
}

int mlp_forward_device(Context& c, const __nv_bfloat16* x, int n, float* score, __nv_bfloat16* h1, __nv_bfloat16* h2) {
  MlpState& M = c.mlp;
  MlpFwdArgs a;
  a.x = x;
  a.w1 = M.w1.as<__nv_bfloat16>();
  a.w2 = M.w2.as<__nv_bfloat16>();
  a.b1 = params(M) + kOffB1;
  a.b2 = params(M) + kOffB2;
  a.w3 = params(M) + kOffW3;
  a.b3 = params(M) + kOffB3;
  a.score = score;
  a.h1 = h1;
  a.h2 = h2;
  a.n = n;
  a.err = M.err.as<int>();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaEvent_t ea;
  c.prof_begin(ea);
  cudaError_t e = launch_mlp_fwd(a, sms, c.stream);
  c.prof_end(ea, 3, (double)n);
  c.prof.kernel_launches += 1;
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "mlp forward launch");
}

// One step over n rows already staged in M.x / M.y / M.wt (padded to rows).
int mlp_train_device(Context& c, int n, int rows, float lr, bool want_grad) {
  MlpState& M = c.mlp;
  cudaStream_t s = c.stream;
  auto bf = [](DevBuf& b) { return b.as<__nv_bfloat16>(); };
  cudaMemsetAsync(M.grad.ptr, 0, (size_t)kMlpParams * 4, s);
  cudaMemsetAsync(M.loss.ptr, 0, 4, s);
  int rc = mlp_forward_device(c, bf(M.x), rows, M.score.as<float>(), bf(M.h1), bf(M.h2));
  if (rc != GP_OK) return rc;
  const int rpb = 64;
  const int hb = (rows + rpb - 1) / rpb;
  float* g = M.grad.as<float>();
  cudaError_t e;
  if ((e = M.hpart.ensure((size_t)hb * kHpCols * 4)) != cudaSuccess) return c.cuda_fail(e, "mlp partial");
  k_bwd_head<<<hb, kMlpHid, 0, s>>>(M.score.as<float>(), M.y.as<float>(), M.wt.as<float>(), bf(M.h2),
                                    params(M) + kOffW3, rows, rpb, 1.0f / (float)n, bf(M.dz2), M.hpart.as<float>());
  const dim3 tb(32, 8);
  k_transpose_bf16<<<dim3(rows / 32, kMlpHid / 32), tb, 0, s>>>(bf(M.dz2), rows, kMlpHid, bf(M.dz2t));
  k_transpose_bf16<<<dim3(rows / 32, kMlpHid / 32), tb, 0, s>>>(bf(M.h1), rows, kMlpHid, bf(M.h1t));
  k_transpose_bf16<<<dim3(rows / 32, kMlpInP / 32), tb, 0, s>>>(bf(M.x), rows, kMlpInP, bf(M.xt));
  // dL/dh1 = dz2 W2, masked by layer 1's ReLU: dz1 (rows x 256)
  GemmArgs ga{};
  ga.a = bf(M.dz2);
  ga.b = bf(M.w2t);
  ga.M = rows;
  ga.N = kMlpHid;
  ga.K = kMlpHid;
  ga.lda = ga.ldb = kMlpHid;
  ga.kchunk = kMlpHid;
  ga.out_b = bf(M.dz1);
  ga.mask = bf(M.h1);
  ga.err = M.err.as<int>();
  e = launch_gemm_tn(ga, 256, 1, 1, s);
  if (e != cudaSuccess) return c.cuda_fail(e, "mlp dH1 launch");
  k_transpose_bf16<<<dim3(rows / 32, kMlpHid / 32), tb, 0, s>>>(bf(M.dz1), rows, kMlpHid, bf(M.dz1t));
  k_colsum<<<hb, kMlpHid, 0, s>>>(bf(M.dz1), rows, rpb, M.hpart.as<float>());
  k_sum_head<<<(kHpCols + 255) / 256, 256, 0, s>>>(M.hpart.as<float>(), hb, g, M.loss.as<float>());
  // weight gradients, split over rows: dW2 = dz2^T h1, dW1 = dz1^T x
  const int kchunk = 2048;
  const int splits = (rows + kchunk - 1) / kchunk;
  if ((e = M.partial.ensure((size_t)splits * kMlpHid * kMlpHid * 4)) != cudaSuccess)
    return c.cuda_fail(e, "mlp partial");
  GemmArgs gw{};
  gw.a = bf(M.dz2t);
  gw.b = bf(M.h1t);
  gw.M = kMlpHid;
  gw.N = kMlpHid;
  gw.K = rows;
  gw.lda = gw.ldb = rows;
  gw.kchunk = kchunk;
  gw.out_f = M.partial.as<float>();
  gw.err = M.err.as<int>();
  if ((e = launch_gemm_tn(gw, 256, 0, splits, s)) != cudaSuccess) return c.cuda_fail(e, "mlp dW2 launch");
  k_sum_splits<<<256, 256, 0, s>>>(M.partial.as<float>(), kMlpHid * kMlpHid, splits, g + kOffW2);
  GemmArgs g1{};
  g1.a = bf(M.dz1t);
  g1.b = bf(M.xt);
  g1.M = kMlpHid;
  g1.N = kMlpInP;
  g1.K = rows;
  g1.lda = g1.ldb = rows;
  g1.kchunk = kchunk;
  g1.out_f = M.partial.as<float>();
  g1.err = M.err.as<int>();
  if ((e = launch_gemm_tn(g1, 64, 0, splits, s)) != cudaSuccess) return c.cuda_fail(e, "mlp dW1 launch");
  k_sum_splits<<<64, 256, 0, s>>>(M.partial.as<float>(), kMlpHid * kMlpInP, splits, g + kOffW1);
  c.prof.kernel_launches += 12;
  (void)want_grad;
  if (lr > 0.f) {
    M.step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)M.step), c2 = 1.f - std::pow(b2, (float)M.step);
    k_adam<<<256, 256, 0, s>>>(params(M), g, M.m.as<float>(), M.v.as<float>(), kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
    pack(c);
    c.prof.kernel_launches += 1;
  }
  return GP_OK;
}

}  // namespace gp

using gp::Context;

static Context* Cx(gp_ctx* c) { return reinterpret_cast<Context*>(c); }

extern "C" {

int32_t gp_mlp_param_count(void) { return gp::kMlpParams; }

int gp_mlp_init(gp_ctx* ctx, uint64_t seed) {
  if (!ctx) return GP_E_ARG;
  Context& c = *Cx(ctx);
  int rc = gp::mlp_ensure(c);
  if (rc != GP_OK) return rc;
  // He-uniform weights (fan-in of the 48 real features, then 256), zero biases;
  // the padded feature columns 48..63 of W1 stay zero.
  std::vector<float> p(gp::kMlpParams, 0.f);
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  const float a1 = std::sqrt(6.f / gp::kMlpIn), a2 = std::sqrt(6.f / gp::kMlpHid), a3 = std::sqrt(3.f / gp::kMlpHid);
  for (int j = 0; j < gp::kMlpHid; ++j)
    for (int f = 0; f < gp::kMlpIn; ++f) p[gp::kOffW1 + j * gp::kMlpInP + f] = a1 * u(g);
  for (int i = 0; i < gp::kMlpHid * gp::kMlpHid; ++i) p[gp::kOffW2 + i] = a2 * u(g);
  for (int j = 0; j < gp::kMlpHid; ++j) p[gp::kOffW3 + j] = a3 * u(g);
  return gp_mlp_set_params(ctx, p.data());
}

int gp_mlp_set_params(gp_ctx* ctx, const float* params) {
  if (!ctx || !params) return GP_E_ARG;
  Context& c = *Cx(ctx);
  int rc = gp::mlp_ensure(c);
  if (rc != GP_OK) return rc;
  for (int j = 0; j < gp::kMlpHid; ++j)
    for (int f = gp::kMlpIn; f < gp::kMlpInP; ++f)
      if (params[gp::kOffW1 + j * gp::kMlpInP + f] != 0.f)
        return (c.fail(GP_E_ARG, "mlp: padded feature columns 48..63 of W1 must be zero"), GP_E_ARG);
  cudaMemcpyAsync(c.mlp.param.ptr, params, (size_t)gp::kMlpParams * 4, cudaMemcpyHostToDevice, c.stream);
  cudaMemsetAsync(c.mlp.m.ptr, 0, (size_t)gp::kMlpParams * 4, c.stream);
  cudaMemsetAsync(c.mlp.v.ptr, 0, (size_t)gp::kMlpParams * 4, c.stream);
  c.mlp.step = 0;
  gp::pack(c);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "mlp set params");
}

int gp_mlp_get_params(gp_ctx* ctx, float* params) {
  if (!ctx || !params) return GP_E_ARG;
  Context& c = *Cx(ctx);
  if (!c.mlp.ready) return (c.fail(GP_E_STATE, "mlp: no parameters (gp_mlp_init)"), GP_E_STATE);
  cudaMemcpyAsync(params, c.mlp.param.ptr, (size_t)gp::kMlpParams * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "mlp get params");
}

static int stage_rows(Context& c, int32_t n, const float* x, int& rows) {
  rows = (n + 127) / 128 * 128;
  int rc = gp::mlp_rows(c, rows);
  if (rc != GP_OK) return rc;
  gp::DevBuf& tmp = c.mlp.xf;
  cudaError_t e = tmp.ensure((size_t)n * gp::kMlpIn * 4);
  if (e != cudaSuccess) return c.cuda_fail(e, "mlp staging");
  cudaMemcpyAsync(tmp.ptr, x, (size_t)n * gp::kMlpIn * 4, cudaMemcpyHostToDevice, c.stream);
  gp::k_feat_bf16<<<512, 256, 0, c.stream>>>(tmp.as<float>(), n, rows, c.mlp.x.as<__nv_bfloat16>());
  c.prof.kernel_launches += 1;
  return GP_OK;
}

int gp_mlp_forward(gp_ctx* ctx, int32_t n, const float* x, float* score, float* h1, float* h2) {
  if (!ctx || n <= 0 || !x || !score) return GP_E_ARG;
  Context& c = *Cx(ctx);
  if (!c.mlp.ready) return (c.fail(GP_E_STATE, "mlp: no parameters (gp_mlp_init)"), GP_E_STATE);
  int rows = 0;
  int rc = stage_rows(c, n, x, rows);
  if (rc != GP_OK) return rc;
  gp::MlpState& M = c.mlp;
  // the hidden activations are written only when the caller asks for them
  rc = gp::mlp_forward_device(c, M.x.as<__nv_bfloat16>(), n, M.score.as<float>(),
                              h1 ? M.h1.as<__nv_bfloat16>() : nullptr, h2 ? M.h2.as<__nv_bfloat16>() : nullptr);
  if (rc != GP_OK) return rc;
  cudaMemcpyAsync(score, M.score.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, c.stream);
  std::vector<__nv_bfloat16> hb;
  if (h1 || h2) hb.resize((size_t)n * gp::kMlpHid);
  rc = gp::check_mlp_err(c, "mlp forward");
  if (rc != GP_OK) return rc;
  for (int k = 0; k < 2; ++k) {
    float* out = k ? h2 : h1;
    if (!out) continue;
    cudaMemcpyAsync(hb.data(), (k ? M.h2 : M.h1).ptr, hb.size() * 2, cudaMemcpyDeviceToHost, c.stream);
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return c.cuda_fail(cudaGetLastError(), "mlp forward");
    for (size_t i = 0; i < hb.size(); ++i) out[i] = __bfloat162float(hb[i]);
  }
  return GP_OK;
}

int gp_mlp_train_step(gp_ctx* ctx, int32_t n, const float* x, const float* y, const float* wt, float lr, float* loss,
                      float* grad) {
  if (!ctx || n <= 0 || !x || !y) return GP_E_ARG;
  Context& c = *Cx(ctx);
  if (!c.mlp.ready) return (c.fail(GP_E_STATE, "mlp: no parameters (gp_mlp_init)"), GP_E_STATE);
  int rows = 0;
  int rc = stage_rows(c, n, x, rows);
  if (rc != GP_OK) return rc;
  gp::MlpState& M = c.mlp;
  std::vector<float> yy(rows, 0.f), ww(rows, 0.f);
  for (int i = 0; i < n; ++i) {
    yy[i] = y[i];
    ww[i] = wt ? wt[i] : 1.f;
  }
  cudaMemcpyAsync(M.y.ptr, yy.data(), (size_t)rows * 4, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(M.wt.ptr, ww.data(), (size_t)rows * 4, cudaMemcpyHostToDevice, c.stream);
  rc = gp::mlp_train_device(c, n, rows, lr, grad != nullptr);
  if (rc != GP_OK) return rc;
  if (grad) cudaMemcpyAsync(grad, M.grad.ptr, (size_t)gp::kMlpParams * 4, cudaMemcpyDeviceToHost, c.stream);
  float l = 0.f;
  cudaMemcpyAsync(&l, M.loss.ptr, 4, cudaMemcpyDeviceToHost, c.stream);
  rc = gp::check_mlp_err(c, "mlp train step");
  if (rc != GP_OK) return rc;
  if (loss) *loss = l;
  return GP_OK;
}

}  // extern "C"
