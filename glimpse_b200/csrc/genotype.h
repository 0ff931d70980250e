// Launchers of the per-site target kernels (kernels_genotype.cu) and of the
// init-stage selection (kernels_init.cu).
#pragma once
#include "internal.h"

namespace gp {

cudaError_t upload_unphred(const float* table);
void launch_hl(const uint8_t* gl, const uint8_t* flat, const int32_t* ploidy, const uint8_t* h0, const uint8_t* h1,
               int n, int L, int stage_init, int hap, float min_gl, float* hl, cudaStream_t s);
void launch_sample(const float* hp, const int32_t* ploidy, int n, int L, uint64_t seed, uint32_t purpose,
                   int iteration, int only_diploid, uint8_t* h, cudaStream_t s);
void launch_gp_store(const float* hp0, const float* hp1, const int32_t* ploidy, int n, int L, int stored_cnt,
                     float* gp0, float* gp1, uint8_t* flags, cudaStream_t s);
void launch_gp_finalize(const int32_t* ploidy, int n, int L, int stored_cnt, const uint8_t* flags, float* gp0,
                        float* gp1, float* ds, uint8_t* gt0, uint8_t* gt1, uint8_t* h0, uint8_t* h1,
                        cudaStream_t s);

// Init-stage selection. sind: per-target rare non-ref GL calls (site lists in
// site order, stride L, counts nsind); bitmap: n x ceil(N/32) words scratch;
// states/nstates: output (stride Kp, sorted).
struct InitSelArgs {
  const uint8_t* gl;
  const uint8_t* flat;
  const int32_t* ploidy;
  const uint8_t* common;
  const uint8_t* lq;
  const uint8_t* major;
  const uint32_t* cref;
  const uint32_t* calt;
  const int64_t* svar_off;   // SvarRef CSR over sites (reference haplotypes carrying the non-major allele)
  const int32_t* svar_haps;
  int32_t* sind;
  int32_t* nsind;
  uint32_t* bitmap;
  uint32_t* states;
  int32_t* nstates;
  int n, L, N, Kp, kinit, max_mac;
  uint64_t seed;
  int iteration;
};
void launch_init_select(const InitSelArgs& a, cudaStream_t s);
cudaError_t upload_unphred_init(const float* table);

}  // namespace gp
