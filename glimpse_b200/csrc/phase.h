// Device data of the phasing HMM (kernels_phase.cu).
#pragma once
#include "internal.h"

namespace gp {

constexpr int kPhaseThreads = 256;
// VAR codes: 0..2 peak het of type n_het % 3, VT_HOM peak hom, VT_FLAT flat het
// (VAR_PEAK_HET / VAR_PEAK_HOM / VAR_FLAT_HET, phasing_hmm.h:40-42); bit 3 = VAR_ALT.
constexpr int VT_HOM = 3;
constexpr int VT_FLAT = 4;

// Per batch entry b: arrays of stride L (VAR entries), L+2 (segments).
struct PhaseVars {
  int32_t* rel;        // VAR_REL: poly index
  uint8_t* code;       // type | alt << 3
  int32_t* seg;        // segment of the entry
  int32_t* miss;       // flat-het index or -1
  int32_t* seg_start;  // first entry of each segment, [nseg] = nvar
  float* yt_prev;      // transition from the previous VAR site (0 for the first)
  float* yt_next;      // transition to the next VAR site (0 for the last)
  uint8_t* flags;      // bit0: first entry of its segment, bit1: last entry of its segment
  // The fields the sweeps read per entry, packed into 16 bytes per direction:
  // x = rel | code << 24 | flags << 28, y = seg, z = miss, w = bits of the
  // transition to the next entry (recb, backward) or from the previous one (recf).
  int4* recb;
  int4* recf;
  int32_t* nvar;
  int32_t* nseg;
  int32_t* nmiss;
  // Per-entry stride of the arrays above and of PhaseStore's per-entry sums:
  // the batch's largest polymorphic-site count (VAR sites are a subset).
  int lv;
};

struct PhaseStore {
  float* pprob;          // pool: [nseg][K][8] per entry at pprob_off[b]
  const int64_t* pprob_off;
  float* pprob_sum;      // [b][L+2][8]
  float* pprob_sumsum;   // [b][L+2]
  float* iprob;          // pool: [nmiss][K][8] per entry at iprob_off[b]
  const int64_t* iprob_off;
  float* iprob_sum;      // [b][L][8]
  float* of1;            // imputeProbOf1s [b][L][8]
  int32_t* dip;          // dip_sampled [b][L+2]
  int32_t* err;          // [b] nonzero when a diplotype draw saw an invalid sum
  const int32_t* order;  // [nb] batch entry of each block of k_phase (heaviest first), or null for the identity
};

void launch_build_vars(const int32_t* tsel, int nb, const int32_t* poly, const int32_t* npoly, const uint8_t* h0,
                       const uint8_t* h1, const uint8_t* flat, const uint8_t* lq, int L, PhaseVars V,
                       cudaStream_t s);
// Per-VAR transition records of all nb entries (before the phasing launches).
void launch_var_records(const int32_t* tsel, int nb, const int32_t* poly, int L, const double* cm,
                        const ModelConst& mc, PhaseVars V, cudaStream_t s);
// k_phase over nb blocks: block i runs entry S.order[i] (S.order may point into
// a longer order, for a chunk of the batch).
int launch_phase(int J, const int32_t* tsel, int nb, const int32_t* nstates, const uint32_t* hvar, int WB, int Kp,
                 const int32_t* poly, const int32_t* npoly, int L, const double* cm, PhaseVars V, PhaseStore S,
                 const ModelConst& mc, uint64_t seed, int iteration, const int32_t* target_ids, cudaStream_t s);
void launch_phase_writeback(const int32_t* tsel, int nb, const int32_t* poly, const int32_t* polyidx, int L,
                            PhaseVars V, PhaseStore S, const ModelConst& mc, uint64_t seed, int iteration,
                            const int32_t* target_ids, uint8_t* h0, uint8_t* h1, cudaStream_t s);

}  // namespace gp
