// PBWT state selection: panel-side precompute (pbwt_host.cpp) and the
// per-iteration device kernels (kernels_pbwt.cu).
#pragma once
#include <string>
#include <vector>

#include "internal.h"

namespace gp {

// Site kinds for the selection sweep.
enum SiteKind : uint8_t { SK_LQ = 0, SK_COMMON = 1, SK_RARE = 2 };

// Panel-side sparse PBWT (ref_haplotype_set.h:70-71) in host memory.
struct SparsePbwt {
  std::vector<uint8_t> ypacked;
  std::vector<int64_t> asmall_off;  // [n_com_hq + 2]
  std::vector<int32_t> asmall;      // positions in the full PBWT order, sorted
};

// Consistency of the panel arrays the PBWT relies on: cref + calt = N, the
// HvarRef row of every common site has calt ones, and every rare site lists as
// many non-major carriers as its counts say. Returns GP_OK or GP_E_DATA (msg set).
int validate_panel(int N, int L, const uint8_t* lq, const uint8_t* common, const uint8_t* major,
                   const uint32_t* cref, const uint32_t* calt, const uint8_t* hvar, const int64_t* svar_off,
                   std::string& msg);

// ref_haplotype_set::build_sparsePBWT (ref_haplotype_set.cpp:47-193) over the
// in-memory panel, restated: pack3 run-length coding of every HQ common column in
// PBWT order, and of every rare column in the order of the small PBWT over the
// haplotypes that carry a rare allele in that run of rare sites.
void build_sparse_pbwt(int N, int L, const uint8_t* lq, const uint8_t* common, const uint8_t* major,
                       const uint32_t* cref, const uint32_t* calt, const uint8_t* hvar, const int64_t* svar_off,
                       const int32_t* svar_haps, SparsePbwt& out);

// Device-resident decode of the sparse PBWT, as the target-side sweep of
// haplotype_set::matchHapsFromCompressedPBWTSmall sees it (haplotype_set.cpp:396-444,
// 562-680): prefix arrays after every HQ common site, the merged prefix array
// where a run of rare sites ends, and the rank (V) arrays of every column.
struct DevPbwt {
  bool ready = false;
  int n_com_hq = 0, Wv = 0, R = 0, n_rare_hq = 0;  // R: words per vrow row, a multiple of 4
  uint32_t* a_after = nullptr;   // [n_com_hq][N]
  int32_t* before_id = nullptr;  // [n_com_hq]: -2 iota, -1 a_after[l-1], >= 0 merged[id]
  uint32_t* merged = nullptr;    // [n_merged][N]
  uint32_t* vrow = nullptr;      // [n_com_hq][R]: V bits (Wv words), then their prefix counts (Wv + 1 words)
  int64_t* svoff = nullptr;      // [n_rare_hq + 1] word offsets of small columns
  uint32_t* svbits = nullptr;    // small-column bits
  uint32_t* svpref = nullptr;    // small-column prefix counts (one more entry per column)
  int64_t* asoff = nullptr;      // [n_com_hq + 2]
  int32_t* asidx = nullptr;
  int32_t* site_info = nullptr;  // [L]: kind | (index << 2); common: l_hq, rare: rare ordinal
  int32_t* site_run = nullptr;   // [L]: rare sites: run index l (A_small_idx row); common: l_all
  int32_t* run_end = nullptr;    // [L]: at the first site of a run of rare sites, the run's last non-LQ site
  // The sweep's event list: every non-LQ common site and every run of rare sites,
  // in site order, as two int4 per event:
  //   common: {k, l, cref[k], asoff[l]}, {sn(l), before_id[l], init_common[l], common2tot[max(l - 1, 0)]}
  //   run:    {k | 1 << 30, l, last site of the run, asoff[l]}, {sn(l), 0, 0, 0}
  int4* events = nullptr;
  int n_events = 0;
  uint8_t* init_common = nullptr;  // [n_com_hq]
  uint32_t* cref = nullptr;      // [L]
  float* cm_pos = nullptr;       // [L]  max(0, (float)cm)
  int32_t* common2tot = nullptr; // [n_com]
};

struct PbwtSelectArgs {
  DevPbwt P;
  int N, L, depth, n_haps, n_targets, cap;
  float modulo;
  const uint8_t* lq;
  const uint8_t* common;
  const uint8_t* major;
  const uint32_t* calt;
  const uint8_t* h0;
  const uint8_t* h1;
  const int32_t* hap_target;  // [n_haps]
  const int32_t* hap_which;   // [n_haps] 0 = H0, 1 = H1
  const int32_t* target_hap0; // [n_targets]
  const int32_t* target_nhap; // [n_targets]
  const int32_t* grp;         // [nstored] group ends (pbwt_grp)
  int nstored;
  uint32_t* stored_bits;      // [ceil(n_com_hq/32)]
  uint32_t* carry;            // [n_haps][Wc]: bit k = non-LQ rare site k where the haplotype has the non-major allele
  int Wc;                     // ceil(L / 32)
  uint32_t* ebits;            // [n_haps][We]: bit (e & 31) of word e >> 5 is, for event e of the sweep, the
                              // haplotype's allele at that HQ common site, or for a run of rare sites, whether it
                              // carries a non-major allele at a non-LQ site of the run
  int We;                     // ceil(n_events / 32)
  int grid_y_cap;             // largest gridDim.y of the event-bit launch (65535, the hardware limit, by default)
  int32_t* start_idx;         // [n_haps] random pbwt_index
  uint8_t* tar_hap;           // [n_haps] persistent across iterations
  uint32_t* push_key;         // [n_haps][depth][cap]
  uint32_t* push_id;          // [n_haps][depth][cap]
  int32_t* push_cnt;          // [n_haps][depth]
  int32_t* overflow;          // [1]
  const int32_t* kpbwt;       // [n_targets] (already min'ed with N)
  uint32_t* bitmap;           // [n_targets][ceil(N/32)]
  int32_t* union_rank;        // [n_targets][N] or null: for every id the union inserts, level << 16 | insertion index
  uint32_t* states;           // [n_targets][Kp]
  int32_t* nstates;
  int Kp;
  uint64_t seed;
  int iteration;
};

// The whole selection: prepare (stream starts, carrier bits, event bits),
// sweep with hpw haplotypes per warp (1, 2, 4, 8 or 16), union.
void launch_pbwt_select(const PbwtSelectArgs& a, int hpw, cudaStream_t s);
void launch_pbwt_prepare(const PbwtSelectArgs& a, cudaStream_t s);
void launch_pbwt_sweep(const PbwtSelectArgs& a, int hpw, cudaStream_t s);

}  // namespace gp
