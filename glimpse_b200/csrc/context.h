// The context object behind gp_ctx.
#pragma once
#include <string>
#include <vector>

#include "internal.h"
#include "learned.h"
#include "mlp.h"
#include "select.h"

namespace gp {

struct HostPanel {
  int N = 0, L = 0, n_com = 0, n_com_hq = 0;
  std::vector<double> cm;
  std::vector<uint32_t> cref, calt;
  std::vector<uint8_t> lq, common, major;
  std::vector<int32_t> comrow;
  std::vector<uint8_t> hvar;
  std::vector<int64_t> shap_off;
  std::vector<int32_t> shap_sites;
  std::vector<int64_t> svar_off;    // SvarRef: per rare site, carriers of the non-major allele
  std::vector<int32_t> svar_haps;
  std::vector<int32_t> common_sites;  // common2tot
  std::vector<float> cm_pos;
  int max_rare_mac = 0;
};

// Target batch state (genotype_set + the per-target-haplotype PBWT bookkeeping).
struct TargetWork {
  int n = 0;
  std::vector<int32_t> ploidy_h, kpbwt_h, diploid;
  std::vector<int32_t> hap_target, hap_which, target_hap0, target_nhap;
  DevBuf gl, flat, ploidy, dip_list;
  DevBuf h0, h1, hl, hp0, hp1;
  DevBuf gp0, gp1, gpflags, ds, gt0, gt1;
  DevBuf sind, nsind, bitmap;
  DevBuf d_hap_target, d_hap_which, d_target_hap0, d_target_nhap, d_kpbwt, tar_hap, d_grp;
  DevBuf push_key, push_id, push_cnt, stored_bits, start_idx, overflow, carry, ebits;
  int stored_cnt = 0;
  bool finalized = false;
  std::vector<DevBuf*> all() {
    return {&gl, &flat, &ploidy, &dip_list, &h0, &h1, &hl, &hp0, &hp1, &gp0, &gp1, &gpflags, &ds, &gt0, &gt1,
            &sind, &nsind, &bitmap, &d_hap_target, &d_hap_which, &d_target_hap0, &d_target_nhap, &d_kpbwt,
            &tar_hap, &d_grp, &push_key, &push_id, &push_cnt, &stored_bits, &start_idx, &overflow, &carry, &ebits};
  }
};

void unphred_table(float* out);

ModelConst model_constants(const gp_config& c, int n_ref_haps);

struct Context {
  gp_config cfg{};
  ModelConst mc{};
  cudaStream_t stream = nullptr;
  std::string err;
  HostPanel host;
  DevPanel panel;
  ImputeWork impute;
  PhaseWork phase;
  DevBuf scratch_h0, scratch_h1, scratch_ids;
  DevBuf glin_src, glin_nval, glin_ploidy, glin_gl, glin_flat, glin_err;  // gp_gl_from_pl / gp_gl_from_float
  DevBuf out_gp, out_site;                                                 // gp_output_records
  DevBuf lig_a, lig_b, lig_s, lig_cnt;                                     // gp_ligate_overlap / gp_ligate_swap
  std::vector<int32_t> host_nstates;   // K per conditioning set of the current batch
  std::vector<int32_t> impute_np;      // poly sites per conditioning set of the current batch
  std::vector<int32_t> last_phase_nseg;
  // Per-target diplotype-draw error flags of the last phasing launch, copied to
  // pinned host memory on the stream and read after the caller's synchronisation.
  int32_t* phase_err_host = nullptr;
  int phase_err_cap = 0, phase_err_n = 0;
  std::vector<int32_t> phase_err_ids;  // target reported for each flag
  int check_phase_errors();
  TargetWork tw;
  MlpState mlp;          // the learned proposal's network (mlp.cu)
  LearnedWork learned;   // the learned proposal around it (learned.cu)
  SparsePbwt sparse;
  DevPbwt pbwt;
  bool pbwt_active = false;
  float pbwt_modulo = 0.1f;
  std::vector<int32_t> pbwt_grp;
  int tw_push_cap = 4096;
  int grid_y_cap = 65535;  // largest gridDim.y of the launches that loop over it (GLIMPSE_B200_GRID_Y_CAP)
  float stage_ms[5] = {0, 0, 0, 0, 0};
  // profiling: events around the hot kernels, resolved at the next host sync
  struct ProfEv {
    cudaEvent_t a, b;
    int kind;  // 0 imputation forward-backward, 1 phasing, 2 selection, 3 network forward
    double cells;
  };
  std::vector<ProfEv> prof_pending;
  gp_profile prof{};
  void prof_begin(cudaEvent_t& a);
  void prof_end(cudaEvent_t a, int kind, double cells);
  void prof_resolve();
  std::vector<void*> owned;  // device allocations freed at destruction

  ~Context();
  Status fail(int code, const std::string& msg);
  int cuda_fail(cudaError_t e, const char* where);
  int create_panel(const gp_panel_desc& d);
  int build_condsets(int n, const std::vector<int64_t>& off, const std::vector<uint32_t>& states);
  int run_impute(const float* d_hl, const uint8_t* d_flat, float* d_hp);
  size_t store_budget(size_t held, size_t need);
  int run_impute_ckpt(const float* d_hl, const uint8_t* d_flat, float* d_hp);
  int precision_mode = GP_PRECISION_FULL;
  DevBuf ckpt, ckpt_sum, ckpt_scratch, loglik;  // checkpointed imputation (kernels_impute_ckpt.cu)
  int loglik_n = 0;                             // entries of the last checkpointed imputation call
  int impute_chunks = 0;  // launches pairs of the last run_impute (1 when the whole batch fit)
  int phase_chunks = 0;   // k_phase launches of the last run_phase
  // Autotuner: launch shapes picked by timing every candidate on the first batch
  // large enough to tell them apart; fixed_* (gp_tuning_set) override it.
  int tune_cpc = 0, tune_hpw = 0;     // chosen chains per CTA / haplotypes per sweep warp (0: not yet)
  int fixed_cpc = 0, fixed_hpw = 0;
  // k_phase placement (1, the default: entries in decreasing order of work; 2:
  // the heaviest alone on an SM, the others paired heavy with light)
  int fixed_porder = 0;
  // phase-1 ms for 1, 2, 4 chains per CTA; sweep ms for 1, 2, 4, 8; k_phase ms for placements 1, 2
  float tune_ms[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int sm_count = 0;
  DevBuf tune_tarhap;
  // --state-list: per target the sorted union of its haplotypes' rows (empty: no lists)
  std::vector<int32_t> list_len;
  DevBuf list_off, list_ids, merged_states;
  int set_state_lists(int n_haps, const int64_t* off, const int32_t* ids);
  int merge_state_lists(int& Kp);
  int set_targets(int n, const uint8_t* gl, const uint8_t* flat, const int32_t* ploidy, const int32_t* kp);
  int build_condsets_device(int n, int Kp);
  int select_states(int stage, int iteration, int& Kp);
  int init_select_states(int iteration, int Kp, int kinit);
  int iteration(int stage, int iteration);
  int finalize();
  int pbwt_prepare_panel();
  int pbwt_prepare_targets(bool reset_state);
  int pbwt_select_states(int stage, int iteration, int Kp);
  int pbwt_states_get(int target, int32_t* counts, int32_t* states, int cap);
  int learned_prepare_panel();
  int learned_features(int Kpc, DevBuf& xout);
  int learned_prepare_features(int Kpc);
  int learned_feature_rows(int Kpc, DevBuf& xout, int t0, int nc);
  int learned_select_states(int stage, int iteration, int& Kp);
  int learned_labels(int Kpc, float kpos, DevBuf& yout, DevBuf& wout);
  int learned_apply_k(bool reset_state = false);
  int run_phase(const int32_t* d_tsel, const std::vector<int32_t>& tsel_host, int nb, uint8_t* d_h0, uint8_t* d_h1,
                const uint8_t* d_flat, int iteration, const int32_t* d_target_ids);
};

}  // namespace gp
