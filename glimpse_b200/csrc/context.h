// The context object behind gp_ctx.
#pragma once
#include <string>
#include <vector>

#include "internal.h"

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
};

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
  std::vector<int32_t> host_nstates;   // K per conditioning set of the current batch
  std::vector<int32_t> impute_np;      // poly sites per conditioning set of the current batch
  std::vector<int32_t> last_phase_nseg;
  std::vector<void*> owned;  // device allocations freed at destruction

  ~Context();
  Status fail(int code, const std::string& msg);
  int cuda_fail(cudaError_t e, const char* where);
  int create_panel(const gp_panel_desc& d);
  int build_condsets(int n, const std::vector<int64_t>& off, const std::vector<uint32_t>& states);
  int run_impute(const float* d_hl, const uint8_t* d_flat, float* d_hp);
  int run_phase(const int32_t* d_tsel, const std::vector<int32_t>& tsel_host, int nb, uint8_t* d_h0, uint8_t* d_h1,
                const uint8_t* d_flat, int iteration, const int32_t* d_target_ids);
};

}  // namespace gp
