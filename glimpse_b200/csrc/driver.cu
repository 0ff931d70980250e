// The batched Gibbs driver: caller::phase_iteration / phase_individual
// (phase/src/caller/caller_algorithm.cpp:53-126) for all targets at once, and
// the target-level C-ABI entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "context.h"
#include "genotype.h"
#include "phase.h"
#include "select.h"

namespace gp {

// unphred[i] = 10^(-i/10) as the reference tabulates it: each value printed with
// seven significant digits, then read back as a float (otools.h:98).
void unphred_table(float* out) {
  for (int i = 0; i < 256; ++i) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.6e", std::pow(10.0, -i / 10.0));
    out[i] = std::strtof(buf, nullptr);
  }
}

int Context::set_targets(int n, const uint8_t* gl, const uint8_t* flat, const int32_t* ploidy, const int32_t* kp) {
  const int L = panel.L;
  TargetWork& T = tw;
  // validate before touching the context, so that a refused call leaves it as it was
  for (int i = 0; i < n; ++i) {
    if (ploidy[i] != 1 && ploidy[i] != 2) return (fail(GP_E_ARG, "ploidy must be 1 or 2"), GP_E_ARG);
    if ((kp ? kp[i] : cfg.kpbwt) < 0) return (fail(GP_E_ARG, "negative Kpbwt"), GP_E_ARG);
  }
  T.n = n;
  list_len.clear();  // state lists belong to a target set
  T.ploidy_h.assign(ploidy, ploidy + n);
  T.kpbwt_h.resize(n);
  T.diploid.clear();
  for (int i = 0; i < n; ++i) {
    T.kpbwt_h[i] = kp ? kp[i] : cfg.kpbwt;
    if (ploidy[i] == 2) T.diploid.push_back(i);
  }
  cudaError_t e;
  const size_t nL = (size_t)n * L;
  for (auto* b : {&T.gl}) if ((e = b->ensure(nL * 3)) != cudaSuccess) return cuda_fail(e, "alloc targets");
  for (auto* b : {&T.flat, &T.h0, &T.h1, &T.gpflags, &T.gt0, &T.gt1})
    if ((e = b->ensure(nL)) != cudaSuccess) return cuda_fail(e, "alloc targets");
  for (auto* b : {&T.hl, &T.hp0, &T.hp1})
    if ((e = b->ensure(nL * 2 * 4)) != cudaSuccess) return cuda_fail(e, "alloc targets");
  for (auto* b : {&T.gp0, &T.gp1, &T.ds, &T.sind})
    if ((e = b->ensure(nL * 4)) != cudaSuccess) return cuda_fail(e, "alloc targets");
  if ((e = T.ploidy.ensure(n * 4)) != cudaSuccess) return cuda_fail(e, "alloc targets");
  if ((e = T.nsind.ensure(n * 4)) != cudaSuccess) return cuda_fail(e, "alloc targets");
  if ((e = T.dip_list.ensure(std::max<size_t>(1, T.diploid.size()) * 4)) != cudaSuccess)
    return cuda_fail(e, "alloc targets");
  if ((e = T.bitmap.ensure((size_t)n * ((panel.N + 31) / 32) * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  cudaMemcpyAsync(T.gl.ptr, gl, nL * 3, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(T.flat.ptr, flat, nL, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(T.ploidy.ptr, ploidy, n * 4, cudaMemcpyHostToDevice, stream);
  if (!T.diploid.empty())
    cudaMemcpyAsync(T.dip_list.ptr, T.diploid.data(), T.diploid.size() * 4, cudaMemcpyHostToDevice, stream);
  // genotype::allocate (genotype.cpp:48-54): H0 = H1 = 0, no stored posteriors
  cudaMemsetAsync(T.h0.ptr, 0, nL, stream);
  cudaMemsetAsync(T.h1.ptr, 0, nL, stream);
  cudaMemsetAsync(T.gpflags.ptr, 0, nL, stream);
  cudaMemsetAsync(T.gp0.ptr, 0, nL * 4, stream);
  cudaMemsetAsync(T.gp1.ptr, 0, nL * 4, stream);
  cudaMemsetAsync(T.hp0.ptr, 0, nL * 8, stream);
  cudaMemsetAsync(T.hp1.ptr, 0, nL * 8, stream);
  T.stored_cnt = 0;
  T.finalized = false;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "targets upload");
  learned.kfinal.clear();  // the caller's Kpbwt becomes the learned mode's conditioning-set size
  return learned_apply_k(true);
}

// Conditioning sets from states already on the device (impute.states with
// stride Kp, impute.nstates): poly sites and Hvar. Copies K and npoly to the host.
// The Hvar words are sized on the batch's largest polymorphic-site count (its
// blocks of 32), not on all panel sites: the counts come back to the host
// before the words are built.
int Context::build_condsets_device(int n, int Kp) {
  ImputeWork& w = impute;
  const int L = panel.L;
  w.n = n;
  w.L = L;
  w.Kp = Kp;
  cudaError_t e;
  if ((e = w.mark.ensure((size_t)n * L)) != cudaSuccess) return cuda_fail(e, "alloc mark");
  if ((e = w.polyidx.ensure((size_t)n * L * 4)) != cudaSuccess) return cuda_fail(e, "alloc polyidx");
  if ((e = w.poly.ensure((size_t)n * L * 4)) != cudaSuccess) return cuda_fail(e, "alloc poly");
  if ((e = w.npoly.ensure(n * 4)) != cudaSuccess) return cuda_fail(e, "alloc npoly");
  launch_mark_poly(panel, w, stream);
  launch_compact_poly(panel, w, stream);
  impute_np.assign(n, 0);
  host_nstates.assign(n, 0);
  cudaMemcpyAsync(impute_np.data(), w.npoly.ptr, n * 4, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(host_nstates.data(), w.nstates.ptr, n * 4, cudaMemcpyDeviceToHost, stream);
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "conditioning set");
  for (int i = 0; i < n; ++i)
    if (host_nstates[i] <= 0)
      return (fail(GP_E_DATA, "States for individual " + std::to_string(i) + " are zero. Error during selection."),
              GP_E_DATA);
  int np_max = 1;
  for (int i = 0; i < n; ++i) np_max = std::max(np_max, impute_np[i]);
  w.WB = (np_max + 31) / 32;
  if ((e = w.hvar.ensure((size_t)n * w.WB * w.Kp * 4)) != cudaSuccess) return cuda_fail(e, "alloc hvar");
  launch_build_hvar(panel, w, stream);
  return GP_OK;
}

// Stage selection into impute.states / impute.nstates. Returns the stride Kp.
// The branches of conditioning_set::compactSelection (conditioning_set.cpp:82-121):
// the init selection at the init stage when Kinit > 0; the whole panel when
// Kpbwt >= n_ref_haps; else the PBWT (or learned) selection, which at the init
// stage (Kinit = 0) or with Kpbwt = 0 is empty. The state lists then join every
// set but the whole panel's.
int Context::select_states(int stage, int iteration, int& Kp) {
  TargetWork& T = tw;
  ImputeWork& w = impute;
  const int n = T.n;
  const int N = panel.N;
  const int kinit = std::min(cfg.kinit, N);
  const bool lists = !list_len.empty();
  cudaError_t e;
  int Kmax = 0;
  bool full_panel = false;
  const bool init_sel = stage == GP_STAGE_INIT && kinit > 0;
  if (init_sel) {
    Kmax = kinit;
  } else {
    for (int i = 0; i < n; ++i) {
      const int k = std::min(T.kpbwt_h[i], N);
      if (k >= N) full_panel = true;
      Kmax = std::max(Kmax, k);
    }
    if (full_panel) Kmax = N;
  }
  // no selection: the init stage without Kinit, or Kpbwt = 0 for every target
  const bool empty_sel = !init_sel && !full_panel && (stage == GP_STAGE_INIT || !pbwt_active);
  if (empty_sel) Kmax = 0;
  if (Kmax <= 0 && !lists)
    return (fail(GP_E_ARG, "Kinit/Kpbwt of zero needs a state list (gp_state_lists_set)"), GP_E_ARG);
  if (Kmax > kMaxStates)
    return (fail(GP_E_ARG, "more than " + std::to_string(kMaxStates) + " conditioning states per target"), GP_E_ARG);
  Kp = std::max(32, (Kmax + 31) / 32 * 32);
  if ((e = w.states.ensure((size_t)n * Kp * 4)) != cudaSuccess) return cuda_fail(e, "alloc states");
  if ((e = w.nstates.ensure((size_t)n * 4)) != cudaSuccess) return cuda_fail(e, "alloc nstates");
  int rc = GP_OK;
  if (empty_sel) {
    cudaMemsetAsync(w.nstates.ptr, 0, (size_t)n * 4, stream);
  } else if (init_sel) {
    rc = init_select_states(iteration, Kp, kinit);
  } else if (learned.on && mlp.ready) {
    rc = learned_select_states(stage, iteration, Kp);
  } else {
    rc = pbwt_select_states(stage, iteration, Kp);
  }
  if (rc != GP_OK || !lists || full_panel) return rc;
  return merge_state_lists(Kp);
}

// Init-stage selection (haplotype_set.cpp:775-833) for every target.
int Context::init_select_states(int iteration, int Kp, int kinit) {
  TargetWork& T = tw;
  ImputeWork& w = impute;
  const int n = T.n;
  InitSelArgs a;
  a.gl = T.gl.as<uint8_t>();
  a.flat = T.flat.as<uint8_t>();
  a.ploidy = T.ploidy.as<int32_t>();
  a.common = panel.common;
  a.lq = panel.lq;
  a.major = panel.major;
  a.cref = panel.cref;
  a.calt = panel.calt;
  a.svar_off = panel.svar_off;
  a.svar_haps = panel.svar_haps;
  a.sind = T.sind.as<int32_t>();
  a.nsind = T.nsind.as<int32_t>();
  a.bitmap = T.bitmap.as<uint32_t>();
  a.states = w.states.as<uint32_t>();
  a.nstates = w.nstates.as<int32_t>();
  a.n = n;
  a.L = panel.L;
  a.N = panel.N;
  a.Kp = Kp;
  a.kinit = kinit;
  a.max_mac = host.max_rare_mac;
  a.seed = cfg.seed;
  a.iteration = iteration;
  launch_init_select(a, stream);
  prof.kernel_launches += 2;
  return GP_OK;
}

int Context::iteration(int stage, int iteration) {
  TargetWork& T = tw;
  if (T.n <= 0) return (fail(GP_E_STATE, "no targets"), GP_E_STATE);
  if (stage < GP_STAGE_INIT || stage > GP_STAGE_MAIN) return (fail(GP_E_ARG, "bad stage"), GP_E_ARG);
  const int n = T.n, L = panel.L;
  struct Events {  // destroyed on every return path
    cudaEvent_t ev[6] = {};
    ~Events() {
      for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    }
  } evs;
  cudaEvent_t* ev = evs.ev;
  phase_err_n = 0;
  for (int i = 0; i < 6; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) return cuda_fail(cudaGetLastError(), "iteration events");
  cudaEventRecord(ev[0], stream);
  int Kp = 0;
  int rc = select_states(stage, iteration, Kp);
  if (rc != GP_OK) return rc;
  rc = build_condsets_device(n, Kp);
  if (rc != GP_OK) return rc;
  cudaEventRecord(ev[1], stream);
  // first haplotype (caller_algorithm.cpp:58-65)
  launch_hl(T.gl.as<uint8_t>(), T.flat.as<uint8_t>(), T.ploidy.as<int32_t>(), T.h0.as<uint8_t>(),
            T.h1.as<uint8_t>(), n, L, stage == GP_STAGE_INIT, 0, mc.min_gl, T.hl.as<float>(), stream);
  prof.kernel_launches += 1;
  rc = run_impute(T.hl.as<float>(), T.flat.as<uint8_t>(), T.hp0.as<float>());
  if (rc != GP_OK) return rc;
  launch_sample(T.hp0.as<float>(), T.ploidy.as<int32_t>(), n, L, cfg.seed, RNG_SAMPLE_H0, iteration, 0,
                T.h0.as<uint8_t>(), stream);
  prof.kernel_launches += 1;
  cudaEventRecord(ev[2], stream);
  if (!T.diploid.empty()) {
    // second haplotype and phasing (caller_algorithm.cpp:66-72)
    launch_hl(T.gl.as<uint8_t>(), T.flat.as<uint8_t>(), T.ploidy.as<int32_t>(), T.h0.as<uint8_t>(),
              T.h1.as<uint8_t>(), n, L, 0, 1, mc.min_gl, T.hl.as<float>(), stream);
    prof.kernel_launches += 1;
    rc = run_impute(T.hl.as<float>(), T.flat.as<uint8_t>(), T.hp1.as<float>());
    if (rc != GP_OK) return rc;
    launch_sample(T.hp1.as<float>(), T.ploidy.as<int32_t>(), n, L, cfg.seed, RNG_SAMPLE_H1, iteration, 1,
                  T.h1.as<uint8_t>(), stream);
    prof.kernel_launches += 1;
    cudaEventRecord(ev[3], stream);
    const bool all = (int)T.diploid.size() == n;
    rc = run_phase(all ? nullptr : T.dip_list.as<int32_t>(), all ? std::vector<int32_t>() : T.diploid,
                   (int)T.diploid.size(), T.h0.as<uint8_t>(), T.h1.as<uint8_t>(), T.flat.as<uint8_t>(), iteration,
                   nullptr);
    if (rc != GP_OK) return rc;
  } else {
    cudaEventRecord(ev[3], stream);
  }
  cudaEventRecord(ev[4], stream);
  if (stage == GP_STAGE_MAIN) {
    launch_gp_store(T.hp0.as<float>(), T.hp1.as<float>(), T.ploidy.as<int32_t>(), n, L, T.stored_cnt,
                    T.gp0.as<float>(), T.gp1.as<float>(), T.gpflags.as<uint8_t>(), stream);
    prof.kernel_launches += 1;
    T.stored_cnt++;
  }
  cudaEventRecord(ev[5], stream);
  cudaError_t e = cudaEventSynchronize(ev[5]);
  if (e != cudaSuccess) return cuda_fail(e, "iteration");
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "iteration launch");
  for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
  prof.select_ms += stage_ms[0];
  prof_resolve();
  return check_phase_errors();
}

int Context::finalize() {
  TargetWork& T = tw;
  if (T.n <= 0) return (fail(GP_E_STATE, "no targets"), GP_E_STATE);
  if (T.stored_cnt == 0) return (fail(GP_E_STATE, "no main iteration ran"), GP_E_STATE);
  launch_gp_finalize(T.ploidy.as<int32_t>(), T.n, panel.L, T.stored_cnt, T.gpflags.as<uint8_t>(), T.gp0.as<float>(),
                     T.gp1.as<float>(), T.ds.as<float>(), T.gt0.as<uint8_t>(), T.gt1.as<uint8_t>(),
                     T.h0.as<uint8_t>(), T.h1.as<uint8_t>(), stream);
  prof.kernel_launches += 1;
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "finalize");
  T.finalized = true;
  return GP_OK;
}

}  // namespace gp

using gp::Context;

static Context* C_(gp_ctx* c) { return reinterpret_cast<Context*>(c); }

extern "C" {

int gp_targets_set(gp_ctx* ctx, int32_t n, const uint8_t* gl, const uint8_t* flat, const int32_t* ploidy,
                   const int32_t* kpbwt) {
  if (!ctx) return GP_E_ARG;
  if (n <= 0 || !gl || !flat || !ploidy) return (C_(ctx)->fail(GP_E_ARG, "targets: bad argument"), GP_E_ARG);
  if (n > GP_MAX_TARGETS)
    return (C_(ctx)->fail(GP_E_ARG, "targets: more than " + std::to_string(GP_MAX_TARGETS) + " targets per context"),
            GP_E_ARG);
  return C_(ctx)->set_targets(n, gl, flat, ploidy, kpbwt);
}

int gp_iteration(gp_ctx* ctx, int32_t stage, int32_t iteration) {
  if (!ctx) return GP_E_ARG;
  return C_(ctx)->iteration(stage, iteration);
}

int gp_select(gp_ctx* ctx, int32_t stage, int32_t iteration) {
  if (!ctx) return GP_E_ARG;
  Context& c = *C_(ctx);
  if (c.tw.n <= 0) return (c.fail(GP_E_STATE, "no targets"), GP_E_STATE);
  int Kp = 0;
  int rc = c.select_states(stage, iteration, Kp);
  if (rc != GP_OK) return rc;
  c.impute.n = c.tw.n;
  c.impute.Kp = Kp;
  c.host_nstates.assign(c.tw.n, 0);
  cudaMemcpyAsync(c.host_nstates.data(), c.impute.nstates.ptr, c.tw.n * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "select");
}

int gp_run(gp_ctx* ctx, int32_t burnin, int32_t main) {
  if (!ctx) return GP_E_ARG;
  Context& c = *C_(ctx);
  if (burnin < 0 || main < 1 || main > 15)
    return (c.fail(GP_E_ARG, "Maximum value for --main is 15"), GP_E_ARG);  // caller_parameters.cpp:139-140
  int it = 0;
  int rc = c.iteration(GP_STAGE_INIT, it++);
  for (int i = 0; rc == GP_OK && i < burnin; ++i) rc = c.iteration(GP_STAGE_BURN, it++);
  for (int i = 0; rc == GP_OK && i < main; ++i) rc = c.iteration(GP_STAGE_MAIN, it++);
  if (rc == GP_OK) rc = c.finalize();
  return rc;
}

int gp_finalize(gp_ctx* ctx) {
  if (!ctx) return GP_E_ARG;
  return C_(ctx)->finalize();
}

int gp_haps_get(gp_ctx* ctx, uint8_t* h0, uint8_t* h1) {
  if (!ctx || !h0 || !h1) return GP_E_ARG;
  Context& c = *C_(ctx);
  const size_t nL = (size_t)c.tw.n * c.panel.L;
  cudaMemcpyAsync(h0, c.tw.h0.ptr, nL, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(h1, c.tw.h1.ptr, nL, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "haps_get");
}

int gp_haps_set(gp_ctx* ctx, const uint8_t* h0, const uint8_t* h1) {
  if (!ctx || !h0 || !h1) return GP_E_ARG;
  Context& c = *C_(ctx);
  const size_t nL = (size_t)c.tw.n * c.panel.L;
  cudaMemcpyAsync(c.tw.h0.ptr, h0, nL, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.tw.h1.ptr, h1, nL, cudaMemcpyHostToDevice, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "haps_set");
}

int gp_posteriors_get(gp_ctx* ctx, int32_t target, float* hp0, float* hp1) {
  if (!ctx || !hp0) return GP_E_ARG;
  Context& c = *C_(ctx);
  if (target < 0 || target >= c.tw.n) return (c.fail(GP_E_ARG, "target out of range"), GP_E_ARG);
  const size_t L2 = (size_t)c.panel.L * 2;
  cudaMemcpyAsync(hp0, c.tw.hp0.as<float>() + target * L2, L2 * 4, cudaMemcpyDeviceToHost, c.stream);
  if (hp1) cudaMemcpyAsync(hp1, c.tw.hp1.as<float>() + target * L2, L2 * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "posteriors_get");
}

int gp_states_get(gp_ctx* ctx, int32_t target, uint32_t* states, int32_t* n_out) {
  if (!ctx || !states || !n_out) return GP_E_ARG;
  Context& c = *C_(ctx);
  if (target < 0 || target >= c.impute.n) return (c.fail(GP_E_ARG, "target out of range"), GP_E_ARG);
  const int K = c.host_nstates[target];
  cudaMemcpyAsync(states, c.impute.states.as<uint32_t>() + (size_t)target * c.impute.Kp, K * 4,
                  cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  *n_out = K;
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "states_get");
}

int gp_gp_get(gp_ctx* ctx, float* gp0, float* gp1, float* ds, uint8_t* gt0, uint8_t* gt1) {
  if (!ctx) return GP_E_ARG;
  Context& c = *C_(ctx);
  if (!c.tw.finalized) return (c.fail(GP_E_STATE, "gp_finalize has not run"), GP_E_STATE);
  const size_t nL = (size_t)c.tw.n * c.panel.L;
  if (gp0) cudaMemcpyAsync(gp0, c.tw.gp0.ptr, nL * 4, cudaMemcpyDeviceToHost, c.stream);
  if (gp1) cudaMemcpyAsync(gp1, c.tw.gp1.ptr, nL * 4, cudaMemcpyDeviceToHost, c.stream);
  if (ds) cudaMemcpyAsync(ds, c.tw.ds.ptr, nL * 4, cudaMemcpyDeviceToHost, c.stream);
  if (gt0) cudaMemcpyAsync(gt0, c.tw.gt0.ptr, nL, cudaMemcpyDeviceToHost, c.stream);
  if (gt1) cudaMemcpyAsync(gt1, c.tw.gt1.ptr, nL, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "gp_get");
}

int gp_gp_accum_get(gp_ctx* ctx, int32_t target, float* gp0, float* gp1, uint8_t* flags) {
  if (!ctx || !gp0 || !gp1 || !flags) return GP_E_ARG;
  Context& c = *C_(ctx);
  if (target < 0 || target >= c.tw.n) return (c.fail(GP_E_ARG, "target out of range"), GP_E_ARG);
  const size_t L = c.panel.L, o = (size_t)target * L;
  cudaMemcpyAsync(gp0, c.tw.gp0.as<float>() + o, L * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(gp1, c.tw.gp1.as<float>() + o, L * 4, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(flags, c.tw.gpflags.as<uint8_t>() + o, L, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return c.cuda_fail(e, "gp_accum_get");
  for (size_t l = 0; l < L; ++l)
    if (!(flags[l] & 1)) gp0[l] = gp1[l] = 0.0f;
  return GP_OK;
}

int gp_targets_reset(gp_ctx* ctx) {
  if (!ctx) return GP_E_ARG;
  Context& c = *C_(ctx);
  gp::TargetWork& T = c.tw;
  if (T.n <= 0) return (c.fail(GP_E_STATE, "no targets"), GP_E_STATE);
  const size_t nL = (size_t)T.n * c.panel.L;
  cudaMemsetAsync(T.h0.ptr, 0, nL, c.stream);
  cudaMemsetAsync(T.h1.ptr, 0, nL, c.stream);
  cudaMemsetAsync(T.gpflags.ptr, 0, nL, c.stream);
  cudaMemsetAsync(T.gp0.ptr, 0, nL * 4, c.stream);
  cudaMemsetAsync(T.gp1.ptr, 0, nL * 4, c.stream);
  cudaMemsetAsync(T.tar_hap.ptr, 0, T.hap_target.size(), c.stream);
  T.stored_cnt = 0;
  T.finalized = false;
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "targets_reset");
}

int gp_profile_get(gp_ctx* ctx, gp_profile* out) {
  if (!ctx || !out) return GP_E_ARG;
  Context& c = *C_(ctx);
  c.prof_resolve();
  *out = c.prof;
  return GP_OK;
}

int gp_profile_reset(gp_ctx* ctx) {
  if (!ctx) return GP_E_ARG;
  Context& c = *C_(ctx);
  c.prof_resolve();
  c.prof = gp_profile{};
  return GP_OK;
}

void* gp_stream(gp_ctx* ctx) { return ctx ? (void*)C_(ctx)->stream : nullptr; }

int gp_stage_times(gp_ctx* ctx, float* ms, int32_t n) {
  if (!ctx || !ms) return GP_E_ARG;
  Context& c = *C_(ctx);
  for (int i = 0; i < n && i < 5; ++i) ms[i] = c.stage_ms[i];
  return GP_OK;
}

}  // extern "C"
