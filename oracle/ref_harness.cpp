// ORACLE — test infrastructure only. Never linked into the product library.
//
// C-ABI harness around the reference's own hot-path classes, compiled
// unmodified from the reference tree (oracle/Makefile). It restates the
// GLIMPSE2_phase driver (phase/src/caller/caller_algorithm.cpp:53-126,223-243)
// without htslib/Boost I/O, fills the panel in memory instead of reading a
// binary archive, and selects the replay-RNG stream before every call that
// draws random numbers, so that the GPU path can be compared call by call.
//
// Used by tests/ (parity), __graft_entry__.smoke() (check only) and bench.py's
// reference arm / cpu_baseline leg (timing of the reference's CPU path).
#include <atomic>
#include <thread>
#include <mutex>
#include <memory>

// Everything the model headers include is pulled in first, so that the
// access-specifier override below only reaches the two model classes (their
// private message buffers are read back for parity checks).
#include <utils/otools.h>
#include "../glimpse_b200/csrc/replay_rng.h"
#include <containers/bitmatrix.h>
#include <containers/variant_map.h>
#include <containers/haplotype_set.h>
#include <containers/conditioning_set.h>
#define private public
#define protected public
#include <models/imputation_hmm.h>
#include <models/phasing_hmm.h>
#undef private
#undef protected
#include <containers/conditioning_set.h>
#include <containers/haplotype_set.h>
#include <containers/genotype_set.h>
#include <containers/variant_map.h>
#include <objects/genotype.h>

thread_local random_number_generator rng;
verbose vrb;
string_utils stb;
timer tac;

namespace {

// Stream control. The replay engine is pointed at the (purpose, iteration,
// target) stream before each call that draws. The native-RNG build (the
// reference's own std::mt19937, GP_NATIVE_RNG) is seeded once, as
// caller_initialise.cpp:49 does, and draws in the reference's call order, so
// both are no-ops there.
#ifdef GP_NATIVE_RNG
constexpr bool kNativeRng = true;
inline void rng_select(uint32_t, uint32_t, uint32_t) {}
inline void rng_reseed(uint64_t) {}
#else
constexpr bool kNativeRng = false;
inline void rng_select(uint32_t purpose, uint32_t iteration, uint32_t target) {
  rng.randomEngine.select(purpose, iteration, target);
}
inline void rng_reseed(uint64_t seed) { rng.randomEngine.seed_with(seed); }
#endif

struct Worker {
  std::unique_ptr<conditioning_set> cond;
  std::unique_ptr<imputation_hmm> hmm;
  std::unique_ptr<phasing_hmm> dmm;
  std::vector<float> HLC, HP0, HP1;
};

struct Oracle {
  variant_map V;
  haplotype_set H;
  genotype_set G;
  // configuration (caller_parameters.cpp defaults unless set)
  int ne = 100000;
  float err_imp = 1e-12f, err_phase = 1e-4f, min_gl = 1e-10f;
  int pbwt_depth = 12;
  float pbwt_modulo_cm = 0.1f;
  int kinit = 1000, kpbwt = 2000;
  std::vector<int> kpbwt_target;  // per-target Kpbwt (conditioning_set::Kpbwt)
  uint64_t seed = 15052011ull;
  bool configured = false;
  // per-target records of the last iteration, for parity checks
  std::vector<std::vector<unsigned int>> last_states;
  std::vector<std::vector<float>> last_HP0, last_HP1;
  std::vector<int> last_npoly;
  std::string err;
};

std::unique_ptr<Worker> make_worker(Oracle& o, int kp) {
  auto w = std::make_unique<Worker>();
  const int kpbwt = std::min(kp, (int)o.H.n_ref_haps);
  const int kinit = std::min(o.kinit, (int)o.H.n_ref_haps);
  const float err_imp = std::clamp(o.err_imp, 1e-12f, 1e-3f);  // caller_initialise.cpp:152
  w->cond.reset(new conditioning_set(o.V, o.H, o.H.n_ref_haps, o.ne, kinit, kpbwt, err_imp, o.err_phase, false));
  w->hmm.reset(new imputation_hmm(w->cond.get()));
  w->dmm.reset(new phasing_hmm(w->cond.get()));
  w->HLC.assign(o.H.n_tot_sites * 2, 0.0f);
  w->HP0.assign(o.H.n_tot_sites * 2, 0.0f);
  w->HP1.assign(o.H.n_tot_sites * 2, 0.0f);
  return w;
}

// caller::phase_individual (caller_algorithm.cpp:53-84) with replay streams.
void phase_individual(Oracle& o, Worker& w, int ind, int stage, int iter_index) {
  genotype* g = o.G.vecG[ind];
  const int ploidy = g->ploidy;
  w.cond->Kpbwt = std::min(o.kpbwt_target[ind], (int)o.H.n_ref_haps);
  w.cond->select(ind, stage);
  if (stage == STAGE_INIT) g->initHaplotypeLikelihoods(w.HLC, o.min_gl);
  else {
    if (ploidy > 1) g->makeHaplotypeLikelihoods(w.HLC, true, o.min_gl);
    else g->initHaplotypeLikelihoods(w.HLC, o.min_gl);
  }
  w.hmm->computePosteriors(w.HLC, g->flat, w.HP0);
  rng_select(gp::RNG_SAMPLE_H0, iter_index, ind);
  g->sampleHaplotypeH0(w.HP0);
  if (ploidy > 1) {
    g->makeHaplotypeLikelihoods(w.HLC, false, o.min_gl);
    w.hmm->computePosteriors(w.HLC, g->flat, w.HP1);
    rng_select(gp::RNG_SAMPLE_H1, iter_index, ind);
    g->sampleHaplotypeH1(w.HP1);
    rng_select(gp::RNG_PHASE, iter_index, ind);
    w.dmm->rephaseHaplotypes(g->H0, g->H1, g->flat);
  }
  if (stage == STAGE_MAIN) {
    if (ploidy > 1) g->storeGenotypePosteriorsAndHaplotypes(w.HP0, w.HP1);
    else g->storeGenotypePosteriorsAndHaplotypes(w.HP0);
  }
  o.last_states[ind] = w.cond->idxHaps_ref;
  o.last_HP0[ind] = w.HP0;
  if (ploidy > 1) o.last_HP1[ind] = w.HP1;
  o.last_npoly[ind] = (int)w.cond->polymorphic_sites.size();
}

// Init-stage selection (haplotype_set.cpp:775-833) run one target at a time so
// that each target draws from its own stream (target index moved to slot 0).
// The native-RNG build runs it over all targets in one call, as
// caller_algorithm.cpp:91 does.
void init_selection(Oracle& o, int iter_index) {
  haplotype_set& H = o.H;
  if (H.Kinit == 0) return;
  if (kNativeRng) {
    H.performSelection_RARE_INIT_GL(o.V);
    return;
  }
  std::vector<std::vector<int>> sind = H.SindTarGL;
  const unsigned int n_tar = H.n_tar_samples;
  std::vector<std::set<int>> result(n_tar);
  std::vector<int> ind2hap = H.tar_ind2hapid;
  for (unsigned int i = 0; i < n_tar; ++i) {
    H.n_tar_samples = 1;
    H.SindTarGL.assign(1, sind[i]);
    H.init_states.assign(1, std::set<int>());
    H.tar_ind2hapid.assign(1, ind2hap[i]);
    rng_select(gp::RNG_INIT_SEL, iter_index, i);
    H.performSelection_RARE_INIT_GL(o.V);
    result[i] = H.init_states[0];
  }
  H.n_tar_samples = n_tar;
  H.tar_ind2hapid = ind2hap;
  H.init_states = result;
  H.SindTarGL.clear();
}

// caller::phase_iteration (caller_algorithm.cpp:86-126) without checkpoint.
void phase_iteration(Oracle& o, int stage, int iter_index, int n_threads) {
  if (kNativeRng && n_threads > 1)
    throw std::runtime_error("the reference's own generator is one global stream: run it on one thread");
  if (stage == STAGE_INIT) {
    o.H.initRareTar(o.G, o.V);
    init_selection(o, iter_index);
  } else {
    o.H.updateHaplotypes(o.G);
    o.H.transposeRareTar();
    rng_select(gp::RNG_PBWT, iter_index, 0);
    o.H.matchHapsFromCompressedPBWTSmall(o.V, stage == STAGE_MAIN);
  }
  const int n_ind = o.G.n_ind;
  if (n_threads <= 1) {
    auto w = make_worker(o, o.kpbwt);
    for (int i = 0; i < n_ind; ++i) phase_individual(o, *w, i, stage, iter_index);
  } else {
    std::atomic<int> next{0};
    std::mutex emu;
    std::string first_err;
    std::vector<std::thread> pool;
    for (int t = 0; t < n_threads; ++t) {
      pool.emplace_back([&]() {
        rng.setSeed((unsigned int)o.seed);
        rng_reseed(o.seed);
        auto w = make_worker(o, o.kpbwt);
        for (;;) {
          const int i = next.fetch_add(1);
          if (i >= n_ind) break;
          try {
            phase_individual(o, *w, i, stage, iter_index);
          } catch (const std::exception& e) {
            std::lock_guard<std::mutex> lk(emu);
            if (first_err.empty()) first_err = e.what();
          }
        }
      });
    }
    for (auto& th : pool) th.join();
    if (!first_err.empty()) throw std::runtime_error(first_err);
  }
  if (stage == STAGE_INIT) {
    o.H.init_states.clear();
    o.H.init_states.shrink_to_fit();
  }
}

template <class F>
int guarded(Oracle* o, F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    if (o) o->err = e.what();
    return 1;
  }
}

}  // namespace

extern "C" {

// Panel in the reference's in-memory representation (ref_haplotype_set.h:60-75,
// variant.h:33-45). hvar: n_com rows of ceil(n_ref_haps/8) bytes, MSB first.
// shap_off/shap_sites: ShapRef as CSR over reference haplotypes.
void* orc_create(int n_ref_haps, int n_sites, const int* bp, const double* cm, const uint32_t* cref,
                 const uint32_t* calt, const uint8_t* lq, const uint8_t* flag_common, const uint8_t* major,
                 const uint8_t* hvar, const int64_t* shap_off, const int32_t* shap_sites) {
  Oracle* o = new Oracle();
  int rc = guarded(o, [&]() {
    haplotype_set& H = o->H;
    for (int l = 0; l < n_sites; ++l) {
      variant* v = new variant(bp[l], std::to_string(l), "A", "C", 1, l, cref[l], calt[l], !lq[l]);
      v->cm = cm[l];
      o->V.push(v);
    }
    H.n_ref_haps = n_ref_haps;
    H.n_tot_sites = n_sites;
    H.n_com_sites = 0;
    H.n_rar_sites = 0;
    H.n_com_sites_hq = 0;
    H.flag_common.clear();
    H.major_alleles.clear();
    H.common2tot.clear();
    for (int l = 0; l < n_sites; ++l) {
      H.flag_common.push_back(flag_common[l] != 0);
      H.major_alleles.push_back(major[l] != 0);
      if (flag_common[l]) {
        H.common2tot.push_back(l);
        H.n_com_sites++;
        if (!lq[l]) H.n_com_sites_hq++;
      } else {
        H.n_rar_sites++;
      }
    }
    H.ref_haplotype_set::allocate();
    const size_t stride = (size_t)H.HvarRef.n_cols / 8;
    const size_t in_stride = ((size_t)n_ref_haps + 7) / 8;
    for (unsigned int r = 0; r < H.n_com_sites; ++r)
      std::memcpy(H.HvarRef.bytes + r * stride, hvar + r * in_stride, in_stride);
    for (int h = 0; h < n_ref_haps; ++h)
      for (int64_t j = shap_off[h]; j < shap_off[h + 1]; ++j) H.ShapRef[h].push_back(shap_sites[j]);
    H.build_sparsePBWT(o->V);
  });
  if (rc) {
    std::fprintf(stderr, "orc_create: %s\n", o->err.c_str());
    delete o;
    return nullptr;
  }
  return o;
}

void orc_destroy(void* p) { delete static_cast<Oracle*>(p); }
const char* orc_last_error(void* p) { return static_cast<Oracle*>(p)->err.c_str(); }

int64_t orc_ypacked(void* p, uint8_t* out, int64_t cap) {
  Oracle* o = static_cast<Oracle*>(p);
  const int64_t n = (int64_t)o->H.Ypacked.size();
  if (out) std::memcpy(out, o->H.Ypacked.data(), std::min(n, cap));
  return n;
}

// A_small_idx as CSR: returns total count; off has n_com_sites_hq + 2 entries.
int64_t orc_asmall(void* p, int64_t* off, int32_t* vals, int64_t cap) {
  Oracle* o = static_cast<Oracle*>(p);
  int64_t tot = 0;
  const auto& A = o->H.A_small_idx;
  for (size_t i = 0; i < A.size(); ++i) {
    if (off) off[i] = tot;
    for (int v : A[i]) {
      if (vals && tot < cap) vals[tot] = v;
      ++tot;
    }
  }
  if (off) off[A.size()] = tot;
  return tot;
}
int orc_asmall_rows(void* p) { return (int)static_cast<Oracle*>(p)->H.A_small_idx.size(); }

// Targets: GL is n_tar x (3 * n_sites) phred bytes, (ploidy+1) used per site;
// flat is n_tar x n_sites.
int orc_targets(void* p, int n_tar, const int* ploidy, const uint8_t* GL, const uint8_t* flat) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    haplotype_set& H = o->H;
    const int L = H.n_tot_sites;
    H.n_tar_samples = n_tar;
    H.tar_ploidy.clear();
    H.tar_ind2hapid.clear();
    H.max_ploidy = 1;
    int hap = 0;
    bool any1 = false, any2 = false;
    for (int i = 0; i < n_tar; ++i) {
      H.tar_ploidy.push_back(ploidy[i]);
      H.tar_ind2hapid.push_back(hap);
      hap += ploidy[i];
      H.max_ploidy = std::max(H.max_ploidy, ploidy[i]);
      (ploidy[i] == 1 ? any1 : any2) = true;
    }
    H.fploidy = (any1 && any2) ? -2 : (any2 ? 2 : 1);
    H.n_tar_haps = hap;
    o->G.n_ind = n_tar;
    o->G.n_site = L;
    o->G.n_hap = hap;
    for (int i = 0; i < n_tar; ++i) {
      genotype* g = new genotype("t" + std::to_string(i), i, L, ploidy[i], H.tar_ind2hapid[i]);
      g->allocate();
      const int pp1 = ploidy[i] + 1;
      for (int l = 0; l < L; ++l) {
        for (int a = 0; a < pp1; ++a) g->GL[pp1 * l + a] = GL[(size_t)i * 3 * L + 3 * l + a];
        g->flat[l] = flat[(size_t)i * L + l] != 0;
      }
      o->G.vecG.push_back(g);
    }
    H.allocate_hap_only();
    H.transposeRareRef();
    o->last_states.assign(n_tar, {});
    o->last_HP0.assign(n_tar, {});
    o->last_HP1.assign(n_tar, {});
    o->last_npoly.assign(n_tar, 0);
  });
}

int orc_config(void* p, int ne, float err_imp, float err_phase, float min_gl, int pbwt_depth, float pbwt_modulo_cm,
               int kinit, int kpbwt, const int* kpbwt_target, uint64_t seed) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    o->ne = ne;
    o->err_imp = err_imp;
    o->err_phase = err_phase;
    o->min_gl = min_gl;
    o->pbwt_depth = pbwt_depth;
    o->pbwt_modulo_cm = pbwt_modulo_cm;
    o->kinit = kinit;
    o->kpbwt = kpbwt;
    o->seed = seed;
    o->kpbwt_target.assign(o->G.n_ind, kpbwt);
    if (kpbwt_target)
      for (int i = 0; i < o->G.n_ind; ++i) o->kpbwt_target[i] = kpbwt_target[i];
    rng.setSeed((unsigned int)seed);
    rng_reseed(seed);
    const int kp = std::min(kpbwt, (int)o->H.n_ref_haps);
    const int ki = std::min(kinit, (int)o->H.n_ref_haps);
    o->H.allocatePBWT(pbwt_depth, pbwt_modulo_cm, o->V, o->G, ki, kp);
    o->configured = true;
  });
}

// One Gibbs iteration: stage 0 init, 1 burn-in, 2 main. iter_index keys the streams.
int orc_iteration(void* p, int stage, int iter_index, int n_threads) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    rng_reseed(o->seed);
    phase_iteration(*o, stage, iter_index, n_threads);
  });
}

// caller::phase_loop tail (caller_algorithm.cpp:239-240).
int orc_finalize(void* p) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    for (auto* g : o->G.vecG) g->sortAndNormAndInferGenotype();
  });
}

int orc_get_haps(void* p, int ind, uint8_t* H0, uint8_t* H1) {
  Oracle* o = static_cast<Oracle*>(p);
  genotype* g = o->G.vecG[ind];
  for (int l = 0; l < g->n_variants; ++l) {
    H0[l] = g->H0[l];
    if (H1) H1[l] = g->ploidy > 1 ? g->H1[l] : 0;
  }
  return 0;
}

int orc_set_haps(void* p, int ind, const uint8_t* H0, const uint8_t* H1) {
  Oracle* o = static_cast<Oracle*>(p);
  genotype* g = o->G.vecG[ind];
  for (int l = 0; l < g->n_variants; ++l) {
    g->H0[l] = H0[l] != 0;
    if (g->ploidy > 1 && H1) g->H1[l] = H1[l] != 0;
  }
  return 0;
}

// Sparse GP storage (genotype.h:38-78) exported densely: stored[l] = 1 where an
// entry exists; gp0/gp1/hds then hold its values; stored_cnt returned.
int orc_get_gp(void* p, int ind, float* gp0, float* gp1, uint8_t* hds, uint8_t* stored) {
  Oracle* o = static_cast<Oracle*>(p);
  genotype* g = o->G.vecG[ind];
  for (int l = 0; l < g->n_variants; ++l) {
    gp0[l] = 1.0f; gp1[l] = 0.0f; hds[l] = 0; stored[l] = 0;
  }
  for (const auto& e : g->stored_data) {
    gp0[e.idx] = e.gp0; gp1[e.idx] = e.gp1; hds[e.idx] = e.hds; stored[e.idx] = 1;
  }
  return g->stored_cnt;
}

int orc_last_states(void* p, int ind, uint32_t* out, int cap) {
  Oracle* o = static_cast<Oracle*>(p);
  const auto& s = o->last_states[ind];
  for (int i = 0; i < (int)s.size() && i < cap; ++i) out[i] = s[i];
  return (int)s.size();
}

int orc_last_hp(void* p, int ind, float* HP0, float* HP1) {
  Oracle* o = static_cast<Oracle*>(p);
  const auto& a = o->last_HP0[ind];
  std::copy(a.begin(), a.end(), HP0);
  if (HP1 && !o->last_HP1[ind].empty()) std::copy(o->last_HP1[ind].begin(), o->last_HP1[ind].end(), HP1);
  return o->last_npoly[ind];
}

// PBWT selection only (haplotype_set.cpp:317-394) from the current target
// haplotypes, then pbwt_states per target and level.
int orc_pbwt_select(void* p, int iter_index, int main_iteration) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    o->H.updateHaplotypes(o->G);
    o->H.transposeRareTar();
    rng_reseed(o->seed);
    rng_select(gp::RNG_PBWT, iter_index, 0);
    o->H.matchHapsFromCompressedPBWTSmall(o->V, main_iteration != 0);
  });
}

int orc_pbwt_levels(void* p, int ind) { return (int)static_cast<Oracle*>(p)->H.pbwt_states[ind].size(); }
int orc_pbwt_states(void* p, int ind, int level, int32_t* out, int cap) {
  Oracle* o = static_cast<Oracle*>(p);
  const auto& v = o->H.pbwt_states[ind][level];
  for (int i = 0; i < (int)v.size() && i < cap; ++i) out[i] = v[i];
  return (int)v.size();
}
int orc_pbwt_nstored(void* p) { return static_cast<Oracle*>(p)->H.nstored; }
float orc_pbwt_modulo(void* p) { return static_cast<Oracle*>(p)->H.pbwt_modulo_cm; }
int orc_pbwt_groups(void* p, int32_t* out, int cap) {
  Oracle* o = static_cast<Oracle*>(p);
  const auto& g = o->H.pbwt_grp;
  for (int i = 0; i < (int)g.size() && i < cap; ++i) out[i] = g[i];
  return (int)g.size();
}

// conditioning_set::select for target ind at `stage` (uses the last PBWT /
// init selection); returns n_states and fills idxHaps_ref.
int orc_select(void* p, int ind, int stage, uint32_t* out, int cap) {
  Oracle* o = static_cast<Oracle*>(p);
  int n = -1;
  guarded(o, [&]() {
    auto w = make_worker(*o, o->kpbwt_target[ind]);
    w->cond->select(ind, stage);
    const auto& s = w->cond->idxHaps_ref;
    for (int i = 0; i < (int)s.size() && i < cap; ++i) out[i] = s[i];
    n = (int)s.size();
  });
  return n;
}

// Init-stage selection only (haplotype_set.cpp:108-169,775-833).
int orc_init_select(void* p, int iter_index) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    o->H.initRareTar(o->G, o->V);
    init_selection(*o, iter_index);
  });
}
// haplotype_set::read_list_states (haplotype_set.cpp:835-857) from memory: row
// h of the --state-list file is ids[off[h] .. off[h+1]). n_haps = 0 clears.
int orc_state_lists(void* p, int n_haps, const int64_t* off, const int32_t* ids) {
  Oracle* o = static_cast<Oracle*>(p);
  return guarded(o, [&]() {
    haplotype_set& H = o->H;
    H.list_states.assign(H.n_tar_haps, std::vector<int>());
    for (int h = 0; h < n_haps && h < (int)H.n_tar_haps; ++h) H.list_states[h].assign(ids + off[h], ids + off[h + 1]);
  });
}

int orc_init_states(void* p, int ind, int32_t* out, int cap) {
  Oracle* o = static_cast<Oracle*>(p);
  const auto& s = o->H.init_states[ind];
  int i = 0;
  for (int v : s) {
    if (i < cap) out[i] = v;
    ++i;
  }
  return (int)s.size();
}

// One imputation_hmm::computePosteriors call (imputation_hmm.cpp:136-141) with
// an explicit conditioning set, passed through the state-list path of
// conditioning_set::compactSelection (conditioning_set.cpp:114-121).
// Also returns the conditioning set's polymorphic site list.
int orc_impute(void* p, const uint32_t* states, int K, const float* HL, const uint8_t* flat, float* HP,
               int32_t* poly_out) {
  Oracle* o = static_cast<Oracle*>(p);
  int npoly = -1;
  guarded(o, [&]() {
    haplotype_set& H = o->H;
    const int L = H.n_tot_sites;
    if (H.list_states.size() < 1) H.list_states.resize(std::max(1u, H.n_tar_haps));
    std::vector<std::vector<int>> saved = H.list_states;
    H.list_states[0].assign(states, states + K);
    if (H.list_states.size() > 1) H.list_states[1].clear();
    const float err_imp = std::clamp(o->err_imp, 1e-12f, 1e-3f);
    conditioning_set C(o->V, H, H.n_ref_haps, o->ne, 0, 0, err_imp, o->err_phase, false);
    C.select(0, STAGE_MAIN);
    H.list_states = saved;
    imputation_hmm M(&C);
    std::vector<float> hl(HL, HL + 2 * L), hp(2 * L, 0.0f);
    std::vector<bool> fl(L);
    for (int l = 0; l < L; ++l) fl[l] = flat[l] != 0;
    M.computePosteriors(hl, fl, hp);
    std::copy(hp.begin(), hp.end(), HP);
    npoly = (int)C.polymorphic_sites.size();
    if (poly_out)
      for (int i = 0; i < npoly; ++i) poly_out[i] = C.polymorphic_sites[i];
  });
  return npoly;
}

// One phasing_hmm::rephaseHaplotypes call (phasing_hmm.cpp:247-302) with an
// explicit conditioning set and the stream (RNG_PHASE, iter_index, target).
// dip_out (optional, cap entries) receives dip_sampled; returns n_segs.
int orc_rephase(void* p, const uint32_t* states, int K, uint8_t* H0, uint8_t* H1, const uint8_t* flat,
                int iter_index, int target, int32_t* dip_out, int cap) {
  Oracle* o = static_cast<Oracle*>(p);
  int nseg = -1;
  guarded(o, [&]() {
    haplotype_set& H = o->H;
    const int L = H.n_tot_sites;
    if (H.list_states.size() < 1) H.list_states.resize(std::max(1u, H.n_tar_haps));
    std::vector<std::vector<int>> saved = H.list_states;
    H.list_states[0].assign(states, states + K);
    if (H.list_states.size() > 1) H.list_states[1].clear();
    const float err_imp = std::clamp(o->err_imp, 1e-12f, 1e-3f);
    conditioning_set C(o->V, H, H.n_ref_haps, o->ne, 0, 0, err_imp, o->err_phase, false);
    C.select(0, STAGE_MAIN);
    H.list_states = saved;
    phasing_hmm D(&C);
    std::vector<bool> h0(L), h1(L), fl(L);
    for (int l = 0; l < L; ++l) {
      h0[l] = H0[l] != 0;
      h1[l] = H1[l] != 0;
      fl[l] = flat[l] != 0;
    }
    rng_reseed(o->seed);
    rng_select(gp::RNG_PHASE, iter_index, target);
    D.rephaseHaplotypes(h0, h1, fl);
    for (int l = 0; l < L; ++l) {
      H0[l] = h0[l];
      H1[l] = h1[l];
    }
    nseg = (int)D.n_segs;
    if (dip_out)
      for (int i = 0; i < (int)D.dip_sampled.size() && i < cap; ++i) dip_out[i] = D.dip_sampled[i];
  });
  return nseg;
}

// Reference unphred table (otools.h:98) for fixture generation.
void orc_unphred(float* out) {
  for (int i = 0; i < 256; ++i) out[i] = unphred[i];
}

// Replay stream words, to check the device generator against the host.
void orc_stream_words(uint64_t seed, uint32_t purpose, uint32_t iteration, uint32_t target, uint64_t start,
                      int n, uint32_t* out) {
  for (int i = 0; i < n; ++i) out[i] = gp::stream_word(seed, purpose, iteration, target, start + i);
}

// Raw Philox4x32-10 block, for known-answer tests of the stream generator.
void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  gp::philox4x32_10(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1], out);
}

#ifndef GP_NATIVE_RNG
// getFloat / getInt through the shimmed reference RNG class (replay build only).
void orc_rng_floats(uint64_t seed, uint32_t purpose, uint32_t iteration, uint32_t target, int n, float* out) {
  random_number_generator r;
  r.randomEngine.seed_with(seed);
  r.randomEngine.select(purpose, iteration, target);
  for (int i = 0; i < n; ++i) out[i] = (float)r.getFloat();
}
void orc_rng_ints(uint64_t seed, uint32_t purpose, uint32_t iteration, uint32_t target, int n, const uint32_t* lo,
                  const uint32_t* hi, uint32_t* out, uint64_t* words_used) {
  random_number_generator r;
  r.randomEngine.seed_with(seed);
  r.randomEngine.select(purpose, iteration, target);
  for (int i = 0; i < n; ++i) out[i] = r.getInt(lo[i], hi[i]);
  *words_used = r.randomEngine.pos;
}
// std::sample over [0, pop) through the shimmed engine (selection sampling).
int orc_std_sample(uint64_t seed, uint32_t purpose, uint32_t iteration, uint32_t target, int pop, int n,
                   int32_t* out, uint64_t* words_used) {
  random_number_generator r;
  r.randomEngine.seed_with(seed);
  r.randomEngine.select(purpose, iteration, target);
  std::vector<int> iota(pop);
  std::iota(iota.begin(), iota.end(), 0);
  std::vector<int> s;
  std::sample(iota.begin(), iota.end(), std::back_inserter(s), n, r.randomEngine);
  for (size_t i = 0; i < s.size(); ++i) out[i] = s[i];
  *words_used = r.randomEngine.pos;
  return (int)s.size();
}
#endif  // GP_NATIVE_RNG

// 1 in the native-RNG build (the reference's own std::mt19937), 0 in the replay build.
int orc_native_rng() { return kNativeRng ? 1 : 0; }

}  // extern "C"
