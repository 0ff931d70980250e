// Context creation, panel upload and the call-level C-ABI entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>

#include "context.h"
#include "phase.h"
#include "genotype.h"

namespace gp {

namespace {

// HvarRef (row = common site, MSB-first bytes, bitmatrix.h:89-119) to
// haplotype-major 32-bit words: refT[h][w] bit i = allele of h at common row 32w+i.
// Thread x is haplotype blockIdx.x * blockDim.x + x; the words run over blockIdx.y
// in steps of gridDim.y, which the launch caps at 65535 (panels with more than
// 2,097,120 common sites need more than one word per block row).
__global__ void k_transpose_panel(const uint8_t* __restrict__ hvar, int n_com, int stride, int N, int W,
                                  uint32_t* __restrict__ refT) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= N) return;
  for (int wi = blockIdx.y; wi < W; wi += gridDim.y) {
    uint32_t word = 0;
    const int r0 = wi * 32;
    const int n = min(32, n_com - r0);
    for (int i = 0; i < n; ++i) {
      const uint8_t byte = hvar[(size_t)(r0 + i) * stride + (h >> 3)];
      word |= (uint32_t)((byte >> (7 - (h & 7))) & 1) << i;
    }
    refT[(size_t)h * W + wi] = word;
  }
}

}  // namespace

ModelConst model_constants(const gp_config& c, int n_ref_haps) {
  ModelConst m;
  const float err_imp = std::clamp(c.err_imp, 1e-12f, 1e-3f);  // caller_initialise.cpp:152
  m.ed_imp = err_imp;
  m.ee_imp = (float)(1.0 - (double)err_imp);                   // conditioning_set.cpp:33-34
  m.ed_phs = c.err_phase;
  m.ee_phs = (float)(1.0 - (double)c.err_phase);
  m.min_gl = c.min_gl;
  m.nrho = (-0.04 * (double)c.ne) / (double)n_ref_haps;       // conditioning_set.cpp:30
  m.one_l = 1.0 - 1e-7;
  return m;
}

void Context::prof_begin(cudaEvent_t& a) {
  cudaEventCreate(&a);
  cudaEventRecord(a, stream);
}

void Context::prof_end(cudaEvent_t a, int kind, double cells) {
  cudaEvent_t b;
  cudaEventCreate(&b);
  cudaEventRecord(b, stream);
  prof_pending.push_back({a, b, kind, cells});
}

// Called after a stream synchronisation: accumulates the event pairs.
void Context::prof_resolve() {
  for (auto& p : prof_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      if (p.kind == 0) {
        prof.impute_ms += ms;
        prof.impute_cells += p.cells;
        prof.impute_bytes += p.cells * 8.25;  // 1/8 B Hvar + 4 B alpha, forward and backward
        prof.impute_launches++;
      } else if (p.kind == 1) {
        prof.phase_ms += ms;
        prof.phase_cells += p.cells;
        prof.phase_launches++;
      } else if (p.kind == 3) {
        prof.mlp_ms += ms;
        prof.mlp_rows += p.cells;
        prof.mlp_launches++;
      } else {
        prof.select_ms += ms;
      }
    }
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  prof_pending.clear();
}

Status Context::fail(int code, const std::string& msg) {
  err = msg;
  Status s;
  s.code = code;
  s.msg = msg;
  return s;
}

int Context::cuda_fail(cudaError_t e, const char* where) {
  err = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? GP_E_NOMEM : GP_E_CUDA;
}

bool inject_alloc_failure() {
  static std::mutex mu;
  static std::string last;
  static long countdown = 0;
  const char* v = std::getenv("GLIMPSE_B200_FAIL_ALLOC");
  std::lock_guard<std::mutex> lk(mu);
  const std::string cur = v ? v : "";
  if (cur != last) {
    last = cur;
    countdown = cur.empty() ? 0 : std::strtol(cur.c_str(), nullptr, 10);
  }
  if (countdown <= 0) return false;
  return --countdown == 0;
}

template <class T>
static cudaError_t upload(T** dst, const T* src, size_t n, std::vector<void*>& owned) {
  *dst = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)dst, n * sizeof(T));
  if (e != cudaSuccess) return e;
  owned.push_back(*dst);
  if (src) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

int Context::create_panel(const gp_panel_desc& d) {
  const int N = d.n_ref_haps, L = d.n_sites;
  if (N <= 0 || L <= 0 || !d.cm || !d.cref || !d.calt || !d.lq || !d.flag_common || !d.major || !d.shap_off)
    return (fail(GP_E_ARG, "panel: missing array or empty panel"), GP_E_ARG);
  if (L >= (1 << 24))
    return (fail(GP_E_ARG, "panel: more than 16,777,215 sites in one chunk"), GP_E_ARG);  // 24-bit site fields
  host.N = N;
  host.L = L;
  host.cm.assign(d.cm, d.cm + L);
  host.cref.assign(d.cref, d.cref + L);
  host.calt.assign(d.calt, d.calt + L);
  host.lq.assign(d.lq, d.lq + L);
  host.common.assign(d.flag_common, d.flag_common + L);
  host.major.assign(d.major, d.major + L);
  host.comrow.assign(L, -1);
  int nc = 0, nchq = 0;
  for (int l = 0; l < L; ++l)
    if (host.common[l]) {
      host.comrow[l] = nc++;
      if (!host.lq[l]) ++nchq;
    }
  host.n_com = nc;
  host.n_com_hq = nchq;
  const int stride = (N + 7) / 8;
  if (nc > 0 && !d.hvar) return (fail(GP_E_ARG, "panel: hvar missing"), GP_E_ARG);
  host.hvar.assign(d.hvar, d.hvar + (size_t)nc * stride);
  const int64_t nnz = d.shap_off[N];
  host.shap_off.assign(d.shap_off, d.shap_off + N + 1);
  host.shap_sites.assign(d.shap_sites, d.shap_sites + nnz);
  for (int64_t j = 0; j < nnz; ++j)
    if (host.shap_sites[j] < 0 || host.shap_sites[j] >= L || host.common[host.shap_sites[j]])
      return (fail(GP_E_DATA, "panel: ShapRef lists a site that is not a rare site"), GP_E_DATA);

  DevPanel& P = panel;
  P.N = N;
  P.L = L;
  P.n_com = nc;
  P.n_com_hq = nchq;
  P.W = std::max(1, (nc + 31) / 32);
  P.shap_nnz = nnz;
  cudaError_t e;
  if ((e = upload(&P.cm, host.cm.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel cm");
  if ((e = upload(&P.lq, host.lq.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel lq");
  if ((e = upload(&P.common, host.common.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel common");
  if ((e = upload(&P.major, host.major.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel major");
  if ((e = upload(&P.cref, host.cref.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel cref");
  if ((e = upload(&P.calt, host.calt.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel calt");
  if ((e = upload(&P.comrow, host.comrow.data(), L, owned)) != cudaSuccess) return cuda_fail(e, "panel comrow");
  if ((e = upload(&P.shap_off, host.shap_off.data(), N + 1, owned)) != cudaSuccess) return cuda_fail(e, "shap_off");
  if ((e = upload(&P.shap_sites, host.shap_sites.data(), (size_t)nnz, owned)) != cudaSuccess)
    return cuda_fail(e, "shap_sites");
  // SvarRef (haplotype_set::transposeRareRef, haplotype_set.cpp:201-214)
  host.svar_off.assign(L + 1, 0);
  for (int64_t j = 0; j < nnz; ++j) host.svar_off[host.shap_sites[j] + 1]++;
  for (int l = 0; l < L; ++l) host.svar_off[l + 1] += host.svar_off[l];
  host.svar_haps.assign(nnz, 0);
  {
    std::vector<int64_t> fill(host.svar_off.begin(), host.svar_off.end() - 1);
    for (int h = 0; h < N; ++h)
      for (int64_t j = host.shap_off[h]; j < host.shap_off[h + 1]; ++j) host.svar_haps[fill[host.shap_sites[j]]++] = h;
  }
  host.common_sites.clear();
  host.max_rare_mac = 0;
  for (int l = 0; l < L; ++l) {
    if (host.common[l]) host.common_sites.push_back(l);
    else host.max_rare_mac = std::max<int>(host.max_rare_mac, (int)std::min(host.cref[l], host.calt[l]));
  }
  if ((e = upload(&P.svar_off, host.svar_off.data(), L + 1, owned)) != cudaSuccess) return cuda_fail(e, "svar_off");
  if ((e = upload(&P.svar_haps, host.svar_haps.data(), (size_t)nnz, owned)) != cudaSuccess)
    return cuda_fail(e, "svar_haps");
  if ((e = upload(&P.refT, (const uint32_t*)nullptr, (size_t)N * P.W, owned)) != cudaSuccess)
    return cuda_fail(e, "refT");
  if (nc > 0) {
    uint8_t* dh = nullptr;
    if ((e = cudaMalloc(&dh, host.hvar.size())) != cudaSuccess) return cuda_fail(e, "hvar staging");
    e = cudaMemcpy(dh, host.hvar.data(), host.hvar.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      dim3 g((N + 255) / 256, std::min(P.W, grid_y_cap));
      k_transpose_panel<<<g, 256, 0, stream>>>(dh, nc, stride, N, P.W, P.refT);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    }
    cudaFree(dh);
    if (e != cudaSuccess) return cuda_fail(e, "panel transpose");
  } else {
    cudaMemsetAsync(P.refT, 0, sizeof(uint32_t) * N * P.W, stream);
  }
  {
    std::string msg;
    if (validate_panel(N, L, host.lq.data(), host.common.data(), host.major.data(), host.cref.data(),
                       host.calt.data(), host.hvar.data(), host.svar_off.data(), msg) != GP_OK)
      return (fail(GP_E_DATA, "panel: " + msg), GP_E_DATA);
  }
  // Sparse PBWT: supplied with the panel (binary panel format) or built here.
  if (d.ypacked && d.asmall_off && d.asmall_idx) {
    sparse.ypacked.assign(d.ypacked, d.ypacked + d.ypacked_len);
    sparse.asmall_off.assign(d.asmall_off, d.asmall_off + nchq + 2);
    sparse.asmall.assign(d.asmall_idx, d.asmall_idx + sparse.asmall_off[nchq + 1]);
  } else {
    build_sparse_pbwt(N, L, host.lq.data(), host.common.data(), host.major.data(), host.cref.data(),
                      host.calt.data(), host.hvar.data(), host.svar_off.data(), host.svar_haps.data(), sparse);
  }
  float tab[256];
  unphred_table(tab);
  if ((e = upload_unphred(tab)) != cudaSuccess) return cuda_fail(e, "unphred");
  if ((e = upload_unphred_init(tab)) != cudaSuccess) return cuda_fail(e, "unphred");
  return pbwt_prepare_panel();
}

Context::~Context() {
  cudaStreamSynchronize(stream);
  for (void* p : owned) cudaFree(p);
  impute.states.release(); impute.nstates.release(); impute.states_off.release();
  impute.mark.release(); impute.polyidx.release(); impute.poly.release(); impute.npoly.release();
  impute.hvar.release(); impute.em.release(); impute.tr.release(); impute.fl.release();
  impute.alpha.release(); impute.alpha_off.release(); impute.split.release(); impute.split_scr.release();
  impute.hl.release(); impute.hp.release(); impute.flat.release();
  prof_resolve();
  for (DevBuf* b : phase.all()) b->release();
  for (DevBuf* b : tw.all()) b->release();
  scratch_h0.release(); scratch_h1.release(); scratch_ids.release();
  glin_src.release(); glin_nval.release(); glin_ploidy.release(); glin_gl.release(); glin_flat.release();
  glin_err.release();
  out_gp.release(); out_site.release();
  lig_a.release(); lig_b.release(); lig_s.release(); lig_cnt.release();
  for (DevBuf* b : mlp.all()) b->release();
  tune_tarhap.release();
  list_off.release(); list_ids.release(); merged_states.release();
  ckpt.release(); ckpt_sum.release(); ckpt_scratch.release(); loglik.release();
  for (DevBuf* b : learned.all()) b->release();
  if (phase_err_host) cudaFreeHost(phase_err_host);
  if (stream) cudaStreamDestroy(stream);
}

// Conditioning sets from explicit state lists (sorted ids per entry): poly
// sites, Hvar words. Leaves npoly on the host in impute_np.
int Context::build_condsets(int n, const std::vector<int64_t>& off, const std::vector<uint32_t>& states) {
  const int L = panel.L;
  int Kmax = 0;
  for (int i = 0; i < n; ++i) Kmax = std::max<int>(Kmax, (int)(off[i + 1] - off[i]));
  for (int i = 0; i < n; ++i)
    if (off[i + 1] == off[i]) return (fail(GP_E_DATA, "conditioning set is empty"), GP_E_DATA);
  if (Kmax > kMaxStates)
    return (fail(GP_E_ARG, "conditioning set larger than " + std::to_string(kMaxStates) + " states"), GP_E_ARG);
  ImputeWork& w = impute;
  w.n = n;
  w.L = L;
  w.Kp = (Kmax + 31) / 32 * 32;
  w.WB = (L + 31) / 32;
  std::vector<uint32_t> hs((size_t)n * w.Kp, 0u);
  std::vector<int32_t> hn(n);
  for (int i = 0; i < n; ++i) {
    hn[i] = (int32_t)(off[i + 1] - off[i]);
    for (int64_t j = off[i]; j < off[i + 1]; ++j) {
      const uint32_t h = states[j];
      if ((int)h >= panel.N) return (fail(GP_E_ARG, "state id out of range"), GP_E_ARG);
      if (j > off[i] && states[j - 1] >= h)
        return (fail(GP_E_ARG, "state ids must be sorted and unique"), GP_E_ARG);
      hs[(size_t)i * w.Kp + (j - off[i])] = h;
    }
  }
  host_nstates = hn;
  cudaError_t e;
  if ((e = w.states.ensure(hs.size() * 4)) != cudaSuccess) return cuda_fail(e, "alloc states");
  if ((e = w.nstates.ensure(n * 4)) != cudaSuccess) return cuda_fail(e, "alloc nstates");
  if ((e = w.mark.ensure((size_t)n * L)) != cudaSuccess) return cuda_fail(e, "alloc mark");
  if ((e = w.polyidx.ensure((size_t)n * L * 4)) != cudaSuccess) return cuda_fail(e, "alloc polyidx");
  if ((e = w.poly.ensure((size_t)n * L * 4)) != cudaSuccess) return cuda_fail(e, "alloc poly");
  if ((e = w.npoly.ensure(n * 4)) != cudaSuccess) return cuda_fail(e, "alloc npoly");
  if ((e = w.hvar.ensure((size_t)n * w.WB * w.Kp * 4)) != cudaSuccess) return cuda_fail(e, "alloc hvar");
  cudaMemcpyAsync(w.states.ptr, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(w.nstates.ptr, hn.data(), n * 4, cudaMemcpyHostToDevice, stream);
  launch_mark_poly(panel, w, stream);
  launch_compact_poly(panel, w, stream);
  launch_build_hvar(panel, w, stream);
  prof.kernel_launches += 5;
  impute_np.assign(n, 0);
  cudaMemcpyAsync(impute_np.data(), w.npoly.ptr, n * 4, cudaMemcpyDeviceToHost, stream);
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "conditioning set");
  return GP_OK;
}

// Bytes a growable store may take when `need` bytes are wanted and `held`
// are already allocated: everything wanted when it fits what is held (no query
// of the device), else half of the device's memory and no more than is free
// now (plus what the store holds) less 8 GiB for the rest of the iteration.
// GLIMPSE_B200_STORE_BUDGET_MB lowers it (tests use it to run the chunked
// paths on small batches).
size_t Context::store_budget(size_t held, size_t need) {
  size_t b = need;
  if (need > held) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
      const size_t reserve = size_t(8) << 30;
      b = std::min(tot / 2, fr + held > reserve ? fr + held - reserve : held);
    } else {
      b = held;
    }
  }
  if (const char* env = std::getenv("GLIMPSE_B200_STORE_BUDGET_MB")) {
    const long long mb = std::atoll(env);
    if (mb > 0) b = std::min(b, (size_t)mb << 20);
  }
  return b;
}

// Forward-backward over the current conditioning sets. The haplotypes run in
// decreasing order of polymorphic sites; when their stores do not fit the
// budget together, they run in consecutive chunks of that order, each chunk's
// stores packed from the start of the buffer.
int Context::run_impute(const float* d_hl, const uint8_t* d_flat, float* d_hp) {
  ImputeWork& w = impute;
  const int n = w.n, L = w.L;
  cudaError_t e;
  if ((e = w.em.ensure((size_t)n * L * 16)) != cudaSuccess) return cuda_fail(e, "alloc em");
  if ((e = w.tr.ensure((size_t)n * L * 8)) != cudaSuccess) return cuda_fail(e, "alloc tr");
  if ((e = w.fl.ensure((size_t)n * L)) != cudaSuccess) return cuda_fail(e, "alloc fl");
  if (precision_mode != GP_PRECISION_FULL) return run_impute_ckpt(d_hl, d_flat, d_hp);
  if ((e = w.alpha_off.ensure((size_t)n * 8)) != cudaSuccess) return cuda_fail(e, "alloc alpha_off");
  int Kmax = 0;
  for (int i = 0; i < n; ++i) Kmax = std::max(Kmax, host_nstates[i]);
  w.Ks = impute_store_stride(Kmax);
  // Chains of the longest haplotypes (most poly sites) are launched first.
  std::vector<int32_t> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return impute_np[x] > impute_np[y]; });
  // chunks of the order whose stores fit the budget
  size_t need_all = 0;
  for (int i = 0; i < n; ++i) need_all += (size_t)impute_np[i] * w.Ks * 4;
  const size_t budget = store_budget(w.alpha.cap, need_all);
  std::vector<int64_t> aoff(n);
  std::vector<int32_t> split(n);
  std::vector<int> chunk_start(1, 0);
  int64_t tot = 0, need = 0;
  for (int j = 0; j < n; ++j) {
    const int i = order[j];
    const int64_t bytes = (int64_t)impute_np[i] * w.Ks * 4;
    if (j > chunk_start.back() && (size_t)(tot + bytes) > budget) {
      chunk_start.push_back(j);
      tot = 0;
    }
    aoff[i] = tot / 4;
    tot += bytes;
    need = std::max(need, tot);
    split[i] = (impute_np[i] / 2) & ~31;  // forward/backward meeting point, a multiple of 32
  }
  chunk_start.push_back(n);
  if ((e = w.alpha.ensure((size_t)std::max<int64_t>(need, 4))) != cudaSuccess) return cuda_fail(e, "alloc alpha");
  if ((e = w.split.ensure((size_t)n * 4)) != cudaSuccess) return cuda_fail(e, "alloc split");
  if ((e = w.split_scr.ensure(((size_t)((2 * n + 3) & ~3) + (size_t)n * w.Ks) * 4)) != cudaSuccess)
    return cuda_fail(e, "alloc split");
  cudaMemcpyAsync(w.alpha_off.ptr, aoff.data(), n * 8, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(w.split.ptr, split.data(), n * 4, cudaMemcpyHostToDevice, stream);
  if ((e = w.order.ensure((size_t)n * 4)) != cudaSuccess) return cuda_fail(e, "alloc order");
  cudaMemcpyAsync(w.order.ptr, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, stream);
  launch_site_records(panel, mc, w, d_hl, d_flat, stream);
  double cells = 0;
  for (int i = 0; i < n; ++i) cells += (double)impute_np[i] * (double)host_nstates[i];
  // one warp per chain: lane-owned states in groups of 8 per lane
  const int J = impute_groups(Kmax);
  cudaEvent_t ea;
  prof_begin(ea);
  int cpc = fixed_cpc ? fixed_cpc : tune_cpc;
  if (!cpc) {
    // Autotune chains per CTA on this batch's first chunk: phase 1 only writes
    // the store, so the runs repeat the same work; the real run follows.
    cpc = 2;
    if (chunk_start[1] >= 16) {
      const int cand[3] = {1, 2, 4};
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      float best = 1e30f;
      for (int ci = 0; ci < 3; ++ci) {
        cudaEventRecord(e0, stream);
        const int lrc = launch_impute_warp(1, J, mc, w, d_hp, stream, 0, chunk_start[1], cand[ci]);
        cudaEventRecord(e1, stream);
        float ms = 1e30f;
        if (lrc == GP_OK && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        else cudaGetLastError();
        tune_ms[ci] = ms < 1e29f ? ms : -1.f;
        if (ms < best) {
          best = ms;
          cpc = cand[ci];
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      tune_cpc = cpc;
      prof.kernel_launches += 3;
    }
  }
  for (size_t c = 0; c + 1 < chunk_start.size(); ++c) {
    const int j0 = chunk_start[c], nc = chunk_start[c + 1] - j0;
    int lrc = launch_impute_warp(1, J, mc, w, d_hp, stream, j0, nc, cpc);
    if (lrc == GP_OK) lrc = launch_impute_warp(2, J, mc, w, d_hp, stream, j0, nc, cpc);
    if (lrc == GP_E_CUDA) return cuda_fail(cudaGetLastError(), "imputation: shared-memory attribute");
    if (lrc != GP_OK) return (fail(GP_E_ARG, "imputation: too many states"), GP_E_ARG);
    prof.kernel_launches += 2;
  }
  prof_end(ea, 0, cells);
  impute_chunks = (int)chunk_start.size() - 1;
  launch_impute_finish(panel, mc, w, d_hl, d_flat, d_hp, stream);
  prof.kernel_launches += 2;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "imputation launch");
  return GP_OK;
}

// The checkpointed variant (kernels_impute_ckpt.cu): checkpoint rows every 32
// polymorphic sites (FP32 or BF16), recompute in the backward pass, FP64 chunk
// log-likelihood per haplotype into d_loglik.
int Context::run_impute_ckpt(const float* d_hl, const uint8_t* d_flat, float* d_hp) {
  ImputeWork& w = impute;
  const int n = w.n;
  const bool bf16 = precision_mode == GP_PRECISION_CKPT_BF16;
  cudaError_t e;
  // alpha and beta checkpoints and their sums, one 32-row scratch per chain,
  // the log-likelihood and its first half
  if ((e = ckpt.ensure((size_t)2 * n * w.WB * w.Kp * (bf16 ? 2 : 4))) != cudaSuccess) return cuda_fail(e, "alloc ckpt");
  if ((e = ckpt_sum.ensure((size_t)2 * n * w.WB * 4)) != cudaSuccess) return cuda_fail(e, "alloc ckpt");
  if ((e = ckpt_scratch.ensure((size_t)2 * n * 32 * w.Kp * 4)) != cudaSuccess) return cuda_fail(e, "alloc ckpt");
  if ((e = loglik.ensure((size_t)2 * n * 8)) != cudaSuccess) return cuda_fail(e, "alloc loglik");
  launch_site_records(panel, mc, w, d_hl, d_flat, stream);
  double cells = 0;
  for (int i = 0; i < n; ++i) cells += (double)impute_np[i] * (double)host_nstates[i];
  cudaEvent_t ea;
  prof_begin(ea);
  if (launch_impute_ckpt(w, bf16, ckpt.ptr, ckpt_sum.as<float>(), ckpt_scratch.as<float>(), loglik.as<double>(),
                         d_hp, stream) != GP_OK)
    return (fail(GP_E_ARG, "imputation: too many states"), GP_E_ARG);
  prof_end(ea, 0, cells);
  launch_impute_finish(panel, mc, w, d_hl, d_flat, d_hp, stream);
  prof.kernel_launches += 4;
  loglik_n = n;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "imputation launch");
  return GP_OK;
}

// After a synchronisation that follows run_phase: GP_E_DATA naming the first
// target whose diplotype draw saw a NaN, infinite or sub-normal sum. The draw
// keeps the previous diplotype there and the run is otherwise complete; the
// reference stops on an assertion (phasing_hmm.cpp:175).
int Context::check_phase_errors() {
  const int n = phase_err_n;
  phase_err_n = 0;
  for (int b = 0; b < n; ++b)
    if (phase_err_host[b])
      return (fail(GP_E_DATA, "phasing: invalid diplotype probabilities (NaN, infinite or zero sum) for target " +
                                  std::to_string(phase_err_ids[b])),
              GP_E_DATA);
  return GP_OK;
}

// Phasing for nb entries of the current conditioning sets (tsel: device list of
// entry indices or null for 0..nb-1; target_ids: device stream targets or null).
int Context::run_phase(const int32_t* d_tsel, const std::vector<int32_t>& tsel_host, int nb, uint8_t* d_h0,
                       uint8_t* d_h1, const uint8_t* d_flat, int iteration, const int32_t* d_target_ids) {
  ImputeWork& w = impute;
  PhaseWork& p = phase;
  const int L = panel.L;
  cudaError_t e;
  // per-entry VAR arrays and sums strided by the batch's largest poly count (VAR sites are poly sites)
  int lv = 1;
  for (int b = 0; b < nb; ++b) lv = std::max(lv, impute_np[tsel_host.empty() ? b : tsel_host[b]]);
  if ((e = p.rel.ensure((size_t)nb * lv * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.code.ensure((size_t)nb * lv)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.seg.ensure((size_t)nb * lv * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.miss.ensure((size_t)nb * lv * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.seg_start.ensure((size_t)nb * (lv + 2) * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.counts.ensure((size_t)nb * 3 * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.ytp.ensure((size_t)nb * lv * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.ytn.ensure((size_t)nb * lv * 4)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.vflags.ensure((size_t)nb * lv)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.recb.ensure((size_t)nb * lv * 16)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  if ((e = p.recf.ensure((size_t)nb * lv * 16)) != cudaSuccess) return cuda_fail(e, "alloc vars");
  PhaseVars V;
  V.rel = p.rel.as<int32_t>();
  V.code = p.code.as<uint8_t>();
  V.seg = p.seg.as<int32_t>();
  V.miss = p.miss.as<int32_t>();
  V.seg_start = p.seg_start.as<int32_t>();
  V.yt_prev = p.ytp.as<float>();
  V.yt_next = p.ytn.as<float>();
  V.flags = p.vflags.as<uint8_t>();
  V.recb = p.recb.as<int4>();
  V.recf = p.recf.as<int4>();
  V.nvar = p.counts.as<int32_t>();
  V.nseg = V.nvar + nb;
  V.nmiss = V.nvar + 2 * nb;
  V.lv = lv;
  launch_build_vars(d_tsel, nb, w.poly.as<int32_t>(), w.npoly.as<int32_t>(), d_h0, d_h1, d_flat, panel.lq, L, V,
                    stream);
  prof.kernel_launches += 1;
  std::vector<int32_t> cnt((size_t)nb * 3);
  cudaMemcpyAsync(cnt.data(), p.counts.ptr, cnt.size() * 4, cudaMemcpyDeviceToHost, stream);
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "phasing vars");
  // Blocks in decreasing order of work (VAR sites x state groups), so that the
  // heaviest targets start first and share an SM with the lightest.
  std::vector<int32_t> order(nb);
  std::vector<double> cost(nb);
  int Kmax = 0;
  for (int b = 0; b < nb; ++b) {
    const int t = tsel_host.empty() ? b : tsel_host[b];
    order[b] = b;
    cost[b] = (double)cnt[b] * (1.0 + (double)((host_nstates[t] + kPhaseThreads - 1) / kPhaseThreads));
    Kmax = std::max(Kmax, host_nstates[t]);
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  // Placement 2, for batches of one to two entries per SM: the CTAs at grid
  // positions i and S + i share an SM (S SMs, two CTAs per SM), so the heaviest
  // 2S - nb entries take positions nb - S .. S - 1 and run alone, and the rest
  // are paired heaviest with lightest.
  if (sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
  }
  const int S_sm = sm_count;
  std::vector<int32_t> order_paired;
  if (nb > S_sm && nb <= 2 * S_sm) {
    const int npair = nb - S_sm, nsolo = S_sm - npair;
    order_paired.assign(nb, 0);
    for (int j = 0; j < nsolo; ++j) order_paired[npair + j] = order[j];
    for (int j = 0; j < npair; ++j) {
      order_paired[j] = order[nsolo + j];
      order_paired[S_sm + j] = order[nb - 1 - j];
    }
  }
  // The per-entry buffers of fixed size come first, so that the budget below
  // sees the memory they leave.
  if ((e = p.offs.ensure((size_t)nb * 2 * 8)) != cudaSuccess) return cuda_fail(e, "alloc offs");
  if ((e = p.pprob_sum.ensure((size_t)nb * (lv + 2) * 8 * 4)) != cudaSuccess) return cuda_fail(e, "alloc psum");
  if ((e = p.pprob_sumsum.ensure((size_t)nb * (lv + 2) * 4)) != cudaSuccess) return cuda_fail(e, "alloc pss");
  if ((e = p.iprob_sum.ensure((size_t)nb * lv * 8 * 4)) != cudaSuccess) return cuda_fail(e, "alloc isum");
  if ((e = p.of1.ensure((size_t)nb * lv * 8 * 4)) != cudaSuccess) return cuda_fail(e, "alloc of1");
  if ((e = p.dip.ensure((size_t)nb * (lv + 2) * 4)) != cudaSuccess) return cuda_fail(e, "alloc dip");
  if ((e = p.err.ensure((size_t)nb * 4)) != cudaSuccess) return cuda_fail(e, "alloc err");
  if ((e = p.order.ensure((size_t)nb * 4)) != cudaSuccess) return cuda_fail(e, "alloc order");
  // The stored segment-start and flat-het messages of every entry, its two
  // regions side by side in one pool, packed per chunk of that order: chunks
  // run one after another when all entries' stores do not fit the memory
  // budget together (low coverage makes many flat hets).
  size_t need_all = 0;
  for (int b = 0; b < nb; ++b) {
    const int K = host_nstates[tsel_host.empty() ? b : tsel_host[b]];
    need_all += ((size_t)cnt[nb + b] + (size_t)cnt[2 * nb + b]) * K * 8 * 4;
  }
  const size_t budget = store_budget(p.pool.cap, need_all);
  std::vector<int64_t> poff(nb), ioff(nb);
  std::vector<int> chunk_start(1, 0);
  int64_t tot = 0, need = 0;
  for (int j = 0; j < nb; ++j) {
    const int b = order[j];
    const int t = tsel_host.empty() ? b : tsel_host[b];
    const int K = host_nstates[t];
    const int64_t pb = (int64_t)cnt[nb + b] * K * 8, ib = (int64_t)cnt[2 * nb + b] * K * 8;
    if (j > chunk_start.back() && (size_t)(tot + pb + ib) * 4 > budget) {
      chunk_start.push_back(j);
      tot = 0;
    }
    poff[b] = tot;
    ioff[b] = tot + pb;
    tot += pb + ib;
    need = std::max(need, tot);
  }
  chunk_start.push_back(nb);
  if ((e = p.pool.ensure((size_t)std::max<int64_t>(need, 1) * 4)) != cudaSuccess) return cuda_fail(e, "alloc phasing store");
  std::vector<int64_t> offs(poff);
  offs.insert(offs.end(), ioff.begin(), ioff.end());
  cudaMemcpyAsync(p.offs.ptr, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, stream);
  const int porder = fixed_porder ? fixed_porder : 1;
  const bool paired_ok = !order_paired.empty() && chunk_start.size() == 2;
  cudaMemcpyAsync(p.order.ptr, (paired_ok && porder == 2 ? order_paired : order).data(), (size_t)nb * 4,
                  cudaMemcpyHostToDevice, stream);
  PhaseStore S;
  S.pprob = p.pool.as<float>();
  S.pprob_off = p.offs.as<int64_t>();
  S.pprob_sum = p.pprob_sum.as<float>();
  S.pprob_sumsum = p.pprob_sumsum.as<float>();
  S.iprob = p.pool.as<float>();
  S.iprob_off = p.offs.as<int64_t>() + nb;
  S.iprob_sum = p.iprob_sum.as<float>();
  S.of1 = p.of1.as<float>();
  S.dip = p.dip.as<int32_t>();
  S.err = p.err.as<int32_t>();
  S.order = p.order.as<int32_t>();
  const int J = std::max(1, (Kmax + kPhaseThreads - 1) / kPhaseThreads);
  double pcells = 0;
  for (int b = 0; b < nb; ++b) {
    const int t = tsel_host.empty() ? b : tsel_host[b];
    pcells += 2.0 * 8.0 * (double)cnt[b] * (double)host_nstates[t];
  }
  launch_var_records(d_tsel, nb, w.poly.as<int32_t>(), L, panel.cm, mc, V, stream);
  cudaEvent_t ea;
  prof_begin(ea);
  for (size_t c = 0; c + 1 < chunk_start.size(); ++c) {
    PhaseStore Sc = S;
    Sc.order = S.order + chunk_start[c];
    if (launch_phase(J, d_tsel, chunk_start[c + 1] - chunk_start[c], w.nstates.as<int32_t>(), w.hvar.as<uint32_t>(),
                     w.WB, w.Kp, w.poly.as<int32_t>(), w.npoly.as<int32_t>(), L, panel.cm, V, Sc, mc, cfg.seed,
                     iteration, d_target_ids, stream) != GP_OK)
      return (fail(GP_E_ARG, "phasing: too many states"), GP_E_ARG);
    prof.kernel_launches += 1;
  }
  prof_end(ea, 1, pcells);
  phase_chunks = (int)chunk_start.size() - 1;
  // SAMPLE_DIP's invalid-sum flags (the reference asserts there, phasing_hmm.cpp:175).
  if (phase_err_cap < nb) {
    if (phase_err_host) cudaFreeHost(phase_err_host);
    phase_err_host = nullptr;
    phase_err_cap = 0;
    if ((e = cudaMallocHost(&phase_err_host, (size_t)nb * 4)) != cudaSuccess) return cuda_fail(e, "alloc err flags");
    phase_err_cap = nb;
  }
  cudaMemcpyAsync(phase_err_host, S.err, (size_t)nb * 4, cudaMemcpyDeviceToHost, stream);
  phase_err_n = nb;
  phase_err_ids.resize(nb);
  for (int b = 0; b < nb; ++b) phase_err_ids[b] = tsel_host.empty() ? b : tsel_host[b];
  launch_phase_writeback(d_tsel, nb, w.poly.as<int32_t>(), w.polyidx.as<int32_t>(), L, V, S, mc, cfg.seed, iteration,
                         d_target_ids, d_h0, d_h1, stream);
  prof.kernel_launches += 3;  // VAR records and the two write-back kernels (k_phase counted per chunk)
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "phasing launch");
  last_phase_nseg.assign(cnt.begin() + nb, cnt.begin() + 2 * nb);
  return GP_OK;
}

}  // namespace gp

using gp::Context;

extern "C" {

void gp_config_defaults(gp_config* c) {
  if (!c) return;
  c->ne = 100000;
  c->err_imp = 1e-12f;
  c->err_phase = 1e-4f;
  c->min_gl = 1e-10f;
  c->pbwt_depth = 12;
  c->pbwt_modulo_cm = 0.1f;
  c->kinit = 1000;
  c->kpbwt = 2000;
  c->seed = 15052011ull;
  c->device = 0;
}

int gp_ctx_create(const gp_panel_desc* panel, const gp_config* cfg, gp_ctx** out) {
  if (!panel || !cfg || !out) return GP_E_ARG;
  *out = nullptr;
  // caller_parameters.cpp:255-258: Kinit and Kpbwt non-negative
  if (cfg->kinit < 0 || cfg->kpbwt < 0) return GP_E_ARG;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= cfg->device) return GP_E_CUDA;
  if (cudaSetDevice(cfg->device) != cudaSuccess) return GP_E_CUDA;
  std::unique_ptr<Context> c(new (std::nothrow) Context());
  if (!c) return GP_E_NOMEM;
  c->cfg = *cfg;
  if (const char* cap = std::getenv("GLIMPSE_B200_GRID_Y_CAP")) {
    // Lowers the largest gridDim.y of the launches that loop over a second grid
    // dimension (tests use it to run those loops on small panels).
    const long v = std::strtol(cap, nullptr, 10);
    if (v >= 1 && v <= 65535) c->grid_y_cap = (int)v;
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return GP_E_CUDA;
  int rc = c->create_panel(*panel);
  if (rc != GP_OK) {
    std::fprintf(stderr, "gp_ctx_create: %s\n", c->err.c_str());
    return rc;
  }
  c->mc = gp::model_constants(*cfg, panel->n_ref_haps);
  *out = reinterpret_cast<gp_ctx*>(c.release());
  return GP_OK;
}

int gp_ctx_destroy(gp_ctx* ctx) {
  delete reinterpret_cast<Context*>(ctx);
  return GP_OK;
}

const char* gp_last_error(const gp_ctx* ctx) {
  return ctx ? reinterpret_cast<const Context*>(ctx)->err.c_str() : "null context";
}

int gp_tuning_set(gp_ctx* ctx, int32_t chains_per_cta, int32_t sweep_haps_per_warp, int32_t phase_placement) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if ((chains_per_cta != 0 && chains_per_cta != 1 && chains_per_cta != 2 && chains_per_cta != 4) ||
      (sweep_haps_per_warp != 0 && sweep_haps_per_warp != 1 && sweep_haps_per_warp != 2 && sweep_haps_per_warp != 4 &&
       sweep_haps_per_warp != 8) ||
      phase_placement < 0 || phase_placement > 2)
    return (c.fail(GP_E_ARG, "tuning: chains per CTA in {0, 1, 2, 4}, haplotypes per sweep warp in {0, 1, 2, 4, 8}, "
                             "phasing placement in {0, 1, 2}"),
            GP_E_ARG);
  c.fixed_cpc = chains_per_cta;
  c.fixed_hpw = sweep_haps_per_warp;
  c.fixed_porder = phase_placement;
  if (!chains_per_cta) c.tune_cpc = 0;
  if (!sweep_haps_per_warp) c.tune_hpw = 0;
  return GP_OK;
}

int gp_tuning_get(gp_ctx* ctx, int32_t* chains_per_cta, int32_t* sweep_haps_per_warp, int32_t* phase_placement,
                  float* ms) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (chains_per_cta) *chains_per_cta = c.fixed_cpc ? c.fixed_cpc : c.tune_cpc;
  if (sweep_haps_per_warp) *sweep_haps_per_warp = c.fixed_hpw ? c.fixed_hpw : c.tune_hpw;
  if (phase_placement) *phase_placement = c.fixed_porder ? c.fixed_porder : 1;
  if (ms)
    for (int i = 0; i < 9; ++i) ms[i] = c.tune_ms[i];
  return GP_OK;
}

int gp_set_precision(gp_ctx* ctx, int32_t mode) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (mode != GP_PRECISION_FULL && mode != GP_PRECISION_CKPT_F32 && mode != GP_PRECISION_CKPT_BF16)
    return (c.fail(GP_E_ARG, "precision: unknown mode"), GP_E_ARG);
  c.precision_mode = mode;
  return GP_OK;
}

int gp_loglik_get(gp_ctx* ctx, int32_t n, double* out) {
  if (!ctx || !out) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (c.loglik_n <= 0) return (c.fail(GP_E_STATE, "loglik: no checkpointed imputation has run"), GP_E_STATE);
  if (n != c.loglik_n) return (c.fail(GP_E_ARG, "loglik: n differs from the last imputation call"), GP_E_ARG);
  cudaMemcpyAsync(out, c.loglik.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, c.stream);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  return e == cudaSuccess ? GP_OK : c.cuda_fail(e, "loglik_get");
}

int gp_impute_batch(gp_ctx* ctx, int32_t n, const int64_t* states_off, const uint32_t* states, const float* hl,
                    const uint8_t* flat, float* hp) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (n <= 0 || n > GP_MAX_BATCH || !states_off || !states || !hl || !flat || !hp)
    return (c.fail(GP_E_ARG, "impute: bad argument"), GP_E_ARG);
  const int L = c.panel.L;
  std::vector<int64_t> off(states_off, states_off + n + 1);
  std::vector<uint32_t> st(states, states + off[n]);
  cudaError_t e;
  gp::ImputeWork& w = c.impute;
  if ((e = w.hl.ensure((size_t)n * 2 * L * 4)) != cudaSuccess) return c.cuda_fail(e, "alloc hl");
  if ((e = w.hp.ensure((size_t)n * 2 * L * 4)) != cudaSuccess) return c.cuda_fail(e, "alloc hp");
  if ((e = w.flat.ensure((size_t)n * L)) != cudaSuccess) return c.cuda_fail(e, "alloc flat");
  cudaMemcpyAsync(w.hl.ptr, hl, (size_t)n * 2 * L * 4, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(w.flat.ptr, flat, (size_t)n * L, cudaMemcpyHostToDevice, c.stream);
  int rc = c.build_condsets(n, off, st);
  if (rc != GP_OK) return rc;
  rc = c.run_impute(w.hl.as<float>(), w.flat.as<uint8_t>(), w.hp.as<float>());
  if (rc != GP_OK) return rc;
  cudaMemcpyAsync(hp, w.hp.ptr, (size_t)n * 2 * L * 4, cudaMemcpyDeviceToHost, c.stream);
  if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return c.cuda_fail(e, "impute");
  c.prof_resolve();
  return GP_OK;
}

int gp_rephase_batch(gp_ctx* ctx, int32_t n, const int64_t* states_off, const uint32_t* states, uint8_t* h0,
                     uint8_t* h1, const uint8_t* flat, int32_t iteration, const int32_t* target_ids) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (n <= 0 || n > GP_MAX_BATCH || !states_off || !states || !h0 || !h1 || !flat)
    return (c.fail(GP_E_ARG, "rephase: bad argument"), GP_E_ARG);
  const int L = c.panel.L;
  std::vector<int64_t> off(states_off, states_off + n + 1);
  std::vector<uint32_t> st(states, states + off[n]);
  int rc = c.build_condsets(n, off, st);
  if (rc != GP_OK) return rc;
  gp::DevBuf& bh0 = c.scratch_h0;
  gp::DevBuf& bh1 = c.scratch_h1;
  gp::DevBuf& bfl = c.impute.flat;
  gp::DevBuf& bid = c.scratch_ids;
  cudaError_t e;
  if ((e = bh0.ensure((size_t)n * L)) != cudaSuccess) return c.cuda_fail(e, "alloc h0");
  if ((e = bh1.ensure((size_t)n * L)) != cudaSuccess) return c.cuda_fail(e, "alloc h1");
  if ((e = bfl.ensure((size_t)n * L)) != cudaSuccess) return c.cuda_fail(e, "alloc flat");
  if ((e = bid.ensure((size_t)n * 4)) != cudaSuccess) return c.cuda_fail(e, "alloc ids");
  std::vector<int32_t> ids(n);
  for (int i = 0; i < n; ++i) ids[i] = target_ids ? target_ids[i] : i;
  cudaMemcpyAsync(bh0.ptr, h0, (size_t)n * L, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(bh1.ptr, h1, (size_t)n * L, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(bfl.ptr, flat, (size_t)n * L, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(bid.ptr, ids.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c.stream);
  rc = c.run_phase(nullptr, {}, n, bh0.as<uint8_t>(), bh1.as<uint8_t>(), bfl.as<uint8_t>(), iteration,
                   bid.as<int32_t>());
  if (rc != GP_OK) return rc;
  cudaMemcpyAsync(h0, bh0.ptr, (size_t)n * L, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(h1, bh1.ptr, (size_t)n * L, cudaMemcpyDeviceToHost, c.stream);
  if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return c.cuda_fail(e, "rephase");
  c.prof_resolve();
  for (int b = 0; b < n; ++b) c.phase_err_ids[b] = ids[b];
  return c.check_phase_errors();
}

int gp_sparse_pbwt_get(gp_ctx* ctx, uint8_t* ypacked, int64_t* ypacked_len, int64_t* asmall_off,
                       int32_t* asmall_idx, int64_t* asmall_len) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (ypacked_len) *ypacked_len = (int64_t)c.sparse.ypacked.size();
  if (asmall_len) *asmall_len = (int64_t)c.sparse.asmall.size();
  if (ypacked) std::memcpy(ypacked, c.sparse.ypacked.data(), c.sparse.ypacked.size());
  if (asmall_off) std::memcpy(asmall_off, c.sparse.asmall_off.data(), c.sparse.asmall_off.size() * 8);
  if (asmall_idx) std::memcpy(asmall_idx, c.sparse.asmall.data(), c.sparse.asmall.size() * 4);
  return GP_OK;
}

}  // extern "C"
