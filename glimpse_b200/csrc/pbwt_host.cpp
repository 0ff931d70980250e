// Panel-side sparse PBWT: the pack3 builder, the one-off decode into
// device-resident prefix/rank arrays, and the host orchestration of the
// per-iteration selection.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>

#include "context.h"
#include "select.h"

namespace gp {

namespace {

// pack3 three-level run-length code (common/src/containers/ref_haplotype_set.h:37-101,
// after R. Durbin's pbwt): byte = symbol << 7 | count code, where codes 0..63 are
// literal run lengths, 64..95 encode (c-64) << 6 and 96..127 encode (c-96) << 11.
constexpr uint32_t kMax1 = 64, kMax2 = (95 - 63) << 6, kMax3 = (127 - 96) << 11;

inline int p3_len(uint8_t b) {
  const int c = b & 0x7f;
  return c < 64 ? c : (c < 96 ? (c - 64) << 6 : (c - 96) << 11);
}

void pack3_add(uint8_t y, uint32_t n, std::vector<uint8_t>& out) {
  const uint8_t s = (uint8_t)(y << 7);
  while (n >= kMax3) {
    out.push_back(s | 0x7f);
    n -= kMax3;
  }
  if (n >= kMax2) {
    out.push_back(s | 0x60 | (uint8_t)(n >> 11));
    n &= 0x7ff;
  }
  if (n >= kMax1) {
    out.push_back(s | 0x40 | (uint8_t)(n >> 6));
    n &= 0x3f;
  }
  if (n) out.push_back(s | (uint8_t)n);
}

inline uint8_t hvar_bit(const uint8_t* hvar, size_t stride, int row, int h) {
  return (hvar[(size_t)row * stride + (h >> 3)] >> (7 - (h & 7))) & 1;
}

// Stable partition of `a` by bits (zeros first), writing runs to `code`.
template <class BitOf>
void column_update(std::vector<uint32_t>& a, std::vector<uint32_t>& b, int zeros, BitOf bit_of,
                   std::vector<uint8_t>& code) {
  const int n = (int)a.size();
  int u = 0, v = zeros;
  int m = 0;
  while (m < n) {
    const uint8_t z = bit_of(a[m]);
    const int m0 = m;
    while (++m < n && bit_of(a[m]) == z) {}
    int& occ = z ? v : u;
    for (int i = m0; i < m; ++i) b[occ++] = a[i];
    pack3_add(z, (uint32_t)(m - m0), code);
  }
  a.swap(b);
}

}  // namespace

int validate_panel(int N, int L, const uint8_t* lq, const uint8_t* common, const uint8_t* major,
                   const uint32_t* cref, const uint32_t* calt, const uint8_t* hvar, const int64_t* svar_off,
                   std::string& msg) {
  (void)lq;
  const size_t stride = ((size_t)N + 7) / 8;
  int row = 0;
  for (int k = 0; k < L; ++k) {
    if ((int64_t)cref[k] + (int64_t)calt[k] != N) {
      msg = "site " + std::to_string(k) + ": cref + calt differs from the number of reference haplotypes";
      return GP_E_DATA;
    }
    if (common[k]) {
      int64_t ones = 0;
      const uint8_t* r = hvar + (size_t)row * stride;
      for (size_t b = 0; b < stride; ++b) ones += __builtin_popcount(r[b]);
      if (ones != (int64_t)calt[k]) {
        msg = "common site " + std::to_string(k) + ": HvarRef row has " + std::to_string(ones) +
              " alternative alleles, calt says " + std::to_string(calt[k]);
        return GP_E_DATA;
      }
      ++row;
    } else {
      const int64_t nc = svar_off[k + 1] - svar_off[k];
      const int64_t want = major[k] ? cref[k] : calt[k];
      if (nc != want) {
        msg = "rare site " + std::to_string(k) + ": ShapRef lists " + std::to_string(nc) +
              " carriers of the non-major allele, the counts say " + std::to_string(want);
        return GP_E_DATA;
      }
    }
  }
  return GP_OK;
}

void build_sparse_pbwt(int N, int L, const uint8_t* lq, const uint8_t* common, const uint8_t* major,
                       const uint32_t* cref, const uint32_t* calt, const uint8_t* hvar, const int64_t* svar_off,
                       const int32_t* svar_haps, SparsePbwt& out) {
  const size_t stride = ((size_t)N + 7) / 8;
  int n_com_hq = 0;
  for (int k = 0; k < L; ++k) n_com_hq += common[k] && !lq[k];
  std::vector<std::vector<int32_t>> asmall(n_com_hq + 1);
  out.ypacked.clear();
  std::vector<uint32_t> A(N), B(N);
  std::iota(A.begin(), A.end(), 0u);
  std::vector<int32_t> rank(N);  // position of each haplotype in the current order
  std::iota(rank.begin(), rank.end(), 0);
  std::vector<uint32_t> sA, sB;  // small PBWT over indices into the run's haplotype set
  std::vector<int32_t> small_of(N, -1);
  std::vector<uint8_t> small_bit;
  int l_hq = 0, l_all = 0, last_k = -1;
  for (int k = 0; k < L; ++k) {
    if (lq[k]) {
      l_all += common[k];
      continue;
    }
    if (common[k]) {
      if (!sA.empty() && !(last_k >= 0 && common[last_k])) {
        // ref_haplotype_set::build_init_common: haplotypes outside the run's set
        // keep their order, the set follows in small-PBWT order.
        const std::vector<int32_t>& pos = asmall[l_hq];
        std::vector<uint8_t> in_small(N, 0);
        for (int p : pos) in_small[p] = 1;
        int nz = 0;
        for (int p = 0; p < N; ++p)
          if (!in_small[p]) B[nz++] = A[p];
        for (size_t i = 0; i < sA.size(); ++i) B[nz++] = A[pos[sA[i]]];
        A.swap(B);
      }
      const int row = l_all;
      column_update(A, B, (int)cref[k], [&](uint32_t h) { return hvar_bit(hvar, stride, row, (int)h); },
                    out.ypacked);
      for (int p = 0; p < N; ++p) rank[A[p]] = p;
      ++l_hq;
      ++l_all;
    } else {
      if (last_k < 0 || common[last_k]) {
        // ref_haplotype_set::init_small_rare: haplotypes carrying a rare allele
        // anywhere in this run, ordered by their position in the full PBWT.
        std::vector<int32_t> haps;
        for (int kk = k; kk < L; ++kk) {
          if (lq[kk]) continue;
          if (common[kk]) break;
          for (int64_t j = svar_off[kk]; j < svar_off[kk + 1]; ++j) haps.push_back(svar_haps[j]);
        }
        std::sort(haps.begin(), haps.end());
        haps.erase(std::unique(haps.begin(), haps.end()), haps.end());
        std::vector<std::pair<int32_t, int32_t>> by_pos;
        by_pos.reserve(haps.size());
        for (int h : haps) by_pos.emplace_back(rank[h], h);
        std::sort(by_pos.begin(), by_pos.end());
        std::vector<int32_t>& pos = asmall[l_hq];
        pos.resize(by_pos.size());
        for (size_t i = 0; i < by_pos.size(); ++i) {
          pos[i] = by_pos[i].first;
          small_of[by_pos[i].second] = (int32_t)i;
        }
        sA.resize(pos.size());
        std::iota(sA.begin(), sA.end(), 0u);
        sB.resize(pos.size());
        small_bit.resize(pos.size());
      }
      std::fill(small_bit.begin(), small_bit.end(), major[k]);
      for (int64_t j = svar_off[k]; j < svar_off[k + 1]; ++j) small_bit[small_of[svar_haps[j]]] = !major[k];
      const int zeros = major[k] ? (int)(N - calt[k]) : (int)(sA.size() - calt[k]);
      column_update(sA, sB, zeros, [&](uint32_t i) { return small_bit[i]; }, out.ypacked);
    }
    last_k = k;
  }
  out.asmall_off.assign(asmall.size() + 1, 0);
  out.asmall.clear();
  for (size_t i = 0; i < asmall.size(); ++i) {
    out.asmall_off[i] = (int64_t)out.asmall.size();
    out.asmall.insert(out.asmall.end(), asmall[i].begin(), asmall[i].end());
  }
  out.asmall_off[asmall.size()] = (int64_t)out.asmall.size();
}

namespace {

template <class T>
cudaError_t dev_alloc(T** p, size_t n, std::vector<void*>& owned) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e == cudaSuccess) owned.push_back(*p);
  return e;
}

template <class T>
cudaError_t dev_upload(T** p, const std::vector<T>& v, std::vector<void*>& owned) {
  cudaError_t e = dev_alloc(p, v.size(), owned);
  if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

// Decodes the sparse PBWT once, replaying the target-independent part of
// matchHapsFromCompressedPBWTSmall: read_full_pbwt_av / read_small_pbwt_av
// (haplotype_set.cpp:396-444), the small prefix array of init_rare (:655-662)
// and the merge of init_common (:640-652).
int Context::pbwt_prepare_panel() {
  const int N = host.N, L = host.L;
  const uint8_t* yp = sparse.ypacked.data();
  const size_t ylen = sparse.ypacked.size();
  size_t pos = 0;
  DevPbwt& D = pbwt;
  const int n_com_hq = host.n_com_hq;
  D.n_com_hq = n_com_hq;
  D.Wv = (N + 1 + 31) / 32;
  // Row l: V bits and their prefix counts (select_common_pd_fg), then the bits and
  // prefix counts of the small-PBWT positions merged at l (init_common); 16-byte
  // rows, staged by the sweep with cp.async.
  D.R = (4 * D.Wv + 2 + 3) / 4 * 4;
  const int Wv = D.Wv, R = D.R;
  cudaError_t e;
  if ((e = dev_alloc(&D.a_after, (size_t)n_com_hq * N, owned)) != cudaSuccess) return cuda_fail(e, "alloc pbwt");
  if ((e = dev_alloc(&D.vrow, (size_t)n_com_hq * R, owned)) != cudaSuccess) return cuda_fail(e, "alloc pbwt");

  std::vector<int32_t> before_id(n_com_hq, -1);
  std::vector<uint8_t> initc(n_com_hq, 0);
  std::vector<uint32_t> merged_host;  // concatenated merged arrays
  std::vector<int64_t> svoff(1, 0);
  std::vector<uint32_t> svbits, svpref;
  std::vector<int32_t> site_info(L, 0), site_run(L, 0), run_end(L, -1), common2tot;
  std::vector<uint32_t> A(N), B(N);
  std::iota(A.begin(), A.end(), 0u);
  std::vector<uint32_t> sA, sB;
  // staged upload of a_after / V rows
  const int chunk = std::max(1, (int)std::min<int64_t>(4096, (512ll << 20) / ((int64_t)N * 4 + 1)));
  std::vector<uint32_t> stage_a((size_t)chunk * N), stage_vr((size_t)chunk * R, 0u);
  int stage_first = 0, stage_n = 0;
  auto flush = [&]() -> cudaError_t {
    if (!stage_n) return cudaSuccess;
    cudaError_t x = cudaMemcpy(D.a_after + (size_t)stage_first * N, stage_a.data(), (size_t)stage_n * N * 4,
                               cudaMemcpyHostToDevice);
    if (x == cudaSuccess)
      x = cudaMemcpy(D.vrow + (size_t)stage_first * R, stage_vr.data(), (size_t)stage_n * R * 4,
                     cudaMemcpyHostToDevice);
    stage_first += stage_n;
    stage_n = 0;
    return x;
  };
  // Decode one column of `n` symbols from the stream into B (stable partition of A)
  // and its rank bits; returns false on a malformed stream.
  auto decode = [&](std::vector<uint32_t>& a, std::vector<uint32_t>& b, int n, int zeros, uint32_t* bits,
                    uint32_t* pref, int W) -> bool {
    if (zeros < 0 || zeros > n) return false;
    int u = 0, v = zeros, m = 0;
    std::fill(bits, bits + W, 0u);
    while (m < n) {
      if (pos >= ylen) return false;
      const uint8_t z = yp[pos++];
      const int len = p3_len(z);
      const int sym = z >> 7;
      if (len <= 0 || m + len > n) return false;
      int& occ = sym ? v : u;
      if (occ + len > (sym ? n : zeros)) return false;  // column counts disagree with cref/calt
      for (int i = m; i < m + len; ++i) {
        b[occ++] = a[i];
        if (sym) bits[i >> 5] |= 1u << (i & 31);
      }
      m += len;
    }
    pref[0] = 0;
    for (int w = 0; w < W; ++w) pref[w + 1] = pref[w] + (uint32_t)__builtin_popcount(bits[w]);
    a.swap(b);
    return true;
  };

  int l_hq = 0, l_all = 0, last_k = -1, rare_ord = 0;
  int run_l = -1, run_k0 = -1;
  for (int k = 0; k < L; ++k) {
    if (host.common[k]) common2tot.push_back(k);
    if (host.lq[k]) {
      site_info[k] = SK_LQ;
      site_run[k] = host.common[k] ? l_all : -1;
      l_all += host.common[k];
      continue;
    }
    if (host.common[k]) {
      const int64_t so = sparse.asmall_off[l_hq], sn = sparse.asmall_off[l_hq + 1] - so;
      if (sn > 0 && !(last_k >= 0 && host.common[last_k])) {
        const int32_t* posv = sparse.asmall.data() + so;
        std::vector<uint8_t> in_small(N, 0);
        for (int64_t i = 0; i < sn; ++i) in_small[posv[i]] = 1;
        int nz = posv[0];
        for (int p = nz + 1; p < N; ++p)
          if (!in_small[p]) A[nz++] = A[p];
        for (size_t i = 0; i < sA.size(); ++i, ++nz) A[nz] = sA[i];
        before_id[l_hq] = (int32_t)(merged_host.size() / N);
        merged_host.insert(merged_host.end(), A.begin(), A.end());
        initc[l_hq] = 1;
      } else {
        before_id[l_hq] = (l_hq == 0) ? -2 : -1;
      }
      if (stage_n == chunk && (e = flush()) != cudaSuccess) return cuda_fail(e, "pbwt upload");
      uint32_t* vb = stage_vr.data() + (size_t)stage_n * R;
      uint32_t* vp = vb + Wv;
      if (!decode(A, B, N, (int)host.cref[k], vb, vp, Wv))
        return (fail(GP_E_DATA, "sparse PBWT stream is malformed at site " + std::to_string(k)), GP_E_DATA);
      {
        uint32_t* sb = vb + 2 * Wv + 1;
        uint32_t* sp = sb + Wv;
        std::fill(sb, sb + 2 * Wv + 1, 0u);
        if (initc[l_hq])
          for (int64_t i = 0; i < sn; ++i) {
            const int32_t q = sparse.asmall[so + i];
            sb[q >> 5] |= 1u << (q & 31);
          }
        for (int w = 0; w < Wv; ++w) sp[w + 1] = sp[w] + (uint32_t)__builtin_popcount(sb[w]);
      }
      std::copy(A.begin(), A.end(), stage_a.begin() + (size_t)stage_n * N);
      ++stage_n;
      site_info[k] = SK_COMMON | (l_hq << 2);
      site_run[k] = l_all;
      ++l_hq;
      ++l_all;
    } else {
      if (last_k < 0 || host.common[last_k]) {
        // init_rare (haplotype_set.cpp:655-662)
        run_l = l_hq;
        run_k0 = k;
        const int64_t so = sparse.asmall_off[l_hq], sn = sparse.asmall_off[l_hq + 1] - so;
        sA.resize(sn);
        sB.resize(sn);
        for (int64_t i = 0; i < sn; ++i) sA[i] = A[sparse.asmall[so + i]];
      }
      const int n = (int)sA.size();
      const int W = (n + 1 + 31) / 32;
      const int zeros = host.major[k] ? (int)host.cref[k] : (int)(n - (int)host.calt[k]);
      const size_t b0 = svbits.size(), p0 = svpref.size();
      svbits.resize(b0 + W);
      svpref.resize(p0 + W + 1);
      if (!decode(sA, sB, n, zeros, svbits.data() + b0, svpref.data() + p0, W))
        return (fail(GP_E_DATA, "sparse PBWT stream is malformed at site " + std::to_string(k)), GP_E_DATA);
      svoff.push_back((int64_t)svbits.size());
      site_info[k] = SK_RARE | (rare_ord << 2);
      site_run[k] = run_l;
      run_end[run_k0] = k;
      ++rare_ord;
    }
    last_k = k;
  }
  if ((e = flush()) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if (pos != ylen)
    return (fail(GP_E_DATA, "sparse PBWT stream has trailing bytes (panel mismatch)"), GP_E_DATA);
  D.n_rare_hq = rare_ord;
  std::vector<float> cmp(L);
  for (int k = 0; k < L; ++k) cmp[k] = std::max(0.0f, (float)host.cm[k]);
  if ((e = dev_upload(&D.before_id, before_id, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.merged, merged_host, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.svoff, svoff, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.svbits, svbits, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.svpref, svpref, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.asoff, sparse.asmall_off, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.asidx, sparse.asmall, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.site_info, site_info, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.site_run, site_run, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.run_end, run_end, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  {
    if (sparse.asmall_off.back() >= ((int64_t)1 << 31))
      return (fail(GP_E_DATA, "sparse PBWT: small-column index list exceeds 2^31 entries"), GP_E_DATA);
    std::vector<int32_t> ev;
    for (int k = 0; k < L; ++k) {
      if (host.lq[k]) continue;
      const int kind = site_info[k] & 3;
      if (kind == SK_COMMON) {
        const int l = site_info[k] >> 2;
        const int64_t so = sparse.asmall_off[l], sn = sparse.asmall_off[l + 1] - so;
        const int32_t a0[8] = {k, l, (int32_t)host.cref[k], (int32_t)so,
                               (int32_t)sn, before_id[l], (int32_t)initc[l], common2tot[l > 0 ? l - 1 : 0]};
        ev.insert(ev.end(), a0, a0 + 8);
      } else if (run_end[k] >= 0) {
        const int l = site_run[k];
        const int64_t so = sparse.asmall_off[l], sn = sparse.asmall_off[l + 1] - so;
        const int32_t a0[8] = {k | (1 << 30), l, run_end[k], (int32_t)so, (int32_t)sn, 0, 0, 0};
        ev.insert(ev.end(), a0, a0 + 8);
        k = run_end[k];
      }
    }
    D.n_events = (int)(ev.size() / 8);
    int32_t* evd = nullptr;
    if ((e = dev_upload(&evd, ev, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
    D.events = reinterpret_cast<int4*>(evd);
  }
  if ((e = dev_upload(&D.init_common, initc, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.cm_pos, cmp, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  if ((e = dev_upload(&D.common2tot, common2tot, owned)) != cudaSuccess) return cuda_fail(e, "pbwt upload");
  D.cref = panel.cref;
  host.cm_pos = cmp;
  D.ready = true;
  return GP_OK;
}

// haplotype_set::allocatePBWT (haplotype_set.cpp:229-315): selection groups by
// rounded cM, halving the modulo for short regions; per-haplotype bookkeeping.
int Context::pbwt_prepare_targets(bool reset_state) {
  TargetWork& T = tw;
  const int N = host.N;
  int kglobal = 0;
  for (int i = 0; i < T.n; ++i) kglobal = std::max(kglobal, std::min(T.kpbwt_h[i], N));
  pbwt_active = (kglobal > 0 && kglobal < N);
  T.hap_target.clear();
  T.hap_which.clear();
  T.target_hap0.assign(T.n, 0);
  T.target_nhap.assign(T.n, 0);
  for (int i = 0; i < T.n; ++i) {
    T.target_hap0[i] = (int)T.hap_target.size();
    T.target_nhap[i] = T.ploidy_h[i];
    for (int j = 0; j < T.ploidy_h[i]; ++j) {
      T.hap_target.push_back(i);
      T.hap_which.push_back(j);
    }
  }
  const int nh = (int)T.hap_target.size();
  cudaError_t e;
  if ((e = T.d_hap_target.ensure(nh * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.d_hap_which.ensure(nh * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.d_target_hap0.ensure(T.n * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.d_target_nhap.ensure(T.n * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.d_kpbwt.ensure(T.n * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.tar_hap.ensure(nh)) != cudaSuccess) return cuda_fail(e, "alloc");
  std::vector<int32_t> kp(T.n);
  for (int i = 0; i < T.n; ++i) kp[i] = std::min(T.kpbwt_h[i], N);
  // on the context's stream, after any work still in flight there
  cudaMemcpyAsync(T.d_hap_target.ptr, T.hap_target.data(), nh * 4, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(T.d_hap_which.ptr, T.hap_which.data(), nh * 4, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(T.d_target_hap0.ptr, T.target_hap0.data(), T.n * 4, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(T.d_target_nhap.ptr, T.target_nhap.data(), T.n * 4, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(T.d_kpbwt.ptr, kp.data(), T.n * 4, cudaMemcpyHostToDevice, stream);
  // tar_hap is zero-initialised once per target set (haplotype_set.cpp:261) and
  // then carried across iterations; changing K (the learned proposal) keeps it
  if (reset_state) cudaMemsetAsync(T.tar_hap.ptr, 0, nh, stream);
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "pbwt targets");
  if (!pbwt_active) return GP_OK;

  // modulo and groups
  const int L = host.L;
  const std::vector<float>& cmp = host.cm_pos;
  float modulo = cfg.pbwt_modulo_cm;
  const float length = cmp[L - 1] - cmp[0];
  const int depth = cfg.pbwt_depth;
  if ((length / modulo) * 2 * depth < kglobal) {
    while ((length / modulo) * 2 * depth < kglobal && modulo > 0.02) modulo /= 2;
  }
  pbwt_modulo = modulo;
  std::vector<int32_t> grp;
  for (int l_hq = 0, l_all = 0, src = 0; l_all < host.n_com; ++l_all) {
    const int k = host.common_sites[l_all];
    if (host.lq[k]) continue;
    const int tmp = (int)std::round(cmp[k] / modulo);
    if (src != tmp) {
      src = tmp;
      if (l_hq > 0) grp.push_back(l_hq);
    }
    ++l_hq;
  }
  if (grp.empty() || grp.back() < host.n_com_hq) grp.push_back(host.n_com_hq);
  pbwt_grp = grp;
  if ((e = T.d_grp.ensure(grp.size() * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  cudaMemcpy(T.d_grp.ptr, grp.data(), grp.size() * 4, cudaMemcpyHostToDevice);
  const size_t cap = (size_t)tw_push_cap;
  if ((e = T.push_key.ensure((size_t)nh * depth * cap * 4)) != cudaSuccess) return cuda_fail(e, "alloc push");
  if ((e = T.push_id.ensure((size_t)nh * depth * cap * 4)) != cudaSuccess) return cuda_fail(e, "alloc push");
  if ((e = T.push_cnt.ensure((size_t)nh * depth * 4)) != cudaSuccess) return cuda_fail(e, "alloc push");
  if ((e = T.stored_bits.ensure(((size_t)host.n_com_hq + 32) / 32 * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.start_idx.ensure((size_t)nh * 4)) != cudaSuccess) return cuda_fail(e, "alloc");
  if ((e = T.overflow.ensure(4)) != cudaSuccess) return cuda_fail(e, "alloc");
  return GP_OK;
}

int Context::pbwt_select_states(int stage, int iteration, int Kp) {
  TargetWork& T = tw;
  ImputeWork& w = impute;
  if (!pbwt_active) {
    // Kpbwt >= n_ref_haps: the whole panel (conditioning_set.cpp:105-113)
    std::vector<uint32_t> hs((size_t)T.n * Kp);
    std::vector<int32_t> hn(T.n, host.N);
    for (int i = 0; i < T.n; ++i)
      for (int k = 0; k < host.N; ++k) hs[(size_t)i * Kp + k] = (uint32_t)k;
    cudaMemcpyAsync(w.states.ptr, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(w.nstates.ptr, hn.data(), T.n * 4, cudaMemcpyHostToDevice, stream);
    return cudaStreamSynchronize(stream) == cudaSuccess ? GP_OK : cuda_fail(cudaGetLastError(), "states");
  }
  PbwtSelectArgs a;
  a.P = pbwt;
  a.N = host.N;
  a.L = host.L;
  a.depth = cfg.pbwt_depth;
  a.n_haps = (int)T.hap_target.size();
  a.n_targets = T.n;
  a.cap = tw_push_cap;
  a.modulo = pbwt_modulo;
  a.lq = panel.lq;
  a.common = panel.common;
  a.major = panel.major;
  a.calt = panel.calt;
  a.h0 = T.h0.as<uint8_t>();
  a.h1 = T.h1.as<uint8_t>();
  a.hap_target = T.d_hap_target.as<int32_t>();
  a.hap_which = T.d_hap_which.as<int32_t>();
  a.target_hap0 = T.d_target_hap0.as<int32_t>();
  a.target_nhap = T.d_target_nhap.as<int32_t>();
  a.grp = T.d_grp.as<int32_t>();
  a.nstored = (int)pbwt_grp.size();
  a.stored_bits = T.stored_bits.as<uint32_t>();
  a.Wc = (host.L + 31) / 32;
  {
    cudaError_t ec = T.carry.ensure((size_t)a.n_haps * a.Wc * 4);
    if (ec != cudaSuccess) return cuda_fail(ec, "alloc carry");
  }
  a.carry = T.carry.as<uint32_t>();
  a.We = (pbwt.n_events + 31) / 32;
  {
    cudaError_t ec = T.ebits.ensure((size_t)a.n_haps * std::max(a.We, 1) * 4);
    if (ec != cudaSuccess) return cuda_fail(ec, "alloc event bits");
  }
  a.ebits = T.ebits.as<uint32_t>();
  a.grid_y_cap = grid_y_cap;
  a.start_idx = T.start_idx.as<int32_t>();
  a.tar_hap = T.tar_hap.as<uint8_t>();
  a.push_key = T.push_key.as<uint32_t>();
  a.push_id = T.push_id.as<uint32_t>();
  a.push_cnt = T.push_cnt.as<int32_t>();
  a.overflow = T.overflow.as<int32_t>();
  a.kpbwt = T.d_kpbwt.as<int32_t>();
  a.bitmap = T.bitmap.as<uint32_t>();
  a.union_rank = nullptr;
  if (learned.on) {
    cudaError_t eu = learned.urank.ensure((size_t)T.n * host.N * 4);
    if (eu != cudaSuccess) return cuda_fail(eu, "alloc union ranks");
    a.union_rank = learned.urank.as<int32_t>();
  }
  a.states = w.states.as<uint32_t>();
  a.nstates = w.nstates.as<int32_t>();
  a.Kp = Kp;
  a.seed = cfg.seed;
  a.iteration = iteration;
  cudaMemsetAsync(T.overflow.ptr, 0, 4, stream);
  int hpw = fixed_hpw ? fixed_hpw : tune_hpw;
  if (!hpw) {
    hpw = 2;
    if (a.n_haps >= 32) {
      // Autotune haplotypes per sweep warp: the sweep's only state carried across
      // iterations is tar_hap, restored before every candidate run.
      cudaError_t et = tune_tarhap.ensure((size_t)a.n_haps);
      if (et != cudaSuccess) return cuda_fail(et, "alloc tuning");
      launch_pbwt_prepare(a, stream);
      cudaMemcpyAsync(tune_tarhap.ptr, a.tar_hap, (size_t)a.n_haps, cudaMemcpyDeviceToDevice, stream);
      const int cand[4] = {1, 2, 4, 8};
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      float best = 1e30f;
      for (int ci = 0; ci < 4; ++ci) {
        cudaMemcpyAsync(a.tar_hap, tune_tarhap.ptr, (size_t)a.n_haps, cudaMemcpyDeviceToDevice, stream);
        cudaEventRecord(e0, stream);
        launch_pbwt_sweep(a, cand[ci], stream);
        cudaEventRecord(e1, stream);
        float ms = 1e30f;
        if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        tune_ms[3 + ci] = ms;
        if (ms < best) {
          best = ms;
          hpw = cand[ci];
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaMemcpyAsync(a.tar_hap, tune_tarhap.ptr, (size_t)a.n_haps, cudaMemcpyDeviceToDevice, stream);
      tune_hpw = hpw;
      prof.kernel_launches += 7;
    }
  }
  launch_pbwt_select(a, hpw, stream);
  prof.kernel_launches += 5;
  int32_t ovf = 0;
  cudaMemcpyAsync(&ovf, T.overflow.ptr, 4, cudaMemcpyDeviceToHost, stream);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "pbwt selection");
  if (ovf) return (fail(GP_E_DATA, "PBWT selection: per-level state list exceeded its capacity"), GP_E_DATA);
  (void)stage;
  return GP_OK;
}

int Context::pbwt_states_get(int target, int32_t* counts, int32_t* states, int cap) {
  TargetWork& T = tw;
  if (target < 0 || target >= T.n) return (fail(GP_E_ARG, "target out of range"), GP_E_ARG);
  const int K = cfg.pbwt_depth, C = tw_push_cap;
  const int h0 = T.target_hap0[target], nh = T.target_nhap[target];
  if (!pbwt_active) {
    for (int lv = 0; lv < K; ++lv) counts[lv] = 0;
    return GP_OK;
  }
  std::vector<int32_t> cnt((size_t)nh * K);
  std::vector<uint32_t> key((size_t)nh * K * C), id((size_t)nh * K * C);
  // copies on the context's stream, which the legacy default stream does not wait for
  cudaMemcpyAsync(cnt.data(), T.push_cnt.as<int32_t>() + (size_t)h0 * K, cnt.size() * 4, cudaMemcpyDeviceToHost,
                  stream);
  cudaMemcpyAsync(key.data(), T.push_key.as<uint32_t>() + (size_t)h0 * K * C, key.size() * 4,
                  cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(id.data(), T.push_id.as<uint32_t>() + (size_t)h0 * K * C, id.size() * 4, cudaMemcpyDeviceToHost,
                  stream);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "pbwt_states_get");
  int w = 0;
  for (int lv = 0; lv < K; ++lv) {
    int p[2] = {0, 0};
    int n = 0;
    while (true) {
      int j = -1;
      for (int q = 0; q < nh; ++q) {
        if (p[q] >= cnt[(size_t)q * K + lv]) continue;
        const uint32_t kq = key[((size_t)q * K + lv) * C + p[q]];
        if (j < 0 || kq < key[((size_t)j * K + lv) * C + p[j]]) j = q;
      }
      if (j < 0) break;
      const uint32_t h = id[((size_t)j * K + lv) * C + p[j]++];
      if (states && w < cap) states[w] = (int32_t)h;
      ++w;
      ++n;
    }
    counts[lv] = n;
  }
  return GP_OK;
}

}  // namespace gp

using gp::Context;

extern "C" {

int gp_pbwt_states_get(gp_ctx* ctx, int32_t target, int32_t* counts, int32_t* states, int32_t cap) {
  if (!ctx || !counts) return GP_E_ARG;
  return reinterpret_cast<Context*>(ctx)->pbwt_states_get(target, counts, states, cap);
}

int gp_build_sparse_pbwt(const gp_panel_desc* d, uint8_t* ypacked, int64_t* ypacked_len, int64_t* asmall_off,
                         int32_t* asmall_idx, int64_t* asmall_len) {
  if (!d || d->n_ref_haps <= 0 || d->n_sites <= 0 || !d->lq || !d->flag_common || !d->major || !d->cref ||
      !d->calt || !d->shap_off)
    return GP_E_ARG;
  const int N = d->n_ref_haps, L = d->n_sites;
  const int64_t nnz = d->shap_off[N];
  std::vector<int64_t> so(L + 1, 0);
  for (int64_t j = 0; j < nnz; ++j) {
    const int s = d->shap_sites[j];
    if (s < 0 || s >= L || d->flag_common[s]) return GP_E_DATA;
    so[s + 1]++;
  }
  for (int l = 0; l < L; ++l) so[l + 1] += so[l];
  std::vector<int32_t> sh(nnz);
  std::vector<int64_t> fill(so.begin(), so.end() - 1);
  for (int h = 0; h < N; ++h)
    for (int64_t j = d->shap_off[h]; j < d->shap_off[h + 1]; ++j) sh[fill[d->shap_sites[j]]++] = h;
  std::string msg;
  if (gp::validate_panel(N, L, d->lq, d->flag_common, d->major, d->cref, d->calt, d->hvar, so.data(), msg) != GP_OK)
    return GP_E_DATA;
  gp::SparsePbwt sp;
  gp::build_sparse_pbwt(N, L, d->lq, d->flag_common, d->major, d->cref, d->calt, d->hvar, so.data(), sh.data(), sp);
  if (ypacked_len) *ypacked_len = (int64_t)sp.ypacked.size();
  if (asmall_len) *asmall_len = (int64_t)sp.asmall.size();
  if (ypacked) std::memcpy(ypacked, sp.ypacked.data(), sp.ypacked.size());
  if (asmall_off) std::memcpy(asmall_off, sp.asmall_off.data(), sp.asmall_off.size() * 8);
  if (asmall_idx) std::memcpy(asmall_idx, sp.asmall.data(), sp.asmall.size() * 4);
  return GP_OK;
}

}  // extern "C"
