// Per-iteration PBWT state selection on the device
// (haplotype_set::matchHapsFromCompressedPBWTSmall, haplotype_set.cpp:317-394,
// with select_common_pd_fg :445-492, select_rare_pd_fg :494-560,
// init_common :562-653, init_rare :655-680, selectK :682-728) followed by the
// state union of conditioning_set::compactSelection (conditioning_set.cpp:96-104).
//
// Given the panel-side prefix/rank arrays (decoded once), every target haplotype's
// sweep over the sites depends only on its own alleles, so one thread runs one
// haplotype. Each selectK push is recorded with the key (site << 1 | phase) so
// that the union can rebuild the per-sample, per-level lists in the reference's
// push order (sites in order, init_common before select_common, haplotypes in
// order, down before up).
#include "select.h"

namespace gp {

namespace {

__device__ __forceinline__ int rank_v(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ pref, int x) {
  const uint32_t w = bits[x >> 5];
  const uint32_t m = (x & 31) ? (w & ((1u << (x & 31)) - 1u)) : 0u;
  return (int)(pref[x >> 5] + __popc(m));
}

// number of entries of the sorted array a[0..n) that are < x (std::lower_bound distance)
__device__ __forceinline__ int lower_count(const int32_t* __restrict__ a, int n, int x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

struct Pusher {
  uint32_t* key;
  uint32_t* id;
  int32_t* cnt;
  int cap;
  int32_t* overflow;
  __device__ void push(int level, uint32_t k, uint32_t h) {
    const int c = cnt[level];
    if (c >= cap) {
      *overflow = 1;
      return;
    }
    key[(size_t)level * cap + c] = k;
    id[(size_t)level * cap + c] = h;
    cnt[level] = c + 1;
  }
};

// haplotype_set::selectK (haplotype_set.cpp:682-728); arr == nullptr means the
// identity order.
__device__ void select_k(int pbwt_idx, int f, int g, int ref_rac, const uint32_t* __restrict__ arr, int a, int K,
                         int N, uint32_t key, Pusher& P) {
  int nh_up = 0, nh_down = 0;
  const int d_up = pbwt_idx - f;
  const int d_down = g - pbwt_idx;
  const int k1 = K;
  if (d_up < k1 && d_down < k1) {
    nh_up = d_up;
    nh_down = d_down;
  } else if (d_up >= k1 && d_down >= k1) {
    nh_up = k1;
    nh_down = k1;
  } else if (d_up < k1) {
    nh_down += k1 - d_up;
  } else if (d_down < k1) {
    nh_up += k1 - d_down;
  }
  const int max_hh = max(nh_up, nh_down);
  for (int o = 0, od = 0, ou = 0; o < max_hh; ++o) {
    if (od < nh_down) {
      const int idx = pbwt_idx + od;
      if (idx < N && ((idx >= ref_rac) == (a != 0))) {
        P.push(o, key, arr ? arr[idx] : (uint32_t)idx);
        ++od;
      }
    }
    if (ou < nh_up) {
      const int idx = pbwt_idx - (ou + 1);
      if (idx >= 0 && ((idx >= ref_rac) == (a != 0))) {
        P.push(o, key, arr ? arr[idx] : (uint32_t)idx);
        ++ou;
      }
    }
  }
}

// pbwt_stored groups and random starting positions (haplotype_set.cpp:336-348).
__global__ void k_pbwt_rng(PbwtSelectArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nw = (a.P.n_com_hq + 32) / 32;
  for (int i = 0; i < nw; ++i) a.stored_bits[i] = 0u;
  StreamCursor g(a.seed, RNG_PBWT, (uint32_t)a.iteration, 0u);
  int loffset = 0;
  for (int i = 0; i < a.nstored; ++i) {
    const uint32_t st = uniform_uint(g, (uint32_t)loffset, (uint32_t)(a.grp[i] - 1));
    a.stored_bits[st >> 5] |= 1u << (st & 31);
    loffset = a.grp[i];
  }
  for (int e = 0; e < a.n_haps; ++e) a.start_idx[e] = (int32_t)uniform_uint(g, 0u, (uint32_t)(a.N - 1));
}

// Per target haplotype, the non-LQ rare sites where it carries the non-major
// allele, as bits: what the init_rare scan of haplotype_set.cpp:655-680 looks
// for, so that the sweep can test a whole run of rare sites at once.
__global__ void k_rare_carriers(PbwtSelectArgs a) {
  const int hp = blockIdx.y;
  const int t = a.hap_target[hp];
  const uint8_t* H = (a.hap_which[hp] ? a.h1 : a.h0) + (size_t)t * a.L;
  for (int wi = blockIdx.x * blockDim.x + threadIdx.x; wi < a.Wc; wi += gridDim.x * blockDim.x) {
    uint32_t bits = 0u;
    const int s0 = wi << 5;
    const int n = min(32, a.L - s0);
    for (int i = 0; i < n; ++i) {
      const int s = s0 + i;
      if (!a.lq[s] && !a.common[s] && H[s] != a.major[s]) bits |= 1u << i;
    }
    a.carry[(size_t)hp * a.Wc + wi] = bits;
  }
}

// Any carrier bit in sites [k0, k1].
__device__ __forceinline__ bool any_carrier(const uint32_t* __restrict__ c, int k0, int k1) {
  const int w0 = k0 >> 5, w1 = k1 >> 5;
  for (int w = w0; w <= w1; ++w) {
    uint32_t v = c[w];
    if (w == w0) v &= ~0u << (k0 & 31);
    if (w == w1) v &= (k1 & 31) == 31 ? ~0u : ((1u << ((k1 & 31) + 1)) - 1u);
    if (v) return true;
  }
  return false;
}

__global__ void k_pbwt_sweep(PbwtSelectArgs a) {
  const int hp = blockIdx.x * blockDim.x + threadIdx.x;
  if (hp >= a.n_haps) return;
  const DevPbwt& P = a.P;
  const int N = a.N, L = a.L, K = a.depth;
  const int t = a.hap_target[hp];
  const uint8_t* H = (a.hap_which[hp] ? a.h1 : a.h0) + (size_t)t * L;
  const uint32_t* carry = a.carry + (size_t)hp * a.Wc;
  Pusher pu{a.push_key + (size_t)hp * K * a.cap, a.push_id + (size_t)hp * K * a.cap, a.push_cnt + (size_t)hp * K,
            a.cap, a.overflow};
  for (int o = 0; o < K; ++o) pu.cnt[o] = 0;
  int idx = a.start_idx[hp], f = 0, g = N;
  int sidx = 0, fs = 0, gs = 0;
  int last_reset = 0, last_rare = 0;
  int tar = a.tar_hap[hp];
  bool in_rare = false;
  int prev_ref_com = 0;
  int last_k = -1;
  const float half_mod = a.modulo / 2.0f;
  const float fifth_mod = a.modulo / 5.0f;
  for (int k = 0; k < L; ++k) {
    const int info = P.site_info[k];
    const int kind = info & 3;
    if (kind == SK_LQ) continue;
    if (kind == SK_COMMON) {
      const int l = info >> 2;
      const uint32_t* a_pre = l > 0 ? P.a_after + (size_t)(l - 1) * N : nullptr;
      if (P.init_common[l]) {
        const int64_t so = P.asoff[l];
        const int sn = (int)(P.asoff[l + 1] - so);
        const int32_t* sm = P.asidx + so;
        int nidx, nf, ng;
        if (in_rare) {
          nidx = N - sn + sidx;
          nf = last_reset >= last_rare ? 0 : N - sn + fs;
          ng = N - sn + gs;
          if (ng <= nf) {
            select_k(idx, f, g, prev_ref_com, a_pre, tar, K, N, (uint32_t)(k << 1), pu);
            nf = 0;
            ng = N;
            last_reset = k - 1;
          }
        } else {
          const int c0 = lower_count(sm, sn, f), c1 = lower_count(sm, sn, g), c2 = lower_count(sm, sn, idx);
          nidx = idx - c2;
          nf = f - c0;
          ng = g - c1;
          if (ng <= nf) {
            const int prev_site = P.common2tot[l > 0 ? l - 1 : 0];  // indexed by the HQ count, as the reference does
            if (__fsub_rn(P.cm_pos[prev_site], P.cm_pos[last_reset]) > fifth_mod)
              select_k(idx, f, g, prev_ref_com, a_pre, tar, K, N, (uint32_t)(k << 1), pu);
            nf = 0;
            ng = N - sn;
            last_reset = prev_site;
          }
        }
        idx = nidx;
        f = nf;
        g = ng;
      }
      // select_common_pd_fg at HQ common site l
      const int ref = (int)P.cref[k];
      const uint32_t* vb = P.vbits + (size_t)l * P.Wv;
      const uint32_t* vp = P.vpref + (size_t)l * (P.Wv + 1);
      const int prev_hap = tar;
      const int al = H[k];
      tar = al;
      const int vi = rank_v(vb, vp, idx), vf = rank_v(vb, vp, f), vg = rank_v(vb, vp, g);
      int nidx = al ? ref + vi : idx - vi;
      int nf = al ? ref + vf : f - vf;
      int ng = al ? ref + vg : g - vg;
      const bool stored = (a.stored_bits[l >> 5] >> (l & 31)) & 1u;
      bool reset = false;
      if (ng <= nf) {
        const int km1 = k > 0 ? k - 1 : 0;
        if (stored || __fsub_rn(P.cm_pos[km1], P.cm_pos[last_reset]) > half_mod) {
          const int bid = P.before_id[l];
          const uint32_t* b_arr = bid >= 0 ? P.merged + (size_t)bid * N : (bid == -1 ? a_pre : nullptr);
          select_k(idx, f, g, prev_ref_com, b_arr, prev_hap, K, N, (uint32_t)((k << 1) | 1), pu);
        }
        nf = al * ref;
        ng = al * N + (1 - al) * ref;
        last_reset = k;
        reset = true;
      }
      idx = nidx;
      f = nf;
      g = ng;
      if (!reset && stored) {
        select_k(idx, f, g, ref, P.a_after + (size_t)l * N, al, K, N, (uint32_t)((k << 1) | 1), pu);
        f = al * ref;
        g = al * N + (1 - al) * ref;
        last_reset = k;
      }
      prev_ref_com = ref;
    } else {
      const int r = info >> 2;
      const int l = P.site_run[k];
      const int64_t so = P.asoff[l];
      const int sn = (int)(P.asoff[l + 1] - so);
      if (last_k < 0 || a.common[last_k]) {
        // init_rare: is this haplotype in rareTarHaps for the run?
        const int kend = max(P.run_end[k], k);  // the run start's own entry is always >= k
        in_rare = sn > 0 && any_carrier(carry, k, kend);
        // Nothing happens at the run's sites for a haplotype outside rareTarHaps.
        // When no haplotype of the warp is in it, the warp continues after the run
        // together, so that its lanes keep walking the sites in step.
        if (__all_sync(__activemask(), !in_rare)) {
          last_k = kend;
          k = kend;
          continue;
        }
        if (in_rare) {
          const int32_t* sm = P.asidx + so;
          int fsn = lower_count(sm, sn, f);
          int gsn = lower_count(sm, sn, g);
          if (gsn <= fsn) {
            fsn = 0;
            gsn = sn;
            last_reset = k;
          }
          sidx = lower_count(sm, sn, idx);
          fs = fsn;
          gs = gsn;
        }
      }
      if (in_rare) {
        const int ref = a.major[k] ? (int)P.cref[k] : sn - (int)a.calt[k];
        const uint32_t* vb = P.svbits + P.svoff[r];
        const uint32_t* vp = P.svpref + (P.svoff[r] + r);
        const int vi = rank_v(vb, vp, sidx), vf = rank_v(vb, vp, fs), vg = rank_v(vb, vp, gs);
        int ns, nfs, ngs;
        if (H[k] != a.major[k]) {
          last_rare = k;
          ns = ref + vi;
          nfs = ref + vf;
          ngs = ref + vg;
          if (ngs <= nfs) {
            nfs = ref;
            ngs = sn;
            last_reset = k;
          }
        } else {
          ns = sidx - vi;
          nfs = fs - vf;
          ngs = gs - vg;
          if (ngs <= nfs) {
            nfs = 0;
            ngs = ref;
            last_reset = k;
          }
        }
        sidx = ns;
        fs = nfs;
        gs = ngs;
      }
    }
    last_k = k;
  }
  a.tar_hap[hp] = (uint8_t)tar;
}

// conditioning_set::compactSelection union (conditioning_set.cpp:96-104): levels
// in order, each level from its last push backwards, until Kpbwt states.
__global__ void k_pbwt_union(PbwtSelectArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_targets) return;
  const int N = a.N, K = a.depth, cap = a.cap;
  const int W = (N + 31) / 32;
  uint32_t* bm = a.bitmap + (size_t)t * W;
  for (int i = 0; i < W; ++i) bm[i] = 0u;
  const int kmax = a.kpbwt[t];
  const int h0 = a.target_hap0[t], nh = a.target_nhap[t];
  int count = 0;
  for (int lv = 0; lv < K && count < kmax; ++lv) {
    int p[2] = {0, 0};
    const uint32_t* keys[2] = {nullptr, nullptr};
    const uint32_t* ids[2] = {nullptr, nullptr};
    for (int j = 0; j < nh; ++j) {
      const int hp = h0 + j;
      p[j] = a.push_cnt[(size_t)hp * K + lv] - 1;
      keys[j] = a.push_key + ((size_t)hp * K + lv) * cap;
      ids[j] = a.push_id + ((size_t)hp * K + lv) * cap;
    }
    while (count < kmax && (p[0] >= 0 || (nh > 1 && p[1] >= 0))) {
      int j;
      if (nh < 2 || p[1] < 0) j = 0;
      else if (p[0] < 0) j = 1;
      else j = (keys[1][p[1]] >= keys[0][p[0]]) ? 1 : 0;
      const uint32_t h = ids[j][p[j]--];
      const uint32_t m = 1u << (h & 31);
      if (!(bm[h >> 5] & m)) {
        bm[h >> 5] |= m;
        ++count;
      }
    }
  }
  int k = 0;
  for (int i = 0; i < W; ++i) {
    uint32_t w = bm[i];
    while (w) {
      const int b = __ffs(w) - 1;
      w &= w - 1;
      if (k < a.Kp) a.states[(size_t)t * a.Kp + k] = (uint32_t)(i * 32 + b);
      ++k;
    }
  }
  a.nstates[t] = k;
}

}  // namespace

void launch_pbwt_select(const PbwtSelectArgs& a, cudaStream_t s) {
  k_pbwt_rng<<<1, 32, 0, s>>>(a);
  k_rare_carriers<<<dim3((a.Wc + 127) / 128, a.n_haps), 128, 0, s>>>(a);
  k_pbwt_sweep<<<(a.n_haps + 63) / 64, 64, 0, s>>>(a);
  k_pbwt_union<<<(a.n_targets + 63) / 64, 64, 0, s>>>(a);
}

}  // namespace gp
