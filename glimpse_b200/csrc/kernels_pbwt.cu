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
#include <algorithm>

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

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(smem))),
               "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all_but(int n) {
  // wait until at most n of this thread's cp.async groups are pending (n < 8)
  switch (n) {
    case 0: asm volatile("cp.async.wait_group 0;\n" ::); break;
    case 1: asm volatile("cp.async.wait_group 1;\n" ::); break;
    case 2: asm volatile("cp.async.wait_group 2;\n" ::); break;
    case 3: asm volatile("cp.async.wait_group 3;\n" ::); break;
    case 4: asm volatile("cp.async.wait_group 4;\n" ::); break;
    case 5: asm volatile("cp.async.wait_group 5;\n" ::); break;
    case 6: asm volatile("cp.async.wait_group 6;\n" ::); break;
    default: asm volatile("cp.async.wait_group 7;\n" ::); break;
  }
}

// Warp-cooperative copy of one vrow row (R words, R a multiple of 4, 16-byte
// aligned) into a ring slot, spread over the live lanes of the warp.
__device__ __forceinline__ void stage_row(uint32_t* slot, const uint32_t* row, int R, int rank, int nlive) {
  for (int c = rank; c < (R >> 2); c += nlive) cp_async16(slot + 4 * c, row + 4 * c);
}

// Per-level push lists of one target haplotype. The counts live in shared
// memory (level-major, one column per lane) while the sweep runs and are
// written back to push_cnt at its end.
struct Pusher {
  uint32_t* key;
  uint32_t* id;
  int32_t* cnt;  // shared: cnt[level * 32]
  int cap;
  int32_t* overflow;
  __device__ __forceinline__ void push(int level, uint32_t k, uint32_t h) {
    const int c = cnt[level * 32];
    if (c >= cap) {
      *overflow = 1;
      return;
    }
    key[(size_t)level * cap + c] = k;
    id[(size_t)level * cap + c] = h;
    cnt[level * 32] = c + 1;
  }
};

// haplotype_set::selectK (haplotype_set.cpp:682-728); arr == nullptr means the
// identity order. The reference walks down (pbwt_idx, pbwt_idx + 1, ...) and up
// (pbwt_idx - 1, ...) one level at a time and stops a side at its first position
// outside [0, N) or on the other side of ref_rac than allele a; positions on the
// allowed side of ref_rac form an interval, so each side pushes a run whose
// length is known up front, and the loads of the run are independent.
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
  const bool alt = a != 0;
  int cd = 0, cu = 0;
  if (pbwt_idx >= 0 && pbwt_idx < N && ((pbwt_idx >= ref_rac) == alt)) {
    const int lim = alt ? N : min(ref_rac, N);
    cd = min(nh_down, lim - pbwt_idx);
  }
  const int p = pbwt_idx - 1;
  if (p >= 0 && p < N && ((p >= ref_rac) == alt)) {
    const int lo = alt ? max(ref_rac, 0) : 0;
    cu = min(nh_up, p - lo + 1);
  }
  const int n = max(cd, cu);
#pragma unroll 4
  for (int o = 0; o < n; ++o) {
    if (o < cd) P.push(o, key, arr ? arr[pbwt_idx + o] : (uint32_t)(pbwt_idx + o));
    if (o < cu) P.push(o, key, arr ? arr[p - o] : (uint32_t)(p - o));
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

// The per-haplotype bit of every sweep event (PbwtSelectArgs::ebits): the
// allele H[k] at an HQ common site k, or for a run of rare sites [k0, kend] the
// init_rare test (haplotype_set.cpp:655-680), sn > 0 and a carrier bit in the run.
// The sweep reads one word per 32 events, a chunk ahead, instead of a scattered
// byte or carrier load per event on its sequential path. Thread x of a block is
// haplotype blockIdx.x * blockDim.x + x, and blockIdx.y the chunk of 32 events,
// so the event records a warp reads are the same for all its lanes.
__global__ void k_event_bits(PbwtSelectArgs a) {
  const int hp = blockIdx.x * blockDim.x + threadIdx.x;
  if (hp >= a.n_haps) return;
  const int nev = a.P.n_events;
  const int t = a.hap_target[hp];
  const uint8_t* H = (a.hap_which[hp] ? a.h1 : a.h0) + (size_t)t * a.L;
  const uint32_t* carry = a.carry + (size_t)hp * a.Wc;
  for (int c = blockIdx.y; c < a.We; c += gridDim.y) {  // gridDim.y is capped at grid_y_cap <= 65535
    uint32_t bits = 0u;
    const int n = min(32, nev - (c << 5));
    for (int i = 0; i < n; ++i) {
      const int e = (c << 5) + i;
      const int4 r0 = a.P.events[2 * e];
      const int4 r1 = a.P.events[2 * e + 1];
      bool b;
      if (!(r0.x & (1 << 30))) b = H[r0.x] != 0;
      else b = r1.x > 0 && any_carrier(carry, r0.x & ~(1 << 30), r0.z);
      if (b) bits |= 1u << i;
    }
    a.ebits[(size_t)hp * a.We + c] = bits;
  }
}

// Haplotypes per sweep warp (hpw, a power of two, chosen by the autotuner).
// Lane l runs haplotype l % hpw of its warp's group: lanes l, l + hpw, ... run
// the same haplotype, take the same branches and write the same values to the
// same addresses, so a warp diverges only over hpw haplotypes while all 32
// lanes share the row staging.
//
// One warp per block; lane l runs target haplotype blockIdx.x * hpw + l % hpw
// (measured at 256 targets: 39 ms per sweep with 32 haplotypes per warp, 33 ms
// with 2, as a warp runs every branch any of its haplotypes takes).
// The lanes of a warp walk the event list (non-LQ common sites and runs of rare sites) in step: every branch
// that skips work is warp-uniform. Shared memory per warp holds
//   ring    D slots, one per HQ common site l, filled by cp.async D common sites
//           ahead with the rank row of l (R words: the V ranks of
//           select_common_pd_fg and the small-PBWT position ranks of init_common);
//   evbuf   two chunks of 32 event records (the next chunk is loaded one chunk ahead);
//   scnt    the per-level push counts, one column per lane.
// D = 0 reads the rows from global memory (panels whose rows do not fit in
// shared memory).
__global__ void __launch_bounds__(32) k_pbwt_sweep(PbwtSelectArgs a, int D, int hpw) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int hp = blockIdx.x * hpw + (lane & (hpw - 1));
  const unsigned live = __ballot_sync(0xffffffffu, hp < a.n_haps);
  if (hp >= a.n_haps) return;
  const int rank = __popc(live & ((1u << lane) - 1u)), nlive = __popc(live);
  const DevPbwt& P = a.P;
  const int R = P.R, Wv = P.Wv, ncom = P.n_com_hq, nev = P.n_events;
  const int N = a.N, K = a.depth;
  uint32_t* ring = smem;
  int4* evbuf = reinterpret_cast<int4*>(smem + (size_t)D * R);  // [2][32][2]
  int32_t* scnt = reinterpret_cast<int32_t*>(evbuf + 2 * 32 * 2) + lane;  // [K][32]

  if (D > 0) {
    for (int j = 0; j < D; ++j) {
      if (j < ncom) stage_row(ring + (size_t)j * R, P.vrow + (size_t)j * R, R, rank, nlive);
      cp_commit();
    }
  }
  int ri = 0;  // ring slot of the next HQ common site
  // Event chunk c (32 records) goes to evbuf[c & 1], spread over the live lanes
  // (the last warp of the grid may have fewer than 32); chunk c + 1 is loaded
  // when chunk c starts.
  auto load_chunk = [&](int c) {
    for (int i = rank; i < 32; i += nlive) {
      const int en = (c << 5) + i;
      if (en < nev) {
        evbuf[((c & 1) * 32 + i) * 2] = P.events[2 * en];
        evbuf[((c & 1) * 32 + i) * 2 + 1] = P.events[2 * en + 1];
      }
    }
  };
  load_chunk(0);
  load_chunk(1);
  __syncwarp(live);

  const int L = a.L;
  const int t = a.hap_target[hp];
  const uint8_t* H = (a.hap_which[hp] ? a.h1 : a.h0) + (size_t)t * L;
  // event bits of the current chunk and of the next one
  const uint32_t* eb = a.ebits + (size_t)hp * a.We;
  uint32_t ebw = a.We > 0 ? eb[0] : 0u;
  uint32_t ebn = a.We > 1 ? eb[1] : 0u;
  Pusher pu{a.push_key + (size_t)hp * K * a.cap, a.push_id + (size_t)hp * K * a.cap, scnt, a.cap, a.overflow};
  for (int o = 0; o < K; ++o) scnt[o * 32] = 0;
  int idx = a.start_idx[hp], f = 0, g = N;
  int sidx = 0, fs = 0, gs = 0;
  int last_reset = 0, last_rare = 0;
  int tar = a.tar_hap[hp];
  bool in_rare = false;
  int prev_ref_com = 0;
  const float half_mod = a.modulo / 2.0f;
  const float fifth_mod = a.modulo / 5.0f;

  for (int e = 0; e < nev; ++e) {
    const int c = e >> 5;
    if ((e & 31) == 0 && e > 0) {
      __syncwarp(live);  // chunk c - 1 is no longer read
      load_chunk(c + 1);
      ebw = ebn;
      ebn = c + 1 < a.We ? eb[c + 1] : 0u;
    }
    const bool ebit = (ebw >> (e & 31)) & 1u;
    const int4 r0 = evbuf[((c & 1) * 32 + (e & 31)) * 2];
    const int4 r1 = evbuf[((c & 1) * 32 + (e & 31)) * 2 + 1];
    const int sn = r1.x;
    if (!(r0.x & (1 << 30))) {
      // ---------------- HQ common site ----------------
      const int k = r0.x, l = r0.y, ref = r0.z;
      const uint32_t* a_pre = l > 0 ? P.a_after + (size_t)(l - 1) * N : nullptr;
      // rank row of l: the ring slot, or global memory without a ring
      const uint32_t* row = P.vrow + (size_t)l * R;
      uint32_t* slot = nullptr;
      if (D > 0) {
        slot = ring + (size_t)ri * R;
        row = slot;
        cp_wait_all_but(D - 1);  // this lane's part of slot l has landed
        __syncwarp(live);        // and every other lane's
      }
      if (r1.z) {  // init_common
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
          // numbers of small-PBWT positions below f, g and idx: ranks in the row's second bit vector
          const uint32_t* sb = row + 2 * Wv + 1;
          const int c0 = rank_v(sb, sb + Wv, f), c1 = rank_v(sb, sb + Wv, g), c2 = rank_v(sb, sb + Wv, idx);
          nidx = idx - c2;
          nf = f - c0;
          ng = g - c1;
          if (ng <= nf) {
            const int prev_site = r1.w;  // common2tot indexed by the HQ count, as the reference does
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
      const int prev_hap = tar;
      const int al = ebit ? 1 : 0;  // H[k]
      tar = al;
      const int vi = rank_v(row, row + Wv, idx), vf = rank_v(row, row + Wv, f), vg = rank_v(row, row + Wv, g);
      if (D > 0) {
        __syncwarp(live);  // the slot is free again
        if (l + D < ncom) stage_row(slot, P.vrow + (size_t)(l + D) * R, R, rank, nlive);
        cp_commit();
        ri = (ri + 1 == D) ? 0 : ri + 1;
      }
      int nidx = al ? ref + vi : idx - vi;
      int nf = al ? ref + vf : f - vf;
      int ng = al ? ref + vg : g - vg;
      const bool stored = (a.stored_bits[l >> 5] >> (l & 31)) & 1u;
      bool reset = false;
      if (ng <= nf) {
        const int km1 = k > 0 ? k - 1 : 0;
        if (stored || __fsub_rn(P.cm_pos[km1], P.cm_pos[last_reset]) > half_mod) {
          const int bid = r1.y;
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
      // ---------------- run of rare sites [k0, kend] ----------------
      const int k0 = r0.x & ~(1 << 30), kend = r0.z, so = r0.w;
      // init_rare: is this haplotype in rareTarHaps for the run?
      in_rare = ebit;  // sn > 0 and a carrier bit in [k0, kend]
      // Nothing happens at the run's sites for a haplotype outside rareTarHaps;
      // when no haplotype of the warp is in it, the warp goes on to the next event.
      if (__all_sync(live, !in_rare)) continue;
      if (in_rare) {
        const int32_t* sm = P.asidx + so;
        int fsn = lower_count(sm, sn, f);
        int gsn = lower_count(sm, sn, g);
        if (gsn <= fsn) {
          fsn = 0;
          gsn = sn;
          last_reset = k0;
        }
        sidx = lower_count(sm, sn, idx);
        fs = fsn;
        gs = gsn;
      }
      for (int k = k0; k <= kend; ++k) {
        const int info = P.site_info[k];
        if ((info & 3) == SK_LQ) continue;
        if (!in_rare) continue;
        const int r = info >> 2;
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
  }
  if (D > 0) cp_wait_all_but(0);
  for (int o = 0; o < K; ++o) a.push_cnt[(size_t)hp * K + o] = scnt[o * 32];
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
        if (a.union_rank) a.union_rank[(size_t)t * N + h] = (lv << 16) | min(count, 0xFFFF);
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

static size_t sweep_smem(const PbwtSelectArgs& a, int& D) {
  // Ring of D rank rows, D <= 8, within 96 KB.
  const size_t slot_bytes = (size_t)a.P.R * 4;
  D = (int)std::min<size_t>(8, (96u << 10) / slot_bytes);
  if (D < 2) D = 0;
  return (size_t)D * slot_bytes + 2 * 32 * 2 * 16 + (size_t)a.depth * 32 * 4;
}

void launch_pbwt_sweep(const PbwtSelectArgs& a, int hpw, cudaStream_t s) {
  int D = 0;
  const size_t smem = sweep_smem(a, D);
  if (smem > (48u << 10)) set_smem_limit_once<k_pbwt_sweep>(200 << 10);
  k_pbwt_sweep<<<(a.n_haps + hpw - 1) / hpw, 32, smem, s>>>(a, D, hpw);
}

void launch_pbwt_select(const PbwtSelectArgs& a, int hpw, cudaStream_t s) {
  launch_pbwt_prepare(a, s);
  launch_pbwt_sweep(a, hpw, s);
  k_pbwt_union<<<(a.n_targets + 63) / 64, 64, 0, s>>>(a);
}

void launch_pbwt_prepare(const PbwtSelectArgs& a, cudaStream_t s) {
  k_pbwt_rng<<<1, 32, 0, s>>>(a);
  k_rare_carriers<<<dim3((a.Wc + 127) / 128, a.n_haps), 128, 0, s>>>(a);
  const int ycap = std::max(1, std::min(a.grid_y_cap, 65535));
  if (a.We > 0) k_event_bits<<<dim3((a.n_haps + 127) / 128, std::min(a.We, ycap)), 128, 0, s>>>(a);
}

}  // namespace gp
