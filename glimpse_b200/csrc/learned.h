// The learned state-selection proposal around the scoring network (mlp.h):
// candidate reference haplotypes come from the PBWT selection run with a larger
// K; each (target, window of 256 common sites, candidate) gets kMlpIn features
// from bit operations on the panel and the target's current haplotypes and
// genotype likelihoods; the network scores them; per window the top kTopR
// candidates are ranked and the conditioning set is their union in rank order,
// cut at the target's K. Training labels are per-window state posteriors of
// the HMM over the whole candidate set.
#pragma once
#include <vector>

#include "internal.h"

namespace gp {

constexpr int kWinWords = 8;                  // 32-bit words (of common rows) per window
constexpr int kWinSites = 32 * kWinWords;     // 256 common sites per window
constexpr int kTopR = 32;                     // ranks per window entering the union
constexpr int kMaxCand = 2048;                // candidates per target
constexpr int kPlanes = 5;                    // target bit planes: hap0, hap1, GL-confident, GL alt, GL ref

struct LearnedWork {
  bool on = false;
  int kcand = 0;                       // PBWT candidates per target
  std::vector<int32_t> kfinal;         // conditioning-set size per target (the caller's Kpbwt)
  DevBuf d_kfinal, planes, cand, ncand, x, score, best, cnt, site_win, nsites, mass0, mass1, astore, aoff;
  DevBuf xall, yall, wall, idx;
  DevBuf urank;                        // [n][N]: PBWT level << 16 | insertion index of every union member
  DevBuf maxs;                         // [n][Kpc]: a candidate's best score over the windows that ranked it
  DevBuf tarhap_save;                  // the targets' PBWT sweep state, kept across a training sweep
  float min_logit = 0.f;               // adaptive size: keep candidates whose best score reaches this logit
  int kmin = 0;                        // adaptive size: at least this many states (0: fixed size, the caller's K)
  int nwin = 0;
  std::vector<DevBuf*> all() {
    return {&d_kfinal, &planes, &cand, &ncand, &x, &score, &best, &cnt, &site_win, &nsites, &mass0, &mass1,
            &astore, &aoff, &xall, &yall, &wall, &idx, &urank, &maxs, &tarhap_save};
  }
};

}  // namespace gp
