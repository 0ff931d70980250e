"""Precision of the imputation posteriors against the FP64 restatement of the
forward-backward (oracle/restate.c, following imputation_hmm.cpp:80-429): the
GPU computes in FP32 with per-site rescaling, as the reference does. The test
prints the largest absolute HP error per panel shape (run pytest with -s to see
it) and bounds it at 1e-5, the parity tolerance against the reference."""
import numpy as np
import pytest

from conftest import init_hl

TOL = 1e-5


def _max_err_vs_fp64(w, Ks, seed):
    from glimpse_b200 import native
    from oracle import oracle as O
    P, T = w.panel, w.targets
    rng = np.random.default_rng(seed)
    ctx = native.Context(P)
    try:
        states, hls, flats = [], [], []
        for i, K in enumerate(Ks):
            t = i % T.n
            states.append(np.sort(rng.choice(P.n_ref_haps, size=K, replace=False)).astype(np.uint32))
            hls.append(init_hl(T.gl[t], T.flat[t]))
            flats.append(T.flat[t])
        hp = ctx.impute_batch(states, np.stack(hls), np.stack(flats))
    finally:
        ctx.close()
    worst = 0.0
    for i in range(len(Ks)):
        ref, _ = O.restate_impute(P, states[i], hls[i], flats[i], precision=64)
        worst = max(worst, float(np.abs(hp[i].astype(np.float64) - ref.astype(np.float64)).max()))
    return worst


@pytest.mark.gpu
def test_small_panel_posteriors_vs_fp64():
    from glimpse_b200 import synth
    # the small workload: 1,000 haplotypes x 20,000 sites, K = 500
    w = synth.workload("small", seed=3)
    err = _max_err_vs_fp64(w, [500, 500, 500, 500], seed=1)
    print(f"\nsmall panel (1,000 x 20,000, K=500): max |HP - HP_fp64| = {err:.3e}")
    assert err <= TOL


@pytest.mark.gpu
def test_batched_panel_posteriors_vs_fp64():
    from glimpse_b200 import synth
    # the batched panel (10,000 haplotypes x 150,000 sites, 80% rare), one target, K at both ends of 400-1200
    w = synth.workload("batched", seed=1, n_targets=1)
    err = _max_err_vs_fp64(w, [400, 1200], seed=2)
    print(f"\nbatched panel (10,000 x 150,000, K=400 and 1200): max |HP - HP_fp64| = {err:.3e}")
    assert err <= TOL
