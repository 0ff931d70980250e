"""Imputation HMM parity: GPU forward-backward vs the reference's
imputation_hmm::computePosteriors (imputation_hmm.cpp:136-141), call by call on
identical HL, flat flags and conditioning sets. Tolerance: 1e-5 absolute on HP."""
import numpy as np
import pytest

from conftest import init_hl, ref_oracle_or_skip

TOL = 1e-5


def _random_states(rng, N, K):
    return np.sort(rng.choice(N, size=K, replace=False)).astype(np.uint32)


@pytest.mark.gpu
def test_impute_matches_reference(small_workload):
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    w = small_workload
    P, T = w.panel, w.targets
    orc = O.RefOracle(P, T, kinit=200, kpbwt=150)
    ctx = native.Context(P)
    rng = np.random.default_rng(11)
    states, hls, flats, refs = [], [], [], []
    for t in range(T.n):
        for K in (5, 8, 37, 256, 300):
            s = _random_states(rng, P.n_ref_haps, K)
            hl = init_hl(T.gl[t], T.flat[t])
            hp_ref, _ = orc.impute(s, hl, T.flat[t])
            states.append(s); hls.append(hl); flats.append(T.flat[t]); refs.append(hp_ref)
    hp = ctx.impute_batch(states, np.stack(hls), np.stack(flats))
    for i, r in enumerate(refs):
        err = np.abs(hp[i] - r).max()
        assert err <= TOL, f"case {i}: max |dHP| = {err}"


@pytest.mark.gpu
def test_impute_every_quad_count_matches_reference():
    """k_impute_warp is instantiated for J = 1..16 quads per lane (one warp per
    chain, J = the launch's largest K / 128 rounded up). One call per J, with
    K = 128 J - 17 for the first haplotype and half of it for the second; HP
    within 1e-5 of computePosteriors on each."""
    O = ref_oracle_or_skip()
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(2048, 6000, 0.5, 0.5, 2, ("uniform", 0.5, 2.0), ("fixed", 200), seed=61,
                                     sparse_maf=0.005)
    P, T = w.panel, w.targets
    orc = O.RefOracle(P, T, kinit=200, kpbwt=150)
    ctx = native.Context(P)
    rng = np.random.default_rng(13)
    try:
        for J in range(1, 17):
            states, hls, flats, refs = [], [], [], []
            for t, K in enumerate((128 * J - 17, (128 * J - 17) // 2)):
                s = _random_states(rng, P.n_ref_haps, K)
                hl = init_hl(T.gl[t], T.flat[t])
                refs.append(orc.impute(s, hl, T.flat[t])[0])
                states.append(s); hls.append(hl); flats.append(T.flat[t])
            hp = ctx.impute_batch(states, np.stack(hls), np.stack(flats))
            for i, r in enumerate(refs):
                err = float(np.abs(hp[i] - r).max())
                assert err <= TOL, f"J={J} haplotype {i}: max |dHP| = {err:.3e}"
    finally:
        ctx.close()


@pytest.mark.gpu
def test_chunked_store_matches_single_launch(small_workload, monkeypatch):
    """When the haplotypes' forward-backward stores do not fit the device-memory
    budget together, they run in consecutive chunks (GLIMPSE_B200_STORE_BUDGET_MB
    lowers the budget so that a small batch takes that path). The posteriors
    must be identical to the single-launch run."""
    from glimpse_b200 import native
    from conftest import init_hl
    w = small_workload
    P, T = w.panel, w.targets
    rng = np.random.default_rng(12)
    states, hls, flats = [], [], []
    for i in range(9):
        t = i % T.n
        states.append(np.sort(rng.choice(P.n_ref_haps, int(rng.integers(40, 500)), replace=False)).astype(np.uint32))
        hls.append(init_hl(T.gl[t], T.flat[t]))
        flats.append(T.flat[t])
    ctx = native.Context(P)
    try:
        whole = ctx.impute_batch(states, np.stack(hls), np.stack(flats))
        monkeypatch.setenv("GLIMPSE_B200_STORE_BUDGET_MB", "4")
        chunked = ctx.impute_batch(states, np.stack(hls), np.stack(flats))
        monkeypatch.delenv("GLIMPSE_B200_STORE_BUDGET_MB")
        assert np.array_equal(whole, chunked)
    finally:
        ctx.close()
