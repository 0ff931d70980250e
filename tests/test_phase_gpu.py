"""Phasing HMM parity: GPU rephase vs the reference's
phasing_hmm::rephaseHaplotypes (phasing_hmm.cpp:247-302) on identical
haplotypes, flat flags, conditioning sets and random streams. The outputs are
discrete (sampled diplotypes and alleles) and must be identical."""
import numpy as np
import pytest

from conftest import ref_oracle_or_skip


def _noisy_haps(rng, truth, p=0.03):
    h = truth.copy()
    flip = rng.random(h.shape) < p
    h[flip] ^= 1
    return h


@pytest.mark.gpu
def test_rephase_matches_reference(small_workload):
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    w = small_workload
    P, T = w.panel, w.targets
    orc = O.RefOracle(P, T, kinit=200, kpbwt=150)
    ctx = native.Context(P)
    rng = np.random.default_rng(5)
    cases = []
    for t in range(T.n):
        for K in (6, 64, 257, 520):
            s = np.sort(rng.choice(P.n_ref_haps, size=K, replace=False)).astype(np.uint32)
            h0 = _noisy_haps(rng, T.truth[t, 0])
            h1 = _noisy_haps(rng, T.truth[t, 1])
            cases.append((s, h0, h1, T.flat[t], t))
    it = 3
    refs = [orc.rephase(s, h0, h1, fl, it, tid) for (s, h0, h1, fl, tid) in cases]
    g0, g1 = ctx.rephase_batch([c[0] for c in cases], np.stack([c[1] for c in cases]),
                               np.stack([c[2] for c in cases]), np.stack([c[3] for c in cases]), it,
                               target_ids=[c[4] for c in cases])
    bad = []
    for i, (r0, r1, dip) in enumerate(refs):
        n0 = int((g0[i] != r0).sum())
        n1 = int((g1[i] != r1).sum())
        if n0 or n1:
            bad.append((i, n0, n1, len(dip)))
    assert not bad, f"haplotype mismatches (case, #H0, #H1, nseg): {bad}"


@pytest.mark.gpu
@pytest.mark.parametrize("K", [200, 900, 1400, 1700, 2000])
def test_rephase_states_per_thread_instances(K):
    """k_phase is instantiated for the smallest J (states per thread, 256 threads)
    that holds the launch's largest K. One K per call reaches J = 1, 4, 6, 7 and 8
    (the test above runs J = 3; the iteration tests J = 2 and 5); the sampled
    haplotypes must equal rephaseHaplotypes' on identical inputs and streams."""
    O = ref_oracle_or_skip()
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(2048, 6000, 0.5, 0.5, 2, ("uniform", 0.5, 2.0), ("fixed", 200), seed=59,
                                     sparse_maf=0.005)
    P, T = w.panel, w.targets
    orc = O.RefOracle(P, T, kinit=200, kpbwt=150)
    ctx = native.Context(P)
    try:
        rng = np.random.default_rng(K)
        cases = []
        for t in range(T.n):
            s = np.sort(rng.choice(P.n_ref_haps, size=K, replace=False)).astype(np.uint32)
            cases.append((s, _noisy_haps(rng, T.truth[t, 0]), _noisy_haps(rng, T.truth[t, 1]), T.flat[t], t))
        it = 2
        refs = [orc.rephase(s, h0, h1, fl, it, tid) for (s, h0, h1, fl, tid) in cases]
        g0, g1 = ctx.rephase_batch([c[0] for c in cases], np.stack([c[1] for c in cases]),
                                   np.stack([c[2] for c in cases]), np.stack([c[3] for c in cases]), it,
                                   target_ids=[c[4] for c in cases])
        for i, (r0, r1, _) in enumerate(refs):
            assert np.array_equal(g0[i], r0) and np.array_equal(g1[i], r1), (K, i)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_invalid_diplotype_sums_return_data_error(small_workload):
    """SAMPLE_DIP with a NaN, infinite or sub-normal sum: the reference stops on
    an assertion (phasing_hmm.cpp:175); the library finishes the call and
    returns GP_E_DATA naming the target. A NaN err_phase makes every emission,
    and so every diplotype sum, NaN. The oracle is not run here (it would abort
    the process at that assertion)."""
    from glimpse_b200 import native
    w = small_workload
    P, T = w.panel, w.targets
    rng = np.random.default_rng(8)
    good = native.Context(P)
    bad = native.Context(P, err_phase=float("nan"))
    try:
        s = np.sort(rng.choice(P.n_ref_haps, size=64, replace=False)).astype(np.uint32)
        h0 = _noisy_haps(rng, T.truth[1, 0])
        h1 = _noisy_haps(rng, T.truth[1, 1])
        good.rephase_batch([s], h0[None], h1[None], T.flat[1][None], 2, target_ids=[1])
        with pytest.raises(native.GpError, match="target 7"):
            bad.rephase_batch([s], h0[None], h1[None], T.flat[1][None], 2, target_ids=[7])
        # the context stays usable: an iteration over the targets reports the same error
        bad.set_targets(T, kpbwt=T.kpbwt)
        with pytest.raises(native.GpError, match="invalid diplotype"):
            bad.iteration(native.STAGE_INIT, 0)
    finally:
        good.close()
        bad.close()


@pytest.mark.gpu
def test_chunked_phasing_matches_single_launch(small_workload, monkeypatch):
    """When the targets' stored phasing messages do not fit the device-memory
    budget together, k_phase runs in consecutive chunks of the batch
    (GLIMPSE_B200_STORE_BUDGET_MB lowers the budget so that a small batch takes
    that path). The rephased haplotypes must be identical."""
    from glimpse_b200 import native
    w = small_workload
    P, T = w.panel, w.targets
    rng = np.random.default_rng(9)
    cases = []
    for i in range(9):
        t = i % T.n
        s = np.sort(rng.choice(P.n_ref_haps, size=int(rng.integers(50, 520)), replace=False)).astype(np.uint32)
        cases.append((s, _noisy_haps(rng, T.truth[t, 0]), _noisy_haps(rng, T.truth[t, 1]), T.flat[t], t))
    args = ([c[0] for c in cases], np.stack([c[1] for c in cases]), np.stack([c[2] for c in cases]),
            np.stack([c[3] for c in cases]), 4)
    ctx = native.Context(P)
    try:
        a0, a1 = ctx.rephase_batch(*args, target_ids=[c[4] for c in cases])
        monkeypatch.setenv("GLIMPSE_B200_STORE_BUDGET_MB", "1")
        b0, b1 = ctx.rephase_batch(*args, target_ids=[c[4] for c in cases])
        monkeypatch.delenv("GLIMPSE_B200_STORE_BUDGET_MB")
        assert np.array_equal(a0, b0) and np.array_equal(a1, b1)
    finally:
        ctx.close()
