"""The learned state-selection proposal through the C-ABI.

  * Label HMM: per-window state posteriors (gp_state_posteriors) against the
    FP64 restatement (oracle/restate.c rs_state_post) on identical inputs.
  * The proposal runs inside a Gibbs iteration: trained on the targets' own
    HMM posteriors, enabled for a burn-in iteration, it yields sorted, unique
    conditioning sets of at most each target's K drawn from the PBWT
    candidates, and posteriors that are probabilities.
  * Plain PBWT selection is restored when the proposal is disabled: the
    iteration matches a context that never enabled it."""
import numpy as np
import pytest

from conftest import init_hl


@pytest.mark.gpu
def test_state_posteriors_match_fp64(small_workload):
    from glimpse_b200 import native
    from oracle import oracle as O
    w = small_workload
    P, T = w.panel, w.targets
    ctx = native.Context(P)
    try:
        rng = np.random.default_rng(4)
        states, hls, flats = [], [], []
        for t, K in zip(range(T.n), (37, 256, 599)):
            states.append(np.sort(rng.choice(P.n_ref_haps, K, replace=False)).astype(np.uint32))
            hls.append(init_hl(T.gl[t], T.flat[t]))
            flats.append(T.flat[t])
        mass, ns = ctx.state_posteriors(states, np.stack(hls), np.stack(flats))
        for i in range(len(states)):
            ref, rns = O.restate_state_post(P, states[i], hls[i], flats[i])
            assert np.array_equal(ns[i], rns)
            # each polymorphic site contributes posteriors that sum to 1
            assert np.allclose(mass[i].sum(1), ns[i], rtol=1e-4, atol=1e-3)
            err = float(np.abs(mass[i] - ref).max())
            assert err <= 2e-4 * max(1, int(ns[i].max())) ** 0.5, f"haplotype {i}: max |dmass| {err:.2e}"
    finally:
        ctx.close()


def _workload():
    from glimpse_b200 import synth
    return synth.make_panel_and_targets(2000, 12000, 1.5, 0.6, 8, ("uniform", 0.5, 2.0), ("fixed", 120), seed=31,
                                        sparse_maf=0.005)


@pytest.mark.gpu
def test_learned_selection_in_iteration():
    from glimpse_b200 import native
    w = _workload()
    P, T = w.panel, w.targets
    kw = dict(kinit=300, kpbwt=120, pbwt_depth=8, pbwt_modulo_cm=0.05)
    ctx = native.Context(P, **kw)
    try:
        ctx.set_targets(T, kpbwt=T.kpbwt)
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
        losses = ctx.learned_train(kcand=512, kpos=8.0, steps=60, batch=4096, lr=1e-3, seed=2)
        assert np.isfinite(losses).all()
        assert losses[-10:].mean() < losses[:10].mean()
        ctx.learned_enable(True, kcand=512)
        ctx.iteration(native.STAGE_BURN, 2)
        for t in range(T.n):
            st = ctx.states(t)
            assert 0 < st.size <= T.kpbwt[t]
            assert np.all(np.diff(st.astype(np.int64)) > 0)
            h0, h1 = ctx.posteriors(t)
            assert np.isfinite(h0).all() and np.isfinite(h1).all()
            assert np.allclose(h0[0::2] + h0[1::2], 1.0, atol=1e-4)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_disabling_restores_plain_selection():
    from glimpse_b200 import native
    w = _workload()
    P, T = w.panel, w.targets
    kw = dict(kinit=300, kpbwt=120, pbwt_depth=8, pbwt_modulo_cm=0.05)
    a, b = native.Context(P, **kw), native.Context(P, **kw)
    try:
        for c in (a, b):
            c.set_targets(T, kpbwt=T.kpbwt)
            c.iteration(native.STAGE_INIT, 0)
        a.mlp_init(5)
        a.learned_enable(True, kcand=400)
        a.learned_enable(False, kcand=400)
        a.iteration(native.STAGE_BURN, 1)
        b.iteration(native.STAGE_BURN, 1)
        for t in range(T.n):
            assert np.array_equal(a.states(t), b.states(t))
        ha, hb = a.haps(), b.haps()
        assert np.array_equal(ha[0], hb[0]) and np.array_equal(ha[1], hb[1])
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_feature_chunks_do_not_change_selection(monkeypatch):
    """The learned selection computes feature rows and their scores in chunks of
    targets when the rows do not fit the memory budget together
    (GLIMPSE_B200_STORE_BUDGET_MB lowers the budget so that each chunk holds one
    or two of these targets). The conditioning sets and haplotypes must be
    identical to the run whose rows fit at once."""
    from glimpse_b200 import native
    w = _workload()
    P, T = w.panel, w.targets
    kw = dict(kinit=300, kpbwt=120, pbwt_depth=8, pbwt_modulo_cm=0.05)
    a, b = native.Context(P, **kw), native.Context(P, **kw)
    try:
        for c in (a, b):
            c.set_targets(T, kpbwt=T.kpbwt)
            c.iteration(native.STAGE_INIT, 0)
            c.mlp_init(5)
            c.learned_enable(True, kcand=400)
        a.iteration(native.STAGE_BURN, 1)
        monkeypatch.setenv("GLIMPSE_B200_STORE_BUDGET_MB", "1")
        b.iteration(native.STAGE_BURN, 1)
        monkeypatch.delenv("GLIMPSE_B200_STORE_BUDGET_MB")
        for t in range(T.n):
            assert np.array_equal(a.states(t), b.states(t))
        ha, hb = a.haps(), b.haps()
        assert np.array_equal(ha[0], hb[0]) and np.array_equal(ha[1], hb[1])
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_autotuned_shapes_do_not_change_results():
    """The autotuner picks chains per CTA (imputation) and haplotypes per warp
    (PBWT sweep) by timing; results must not depend on either. Two contexts
    with opposite fixed shapes give identical states, posteriors and
    haplotypes, and an autotuned context reports the shapes it chose."""
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(1500, 8000, 1.0, 0.5, 20, ("uniform", 0.5, 2.0), ("uniform", 100, 300),
                                     seed=41, sparse_maf=0.005)
    P, T = w.panel, w.targets
    kw = dict(kinit=250, kpbwt=int(T.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    ctxs = [native.Context(P, **kw) for _ in range(3)]
    try:
        ctxs[0].tuning_set(1, 1)
        ctxs[1].tuning_set(4, 8)
        for c in ctxs:
            c.set_targets(T, kpbwt=T.kpbwt)
            c.iteration(native.STAGE_INIT, 0)
            c.iteration(native.STAGE_BURN, 1)
        for t in range(T.n):
            a, b = ctxs[0].posteriors(t), ctxs[1].posteriors(t)
            assert np.array_equal(ctxs[0].states(t), ctxs[1].states(t))
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            assert np.array_equal(ctxs[0].states(t), ctxs[2].states(t))
        h = [c.haps() for c in ctxs]
        assert np.array_equal(h[0][0], h[1][0]) and np.array_equal(h[0][1], h[2][1])
        cpc, hpw, _, ms = ctxs[2].tuning()
        assert cpc in (1, 2, 4) and hpw in (1, 2, 4, 8)
        assert (ms[:3] != 0).any() and (ms[3:7] > 0).all()
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.gpu
def test_phasing_placement_does_not_change_results():
    """A batch of one to two targets per SM: the phasing placements (decreasing
    work, the default; heaviest alone, the rest paired) give identical haplotypes."""
    import torch
    from glimpse_b200 import native, synth
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n = sms + sms // 2
    w = synth.make_panel_and_targets(600, 3000, 0.3, 0.5, n, ("uniform", 0.5, 2.0), ("uniform", 60, 300), seed=43,
                                     sparse_maf=0.01)
    P, T = w.panel, w.targets
    kw = dict(kinit=150, kpbwt=int(T.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    ctxs = [native.Context(P, **kw) for _ in range(3)]
    try:
        ctxs[0].tuning_set(0, 0, 1)
        ctxs[1].tuning_set(0, 0, 2)
        for c in ctxs:
            c.set_targets(T, kpbwt=T.kpbwt)
            c.iteration(native.STAGE_INIT, 0)
            c.iteration(native.STAGE_BURN, 1)
        h = [c.haps() for c in ctxs]
        for i in (1, 2):
            assert np.array_equal(h[0][0], h[i][0]) and np.array_equal(h[0][1], h[i][1])
        assert ctxs[2].tuning()[2] == 1 and ctxs[1].tuning()[2] == 2
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.gpu
def test_adaptive_set_size_stays_in_bounds():
    """With gp_learned_size(min_prob, kmin) the network sizes each conditioning
    set: between kmin and the target's K, and fewer states when min_prob rises."""
    from glimpse_b200 import native
    w = _workload()
    P, T = w.panel, w.targets
    ctx = native.Context(P, kinit=300, kpbwt=200, pbwt_depth=8, pbwt_modulo_cm=0.05)
    try:
        ctx.set_targets(T, kpbwt=np.full(T.n, 200, np.int32))
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
        ctx.learned_train(kcand=512, kpos=8.0, steps=80, batch=4096, lr=1e-3, seed=3)
        ctx.learned_enable(True, kcand=512)
        sizes = {}
        for prob in (0.2, 0.8):
            ctx.learned_size(prob, 16)
            ctx.iteration(native.STAGE_BURN, 2)
            sizes[prob] = np.array([ctx.states(t).size for t in range(T.n)])
            assert (sizes[prob] >= 16).all() and (sizes[prob] <= 200).all()
        assert sizes[0.8].sum() <= sizes[0.2].sum()
    finally:
        ctx.close()


@pytest.mark.gpu
def test_training_is_deterministic():
    """The training step's sums run in a fixed order (split-K partials and the
    loss head's per-block partials added in block order, no float atomics), so
    the same start gives the same parameters and losses on every run."""
    from glimpse_b200 import native
    w = _workload()
    P, T = w.panel, w.targets
    ctx = native.Context(P, kinit=300, kpbwt=120, pbwt_depth=8, pbwt_modulo_cm=0.05)
    try:
        ctx.set_targets(T, kpbwt=T.kpbwt)
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
        runs = []
        for _ in range(2):
            ctx.mlp_init(5)
            losses = ctx.learned_train(kcand=256, kpos=8.0, steps=20, batch=4096, lr=1e-3, seed=3)
            runs.append((losses, ctx.mlp_params()))
        assert np.array_equal(runs[0][0], runs[1][0])
        assert np.array_equal(runs[0][1], runs[1][1])
    finally:
        ctx.close()
