"""The reference's --state-list (caller_parameters.cpp:73; haplotype_set::read_list_states,
haplotype_set.cpp:835-857; conditioning_set::compactSelection, conditioning_set.cpp:114-121)
through gp_state_lists_set, against the reference driver given the same lists.

An init and a burn-in iteration are compared call by call (identical
conditioning sets, posteriors within 1e-5, identical haplotypes after the init
iteration): with the selection plus the lists, with the lists alone (Kinit =
Kpbwt = 0) and with the whole panel (Kpbwt = n_ref_haps, where the reference
leaves the lists out)."""
import numpy as np
import pytest

from conftest import ref_oracle_or_skip

TOL = 1e-5


def _lists(n_ref_haps, ploidy, seed, lo=1, hi=40):
    rng = np.random.default_rng(seed)
    return [np.sort(rng.choice(n_ref_haps, int(rng.integers(lo, hi)), replace=False)).astype(np.int32)
            for _ in range(int(np.sum(ploidy)))]


@pytest.mark.gpu
@pytest.mark.parametrize("kinit,kpbwt", [(200, None), (0, 0), (200, "panel")])
def test_state_lists_iterations_match_reference(small_workload, kinit, kpbwt):
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    P, T = small_workload.panel, small_workload.targets
    if kpbwt is None:
        kp = np.asarray(T.kpbwt, np.int32)
    elif kpbwt == "panel":
        kp = np.full(T.n, P.n_ref_haps, np.int32)
    else:
        kp = np.full(T.n, kpbwt, np.int32)
    kw = dict(kinit=kinit, kpbwt=int(kp.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc = O.RefOracle(P, T, kpbwt_target=kp, **kw)
    ctx = native.Context(P, **kw)
    try:
        ctx.set_targets(T, kpbwt=kp)
        lists = _lists(P.n_ref_haps, T.ploidy, 3)
        orc.set_state_lists(lists)
        ctx.set_state_lists(lists)
        first = np.concatenate([[0], np.cumsum(T.ploidy)])
        for stage, it in ((O.STAGE_INIT, 0), (O.STAGE_BURN, 1)):
            if stage == O.STAGE_BURN:  # start the burn-in iteration from identical haplotypes
                h0, h1 = ctx.haps()
                for t in range(T.n):
                    h0[t], h1[t] = orc.haps(t)
                ctx.set_haps(h0, h1)
            orc.iteration(stage, it)
            ctx.iteration(stage, it)
            gh0, gh1 = ctx.haps()
            for t in range(T.n):
                s = ctx.states(t)
                rows = np.unique(np.concatenate(lists[first[t]:first[t + 1]]))
                if kpbwt == "panel" and stage == O.STAGE_BURN:
                    # the reference builds the whole-panel set once per worker and
                    # leaves idxHaps_ref empty on later calls (conditioning_set.cpp:105-113)
                    assert np.array_equal(s, np.arange(P.n_ref_haps))
                else:
                    assert np.array_equal(orc.last_states(t), s), (stage, t)
                    assert np.isin(rows, s).all()
                if kinit == 0:
                    assert np.array_equal(s, rows)
                r0, r1, _ = orc.last_hp(t)
                g0, g1 = ctx.posteriors(t)
                assert np.abs(r0 - g0).max() <= TOL
                if T.ploidy[t] == 2:
                    assert np.abs(r1 - g1).max() <= TOL
                if stage == O.STAGE_INIT:
                    o0, o1 = orc.haps(t)
                    assert np.array_equal(o0, gh0[t]) and np.array_equal(o1, gh1[t])
    finally:
        ctx.close()


@pytest.mark.gpu
def test_state_list_arguments(small_workload):
    from glimpse_b200 import native
    P, T = small_workload.panel, small_workload.targets
    ctx = native.Context(P, kinit=0, kpbwt=0, pbwt_depth=8, pbwt_modulo_cm=0.05)
    try:
        ctx.set_targets(T, kpbwt=np.zeros(T.n, np.int32))
        lists = _lists(P.n_ref_haps, T.ploidy, 5)
        with pytest.raises(native.GpError, match="rows"):
            ctx.set_state_lists(lists[:-1])
        bad = [x.copy() for x in lists]
        bad[1] = np.zeros(0, np.int32)
        with pytest.raises(native.GpError, match="is empty"):
            ctx.set_state_lists(bad)
        bad[1] = np.array([P.n_ref_haps], np.int32)
        with pytest.raises(native.GpError, match="impossible value"):
            ctx.set_state_lists(bad)
        # refused calls leave no lists: Kinit = Kpbwt = 0 is refused
        with pytest.raises(native.GpError, match="state list"):
            ctx.iteration(native.STAGE_INIT, 0)
        ctx.set_state_lists(lists)
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
        # a new target set clears the lists
        ctx.set_targets(T, kpbwt=np.zeros(T.n, np.int32))
        with pytest.raises(native.GpError, match="state list"):
            ctx.iteration(native.STAGE_INIT, 0)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_state_lists_join_the_learned_selection():
    """With the learned proposal on, the lists still join every set: each set
    is the proposal's choice (at most the target's K) plus the target's rows,
    sorted and without duplicates."""
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(2000, 12000, 1.5, 0.6, 6, ("uniform", 0.5, 2.0), ("fixed", 120), seed=33,
                                     sparse_maf=0.005)
    P, T = w.panel, w.targets
    ctx = native.Context(P, kinit=300, kpbwt=120, pbwt_depth=8, pbwt_modulo_cm=0.05)
    try:
        ctx.set_targets(T, kpbwt=T.kpbwt)
        lists = _lists(P.n_ref_haps, T.ploidy, 9, lo=5, hi=30)
        ctx.set_state_lists(lists)
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
        ctx.learned_train(kcand=512, kpos=8.0, steps=40, batch=4096, lr=1e-3, seed=3)
        ctx.learned_enable(True, kcand=512)
        ctx.iteration(native.STAGE_BURN, 2)
        first = np.concatenate([[0], np.cumsum(T.ploidy)])
        for t in range(T.n):
            s = ctx.states(t).astype(np.int64)
            rows = np.unique(np.concatenate(lists[first[t]:first[t + 1]]))
            assert np.all(np.diff(s) > 0)
            assert np.isin(rows, s).all()
            assert s.size <= int(T.kpbwt[t]) + rows.size
        h0, h1 = ctx.haps()
        assert h0.shape == (T.n, P.n_sites)
    finally:
        ctx.close()
