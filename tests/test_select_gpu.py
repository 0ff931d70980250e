"""State selection parity (bit-exact):
  * init stage: haplotype_set::initRareTar + performSelection_RARE_INIT_GL
    (haplotype_set.cpp:108-169,775-833), per-target std::sample streams;
  * burn-in/main: matchHapsFromCompressedPBWTSmall (haplotype_set.cpp:317-394),
    every pbwt_states level list, and the conditioning_set::compactSelection
    union (conditioning_set.cpp:96-104)."""
import dataclasses

import numpy as np
import pytest

from conftest import ref_oracle_or_skip


def _noisy(rng, h, p):
    h = h.copy()
    h[rng.random(h.shape) < p] ^= 1
    return h


@pytest.fixture(scope="module")
def pair(small_workload):
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    w = small_workload
    kw = dict(kinit=200, kpbwt=int(w.targets.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc = O.RefOracle(w.panel, w.targets, kpbwt_target=w.targets.kpbwt, **kw)
    ctx = native.Context(w.panel, **kw)
    ctx.set_targets(w.targets, kpbwt=w.targets.kpbwt)
    return w, orc, ctx, O


@pytest.mark.gpu
def test_init_selection_matches_reference(pair):
    w, orc, ctx, O = pair
    orc.init_select(0)
    ctx.select(O.STAGE_INIT, 0)
    for t in range(w.targets.n):
        ref = np.sort(orc.init_states(t)).astype(np.uint32)
        got = ctx.states(t)
        assert np.array_equal(ref, got), f"target {t}: {len(ref)} vs {len(got)} states"


@pytest.mark.gpu
@pytest.mark.parametrize("it,noise", [(1, 0.0), (4, 0.02), (9, 0.1)])
def test_pbwt_selection_matches_reference(pair, it, noise):
    w, orc, ctx, O = pair
    rng = np.random.default_rng(it)
    T = w.targets
    h0 = np.stack([_noisy(rng, T.truth[t, 0], noise) for t in range(T.n)])
    h1 = np.stack([_noisy(rng, T.truth[t, 1], noise) for t in range(T.n)])
    for t in range(T.n):
        orc.set_haps(t, h0[t], h1[t])
    ctx.set_haps(h0, h1)
    orc.pbwt_select(it, main_iteration=False)
    ctx.select(O.STAGE_BURN, it)
    for t in range(T.n):
        ref_lv = orc.pbwt_states(t)
        got_lv = ctx.pbwt_states(t, depth=len(ref_lv))
        for lv, (r, g) in enumerate(zip(ref_lv, got_lv)):
            assert np.array_equal(r, g), f"target {t} level {lv}: {r[:10]} vs {g[:10]} ({len(r)} vs {len(g)})"
        ref_states = orc.select(t, O.STAGE_BURN)
        assert np.array_equal(ref_states, ctx.states(t)), f"target {t} union differs"


@pytest.fixture(scope="module")
def pair_haploid(small_workload):
    """The small workload with target 1 haploid: 5 target haplotypes, an odd count,
    so the last warp of the PBWT sweep runs a partial group."""
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    w = small_workload
    T = dataclasses.replace(w.targets, ploidy=w.targets.ploidy.copy())
    T.ploidy[1] = 1
    kw = dict(kinit=200, kpbwt=int(T.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc = O.RefOracle(w.panel, T, kpbwt_target=T.kpbwt, **kw)
    ctx = native.Context(w.panel, **kw)
    ctx.set_targets(T, kpbwt=T.kpbwt)
    return w, T, orc, ctx, O


@pytest.mark.gpu
def test_pbwt_selection_haploid_target_matches_reference(pair_haploid):
    w, T, orc, ctx, O = pair_haploid
    rng = np.random.default_rng(11)
    h0 = np.stack([_noisy(rng, T.truth[t, 0], 0.02) for t in range(T.n)])
    h1 = np.stack([_noisy(rng, T.truth[t, 1], 0.02) for t in range(T.n)])
    for t in range(T.n):
        orc.set_haps(t, h0[t], h1[t])
    ctx.set_haps(h0, h1)
    orc.pbwt_select(4, main_iteration=False)
    ctx.select(O.STAGE_BURN, 4)
    for t in range(T.n):
        ref_lv = orc.pbwt_states(t)
        got_lv = ctx.pbwt_states(t, depth=len(ref_lv))
        for lv, (r, g) in enumerate(zip(ref_lv, got_lv)):
            assert np.array_equal(r, g), f"target {t} level {lv}: {len(r)} vs {len(g)}"
        assert np.array_equal(orc.select(t, O.STAGE_BURN), ctx.states(t)), f"target {t} union differs"


@pytest.mark.gpu
def test_selection_with_capped_grid_matches_reference(small_workload, monkeypatch):
    """The event-bit and panel-transpose kernels loop over their second grid
    dimension when it would pass the hardware's 65,535 (panels with more than
    about 2M events or common sites). GLIMPSE_B200_GRID_Y_CAP=2 makes a small
    panel take those loops; selection must stay bit-exact and posteriors (which
    read the transposed panel) within 1e-5 of the reference."""
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    from conftest import init_hl
    w = small_workload
    T = w.targets
    kw = dict(kinit=200, kpbwt=int(T.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    monkeypatch.setenv("GLIMPSE_B200_GRID_Y_CAP", "2")
    ctx = native.Context(w.panel, **kw)
    monkeypatch.delenv("GLIMPSE_B200_GRID_Y_CAP")
    orc = O.RefOracle(w.panel, T, kpbwt_target=T.kpbwt, **kw)
    try:
        ctx.set_targets(T, kpbwt=T.kpbwt)
        rng = np.random.default_rng(17)
        h0 = np.stack([_noisy(rng, T.truth[t, 0], 0.02) for t in range(T.n)])
        h1 = np.stack([_noisy(rng, T.truth[t, 1], 0.02) for t in range(T.n)])
        for t in range(T.n):
            orc.set_haps(t, h0[t], h1[t])
        ctx.set_haps(h0, h1)
        orc.pbwt_select(3, main_iteration=False)
        ctx.select(O.STAGE_BURN, 3)
        for t in range(T.n):
            ref_lv = orc.pbwt_states(t)
            got_lv = ctx.pbwt_states(t, depth=len(ref_lv))
            for lv, (r, g) in enumerate(zip(ref_lv, got_lv)):
                assert np.array_equal(r, g), f"target {t} level {lv}"
            assert np.array_equal(orc.select(t, O.STAGE_BURN), ctx.states(t)), f"target {t} union differs"
        s = ctx.states(0)
        hl = init_hl(T.gl[0], T.flat[0])
        got = ctx.impute_batch([s], hl[None], T.flat[0][None])[0]
        ref, _ = orc.impute(s, hl, T.flat[0])
        assert float(np.abs(got - ref).max()) <= 1e-5
    finally:
        ctx.close()
