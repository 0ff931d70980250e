"""Whole Gibbs iterations through the C-ABI against the reference driver
(caller_algorithm.cpp:53-126) on the same targets and streams.

The init iteration is compared call by call: identical conditioning sets,
per-site posteriors within 1e-5 and identical sampled/phased haplotypes. Over a
full run (1 init + burn-in + main) trajectories can part where a uniform falls
within float rounding of a posterior, so the run is compared by dosage r^2
against the simulated truth (the bar: within 0.002 of the reference's r^2)."""
import numpy as np
import pytest

from conftest import ref_oracle_or_skip
from glimpse_b200 import synth

TOL = 1e-5


def _make(w, **kw):
    O = ref_oracle_or_skip()
    from glimpse_b200 import native
    orc = O.RefOracle(w.panel, w.targets, kpbwt_target=w.targets.kpbwt, **kw)
    ctx = native.Context(w.panel, **kw)
    ctx.set_targets(w.targets, kpbwt=w.targets.kpbwt)
    return orc, ctx, O


@pytest.mark.gpu
def test_init_iteration_matches_reference(small_workload):
    w = small_workload
    orc, ctx, O = _make(w, kinit=200, kpbwt=int(w.targets.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc.iteration(O.STAGE_INIT, 0)
    ctx.iteration(O.STAGE_INIT, 0)
    h0, h1 = ctx.haps()
    for t in range(w.targets.n):
        assert np.array_equal(orc.last_states(t), ctx.states(t))
        r0, r1, _ = orc.last_hp(t)
        g0, g1 = ctx.posteriors(t)
        assert np.abs(r0 - g0).max() <= TOL
        assert np.abs(r1 - g1).max() <= TOL
        o0, o1 = orc.haps(t)
        assert np.array_equal(o0, h0[t]) and np.array_equal(o1, h1[t])


@pytest.mark.gpu
def test_burn_iteration_matches_reference(small_workload):
    w = small_workload
    orc, ctx, O = _make(w, kinit=200, kpbwt=int(w.targets.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc.iteration(O.STAGE_INIT, 0)
    ctx.iteration(O.STAGE_INIT, 0)
    # start the burn-in iteration from identical haplotypes
    for t in range(w.targets.n):
        o0, o1 = orc.haps(t)
        ctx_h0, ctx_h1 = ctx.haps()
        ctx_h0[t], ctx_h1[t] = o0, o1
        ctx.set_haps(ctx_h0, ctx_h1)
    orc.iteration(O.STAGE_BURN, 1)
    ctx.iteration(O.STAGE_BURN, 1)
    for t in range(w.targets.n):
        assert np.array_equal(orc.last_states(t), ctx.states(t))
        r0, r1, _ = orc.last_hp(t)
        g0, g1 = ctx.posteriors(t)
        assert np.abs(r0 - g0).max() <= TOL
        assert np.abs(r1 - g1).max() <= TOL


@pytest.mark.gpu
def test_full_run_dosage_r2():
    w = synth.make_panel_and_targets(800, 6000, 0.6, 0.6, 4, ("uniform", 0.5, 2.0), ("uniform", 150, 400), seed=21,
                                     sparse_maf=0.01)
    orc, ctx, O = _make(w, kinit=300, kpbwt=int(w.targets.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
    orc.run(burnin=3, main=5)
    ctx.run(burnin=3, main=5)
    gp0, gp1, ds, gt0, gt1 = ctx.gp()
    truth = w.targets.truth.sum(1)
    r2_gpu = synth.dosage_r2(ds, truth)
    ref_ds = []
    for t in range(w.targets.n):
        g0, g1, hds, st, cnt = orc.gp(t)
        g2 = np.clip(1.0 - g1 - g0, 0.0, 1.0)
        ref_ds.append(np.round((g1 + 2.0 * g2) * 1000.0) / 1000.0)
    r2_ref = synth.dosage_r2(np.stack(ref_ds), truth)
    assert abs(r2_gpu - r2_ref) <= 0.002, (r2_gpu, r2_ref)
