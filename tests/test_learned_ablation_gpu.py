"""Ablation of the learned state-selection proposal: what the trained network
gains over the method without it.

One panel, two sets of simulated targets: the network is trained on the first
set (its own plain iterations give the haplotypes, the HMM's window posteriors
over the PBWT candidates give the labels) and judged on the second by complete
Gibbs runs (1 init + 3 burn-in + 5 main) at a small conditioning-set size, where
selection matters, with three selections from the same PBWT candidates:
  * plain PBWT selection at that K (the method without the network);
  * the trained network at that K;
  * the same network with untrained (random) weights at that K.
Dosage r^2 against the simulated truth is printed for all three (pytest -s).
Asserted: training lowers the loss, the trained network's loss on a labelled
batch of the training targets is below the untrained network's on the same
batch, and the trained proposal's r^2 stays within 0.01 of plain PBWT
selection. (Single-seed r^2 differences between the two networks are within
the Gibbs runs' spread, so they are reported, not asserted.)"""
import types

import numpy as np
import pytest


def _split(T, idx):
    return types.SimpleNamespace(n=len(idx), ploidy=T.ploidy[idx], gl=T.gl[idx], flat=T.flat[idx],
                                 truth=T.truth[idx], kpbwt=T.kpbwt[idx], coverage=T.coverage[idx])


@pytest.mark.gpu
def test_trained_network_gains_over_untrained_and_matches_pbwt():
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(3000, 20000, 2.0, 0.6, 32, ("uniform", 0.5, 2.0), ("fixed", 40), seed=51,
                                     sparse_maf=0.004)
    P, T = w.panel, w.targets
    train, test = _split(T, np.arange(16)), _split(T, np.arange(16, 32))
    K, kcand = 40, 400
    ctx = native.Context(P, kinit=300, kpbwt=kcand, pbwt_depth=8, pbwt_modulo_cm=0.05)
    try:
        ctx.set_targets(train, kpbwt=np.full(train.n, kcand, np.int32))
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
        ctx.iteration(native.STAGE_BURN, 2)
        losses = ctx.learned_train(kcand=kcand, kpos=8.0, steps=200, batch=8192, lr=1e-3, seed=5)
        trained = ctx.mlp_params()
        # the same labelled batch (same seed), no update (lr 0): trained against untrained weights
        eval_kw = dict(kcand=kcand, kpos=8.0, steps=1, batch=8192, lr=0.0, seed=77)
        loss_trained = float(ctx.learned_train(**eval_kw)[0])
        ctx.mlp_init(99)
        untrained = ctx.mlp_params()
        loss_untrained = float(ctx.learned_train(**eval_kw)[0])
        truth = test.truth.sum(1)

        def r2(learned, params=None):
            ctx.learned_enable(False, kcand=kcand)
            if params is not None:
                ctx.mlp_set_params(params)
            ctx.set_targets(test, kpbwt=np.full(test.n, K, np.int32))
            if learned:
                ctx.learned_enable(True, kcand=kcand)
            ctx.run(3, 5)
            return synth.dosage_r2(ctx.gp()[2], truth)

        r2_plain = r2(False)
        r2_trained = r2(True, trained)
        r2_random = r2(True, untrained)
        print(f"\nablation at K={K} (candidates {kcand}): plain PBWT r2 {r2_plain:.5f}, trained network "
              f"{r2_trained:.5f}, untrained network {r2_random:.5f}; training loss {losses[:10].mean():.4f} -> "
              f"{losses[-10:].mean():.4f}; labelled-batch loss trained {loss_trained:.4f}, untrained "
              f"{loss_untrained:.4f}")
        assert losses[-10:].mean() < losses[:10].mean()
        assert loss_trained < loss_untrained
        assert r2_trained >= r2_plain - 0.01
    finally:
        ctx.close()
