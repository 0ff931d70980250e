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


def _impute_modes(w, Ks, seed, modes):
    """HP (and the FP64 chunk log-likelihood of checkpointed modes) for the same
    haplotypes under each precision mode, with the FP64 restatement's."""
    from glimpse_b200 import native
    from oracle import oracle as O
    P, T = w.panel, w.targets
    rng = np.random.default_rng(seed)
    states, hls, flats = [], [], []
    for i, K in enumerate(Ks):
        t = i % T.n
        states.append(np.sort(rng.choice(P.n_ref_haps, size=K, replace=False)).astype(np.uint32))
        hls.append(init_hl(T.gl[t], T.flat[t]))
        flats.append(T.flat[t])
    ctx = native.Context(P)
    out = {}
    try:
        for m in modes:
            ctx.set_precision(m)
            hp = ctx.impute_batch(states, np.stack(hls), np.stack(flats))
            ll = ctx.loglik(len(Ks)) if m != native.PRECISION_FULL else None
            out[m] = (hp, ll)
    finally:
        ctx.close()
    ref = [O.restate_impute(P, states[i], hls[i], flats[i], precision=64) for i in range(len(Ks))]
    return out, ref


@pytest.mark.gpu
def test_checkpointed_fp32_posteriors_and_loglik():
    """FP32 checkpoints with recompute: posteriors within 1e-5 of FP64 (as the
    full store), and the FP64 chunk log-likelihood sum_l log AlphaSum_l within
    1e-6 per site of the FP64 restatement's."""
    from glimpse_b200 import native, synth
    w = synth.workload("small", seed=3)
    out, ref = _impute_modes(w, [500, 37, 256], 4, [native.PRECISION_FULL, native.PRECISION_CKPT_F32])
    hp_full, _ = out[native.PRECISION_FULL]
    hp_ck, ll = out[native.PRECISION_CKPT_F32]
    for i, (hr, llr) in enumerate(ref):
        e = float(np.abs(hp_ck[i].astype(np.float64) - hr.astype(np.float64)).max())
        assert e <= TOL, f"haplotype {i}: max |HP - HP_fp64| = {e:.3e}"
        assert float(np.abs(hp_ck[i] - hp_full[i]).max()) <= TOL
        n_poly = w.panel.n_sites
        assert abs(ll[i] - llr) <= 1e-6 * n_poly, (i, ll[i], llr)


@pytest.mark.gpu
@pytest.mark.parametrize("K", [700, 1000, 1500, 2000])
def test_checkpointed_states_per_thread_instances(K):
    """Each launch instantiates the checkpointed kernel for the smallest J (states
    per thread, 256 threads) that holds its largest K: K = 700, 1000, 1500 and 2000
    reach J = 3, 4, 6 and 8, the instances the other tests (J = 2 and 5) do not.
    FP32 checkpoints: HP within 1e-5 of the FP64 restatement and of the full
    store, the chunk log-likelihood within 1e-6 per site. The full store's own
    kernel (one warp per chain, J = K / 128 quads rounded up) runs at J = 6, 8, 12
    and 16 here, and its HP must be within 1e-5 of FP64 as well."""
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(2048, 6000, 0.5, 0.5, 2, ("uniform", 0.5, 2.0), ("fixed", 200), seed=53,
                                     sparse_maf=0.005)
    out, ref = _impute_modes(w, [K, K // 3], 6, [native.PRECISION_FULL, native.PRECISION_CKPT_F32])
    hp_full, _ = out[native.PRECISION_FULL]
    hp_ck, ll = out[native.PRECISION_CKPT_F32]
    for i, (hr, llr) in enumerate(ref):
        e = float(np.abs(hp_ck[i].astype(np.float64) - hr.astype(np.float64)).max())
        assert e <= TOL, f"K={K} haplotype {i}: max |HP - HP_fp64| = {e:.3e}"
        ef = float(np.abs(hp_full[i].astype(np.float64) - hr.astype(np.float64)).max())
        assert ef <= TOL, f"K={K} haplotype {i}, full store: max |HP - HP_fp64| = {ef:.3e}"
        assert float(np.abs(hp_ck[i] - hp_full[i]).max()) <= TOL
        assert abs(ll[i] - llr) <= 1e-6 * w.panel.n_sites, (i, ll[i], llr)


def _dosage(hp0, hp1):
    return hp0[1::2].astype(np.float64) + hp1[1::2].astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["small", "batched"])
def test_checkpointed_bf16_error_vs_fp64(shape):
    """BF16 checkpoints (the memory-lean variant): the largest posterior error
    and the largest error of the dosage formed from the two haplotypes'
    posteriors (DS = P(alt | hap 0) + P(alt | hap 1)), against FP64 on the same
    inputs. Printed (pytest -s) and bounded."""
    from glimpse_b200 import native, synth
    w = synth.workload("small", seed=3) if shape == "small" else synth.workload("batched", seed=1, n_targets=2)
    Ks = [500, 500, 500, 500] if shape == "small" else [400, 400, 1200, 1200]
    out, ref = _impute_modes(w, Ks, 5, [native.PRECISION_CKPT_BF16, native.PRECISION_CKPT_F32])
    hp, ll = out[native.PRECISION_CKPT_BF16]
    e_hp = max(float(np.abs(hp[i].astype(np.float64) - ref[i][0].astype(np.float64)).max()) for i in range(len(Ks)))
    e_ds = 0.0
    for i in range(0, len(Ks), 2):
        ds = _dosage(hp[i], hp[i + 1])
        ds64 = _dosage(ref[i][0], ref[i + 1][0])
        e_ds = max(e_ds, float(np.abs(ds - ds64).max()))
    e_ll = max(abs(ll[i] - ref[i][1]) / abs(ref[i][1]) for i in range(len(Ks)))
    print(f"\n{shape}: BF16 checkpoints: max |HP - HP_fp64| = {e_hp:.3e}, max |DS - DS_fp64| = {e_ds:.3e}, "
          f"max relative loglik error {e_ll:.2e}")
    assert e_hp <= 5e-3 and e_ds <= 1e-2 and e_ll <= 1e-4


@pytest.mark.gpu
def test_checkpointed_bf16_full_run_r2():
    """A complete Gibbs run on the small workload with BF16 checkpoints against
    the same run with every row kept: dosage r^2 within 0.002."""
    from glimpse_b200 import native, synth
    w = synth.make_panel_and_targets(800, 6000, 0.6, 0.6, 4, ("uniform", 0.5, 2.0), ("uniform", 150, 400), seed=21,
                                     sparse_maf=0.01)
    truth = w.targets.truth.sum(1)
    r2 = {}
    for m in (native.PRECISION_FULL, native.PRECISION_CKPT_BF16):
        ctx = native.Context(w.panel, kinit=300, kpbwt=int(w.targets.kpbwt.max()), pbwt_depth=8, pbwt_modulo_cm=0.05)
        try:
            ctx.set_precision(m)
            ctx.set_targets(w.targets, kpbwt=w.targets.kpbwt)
            ctx.run(3, 5)
            r2[m] = synth.dosage_r2(ctx.gp()[2], truth)
        finally:
            ctx.close()
    d = r2[native.PRECISION_CKPT_BF16] - r2[native.PRECISION_FULL]
    print(f"\nfull run r2: all rows {r2[native.PRECISION_FULL]:.5f}, BF16 checkpoints "
          f"{r2[native.PRECISION_CKPT_BF16]:.5f} (delta {d:+.5f})")
    assert abs(d) <= 0.002
