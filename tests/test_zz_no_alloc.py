"""gp_impute_one_static (scratch in the library's fixed device region, no
allocation during the call) against gp_impute_batch on the same haplotypes,
called twice in a row, plus the size check that refuses oversized calls.
Tolerance: 1e-6 absolute on HP (both paths run the same kernels)."""
import numpy as np
import pytest

from conftest import init_hl

TOL = 1e-6


@pytest.mark.gpu
def test_static_scratch_matches_batch(small_workload):
    from glimpse_b200 import native
    w = small_workload
    P, T = w.panel, w.targets
    ctx = native.Context(P)
    rng = np.random.default_rng(23)
    try:
        for call in range(2):
            for t in range(min(T.n, 2)):
                for K in (7, 64, 300):
                    s = np.sort(rng.choice(P.n_ref_haps, size=K, replace=False)).astype(np.uint32)
                    hl = init_hl(T.gl[t], T.flat[t])
                    want = ctx.impute_batch([s], hl[None], T.flat[t][None])[0]
                    got = ctx.impute_one_static(s, hl, T.flat[t])
                    err = float(np.abs(got - want).max())
                    assert err <= TOL, f"call {call}, target {t}, K={K}: max |dHP| = {err}"
    finally:
        ctx.close()


@pytest.mark.gpu
def test_static_scratch_refuses_oversized_call():
    from glimpse_b200 import native, synth
    # 9,000 sites x 2,048 states need a 72 MiB alpha store: above the 64 MiB region
    w = synth.make_panel_and_targets(2100, 9000, 0.9, 0.5, 1, ("fixed", 1.0), ("fixed", 500), seed=5)
    P, T = w.panel, w.targets
    ctx = native.Context(P)
    try:
        s = np.arange(2048, dtype=np.uint32)
        hl = init_hl(T.gl[0], T.flat[0])
        with pytest.raises(native.GpError, match="64 MiB"):
            ctx.impute_one_static(s, hl, T.flat[0])
        # a call that fits still runs after the refusal
        s = np.arange(0, 2100, 7, dtype=np.uint32)
        hp = ctx.impute_one_static(s, hl, T.flat[0])
        assert np.isfinite(hp).all()
        assert np.allclose(hp[0::2] + hp[1::2], 1.0, atol=1e-5)
    finally:
        ctx.close()
