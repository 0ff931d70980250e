"""Failure handling through the C-ABI, with every failure made on the host:
invalid target arguments and an allocation failure injected in place of a
device allocation (GLIMPSE_B200_FAIL_ALLOC=n makes the n-th buffer growth
report out-of-memory without calling cudaMalloc). Each call returns its status
and the context stays usable; no GPU fault is involved."""
import numpy as np
import pytest


def _ctx_and_targets(small_workload, **kw):
    from glimpse_b200 import native
    w = small_workload
    return native, native.Context(w.panel, kinit=200, kpbwt=150, pbwt_depth=8, pbwt_modulo_cm=0.05, **kw), w.targets


@pytest.mark.gpu
def test_invalid_target_arguments_are_refused(small_workload):
    native, ctx, T = _ctx_and_targets(small_workload)
    try:
        with pytest.raises(native.GpError, match="negative Kpbwt"):
            ctx.set_targets(T, kpbwt=np.full(T.n, -1, np.int32))
        bad = np.array(T.ploidy, np.int32, copy=True)
        bad[0] = 3
        with pytest.raises(native.GpError, match="ploidy"):
            ctx.set_targets_raw(T.n, T.gl.ctypes.data, T.flat.ctypes.data, bad.ctypes.data, 0)
        # Kpbwt 0 without a state list (gp_state_lists_set) is refused
        ctx.set_targets(T, kpbwt=np.zeros(T.n, np.int32))
        ctx.iteration(native.STAGE_INIT, 0)
        with pytest.raises(native.GpError, match="state list"):
            ctx.iteration(native.STAGE_BURN, 1)
        # the context still runs a valid batch
        ctx.set_targets(T, kpbwt=T.kpbwt)
        ctx.iteration(native.STAGE_INIT, 0)
        ctx.iteration(native.STAGE_BURN, 1)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_injected_allocation_failure_returns_nomem(small_workload, monkeypatch):
    native, ctx, T = _ctx_and_targets(small_workload)
    ref_native, ref, _ = _ctx_and_targets(small_workload)
    try:
        for c in (ctx, ref):
            c.set_targets(T, kpbwt=T.kpbwt)
            c.iteration(native.STAGE_INIT, 0)
        # the burn-in iteration grows buffers (PBWT selection scratch, stores):
        # fail the first growth
        monkeypatch.setenv("GLIMPSE_B200_FAIL_ALLOC", "1")
        with pytest.raises(native.GpError, match="status -3"):
            ctx.iteration(native.STAGE_BURN, 1)
        monkeypatch.delenv("GLIMPSE_B200_FAIL_ALLOC")
        # the same iteration then runs, and gives what an undisturbed context gives
        ctx.iteration(native.STAGE_BURN, 1)
        ref.iteration(native.STAGE_BURN, 1)
        for t in range(T.n):
            assert np.array_equal(ctx.states(t), ref.states(t))
            a, b = ctx.posteriors(t), ref.posteriors(t)
            assert np.array_equal(a[0], b[0])
    finally:
        ctx.close()
        ref.close()


@pytest.mark.gpu
def test_invalid_configuration_and_tuning_are_refused(small_workload):
    """A negative Kinit or Kpbwt is refused at context creation (the reference
    exits there, caller_parameters.cpp:255-256), and tuning shapes outside their
    candidates are refused without changing the context."""
    from glimpse_b200 import native
    w = small_workload
    for kw in (dict(kinit=-1), dict(kpbwt=-5)):
        with pytest.raises(native.GpError, match="status -1"):
            native.Context(w.panel, pbwt_depth=8, pbwt_modulo_cm=0.05, **kw)
    ctx = native.Context(w.panel, kinit=200, kpbwt=150, pbwt_depth=8, pbwt_modulo_cm=0.05)
    try:
        for args in ((3, 0, 0), (0, 3, 0), (0, 0, 3), (0, 0, -1)):
            with pytest.raises(native.GpError, match="tuning"):
                ctx.tuning_set(*args)
        ctx.tuning_set(2, 1, 2)
        assert ctx.tuning()[:3] == (2, 1, 2)
    finally:
        ctx.close()
