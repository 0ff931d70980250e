"""The learned proposal's scoring network (48 -> 256 -> 256 -> 1, ReLU).

CPU: the FP32 oracle's backward formulas against central finite differences of
the exact (float64, unrounded) loss.
GPU, through the C-ABI:
  * the tensor-core forward (k_mlp_fwd) against a plain torch FP32 reference of
    the same network with the same BF16 rounding points: hidden activations
    and scores;
  * the tensor-core backward (k_gemm_tn and the loss head) against the CPU
    FP32 oracle: every gradient block within 1 % relative (Frobenius), the
    loss within 1e-4;
  * training with the device's Adam steps drives the loss of a learnable
    problem down."""
import numpy as np
import pytest

from oracle import mlp as M


def _problem(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, M.N_IN)).astype(np.float32)
    wtrue = rng.normal(0, 1, M.N_IN)
    logit = x @ wtrue / np.sqrt(M.N_IN) * 3 + 0.5 * np.sin(3 * x[:, 0])
    y = (rng.random(n) < 1 / (1 + np.exp(-logit))).astype(np.float32)
    wt = rng.uniform(0.5, 2.0, n).astype(np.float32)
    return x, y, wt


def test_oracle_gradient_matches_finite_differences():
    x, y, wt = _problem(16, 3)
    p = M.init_params(5)
    p[M.OFF_B1:M.OFF_W2] = 0.05  # keep units active so the check is not dominated by ReLU kinks
    p[M.OFF_B2:M.OFF_W3] = 0.05
    # the exact gradient: the oracle's formulas without BF16 rounding
    M_bf16 = M.bf16
    try:
        M.bf16 = lambda a: np.asarray(a, np.float32)
        _, g = M.loss_and_grad(p, x, y, wt)
    finally:
        M.bf16 = M_bf16
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(np.flatnonzero((np.arange(M.OFF_B1) % M.N_INP) < M.N_IN), 12),
                          M.OFF_B1 + rng.choice(M.N_HID, 4), M.OFF_W2 + rng.choice(M.N_HID * M.N_HID, 12),
                          M.OFF_B2 + rng.choice(M.N_HID, 4), M.OFF_W3 + rng.choice(M.N_HID, 4), [M.OFF_B3]])
    eps = 1e-3
    for i in idx:
        pp, pm = p.astype(np.float64), p.astype(np.float64)
        pp = pp.copy(); pm = pm.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (M.loss_exact(pp, x, y, wt) - M.loss_exact(pm, x, y, wt)) / (2 * eps)
        assert abs(fd - g[i]) <= 2e-4 + 2e-2 * abs(fd), (int(i), fd, float(g[i]))


def _blocks():
    return [("W1", M.OFF_W1, M.OFF_B1), ("b1", M.OFF_B1, M.OFF_W2), ("W2", M.OFF_W2, M.OFF_B2),
            ("b2", M.OFF_B2, M.OFF_W3), ("w3", M.OFF_W3, M.OFF_B3), ("b3", M.OFF_B3, M.N_PARAMS)]


@pytest.fixture(scope="module")
def ctx(small_workload):
    from glimpse_b200 import native
    c = native.Context(small_workload.panel)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 128, 300, 5000])
def test_forward_matches_torch_fp32(ctx, n):
    import torch
    x, _, _ = _problem(n, n)
    p = M.init_params(7)
    p[M.OFF_B1:M.OFF_W2] = np.random.default_rng(1).normal(0, 0.1, M.N_HID)
    p[M.OFF_B2:M.OFF_W3] = np.random.default_rng(2).normal(0, 0.1, M.N_HID)
    p[M.OFF_B3] = 0.3
    ctx.mlp_set_params(p)
    score, h1, h2 = ctx.mlp_forward(x, hidden=True)
    P = M.unpack(p)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32))
    xb = torch.zeros(n, M.N_INP)
    xb[:, :M.N_IN] = t(M.bf16(x))
    z1 = xb @ t(M.bf16(P["W1"])).T + t(P["b1"])
    h1_ref = t(M.bf16(torch.relu(z1).numpy()))
    z2 = h1_ref @ t(M.bf16(P["W2"])).T + t(P["b2"])
    h2_ref = torch.relu(z2)
    s_ref = (h2_ref @ t(P["w3"]) + float(P["b3"][0])).numpy()
    # BF16 roundings may flip by one unit where the FP32 sums differ in the last bits
    assert np.abs(h1 - h1_ref.numpy()).max() <= 1e-2 * max(1.0, float(np.abs(h1_ref).max()))
    assert np.mean(h1 != h1_ref.numpy()) <= 1e-3
    assert np.abs(h2 - M.bf16(h2_ref.numpy())).max() <= 1e-2 * max(1.0, float(h2_ref.abs().max()))
    err = np.abs(score - s_ref)
    assert err.max() <= 1e-3 * max(1.0, float(np.abs(s_ref).max())), float(err.max())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [256, 3000])
def test_backward_matches_cpu_oracle(ctx, n):
    x, y, wt = _problem(n, 11 + n)
    p = M.init_params(9)
    p[M.OFF_B1:M.OFF_W2] = 0.02
    p[M.OFF_B2:M.OFF_W3] = 0.02
    ctx.mlp_set_params(p)
    loss, g = ctx.mlp_train_step(x, y, wt, lr=0.0, grad=True)
    loss_ref, g_ref = M.loss_and_grad(p, x, y, wt)
    assert abs(loss - loss_ref) <= 1e-4 * max(1.0, abs(loss_ref)), (loss, loss_ref)
    for name, a, b in _blocks():
        d = np.linalg.norm(g[a:b] - g_ref[a:b])
        r = np.linalg.norm(g_ref[a:b])
        assert d <= 1e-2 * r + 1e-7, f"{name}: |dg| {d:.3e} vs |g| {r:.3e}"
    # the parameters are unchanged by a step with lr = 0
    assert np.array_equal(ctx.mlp_params(), p)


@pytest.mark.gpu
def test_training_reduces_loss(ctx):
    x, y, wt = _problem(8192, 21)
    ctx.mlp_init(3)
    l0, _ = ctx.mlp_train_step(x, y, wt, lr=0.0)
    for _ in range(150):
        ctx.mlp_train_step(x, y, wt, lr=2e-3)
    l1, _ = ctx.mlp_train_step(x, y, wt, lr=0.0)
    assert l1 < 0.8 * l0, (l0, l1)
    # the oracle agrees on the trained parameters' loss
    lr_, _ = M.loss_and_grad(ctx.mlp_params(), x, y, wt)
    assert abs(lr_ - l1) <= 1e-3 * max(1.0, abs(l1))
