"""CPU checks of the learned filter's network oracle (oracle/mlp_oracle.py)."""
import numpy as np
import torch

from oracle import mlp_oracle as M


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(20000).astype(np.float32) * 10.0 ** rng.integers(-6, 6, 20000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0, 3.0e38], np.float32)])
    ours = M.bf16(x)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 8)).astype(np.float32)
    y = (rng.random(n) < 0.2).astype(np.float32)
    return x, y


def test_backward_matches_finite_differences_without_rounding():
    p = M.init_params(3).astype(np.float64)
    p[M.O_B1:M.O_W2] = 0.05
    p[M.O_B2:M.O_W3] = 0.05
    x, y = _data(64, 4)
    _, g = M.loss_and_grad(p, x, y, 3.0, rounding=False)
    rng = np.random.default_rng(5)
    idx = np.concatenate([rng.choice(M.N_PARAMS, 60, replace=False), [M.O_B3]])
    eps = 1e-6
    for q in idx:
        pp, pm = p.copy(), p.copy()
        pp[q] += eps
        pm[q] -= eps
        lp, _ = M.loss_and_grad(pp, x, y, 3.0, rounding=False)
        lm, _ = M.loss_and_grad(pm, x, y, 3.0, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[q]) <= 1e-6 + 1e-4 * abs(fd), (q, fd, g[q])


def test_adam_step_reduces_loss():
    p = M.init_params(7)
    x, y = _data(512, 8)
    m = np.zeros(M.N_PARAMS, np.float32)
    v = np.zeros(M.N_PARAMS, np.float32)
    l0, _ = M.loss_and_grad(p, x, y, 2.0)
    for t in range(1, 51):
        _, g = M.loss_and_grad(p, x, y, 2.0)
        p, m, v = M.adam_step(p, m, v, g.astype(np.float32), t, 1e-2)
    l1, _ = M.loss_and_grad(p, x, y, 2.0)
    assert l1 < l0
