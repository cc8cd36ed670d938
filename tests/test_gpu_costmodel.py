"""Cost-model kernels vs the numpy oracle; training; host inference."""
import numpy as np
import pytest
import torch

import mlp_oracle
from jacquard_b200 import costmodel

pytestmark = pytest.mark.gpu


def rand_problem(n=700, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 24)).astype(np.float32)
    w = rng.normal(size=24).astype(np.float32)
    T = (np.tanh(X @ w / 5) * 2 + 0.3 * np.sin(X[:, 0])).astype(np.float32)
    return X, T


def test_gradient_matches_oracle():
    X, T = rand_problem()
    m = costmodel.CostModel(seed=3, scratch_ctas=16)
    m.mean[:] = 0
    m.inv_std[:] = 1
    Xd = m.features_to_device(X)
    Td = torch.from_numpy(T).cuda()
    idx = torch.arange(X.shape[0], dtype=torch.int32, device="cuda")
    g, loss = m.grad(Xd, Td, idx)
    g = g.cpu().numpy()
    theta = m.theta.cpu().numpy()
    want, wloss = mlp_oracle.grad(theta, mlp_oracle.bf16(X), T)
    scale = np.abs(want).max()
    assert abs(float(loss.item()) - wloss) <= 1e-4 * max(1.0, wloss)
    # fp32 accumulation order differs; tolerance relative to the largest entry
    assert np.max(np.abs(g - want)) <= 2e-3 * scale, np.max(np.abs(g - want)) / scale


def test_forward_matches_oracle_and_host():
    X, T = rand_problem(300, seed=2)
    m = costmodel.CostModel(seed=4)
    m.mean[:] = 0
    m.inv_std[:] = 1
    y = m.predict(X)
    want, _ = mlp_oracle.forward(m.theta.cpu().numpy(), mlp_oracle.bf16(X))
    assert np.allclose(y, want, rtol=1e-4, atol=1e-4)
    from jacquard_b200.frontend import _lib
    packed = m.pack()
    host = np.zeros(X.shape[0], np.float32)
    _lib().jqf_cost_model_predict(packed.ctypes.data, np.ascontiguousarray(X).ctypes.data, X.shape[0],
                                  host.ctypes.data)
    assert np.allclose(host, want, rtol=1e-4, atol=1e-4)


def test_training_reduces_loss():
    X, T = rand_problem(2000, seed=5)
    m = costmodel.CostModel(seed=6)
    hist = m.fit(X, T, steps=400, batch=256, lr=1e-3)
    assert hist[-1][1] < 0.25 * hist[0][1], hist
