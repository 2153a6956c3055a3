"""The learned cost model: its hand-written GPU kernels against the float64 CPU
oracle (oracle/mlp_oracle.py), training, and what it gains over the fixed
heuristic on autotuner timings."""
import os

import numpy as np
import pytest

import mlp_oracle as MO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DB = os.path.join(ROOT, "platform-independent-lcs_b200", "slcs", "data", "timings.npz")


def _random_problem(seed, n=200, k=7):
    rng = np.random.default_rng(seed)
    X = rng.uniform(6, 18, (n, 4)).astype(np.float32)
    W = rng.normal(size=(4, k))
    T = (np.sin(X @ W / 8) + 0.1 * rng.normal(size=(n, k))).astype(np.float32)
    M = (rng.random((n, k)) < 0.85).astype(np.uint8)
    p = np.zeros(MO.param_count(k))
    p[:4] = X.mean(0)
    p[4:8] = X.std(0)
    p[8:] = rng.normal(size=len(p) - 8) * 0.2
    return p, X, T, M, k


def test_oracle_gradient_matches_finite_differences():
    p, X, T, M, k = _random_problem(0, n=40, k=3)
    loss, g = MO.loss_and_grad(p, k, X, T, M)
    rng = np.random.default_rng(1)
    for idx in rng.choice(np.arange(8, len(p)), 40, replace=False):
        e = np.zeros_like(p)
        e[idx] = 1e-6
        num = (MO.loss_and_grad(p + e, k, X, T, M)[0] - MO.loss_and_grad(p - e, k, X, T, M)[0]) / 2e-6
        assert abs(num - g[idx]) <= 1e-6 + 1e-4 * abs(g[idx]), idx


@pytest.mark.gpu
def test_device_gradient_and_forward_match_oracle(cuda):
    from slcs import costmodel as CM
    p, X, T, M, k = _random_problem(2)
    p32 = p.astype(np.float32)
    loss, g = CM.gradient(p32, X, T, M)
    want_loss, want_g = MO.loss_and_grad(p32.astype(np.float64), k, X, T, M)
    # FP32 device sums against the float64 oracle
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss))
    scale = np.abs(want_g).max()
    np.testing.assert_allclose(g, want_g, atol=2e-4 * scale, rtol=2e-3)
    y = CM.predict(p32, k, X)
    np.testing.assert_allclose(y, MO.forward(p32.astype(np.float64), k, X)[0], atol=1e-4, rtol=1e-4)


@pytest.mark.gpu
def test_training_reduces_loss(cuda):
    from slcs import costmodel as CM
    _, X, T, M, k = _random_problem(3, n=500)
    p = CM.init_params(k, X, seed=5)
    loss0, _ = CM.gradient(p, X, T, M)
    loss1 = CM.train(p, X, T, M, epochs=800, lr=3e-3)
    assert loss1 < 0.5 * loss0
    assert loss1 < 0.05


@pytest.mark.gpu
def test_model_beats_fixed_heuristic_on_autotuner_timings(cuda):
    """Trained on the autotuner's training shapes, the model's choices on the
    disjoint test shapes lose less time than the fixed heuristic's."""
    if not os.path.exists(DB):
        pytest.skip("no autotuner timing database committed")
    from slcs import autotune as AT
    from slcs import costmodel as CM
    db = np.load(DB)
    if list(db["variants"]) != [v["name"] for v in CM.VARIANTS]:
        pytest.skip("the committed timings were taken for another variant list")
    model, loss = AT.fit(db["train_X"], db["train_ms"], epochs=1500)
    rep = AT.report(model, db["test_X"], db["test_ms"])
    assert rep["model"]["total_time_ratio"] < rep["heuristic"]["total_time_ratio"]
    assert rep["model"]["mean"] < rep["heuristic"]["mean"]
    assert bool(db["train_agree"].all()) and bool(db["test_agree"].all())
