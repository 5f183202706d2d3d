"""CPU checks of the cost model's host side: the numpy MLP reference against
finite differences, and the schedule helpers."""
import numpy as np

from mlp_ref import loss_grad
from blastp_b200 import costmodel


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    shape = (5, 7, 2)
    n_p = 5 * 7 + 7 + 7 * 2 + 2
    p = rng.normal(size=n_p) * 0.5
    X = rng.normal(size=(11, 5))
    T = rng.normal(size=(11, 2))
    _, g = loss_grad(p, X, T, shape)
    eps = 1e-6
    for k in range(n_p):
        d = np.zeros(n_p)
        d[k] = eps
        fd = (loss_grad(p + d, X, T, shape)[0] - loss_grad(p - d, X, T, shape)[0]) / (2 * eps)
        assert abs(fd - g[k]) < 1e-6 + 1e-5 * abs(g[k])


def test_chunk_sums_and_makespan():
    counters = np.array([[1, 0, 2], [3, 1, 1], [0, 0, 0], [5, 2, 4]], dtype=np.int32)
    first = np.array([0, 2, 4])
    assert costmodel.chunk_sums(counters, first).tolist() == [[4, 1, 3], [5, 2, 4]]
    assert costmodel.makespan(np.array([1.0, 2.0, 3.0, 4.0]), np.array([0, 1, 0, 1])) == 6.0
    assert costmodel.makespan(np.array([1.0]), np.array([-1])) == 0.0


def test_relative_error_and_cost_weights():
    e = costmodel.relative_error(np.array([10.0, 0.0]), np.array([8.0, 0.0]))
    assert abs(e["median"] - 0.125) < 1e-12
    rng = np.random.default_rng(1)
    A = rng.uniform(1, 100, size=(40, 3))
    w_true = np.array([0.01, 0.2, 3.0])
    timing = np.concatenate([A, (A @ w_true)[:, None]], axis=1)
    w = costmodel.fit_cost_weights(timing)
    assert np.allclose(w, w_true, rtol=1e-6)


def test_cosched_split_balances_device_and_cpu():
    rng = np.random.default_rng(4)
    costs = rng.uniform(0.5, 2.0, size=400)
    for f in (0.5, 4.0, 40.0):
        k = costmodel.cosched_split_chunk(costs, f)
        gpu, cpu = costs[:k].sum(), f * costs[k:].sum()
        best = min(max(costs[:j].sum(), f * costs[j:].sum()) for j in range(401))
        assert max(gpu, cpu) == best
        assert abs(gpu - cpu) <= max(costs) * max(1.0, f)
    assert costmodel.cosched_split_chunk(costs, 0.0) == 400      # no CPU share
    assert costmodel.cosched_split_chunk([], 3.0) == 0
