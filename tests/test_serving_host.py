"""CPU checks of the serving driver's arrival process and percentile rule."""
import numpy as np

from blastp_b200 import serving


def test_poisson_arrivals_rate_and_order():
    rng = np.random.default_rng(0)
    a = serving.poisson_arrivals(rng, 1000.0, 20000)
    assert a[0] == 0.0 and np.all(np.diff(a) >= 0)
    assert abs(np.mean(np.diff(a)) - 1e-3) < 5e-5
    assert len(serving.poisson_arrivals(rng, 5.0, 0)) == 0


def test_percentile_nearest_rank():
    v = list(range(1, 101))
    assert serving.percentile(v, 50) == 50
    assert serving.percentile(v, 99) == 99
    assert serving.percentile([7.0], 99) == 7.0
    assert serving.percentile([], 50) == 0.0
