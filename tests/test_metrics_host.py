"""The harness's 99th density percentile from two order statistics equals
numpy.percentile(rho, 99) bit for bit (the device returns the two values,
the host interpolates as numpy does)."""

import numpy as np

from fluid_simulation_b200.dam_break import percentile99, percentile99_ranks


def test_percentile_from_order_statistics_matches_numpy():
    rng = np.random.default_rng(7)
    for _ in range(2000):
        n = int(rng.integers(1, 8000))
        a = (1000.0 + rng.normal(size=n) * rng.uniform(0.01, 80.0)).astype(np.float32)
        k, k1 = percentile99_ranks(n)
        s = np.sort(a)
        assert percentile99(s[k], s[k1], n) == np.percentile(a, 99)
    assert percentile99_ranks(1) == (0, 0)
