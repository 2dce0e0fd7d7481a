"""bench.py's own chi-squared (the parity block of the bench line) against the
oracle's batched chi-squared, on seeded synthetic batch means (no GPU)."""

from __future__ import annotations

import numpy as np

import bench
from oracle import stats


def test_bench_chi2_matches_the_oracle():
    rng = np.random.default_rng(11)
    a = rng.uniform(1.0, 2.0, 500)
    b = a + rng.normal(0.0, 0.02, 500)
    sa, sb = rng.uniform(0.01, 0.03, 500), rng.uniform(0.01, 0.03, 500)
    chi2, mean, p = bench.batched_chi2(a, sa, 10, b, sb, 20)
    r = stats.chi2_batched(a, sa, 10, b, sb, 20)
    assert np.isclose(chi2, r["chi2"]) and np.isclose(mean, r["null_mean"])
    assert np.isclose(p, r["p_value"], rtol=1e-9, atol=1e-12)
