"""The two-sample chi-square that bench.py reports for visit counts: it must
not reject two samples of one law (independent draws), and it must reject a
law shifted by a few percent at the sample sizes the bench uses."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _law(n, rng):
    w = rng.pareto(1.2, n) + 1.0  # heavy-tailed, like degree-proportional visits
    return w / w.sum()


def test_same_law_is_not_rejected():
    rng = np.random.default_rng(3)
    n = 50_000
    p = _law(n, rng)
    pvals = []
    for _ in range(20):
        a = np.bincount(rng.choice(n, 200_000, p=p), minlength=n)
        b = np.bincount(rng.choice(n, 300_000, p=p), minlength=n)
        stat, df, pv = bench.two_sample_chi2(a, b)
        assert df > 1000
        pvals.append(pv)
    pvals = np.array(pvals)
    assert pvals.min() > 1e-4           # no false alarm at the bench's sizes
    assert 0.2 < np.median(pvals) < 0.8  # roughly uniform under the null


def test_shifted_law_is_rejected():
    rng = np.random.default_rng(4)
    n = 50_000
    p = _law(n, rng)
    q = p.copy()
    q[: n // 10] *= 1.3  # a tenth of the vertices 30 % more likely
    q /= q.sum()
    a = np.bincount(rng.choice(n, 1_000_000, p=p), minlength=n)
    b = np.bincount(rng.choice(n, 1_000_000, p=q), minlength=n)
    assert bench.two_sample_chi2(a, b)[2] < 1e-6


def test_pooling_keeps_every_visit():
    # sparse counts are pooled into bins; the statistic still sees every visit
    a = np.zeros(1000, dtype=np.int64)
    b = np.zeros(1000, dtype=np.int64)
    a[::3] = 1
    b[1::3] = 1
    stat, df, pv = bench.two_sample_chi2(a, b)
    assert df >= 1 and np.isfinite(stat) and 0.0 <= pv <= 1.0
