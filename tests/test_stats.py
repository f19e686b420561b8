"""Host statistics of the library (no GPU) against plain numpy."""
import numpy as np

import qcd_2d_gpu_b200 as q


def ar1(n, rho, seed=0):
    rng = np.random.default_rng(seed)
    x = np.empty(n)
    x[0] = rng.normal()
    for i in range(1, n):
        x[i] = rho * x[i - 1] + np.sqrt(1 - rho * rho) * rng.normal()
    return x


def test_mean_variance_is_the_reference_estimator():
    x = ar1(1000, 0.3)
    m, v = q.mean_variance(x)
    # statistics.h:30-39: population variance s2/N - mean^2
    assert np.isclose(m, x.mean(), rtol=0, atol=1e-14)
    assert np.isclose(v, (x * x).mean() - x.mean() ** 2, rtol=1e-12)


def test_autocorrelation_is_the_reference_estimator():
    x = ar1(2000, 0.6, seed=1)
    m, v = q.mean_variance(x)
    r = q.autocorrelation(x, 10, m, v)
    ref = [np.sum((x[:-k] - m) * (x[k:] - m)) / (len(x) - k) / v for k in range(1, 11)]
    assert np.allclose(r, ref, rtol=1e-12, atol=1e-14)
    assert abs(r[0] - 0.6) < 0.08  # AR(1): rho(1) = 0.6


def test_binned_error_matches_numpy():
    x = ar1(1200, 0.0, seed=2)
    m, e = q.binned(x, 10)
    b = x.reshape(120, 10).mean(1)
    assert np.isclose(m, b.mean(), atol=1e-14)
    assert np.isclose(e, b.std(ddof=1) / np.sqrt(120), rtol=1e-10)


def test_tau_int_of_ar1_process():
    # AR(1) with coefficient rho: tau_int = (1 + rho) / (2 (1 - rho))
    for rho in (0.0, 0.5, 0.8):
        x = ar1(200000, rho, seed=3)
        tau, w, dtau = q.tau_int(x, 6.0)
        exact = (1 + rho) / (2 * (1 - rho))
        assert abs(tau - exact) < 4 * dtau + 0.02, (rho, tau, exact, dtau)
        assert w >= 1
