"""Autocorrelation analysis used for the ESS comparison (host logic)."""
import numpy as np
import pytest

from cudacode_b200 import stats


def ar1(phi, n, seed):
    rng = np.random.default_rng(seed)
    x = np.empty(n)
    x[0] = rng.normal() / np.sqrt(1 - phi * phi)
    eps = rng.normal(size=n)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + eps[i]
    return x


@pytest.mark.parametrize("phi", [0.0, 0.5, 0.9, 0.98])
def test_tau_int_of_ar1(phi):
    exact = (1 + phi) / (2 * (1 - phi))
    x = ar1(phi, 200_000, seed=int(phi * 100))
    assert stats.tau_int(x) == pytest.approx(exact, rel=0.1)


def test_effective_samples_and_error():
    x = ar1(0.9, 100_000, 1)
    n_eff = stats.effective_samples(x)
    assert n_eff == pytest.approx(100_000 / (2 * 9.5), rel=0.15)
    m, err = stats.mean_error(x)
    assert abs(m) < 5 * err


def test_constant_series():
    assert stats.tau_int(np.ones(100)) == 0.5
