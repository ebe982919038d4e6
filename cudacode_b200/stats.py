"""Statistics of Monte Carlo time series: integrated autocorrelation time
with Sokal's automatic windowing, effective sample size, and error bars.

tau_int = 1/2 + sum_{t=1}^{M} rho(t), with the window M the smallest value
satisfying M >= c * tau_int(M) (A. D. Sokal, "Monte Carlo methods in
statistical mechanics: foundations and new algorithms", 1989; c = 5).
The variance of the mean of n correlated samples is 2 tau_int sigma^2 / n,
so the effective number of independent samples is n / (2 tau_int).
"""
from __future__ import annotations

import numpy as np


def autocorrelation(x: np.ndarray) -> np.ndarray:
    """Normalised autocorrelation rho(t), t = 0..n-1, by FFT."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    d = x - x.mean()
    f = np.fft.rfft(d, 2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n]
    if acf[0] <= 0.0:
        return np.zeros(n)
    return acf / acf[0]


def tau_int(x: np.ndarray, c: float = 5.0) -> float:
    """Integrated autocorrelation time (Sokal's automatic window)."""
    rho = autocorrelation(x)
    n = len(rho)
    if n < 2 or rho[0] == 0.0:
        return 0.5
    taus = 0.5 + np.cumsum(rho[1:])
    for m in range(1, n):
        if m >= c * taus[m - 1]:
            return float(max(taus[m - 1], 0.5))
    return float(max(taus[-1], 0.5))


def effective_samples(x: np.ndarray, c: float = 5.0) -> float:
    return len(x) / (2.0 * tau_int(x, c))


def mean_error(x: np.ndarray, c: float = 5.0) -> tuple[float, float]:
    """Mean and its standard error accounting for autocorrelation."""
    x = np.asarray(x, dtype=np.float64)
    var = x.var(ddof=1) if len(x) > 1 else 0.0
    return float(x.mean()), float(np.sqrt(2.0 * tau_int(x, c) * var / len(x)))


def specific_heat(energies: np.ndarray, T: float, n_sites: int) -> float:
    """C/N = (<E^2> - <E>^2) / (N T^2)."""
    e = np.asarray(energies, dtype=np.float64)
    return float(e.var() / (n_sites * T * T))
