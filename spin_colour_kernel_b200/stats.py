"""Chain statistics on the host (FP64): integrated autocorrelation time and bootstrap intervals.

`integrated_tau` follows the reference's `exp_core.integrated_tau` (`src/Spin_Colour_Kernel/exp_core.py:157-173`):
the autocorrelation of each chain (mean removed per chain) by a zero-padded FFT, averaged over chains and
normalised at lag 0, summed up to Sokal's automatic window — the first M with M >= c * tau(M), where
tau(M) = 1 + 2 sum_{k=1..M} rho(k) — and floored at 0.5; a constant or non-finite series gives 1. `boot_ci`
follows `exp_perf.boot_ci` (`src/Spin_Colour_Kernel/exp_perf.py:33-38`): percentile interval of a statistic over
resamples drawn with NumPy's PCG64 generator from the given seed. `effective_rate` turns a sample rate and tau into
effective independent samples per second (rate / (2 tau), the variance-inflation convention of Sokal's tau).
"""

from __future__ import annotations

import numpy as np


def autocorrelation(x: np.ndarray) -> np.ndarray:
    """Chain-averaged autocorrelation rho(k), k = 0..n-1, of a (time, chains) series (rho(0) = 1)."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    x = x - x.mean(axis=0)
    n = x.shape[0]
    spec = np.fft.rfft(x, n=2 * n, axis=0)
    acov = np.fft.irfft(spec * np.conj(spec), n=2 * n, axis=0)[:n].mean(axis=1)
    return acov / acov[0]


def integrated_tau(x: np.ndarray, c: float = 6.0) -> float:
    """Integrated autocorrelation time of a (time, chains) series with Sokal's automatic window."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    d = x - x.mean(axis=0)
    if not np.all(np.isfinite(d)) or float((d * d).sum()) == 0.0:
        return 1.0
    rho = autocorrelation(x)
    n = rho.shape[0]
    if n < 2 or not np.all(np.isfinite(rho)):
        return 1.0
    taus = 1.0 + 2.0 * np.cumsum(rho[1:])            # tau(M) for M = 1..n-1
    M = np.arange(1, n)
    hit = np.nonzero(M >= c * taus)[0]
    tau = taus[hit[0]] if hit.size else taus[-1]
    return max(float(tau), 0.5)


def boot_ci(x: np.ndarray, stat=np.mean, n: int = 2000, seed: int = 0, level: float = 0.95):
    """(stat(x), lower, upper): percentile bootstrap interval over n resamples."""
    rng = np.random.default_rng(seed)
    x = np.asarray(x)
    draws = np.empty(n)
    for i in range(n):
        draws[i] = stat(x[rng.integers(0, len(x), len(x))])
    lo, hi = np.quantile(draws, [(1.0 - level) / 2.0, 1.0 - (1.0 - level) / 2.0])
    return float(stat(x)), float(lo), float(hi)


def effective_rate(samples_per_second: float, tau: float) -> float:
    """Effective independent samples per second of an observable with integrated time tau (in samples)."""
    return samples_per_second / (2.0 * tau)
