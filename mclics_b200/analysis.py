"""Time-series analysis of per-sweep observables: integrated autocorrelation time and effective sample size.

    tau, window = tau_int(series)          # Sokal's automatic windowing, c = 5
    n_eff = ess(series)                    # N / (2 tau)

The normalised autocorrelation rho(t) comes from one FFT of the mean-subtracted series (zero-padded to twice its
length, so it is the plain lagged sum, not a circular one); tau(W) = 1/2 + sum_{t=1..W} rho(t), and the window is
the smallest W with W >= c tau(W) (A. D. Sokal, "Monte Carlo methods in statistical mechanics", 1996).
"""
import numpy as np


def autocorr(x):
    """rho(t) for t = 0 .. N-1 (rho(0) = 1)."""
    x = np.asarray(x, np.float64)
    n = x.size
    d = x - x.mean()
    m = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(d, m)
    acov = np.fft.irfft(f * np.conj(f), m)[:n] / n
    if acov[0] == 0:
        return np.zeros(n)
    return acov / acov[0]


def tau_int(x, c=5.0):
    """(tau_int, window) of a series; tau_int = 1/2 for uncorrelated data."""
    x = np.asarray(x, np.float64)
    if x.size < 2:
        return 0.5, 0
    rho = autocorr(x)
    if rho[0] == 0:
        return 0.5, 0
    tau = 0.5 + np.cumsum(rho[1:])
    w = np.arange(1, x.size)
    ok = np.nonzero(w >= c * tau)[0]
    if ok.size == 0:
        return float(tau[-1]), x.size - 1
    i = ok[0]
    return float(tau[i]), int(w[i])


def ess(x, c=5.0):
    """Effective number of independent samples N / (2 tau_int)."""
    tau, _ = tau_int(x, c)
    return len(x) / (2.0 * tau)


def mean_and_error(x, c=5.0):
    """Mean and its standard error sqrt(var * 2 tau / N)."""
    x = np.asarray(x, np.float64)
    tau, _ = tau_int(x, c)
    return float(x.mean()), float(np.sqrt(x.var() * 2.0 * tau / x.size))


def block_error(x, n_blocks=16):
    """Standard error of the mean from the spread of n_blocks consecutive block means (batch means): a check on
    mean_and_error that uses no autocorrelation estimate, valid once a block spans many tau_int."""
    x = np.asarray(x, np.float64)
    b = x.size // n_blocks
    if b < 1 or n_blocks < 2:
        return float("nan")
    m = x[:b * n_blocks].reshape(n_blocks, b).mean(axis=1)
    return float(m.std(ddof=1) / np.sqrt(n_blocks))
