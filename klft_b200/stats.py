"""Error analysis for Markov-chain time series: integrated autocorrelation time
(Madras-Sokal automatic windowing) and binned jackknife errors.

Used to compare ensemble means of two chains (for example this library's GPU
chain and the reference code's CPU chain, or the mixed and FP64 forms): the
means agree when their difference is within a few combined standard errors,
with the errors corrected for autocorrelation by binning over 2 tau_int.
"""
from __future__ import annotations

import math
from typing import Dict, Sequence, Tuple

import numpy as np


def tau_int(x: Sequence[float], c: float = 6.0) -> Tuple[float, int]:
    """Integrated autocorrelation time tau = 1/2 + sum_{t=1}^{W} rho(t), with the
    window W the smallest t >= c * tau(t) (Madras & Sokal, J. Stat. Phys. 50
    (1988) 109).  Returns (tau, W); tau = 0.5 for uncorrelated data."""
    a = np.asarray(x, dtype=np.float64)
    n = a.size
    if n < 4:
        return 0.5, 0
    d = a - a.mean()
    var = float(np.dot(d, d) / n)
    if var == 0.0:
        return 0.5, 0
    # autocovariance by FFT (zero-padded)
    f = np.fft.rfft(d, 2 * n)
    acov = np.fft.irfft(f * np.conj(f))[:n] / n
    rho = acov / var
    tau = 0.5
    for t in range(1, n // 2):
        tau += rho[t]
        if t >= c * tau:
            return max(tau, 0.5), t
    return max(tau, 0.5), n // 2


def jackknife(x: Sequence[float], bin_size: int = 1) -> Tuple[float, float]:
    """Mean and jackknife error of the mean over bins of bin_size consecutive
    values (a trailing partial bin is dropped)."""
    a = np.asarray(x, dtype=np.float64)
    b = max(1, int(bin_size))
    nb = a.size // b
    if nb < 2:
        return float(a.mean()), float("nan")
    bins = a[: nb * b].reshape(nb, b).mean(axis=1)
    total = bins.sum()
    jk = (total - bins) / (nb - 1)
    m = float(jk.mean())
    err = math.sqrt((nb - 1) / nb * float(np.sum((jk - m) ** 2)))
    return float(bins.mean()), err


def mean_error(x: Sequence[float]) -> Dict[str, float]:
    """Mean, autocorrelation-corrected jackknife error (bins of ceil(2 tau_int)),
    tau_int and the number of bins."""
    tau, _ = tau_int(x)
    b = max(1, int(math.ceil(2.0 * tau)))
    m, e = jackknife(x, b)
    return {"mean": m, "err": e, "tau_int": tau, "bin": b, "n": len(x)}


def compare(x: Sequence[float], y: Sequence[float]) -> Dict[str, float]:
    """Difference of two independent chains' means in units of the combined error."""
    a, b = mean_error(x), mean_error(y)
    sig = math.sqrt(a["err"] ** 2 + b["err"] ** 2)
    return {"mean_a": a["mean"], "err_a": a["err"], "mean_b": b["mean"], "err_b": b["err"],
            "diff": a["mean"] - b["mean"], "sigma": sig, "z": (a["mean"] - b["mean"]) / sig if sig > 0 else 0.0,
            "tau_a": a["tau_int"], "tau_b": b["tau_int"]}
