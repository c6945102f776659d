"""The error analysis used by the ensemble comparisons, checked on series with
known answers (no GPU)."""
import numpy as np

from klft_b200.stats import compare, jackknife, mean_error, tau_int


def ar1(n, phi, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros(n)
    e = rng.normal(size=n)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    return x


def test_tau_int_of_white_noise_and_ar1():
    rng = np.random.default_rng(1)
    t, _ = tau_int(rng.normal(size=20000))
    assert 0.4 < t < 0.65
    # AR(1): tau = (1 + phi) / (2 (1 - phi)) = 4.5 for phi = 0.8
    t, _ = tau_int(ar1(200000, 0.8, 2))
    assert 4.0 < t < 5.0


def test_jackknife_error_of_independent_data():
    rng = np.random.default_rng(3)
    x = rng.normal(size=10000)
    m, e = jackknife(x, 1)
    assert abs(m - x.mean()) < 1e-12
    assert abs(e - x.std(ddof=1) / np.sqrt(x.size)) < 1e-9


def test_binning_corrects_for_autocorrelation():
    x = ar1(200000, 0.9, 4)  # tau = 9.5, true error of the mean ~ sqrt(2 tau / n) * sd
    sd = x.std()
    me = mean_error(x)
    want = np.sqrt(2 * 9.5 / x.size) * sd
    assert 0.7 * want < me["err"] < 1.3 * want
    naive = sd / np.sqrt(x.size)
    assert me["err"] > 3 * naive


def test_compare_independent_chains():
    a, b = ar1(50000, 0.5, 5), ar1(50000, 0.5, 6)
    c = compare(a, b)
    assert abs(c["z"]) < 3
    c2 = compare(a + 0.5, b)
    assert c2["z"] > 5


def test_ensemble_summary_is_the_standard_error_of_chain_means():
    from klft_b200.ensemble import summary
    rng = np.random.default_rng(3)
    means = 0.59 + 1e-4 * rng.normal(size=4000)
    m, e = summary(means)
    assert abs(m - 0.59) < 5 * e
    assert abs(e - 1e-4 / np.sqrt(4000)) < 0.1 * e
