"""CPU tests of the HMC oracle (the reference HMC stack does not compile, so
HMC parity rests on these identities): reversibility, dH ~ dt^2 for the
leapfrog, <exp(-dH)> = 1, force = -dS/dA by finite differences."""
import numpy as np
import pytest

from oracle.oracle import INTEGRATOR_LEAPFROG, INTEGRATOR_OMELYAN, INTEGRATOR_REFERENCE_LEAPFROG, Lat


@pytest.mark.parametrize("nc", [1, 2, 3])
@pytest.mark.parametrize("integ", [INTEGRATOR_REFERENCE_LEAPFROG, INTEGRATOR_LEAPFROG, INTEGRATOR_OMELYAN])
def test_reversibility(oracle, nc, integ):
    lat = Lat(nc, [4, 4, 4, 4])
    U = oracle.init(lat, True, 3)
    U0 = U.copy()
    P = oracle.momenta(lat, 5, 0, 0)
    oracle.integrate(lat, U, P, 2.0, 0.5, 5, integ)
    P *= -1.0
    oracle.integrate(lat, U, P, 2.0, 0.5, 5, integ)
    assert np.max(np.abs(U - U0)) < 1e-10


@pytest.mark.parametrize("nc", [2, 3])
def test_dH_scales_as_dt_squared(oracle, nc):
    lat = Lat(nc, [4, 4, 4, 4])
    beta = {2: 2.3, 3: 5.7}[nc]
    U0 = oracle.init(lat, True, 8)
    # thermalise a little so the force is typical
    oracle.metropolis(lat, U0, beta, 0.3 if nc == 2 else 0.0, 5, 5, 8, proposal=1 if nc == 3 else 0, eps=0.3)
    dHs = []
    for n in (40, 80):  # asymptotic regime; averaged over four momentum draws
        r = []
        for seed in range(4):
            U = U0.copy()
            P = oracle.momenta(lat, 9 + seed, 0, 0)
            h0 = 0.5 * np.sum(P * P) + oracle.gauge_action(lat, U, beta)
            oracle.integrate(lat, U, P, beta, 0.5, n, INTEGRATOR_LEAPFROG)
            h1 = 0.5 * np.sum(P * P) + oracle.gauge_action(lat, U, beta)
            r.append(abs(h1 - h0))
        dHs.append(np.mean(r))
    assert 3.2 < dHs[0] / dHs[1] < 4.8


def test_exp_minus_dH_averages_to_one(oracle):
    lat = Lat(2, [4, 4, 4, 4])
    U = oracle.init(lat, True, 11)
    dH, acc = oracle.hmc(lat, U, 2.3, 1.0, 20, INTEGRATOR_LEAPFROG, 11, 0, 0, 80)
    e = np.exp(-dH[10:])
    assert abs(e.mean() - 1.0) < 4 * e.std() / np.sqrt(len(e))
    assert acc.mean() > 0.5


@pytest.mark.parametrize("nc", [1, 2, 3])
def test_force_is_minus_action_gradient(oracle, nc):
    """P -= dt F must decrease H: F_a(x, mu) = d S / d w_a for U -> exp(i w t_a) U."""
    lat = Lat(nc, [4, 4, 2, 2])
    beta = 1.7
    U = oracle.init(lat, True, 13)
    F = oracle.gauge_force(lat, U, beta)
    rng = np.random.default_rng(1)
    for _ in range(3):
        s, mu = int(rng.integers(lat.V)), int(rng.integers(lat.nd))
        a = int(rng.integers(F.shape[2]))
        h = 1e-6
        vals = []
        for sign in (+1, -1):
            V = U.copy()
            P = np.zeros_like(F)
            P[s, mu, a] = sign * h
            # a gauge update with dt = 1 applies exp(i P t) to every link; P is zero elsewhere
            oracle.integrate(lat, V, P, 0.0, 1.0, 1, INTEGRATOR_LEAPFROG)
            vals.append(oracle.gauge_action(lat, V, beta))
        grad = (vals[0] - vals[1]) / (2 * h)
        assert grad == pytest.approx(F[s, mu, a], rel=1e-5, abs=1e-8)
