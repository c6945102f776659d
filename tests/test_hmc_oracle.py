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


@pytest.mark.parametrize("nc", [1, 2, 3])
@pytest.mark.parametrize("integ", [INTEGRATOR_REFERENCE_LEAPFROG, INTEGRATOR_LEAPFROG, INTEGRATOR_OMELYAN])
def test_half_generators_equal_reference_at_half_tau(oracle, nc, integ):
    """t_a / 2 generators (force halved, exponent halved) integrate exactly the
    reference trajectory of half the length: the scale 1/2 is exact in binary,
    so the two agree bit for bit."""
    lat = Lat(nc, [4, 4, 2, 4])
    U0 = oracle.init(lat, True, 17)
    P0 = oracle.momenta(lat, 18, 0, 0)
    Ua, Pa, Ub, Pb = U0.copy(), P0.copy(), U0.copy(), P0.copy()
    try:
        oracle.set_generators(True)
        oracle.integrate(lat, Ua, Pa, 2.1, 0.8, 4, integ)
        Fh = oracle.gauge_force(lat, U0, 2.1)
    finally:
        oracle.set_generators(False)
    oracle.integrate(lat, Ub, Pb, 2.1, 0.4, 4, integ)
    assert np.array_equal(Ua, Ub) and np.array_equal(Pa, Pb)
    assert np.array_equal(Fh, 0.5 * oracle.gauge_force(lat, U0, 2.1))


def test_half_generators_accept_more_at_the_same_step_count(oracle):
    """SU(2) at beta 2.3, tau 1, 10 leapfrog steps: the t_a / 2 normalisation
    (half the effective step) gives a smaller |dH| than klft's Pauli one, and
    <exp(-dH)> stays 1 within errors."""
    lat = Lat(2, [4, 4, 4, 4])
    out = {}
    for half in (False, True):
        U = oracle.init(lat, True, 23)
        oracle.metropolis(lat, U, 2.3, 0.3, 5, 20, 23)
        try:
            oracle.set_generators(half)
            dH, acc = oracle.hmc(lat, U, 2.3, 1.0, 10, INTEGRATOR_LEAPFROG, 24, 0, 0, 60)
        finally:
            oracle.set_generators(False)
        out[half] = (np.mean(np.abs(dH)), acc.mean(), np.exp(-dH))
    assert out[True][0] < 0.25 * out[False][0]
    assert out[True][1] >= out[False][1]
    e = out[True][2]
    assert abs(e.mean() - 1.0) < 4 * e.std() / np.sqrt(len(e)) + 1e-3
