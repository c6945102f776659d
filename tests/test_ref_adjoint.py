"""The oracle's HMC Lie-algebra maps against klft's own AdjointGroup.hpp code
(compiled unchanged on the Kokkos-API shim, oracle/_ref): the adjoint
projection Adj(M) of the force, the exponential map of the gauge update and
the SU(2) product exp(dt P) U, for U(1) and SU(2) (the groups klft's HMC has).
CPU only: these pin the maps the GPU HMC kernels are checked against."""
import numpy as np
import pytest


def rand_su2(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    return np.array([[q[0] + 1j * q[3], q[2] + 1j * q[1]], [-q[2] + 1j * q[1], q[0] - 1j * q[3]]])


def test_su2_adjoint_matches_klft(oracle, refadj):
    rng = np.random.default_rng(1)
    for _ in range(200):
        # a staple product U S is a real multiple of an SU(2) matrix; also a general matrix
        M = rng.uniform(0.1, 6.0) * rand_su2(rng)
        G = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        for m in (M, G):
            np.testing.assert_allclose(oracle.adjoint(m), refadj.adjoint(m), rtol=0, atol=1e-15)


def test_su2_exp_matches_klft(oracle, refadj):
    rng = np.random.default_rng(2)
    for _ in range(200):
        p = rng.normal(size=3)
        t = rng.uniform(-0.2, 0.2)
        np.testing.assert_allclose(oracle.expmap(2, p, t), refadj.expmap(2, p, t), rtol=0, atol=1e-15)
    # large arguments wrap around the group
    for scale in (1.0, 3.0, 10.0):
        p = scale * rng.normal(size=3)
        np.testing.assert_allclose(oracle.expmap(2, p, 1.0), refadj.expmap(2, p, 1.0), rtol=0, atol=1e-14)


def test_su2_gauge_update_product_matches_klft(oracle, refadj):
    """exp(dt P) U with klft's SU2 product (GaugeGroup.hpp:376-383) equals the
    generic complex product the oracle and the GPU use, on group elements."""
    rng = np.random.default_rng(3)
    for _ in range(200):
        X = refadj.expmap(2, rng.normal(size=3), 0.05)
        U = rand_su2(rng)
        np.testing.assert_allclose(refadj.su2_mul(X, U), X @ U, rtol=0, atol=2e-16 * 8)


def test_u1_maps_match_klft(oracle, refadj):
    rng = np.random.default_rng(4)
    for _ in range(200):
        M = np.array([[rng.normal() + 1j * rng.normal()]])
        np.testing.assert_allclose(oracle.adjoint(M), refadj.adjoint(M), rtol=0, atol=1e-15)
        p, t = rng.normal(size=1), rng.uniform(-0.3, 0.3)
        np.testing.assert_allclose(oracle.expmap(1, p, t), refadj.expmap(1, p, t), rtol=0, atol=1e-15)


@pytest.mark.parametrize("nc", [1, 2])
def test_oracle_force_is_klft_adjoint_of_u_times_staple(oracle, refadj, nc):
    """F(x, mu) = (beta/Nc) Adj(U_mu(x) S_mu(x)) (GaugeMonomial.hpp:27-37) with
    klft's own Adj, on the oracle's staples (pinned to klft's staple code)."""
    from oracle.oracle import Lat
    lat = Lat(nc, [4, 4, 2, 4])
    U = oracle.init(lat, True, 9)
    beta = 2.2
    F = oracle.gauge_force(lat, U, beta)
    S = oracle.staple_field(lat, U)
    for s in range(0, lat.V, 7):
        for mu in range(lat.nd):
            ref = (beta / nc) * refadj.adjoint(U[s, mu] @ S[s, mu])
            np.testing.assert_allclose(F[s, mu], ref, rtol=0, atol=1e-13)
