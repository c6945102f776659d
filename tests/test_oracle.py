"""CPU tests of the checker: the oracle against klft's own code (golden
fixtures generated by the reference headers on the Kokkos-API shim), the
reference's known answers (cold start: plaquette = W(L,T) = 1) and physics
identities."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import PROPOSAL_EXP, Lat

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


def test_philox_known_answers(oracle):
    # Random123 known-answer vectors for Philox4x32-10
    assert [hex(x) for x in oracle.philox([0, 0, 0, 0], [0, 0])] == ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                          [0xA4093822, 0x299F31D0])] == ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_uniform_stream_range(oracle):
    u = oracle.uniforms(7, 3, 11, 2, 1, 0, 4096)
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.02


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_reference_golden(oracle, path):
    g = np.load(path)
    lat = Lat(int(g["nc"]), list(g["L"]))
    U = oracle.init(lat, True, int(g["seed"]))
    assert oracle.plaquette(lat, U) == pytest.approx(float(g["plaquette"]), rel=1e-13, abs=1e-15)
    np.testing.assert_allclose(oracle.wilson_temporal(lat, U, g["pairs"]), g["W_temp"], rtol=1e-12, atol=1e-15)
    for (m, n), w in zip(g["munu"], g["W_mu_nu"]):
        np.testing.assert_allclose(oracle.wilson_mu_nu(lat, U, int(m), int(n), g["pairs"]), w, rtol=1e-12, atol=1e-15)
    if lat.nd == 4:
        st = oracle.staple_field(lat, U)
        np.testing.assert_allclose(st.sum(axis=(2, 3)), g["staple_sum"], rtol=0, atol=1e-13)
        np.testing.assert_allclose(st[:4], g["staple_first"], rtol=0, atol=1e-13)
    U2 = U.copy()
    acc = oracle.metropolis(lat, U2, float(g["beta"]), float(g["delta"]), int(g["nhits"]), 3, int(g["seed"]))
    np.testing.assert_array_equal(acc, g["acc"])
    assert oracle.plaquette(lat, U2) == pytest.approx(float(g["plaquette_after"]), rel=1e-12, abs=1e-14)
    np.testing.assert_allclose(U2.sum(axis=(2, 3)), g["links_after_sum"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(U2[:8], g["links_after_first"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("nd,nc", [(2, 1), (3, 2), (4, 3), (4, 1)])
def test_oracle_matches_reference_live(oracle, refshim, nd, nc):
    L = {2: [6, 8], 3: [4, 6, 4], 4: [4, 4, 2, 6]}[nd]
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 555 + nd * 10 + nc)
    assert oracle.plaquette(lat, U) == pytest.approx(refshim.plaquette(lat, U), rel=1e-13, abs=1e-15)
    pairs = [(1, 1), (2, 3), (3, 1)]
    np.testing.assert_allclose(oracle.wilson_temporal(lat, U, pairs), refshim.wilson_temporal(lat, U, pairs),
                               rtol=1e-12, atol=1e-15)
    Ua, Ub = U.copy(), U.copy()
    np.testing.assert_array_equal(oracle.metropolis(lat, Ua, 2.0, 0.2, 3, 2, 77),
                                  refshim.metropolis(lat, Ub, 2.0, 0.2, 3, 2, 77))
    assert np.array_equal(Ua, Ub)


@pytest.mark.parametrize("nd,nc", [(2, 1), (2, 2), (2, 3), (3, 1), (3, 2), (3, 3), (4, 1), (4, 2), (4, 3)])
def test_cold_start_known_answers(oracle, nd, nc):
    # plaq_bench.cpp:88-89 and wloop_temporal_bench.cpp:96-99: identity links give 1
    lat = Lat(nc, [4] * nd)
    U = oracle.init(lat, False)
    assert oracle.plaquette(lat, U) == 1.0
    np.testing.assert_array_equal(oracle.wilson_temporal(lat, U, [(1, 1), (2, 2), (2, 3)]), 1.0)


def _random_gauge(oracle, lat, seed):
    G = oracle.init(Lat(lat.nc, lat.L + ([] if lat.nd == 4 else [])), True, seed)
    return G[:, 0]  # one random group element per site


def _transform(lat, U, g):
    """U_mu(x) -> g(x) U_mu(x) g(x+mu)^+."""
    V = np.empty_like(U)
    coords = np.array(np.unravel_index(np.arange(lat.V), lat.L[::-1]))[::-1].T  # x0 fastest
    for mu in range(lat.nd):
        xp = coords.copy()
        xp[:, mu] = (xp[:, mu] + 1) % lat.L[mu]
        sp = np.ravel_multi_index(xp.T[::-1], lat.L[::-1])
        V[:, mu] = g @ U[:, mu] @ np.conj(np.transpose(g[sp], (0, 2, 1)))
    return V


@pytest.mark.parametrize("nd,nc", [(2, 2), (3, 3), (4, 3), (4, 1)])
def test_gauge_invariance(oracle, nd, nc):
    lat = Lat(nc, [4] * nd)
    U = oracle.init(lat, True, 5)
    g = _random_gauge(oracle, lat, 9)
    V = _transform(lat, U, g)
    assert oracle.plaquette(lat, V) == pytest.approx(oracle.plaquette(lat, U), abs=1e-13)
    pairs = [(1, 2), (2, 2), (3, 1)]
    np.testing.assert_allclose(oracle.wilson_temporal(lat, V, pairs), oracle.wilson_temporal(lat, U, pairs),
                               atol=1e-13)


def test_expi_su3_is_unitary_and_matches_eigen(oracle):
    rng = np.random.default_rng(0)
    for _ in range(20):
        A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        Q = (A + A.conj().T) / 2
        Q -= np.trace(Q) / 3 * np.eye(3)
        Q *= rng.uniform(0.01, 2.0)
        X = oracle.expi_su3(Q)
        w, v = np.linalg.eigh(Q)
        ref = v @ np.diag(np.exp(1j * w)) @ v.conj().T
        np.testing.assert_allclose(X, ref, atol=1e-13)
        assert abs(np.linalg.det(X) - 1) < 1e-13


def test_metropolis_keeps_links_unitary(oracle):
    lat = Lat(3, [4, 4, 4, 4])
    U = oracle.init(lat, True, 3)
    oracle.metropolis(lat, U, 6.0, 0.1, 4, 3, 3, proposal=PROPOSAL_EXP, eps=0.3)
    assert oracle.unitarity(lat, U) < 1e-13


def test_u1_2d_exact_plaquette(oracle):
    # 2D U(1), infinite volume: <P> = I1(beta)/I0(beta)
    from scipy.special import iv
    lat = Lat(1, [16, 16])
    U = oracle.init(lat, True, 12)
    beta = 2.0
    oracle.metropolis(lat, U, beta, 0.5, 10, 100, 12)
    ps = []
    for k in range(400):
        oracle.metropolis(lat, U, beta, 0.5, 10, 1, 12, sweep0=100 + k)
        ps.append(oracle.plaquette(lat, U))
    assert np.mean(ps) == pytest.approx(iv(1, beta) / iv(0, beta), abs=0.01)


def test_su2_2d_exact_plaquette(oracle):
    # 2D SU(2): <(1/2) Re Tr P> = I2(beta)/I1(beta)
    from scipy.special import iv
    lat = Lat(2, [16, 16])
    U = oracle.init(lat, True, 21)
    beta = 3.0
    oracle.metropolis(lat, U, beta, 0.4, 10, 100, 21)
    ps = []
    for k in range(400):
        oracle.metropolis(lat, U, beta, 0.4, 10, 1, 21, sweep0=100 + k)
        ps.append(oracle.plaquette(lat, U))
    assert np.mean(ps) == pytest.approx(iv(2, beta) / iv(1, beta), abs=0.01)


@pytest.mark.parametrize("nd,nc", [(4, 3), (3, 2), (2, 1)])
def test_legacy_gaugevector_loop_matches_wilson_mu_nu(oracle, nd, nc):
    """The legacy whole-field path (GaugeVector.hpp:237-262) and the per-site
    WilsonLoop_mu_nu restatement (pinned against klft's headers) agree on every
    plane, for loops longer than the extent and with mu > nu; Normalize=false is
    the Re Tr sum, V * Nc times the normalised value; identity links give 1."""
    L = [4, 6, 4, 6][:nd]
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 77)
    V = int(np.prod(L))
    for mu in range(nd):
        for nu in range(nd):
            if mu == nu:
                continue
            for Lmu, Lnu in [(1, 1), (2, 3), (5, 1), (0, 2)]:
                w = oracle.wilson_legacy(lat, U, mu, nu, Lmu, Lnu)
                ref = oracle.wilson_mu_nu(lat, U, mu, nu, [(Lmu, Lnu)])[0]
                assert abs(w - ref) < 1e-13
                raw = oracle.wilson_legacy(lat, U, mu, nu, Lmu, Lnu, normalize=False)
                assert abs(raw - w * V * nc) < 1e-10 * V
    assert abs(oracle.wilson_legacy(lat, oracle.init(lat, False), 0, nd - 1, 3, 2) - 1.0) < 1e-15
