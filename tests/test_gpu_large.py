"""GPU parity at the benchmark sizes: SU(3) 32^4, PTBC SU(3) 16^4 replicas
and SU(2) 24^4 HMC, through the C ABI, against klft's own code (compiled on
the Kokkos-API host shim, all host threads) and against the oracle.

Layout and index arithmetic that small lattices never reach (32-bit site
decode, parity-class blocked offsets beyond 2^24 elements, persistent Wilson
tiles over 32,768 columns, multi-chain CTA tables) are exercised here.  Each
CPU side runs one sweep or one trajectory, on OpenMP threads.

Tolerances: FP64 form hit by hit (identical acceptance, links within 1e-11),
plaquette 1e-12 relative, the 64 temporal Wilson loops 1e-12 relative; the
mixed form within 2e-6 absolute of klft's observables; HMC energies within
1e-13 relative of the oracle's compensated sums, links within 1e-11.
"""
import os

import numpy as np
import pytest

from oracle.oracle import INTEGRATOR_LEAPFROG, PROPOSAL_EXP, Lat

pytestmark = pytest.mark.gpu

PAIRS_8x8 = [(L, T) for L in range(1, 9) for T in range(1, 9)]


def gf(L, nc, precision="fp64", start="cold", seed=0):
    import klft_b200
    return klft_b200.GaugeField(L, nc, precision, start, seed)


@pytest.fixture(scope="module")
def su3_32(refshim):
    """One SU(3) 32^4 FP64 hot start after one reference-proposal sweep on the
    GPU, and the same sweep by klft's own code."""
    refshim.set_threads(os.cpu_count() or 1)
    lat = Lat(3, [32, 32, 32, 32])
    g = gf(lat.L, 3, "fp64", "hot", 32091)
    U = g.download()
    g.set_stream(32091, 0)
    acc_g = g.metropolis(6.0, 0.1, 10, 1)
    acc_r = refshim.metropolis(lat, U, 6.0, 0.1, 10, 1, 32091)
    yield lat, g, U, acc_g, acc_r
    g.close()


def test_su3_32x4_reference_sweep_matches_klft_code(su3_32):
    lat, g, U, acc_g, acc_r = su3_32
    np.testing.assert_array_equal(acc_g, acc_r)
    Ug = g.download()
    assert np.max(np.abs(Ug - U)) < 1e-11
    # a checksum of checksums: per-direction sums over the whole lattice
    np.testing.assert_allclose(Ug.sum(axis=(0, 2, 3)), U.sum(axis=(0, 2, 3)), rtol=1e-12)


def test_su3_32x4_observables_match_klft_code(su3_32, refshim):
    lat, g, U, _, _ = su3_32
    p_ref = refshim.plaquette(lat, U)
    assert g.plaquette() == pytest.approx(p_ref, rel=1e-12)
    w_ref = refshim.wilson_temporal(lat, U, PAIRS_8x8)
    np.testing.assert_allclose(g.wilson_loop_temporal(PAIRS_8x8), w_ref, rtol=1e-12, atol=1e-15)
    # the mixed form on the same configuration (FP32 links, FP64 sums)
    m = gf(lat.L, 3, "mixed")
    m.upload(U)
    assert abs(m.plaquette() - p_ref) < 2e-6
    np.testing.assert_allclose(m.wilson_loop_temporal(PAIRS_8x8), w_ref, rtol=0, atol=2e-6)
    m.close()


def test_su3_32x4_exp_sweep_matches_oracle(oracle):
    """One exp(i eps H) sweep (eps 0.25, 10 hits) from a hot start, FP64."""
    lat = Lat(3, [32, 32, 32, 32])
    g = gf(lat.L, 3, "fp64", "hot", 4711)
    U = g.download()
    g.set_stream(4711, 2)
    acc_g = g.metropolis(6.0, 0.0, 10, 1, "exp", 0.25)
    acc_o = oracle.metropolis(lat, U, 6.0, 0.0, 10, 1, 4711, chain=2, proposal=PROPOSAL_EXP, eps=0.25)
    np.testing.assert_array_equal(acc_g, acc_o)
    assert np.max(np.abs(g.download() - U)) < 1e-11
    assert g.plaquette() == pytest.approx(oracle.plaquette(lat, U), rel=1e-12)
    g.close()


DEFECT_16 = [4, 0, 0, 0]  # L_d = 4 at the origin


def test_ptbc_16x4_replica_sweep_and_defect_sums_match_oracle(oracle):
    lat = Lat(3, [16, 16, 16, 16])
    g = gf(lat.L, 3, "fp64", "hot", 5003)
    U = g.download()
    g.set_defect(DEFECT_16[0], DEFECT_16[1:], 1.0 - 3 / 11)
    g.set_stream(5000, 3)
    acc_g = g.metropolis(6.0, 0.0, 10, 1, "exp", 0.25)
    acc_o = oracle.metropolis(lat, U, 6.0, 0.0, 10, 1, 5000, chain=3, proposal=PROPOSAL_EXP, eps=0.25,
                              defect=DEFECT_16, defect_c=1.0 - 3 / 11)
    np.testing.assert_array_equal(acc_g, acc_o)
    assert np.max(np.abs(g.download() - U)) < 1e-11
    np.testing.assert_allclose(g.defect_sums(6.0), oracle.defect_sums(lat, U, DEFECT_16, 6.0), rtol=1e-12)
    g.close()


def test_ptbc_16x4_batch_with_uneven_chains_equals_chains_alone(oracle):
    """Two 16^4 replicas and SU(2) chains of uneven extents in one captured
    cycle: bit for bit what each does alone, and the swap the oracle makes from
    the replicas' defect sums."""
    import klft_b200
    c = [1.0, 0.5]
    b = klft_b200.Batch()
    solo, batch, ids = [], [], []
    for r in range(2):
        pair = []
        for _ in range(2):
            g = gf([16] * 4, 3, "mixed", "hot", 5000 + r)
            g.set_stream(5000, r)
            g.set_defect(DEFECT_16[0], DEFECT_16[1:], c[r])
            pair.append(g)
        ids.append(b.add(pair[0], 6.0, 0.0, 10, "exp", 0.25))
        batch.append(pair[0])
        solo.append(pair[1])
    chains = [([8, 12, 16, 20], 2.3), ([24, 24, 24, 24], 2.5), ([20, 8, 24, 12], 2.2)]
    for k, (L, beta) in enumerate(chains):
        pair = []
        for _ in range(2):
            g = gf(L, 2, "mixed", "hot", 7000 + k)
            g.set_stream(7000, k)
            pair.append(g)
        b.add(pair[0], beta, 0.3, 10)
        batch.append(pair[0])
        solo.append(pair[1])
    b.set_ptbc(ids, c, 6.0, 99)
    acc, plaq, labels, _ = b.run(2, True, True)
    lab = np.arange(2)
    for cyc in range(2):
        for r in range(2):
            assert acc[cyc, r] == solo[r].metropolis(6.0, 0.0, 10, 1, "exp", 0.25)[0]
        for k, (L, beta) in enumerate(chains):
            assert acc[cyc, 2 + k] == solo[2 + k].metropolis(beta, 0.3, 10, 1)[0]
            assert plaq[cyc, 2 + k] == solo[2 + k].plaquette()
        A = np.array([s.defect_sums(6.0) for s in solo[:2]])
        lab_o, _ = oracle.ptbc_swap(np.array(c), A, lab, 99, cyc)
        lab, _ = klft_b200.ptbc_swap(solo[:2], c, lab, 6.0, 99, cyc)
        np.testing.assert_array_equal(lab, lab_o)
        np.testing.assert_array_equal(labels[cyc], lab)
    for x, y in zip(batch, solo):
        np.testing.assert_array_equal(x.download(), y.download())
    b.close()
    for g in batch + solo:
        g.close()


@pytest.mark.parametrize("generators", ["reference", "half"])
def test_su2_24x4_hmc_trajectory_matches_oracle(oracle, generators):
    """The benchmark HMC trajectory (SU(2) 24^4, beta 2.3, tau 1, 20 leapfrog
    steps) from one Haar-random start: force, energies before and after the
    trajectory, links and momenta, FP64; both generator normalisations."""
    lat = Lat(2, [24, 24, 24, 24])
    beta = 2.3
    g = gf(lat.L, 2, "fp64", "hot", 2424)
    g.set_hmc_generators(generators)
    U = g.download()
    half = generators == "half"
    oracle.set_generators(half)
    try:
        np.testing.assert_allclose(g.gauge_force(beta), oracle.gauge_force(lat, U, beta), rtol=0, atol=1e-12)
        g.set_stream(11, 0)
        g.set_counters(0, 3)
        g.refresh_momenta()
        P = oracle.momenta(lat, 11, 0, 3)
        # Box-Muller through the device's and the host's log / sincos: a few ulp
        np.testing.assert_allclose(g.momenta(), P, rtol=0, atol=1e-14)
        g.set_momenta(P)  # the trajectory starts from identical momenta
        k0, s0 = g.hmc_energies(beta)
        h0_o = 0.5 * np.sum(P * P) + oracle.gauge_action(lat, U, beta)  # numpy's pairwise sum
        assert k0 + s0 == pytest.approx(h0_o, rel=1e-13)
        g.hmc_integrate(beta, 1.0, 20, "leapfrog")
        oracle.integrate(lat, U, P, beta, 1.0, 20, INTEGRATOR_LEAPFROG)
        assert np.max(np.abs(g.download() - U)) < 1e-11
        assert np.max(np.abs(g.momenta() - P)) < 1e-10
        k1, s1 = g.hmc_energies(beta)
        h1_o = 0.5 * np.sum(P * P) + oracle.gauge_action(lat, U, beta)
        assert k1 + s1 == pytest.approx(h1_o, rel=1e-13)
        # dH agrees to the rounding of H itself (|H| ~ 1e6 here)
        assert abs((k1 + s1 - k0 - s0) - (h1_o - h0_o)) < 1e-12 * abs(h0_o)
    finally:
        oracle.set_generators(False)
    g.close()
