"""GPU parity of HMC against the oracle (FP64 form to round-off; the mixed form
to FP32 accuracy) and the HMC identities on the device."""
import numpy as np
import pytest

from oracle.oracle import INTEGRATOR_LEAPFROG, INTEGRATOR_OMELYAN, INTEGRATOR_REFERENCE_LEAPFROG, Lat

pytestmark = pytest.mark.gpu

INTEG = {"reference": INTEGRATOR_REFERENCE_LEAPFROG, "leapfrog": INTEGRATOR_LEAPFROG, "omelyan": INTEGRATOR_OMELYAN}
COMBOS = [(1, [6, 4, 4, 4]), (2, [4, 4, 4, 4]), (3, [4, 4, 2, 4]), (2, [6, 8]), (3, [4, 4, 4])]


def gf(L, nc, precision="fp64", start="cold", seed=0):
    import klft_b200
    return klft_b200.GaugeField(L, nc, precision, start, seed)


@pytest.mark.parametrize("nc,L", COMBOS)
def test_force_and_momenta_match_oracle(oracle, nc, L):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 31)
    g = gf(L, nc)
    g.upload(U)
    np.testing.assert_allclose(g.gauge_force(2.1), oracle.gauge_force(lat, U, 2.1), rtol=0, atol=1e-12)
    g.set_stream(77, 3)
    g.set_counters(0, 5)
    g.refresh_momenta()
    np.testing.assert_allclose(g.momenta(), oracle.momenta(lat, 77, 3, 5), rtol=0, atol=1e-14)
    k, s = g.hmc_energies(2.1)
    P = oracle.momenta(lat, 77, 3, 5)
    assert k == pytest.approx(0.5 * np.sum(P * P), rel=1e-13)
    assert s == pytest.approx(oracle.gauge_action(lat, U, 2.1), rel=1e-12)


@pytest.mark.parametrize("nc,L", COMBOS)
@pytest.mark.parametrize("integ", ["reference", "leapfrog", "omelyan"])
def test_integrate_matches_oracle(oracle, nc, L, integ):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 41)
    P = oracle.momenta(lat, 42, 0, 0)
    g = gf(L, nc)
    g.upload(U)
    g.set_momenta(P)
    g.hmc_integrate(2.0, 0.6, 6, integ)
    oracle.integrate(lat, U, P, 2.0, 0.6, 6, INTEG[integ])
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=1e-12)
    np.testing.assert_allclose(g.momenta(), P, rtol=0, atol=1e-11)


# dH = H_new - H_old is a difference of lattice sums of size ~V: its rounding
# floor is ~1e-16 of H, not of dH, hence the absolute term for small dH.
DH_RTOL, DH_ATOL, LINK_ATOL = 1e-12, 1e-12, 1e-12


@pytest.mark.parametrize("nc,L", COMBOS[:3] + [(2, [8, 8, 8, 8]), (3, [8, 8, 8, 8])])
@pytest.mark.parametrize("integ", ["leapfrog", "omelyan"])
def test_trajectories_match_oracle(oracle, nc, L, integ):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 51)
    g = gf(L, nc)
    g.upload(U)
    g.set_stream(1001, 7)
    beta = {1: 1.0, 2: 2.3, 3: 5.5}[nc]
    dH_g, acc_g = g.hmc(beta, 1.0, 8, 4, integ)
    dH_o, acc_o = oracle.hmc(lat, U, beta, 1.0, 8, INTEG[integ], 1001, 7, 0, 4)
    np.testing.assert_array_equal(acc_g, acc_o)
    np.testing.assert_allclose(dH_g, dH_o, rtol=DH_RTOL, atol=DH_ATOL)
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=LINK_ATOL)
    assert g.counters()[1] == 4


def test_gpu_reversibility_and_mixed_dH():
    import klft_b200
    for precision, tol in (("fp64", 1e-11), ("mixed", 5e-5)):
        g = klft_b200.GaugeField([8, 8, 8, 8], 2, precision, "hot", 3)
        U0 = g.download()
        g.refresh_momenta()
        g.hmc_integrate(2.3, 0.5, 10, "leapfrog")
        g.set_momenta(-g.momenta())
        g.hmc_integrate(2.3, 0.5, 10, "leapfrog")
        assert np.max(np.abs(g.download() - U0)) < tol
        g.close()
    # mixed form: dH of a trajectory within FP32 round-off of the FP64 form from the same state
    out = {}
    for precision in ("fp64", "mixed"):
        g = klft_b200.GaugeField([8, 8, 8, 8], 2, precision, "hot", 5)
        g.set_stream(12, 0)
        out[precision] = g.hmc(2.3, 1.0, 20, 1, "leapfrog")[0][0]
        g.close()
    assert abs(out["fp64"] - out["mixed"]) < 2e-2


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("generators,integrator", [("half", "leapfrog"), ("reference", "omelyan"),
                                                   ("half", "omelyan")])
def test_su2_8x4_hmc_chain_accepts_and_exp_minus_dH_is_one(precision, generators, integrator):
    """SU(2) 8^4 at beta 2.3, tau 1, 20 steps after a Metropolis
    thermalisation: acceptance above one half and <exp(-dH)> = 1 within three
    standard errors over 140 trajectories, in both forms.  (klft's Pauli
    normalisation with the 20-step leapfrog doubles the effective step and
    accepts about half of the trajectories at this volume, none at 24^4.)"""
    import klft_b200
    g = klft_b200.GaugeField([8, 8, 8, 8], 2, precision, "hot", 808)
    g.set_stream(808, 1)
    g.metropolis(2.3, 0.3, 5, 100)
    g.set_hmc_generators(generators)
    g.hmc(2.3, 1.0, 20, 10, integrator)
    dH, acc = g.hmc(2.3, 1.0, 20, 140, integrator)
    e = np.exp(-dH)
    assert acc.mean() > 0.5
    assert abs(e.mean() - 1.0) < 3.0 * e.std(ddof=1) / np.sqrt(len(e))
    assert 0.55 < g.plaquette() < 0.65
    g.close()


def test_half_generators_are_the_reference_at_half_tau_on_gpu():
    import klft_b200
    out = []
    for generators, tau in (("half", 0.8), ("reference", 0.4)):
        g = klft_b200.GaugeField([4, 4, 4, 6], 3, "fp64", "hot", 77)
        g.set_hmc_generators(generators)
        g.set_stream(3, 0)
        dH, acc = g.hmc(5.5, tau, 6, 3, "omelyan")
        out.append((dH, acc, g.download()))
        g.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][2], out[1][2])
