"""GPU parity: libklft_b200 (through its C ABI) against the oracle and against
the golden fixtures produced by klft's own code.

Tolerances: the plain FP64 form must reproduce deterministic kernels to 1e-12
relative and Metropolis trajectories hit by hit (identical acceptance counts,
links within 1e-11).  The mixed form (FP32 links, FP64 reductions) is held to
FP32 round-off: 2e-6 on observables of a given configuration.
"""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import PROPOSAL_EXP, Lat

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))
COMBOS = [(2, 1, [8, 6]), (2, 2, [6, 4]), (2, 3, [4, 6]), (3, 1, [4, 4, 6]), (3, 2, [4, 6, 4]), (3, 3, [4, 4, 4]),
          (4, 1, [4, 4, 4, 4]), (4, 2, [4, 2, 4, 6]), (4, 3, [4, 4, 2, 4])]
IDS = [f"{nd}d-nc{nc}" for nd, nc, _ in COMBOS]


def gf(L, nc, precision="fp64", start="cold", seed=0):
    import klft_b200
    return klft_b200.GaugeField(L, nc, precision, start, seed)


@pytest.mark.parametrize("nd,nc,L", COMBOS, ids=IDS)
def test_hot_start_matches_oracle(oracle, nd, nc, L):
    g = gf(L, nc, start="hot", seed=4242)
    U = oracle.init(Lat(nc, L), True, 4242)
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=1e-14)
    g.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 0.0), ("mixed", 3e-7)])
def test_upload_download_roundtrip(oracle, precision, tol):
    lat = Lat(3, [4, 6, 4, 2])
    U = oracle.init(lat, True, 1)
    g = gf(lat.L, 3, precision)
    g.upload(U)
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=tol)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_reference_golden_on_gpu(oracle, path):
    """klft's own outputs (golden fixtures) reproduced by the FP64 GPU form."""
    gd = np.load(path)
    nc, L, seed = int(gd["nc"]), [int(x) for x in gd["L"]], int(gd["seed"])
    g = gf(L, nc, start="hot", seed=seed)
    assert g.plaquette() == pytest.approx(float(gd["plaquette"]), rel=1e-12, abs=1e-14)
    np.testing.assert_allclose(g.wilson_loop_temporal(gd["pairs"]), gd["W_temp"], rtol=1e-12, atol=1e-14)
    for (m, n), w in zip(gd["munu"], gd["W_mu_nu"]):
        np.testing.assert_allclose(g.wilson_loop_mu_nu(int(m), int(n), gd["pairs"]), w, rtol=1e-12, atol=1e-14)
    if len(L) == 4:
        st = g.staple_field()
        np.testing.assert_allclose(st.sum(axis=(2, 3)), gd["staple_sum"], rtol=0, atol=1e-12)
    g.set_stream(seed, 0)
    acc = g.metropolis(float(gd["beta"]), float(gd["delta"]), int(gd["nhits"]), 3)
    np.testing.assert_array_equal(acc, gd["acc"])
    assert g.plaquette() == pytest.approx(float(gd["plaquette_after"]), rel=1e-11, abs=1e-13)
    U2 = g.download()
    np.testing.assert_allclose(U2.sum(axis=(2, 3)), gd["links_after_sum"], rtol=0, atol=1e-11)
    g.close()


@pytest.mark.parametrize("nd,nc,L", COMBOS, ids=IDS)
def test_observables_match_oracle(oracle, nd, nc, L):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 99)
    pairs = [(1, 1), (2, 1), (1, 2), (2, 2), (3, 3), (4, 2)]
    for precision, rtol, atol in (("fp64", 1e-12, 1e-14), ("mixed", 0.0, 2e-6)):
        g = gf(L, nc, precision)
        g.upload(U)
        assert g.plaquette() == pytest.approx(oracle.plaquette(lat, U), rel=rtol, abs=atol)
        np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs),
                                   rtol=rtol, atol=atol)
        np.testing.assert_allclose(g.wilson_loop_mu_nu(0, nd - 1, pairs), oracle.wilson_mu_nu(lat, U, 0, nd - 1, pairs),
                                   rtol=rtol, atol=atol)
        np.testing.assert_allclose(g.staple_field(), oracle.staple_field(lat, U), rtol=0,
                                   atol=1e-12 if precision == "fp64" else 2e-5)
        g.close()


@pytest.mark.parametrize("nd,nc,L", COMBOS, ids=IDS)
def test_metropolis_trajectory_matches_oracle(oracle, nd, nc, L):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, 7)
    g = gf(L, nc)
    g.upload(U)
    g.set_stream(31337, 5)
    beta = {1: 1.0, 2: 2.2, 3: 5.5}[nc]
    acc_g = g.metropolis(beta, 0.25, 5, 4)
    acc_o = oracle.metropolis(lat, U, beta, 0.25, 5, 4, 31337, chain=5)
    np.testing.assert_array_equal(acc_g, acc_o)
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=1e-11)
    assert g.counters()[0] == 4
    g.close()


@pytest.mark.parametrize("L", [[4, 4, 4, 4], [6, 4, 2, 4], [6, 4, 6, 4], [10, 6, 4], [8, 6], [4, 12], [12, 10, 6, 4]])
def test_metropolis_su3_exp_proposal_matches_oracle(oracle, L):
    """The exp(i eps H) link passes hit by hit against the oracle, in 2, 3 and 4
    dimensions and with half-volumes that are not multiples of the 32-site
    chunks a pass is laid out in (6, 36, 60, 12, 180 ...)."""
    lat = Lat(3, L)
    U = oracle.init(lat, True, 8)
    g = gf(L, 3)
    g.upload(U)
    g.set_stream(2024, 0)
    acc_g = g.metropolis(6.0, 0.0, 6, 3, proposal="exp", eps=0.35)
    acc_o = oracle.metropolis(lat, U, 6.0, 0.0, 6, 3, 2024, proposal=PROPOSAL_EXP, eps=0.35)
    np.testing.assert_array_equal(acc_g, acc_o)
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=1e-11)
    assert g.unitarity() < 1e-13
    # the mixed form on the same start follows within FP32 rounding for one sweep
    m = gf(L, 3, "mixed")
    m.upload(oracle.init(lat, True, 8))
    m.set_stream(2024, 0)
    acc_m = m.metropolis(6.0, 0.0, 6, 1, proposal="exp", eps=0.35)
    assert abs(acc_m[0] - acc_g[0]) < 0.02
    m.close()


def test_mixed_form_follows_fp64_chain(oracle):
    """FP32 links: one sweep from the same start stays within FP32 round-off of FP64."""
    lat = Lat(3, [8, 8, 8, 8])
    U = oracle.init(lat, True, 5)
    out = {}
    for precision in ("fp64", "mixed"):
        g = gf(lat.L, 3, precision)
        g.upload(U)
        g.set_stream(77, 0)
        acc = g.metropolis(6.0, 0.0, 10, 1, proposal="exp", eps=0.3)
        out[precision] = (acc[0], g.plaquette(), g.unitarity())
        g.close()
    assert abs(out["fp64"][0] - out["mixed"][0]) < 2e-3
    assert abs(out["fp64"][1] - out["mixed"][1]) < 1e-4
    assert out["mixed"][2] < 1e-5


def test_cold_start_gpu_known_answers():
    for nd, nc, L in COMBOS:
        for precision in ("fp64", "mixed"):
            g = gf(L, nc, precision)
            assert g.plaquette() == 1.0
            np.testing.assert_array_equal(g.wilson_loop_temporal([(1, 1), (2, 2), (2, 3)]), 1.0)
            g.close()


def test_invalid_arguments_raise():
    import klft_b200
    g = gf([4, 4, 4, 4], 2)
    with pytest.raises(klft_b200.KlftError):
        g.wilson_loop_mu_nu(0, 0, [(1, 1)])
    with pytest.raises(klft_b200.KlftError):
        g.wilson_loop_mu_nu(0, 4, [(1, 1)])
    with pytest.raises(klft_b200.KlftError):
        g.wilson_loop_temporal([(-1, 2)])
    with pytest.raises(klft_b200.KlftError):
        g.metropolis(1.0, float("nan"), 1, 1)
    g.close()


@pytest.mark.parametrize("precision,rtol,atol", [("fp64", 1e-12, 1e-14), ("mixed", 0.0, 2e-6)])
def test_wilson_loops_longer_than_lattice(oracle, precision, rtol, atol):
    """Gauge-fixed loops that wrap the lattice once or twice in either direction."""
    lat = Lat(3, [4, 6, 4, 6])
    U = oracle.init(lat, True, 17)
    g = gf(lat.L, 3, precision)
    g.upload(U)
    pairs = [(1, 1), (4, 3), (5, 6), (7, 13), (2, 12), (9, 1)]
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs), rtol=rtol,
                               atol=atol)
    for mu, nu in [(3, 0), (1, 2), (0, 3)]:
        np.testing.assert_allclose(g.wilson_loop_mu_nu(mu, nu, pairs), oracle.wilson_mu_nu(lat, U, mu, nu, pairs),
                                   rtol=rtol, atol=atol)


@pytest.mark.parametrize("L", [[6, 4, 4, 12], [4, 4, 20], [10, 6]])
def test_wilson_loops_uneven_extents(oracle, L):
    """Temporal extents that do not divide the warp (columns straddle warps)."""
    lat = Lat(2, L)
    U = oracle.init(lat, True, 23)
    g = gf(L, 2)
    g.upload(U)
    pairs = [(l, t) for l in range(1, 5) for t in range(1, 6)]
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs), rtol=1e-12,
                               atol=1e-14)


def test_wilson_degenerate_pairs(oracle):
    """Zero-extent loops (routed to the direct kernel) equal 1 up to round-off."""
    lat = Lat(3, [4, 4, 4, 4])
    U = oracle.init(lat, True, 29)
    g = gf(lat.L, 3)
    g.upload(U)
    pairs = [(0, 2), (2, 0), (0, 0), (2, 2)]
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs), rtol=1e-12,
                               atol=1e-14)


def test_mixed_form_dS_error_is_at_fp32_rounding():
    """The mixed form's action change against FP64 with the same proposals, hit
    by hit, on a thermalised SU(3) configuration: errors at FP32 rounding of the
    local action (|d| well below 1e-3, rms below 1e-4), no systematic relative
    error above 1e-5, and accept decisions that differ on a tiny fraction of hits."""
    import klft_b200
    g = klft_b200.GaugeField([8, 8, 8, 8], 3, "fp64", "hot", 61)
    g.set_stream(61, 0)
    g.metropolis(6.0, 0.0, 10, 60, "exp", 0.25)
    U = g.download()
    r = g.exp_dS_error(6.0, 0.25, 10)
    assert r["hits"] == 8 ** 4 * 4 * 10
    assert r["rms"] < 1e-4 and r["max_abs"] < 1e-3
    assert abs(r["slope"]) < 1e-5
    assert r["decision_flip_fraction"] < 1e-3
    np.testing.assert_array_equal(g.download(), U)  # the diagnostic changes no link
    g.close()
