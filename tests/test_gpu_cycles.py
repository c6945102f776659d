"""klft_run_cycles (the run_metropolis loop, Metropolis.hpp:204-218) against the
same steps through the single-call API: sweep, GaugePlaquette, WilsonLoop_temporal.
With (1, 1) among the temporal pairs the cycle takes the temporal plaquettes from
those loop sums, so both pair lists are checked."""
import numpy as np
import pytest

from klft_b200 import GaugeField

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,nc", [([4, 4, 6, 8], 3), ([6, 4, 8], 2), ([8, 6], 1), ([4, 6, 4, 4], 2)])
# the 64 pairs of 1..8 x 1..8: the step's results outgrow the handle's page-locked slots
@pytest.mark.parametrize("pairs", [[(1, 1), (2, 3), (1, 2)], [(2, 2), (3, 1)],
                                   [(l, t) for l in range(1, 9) for t in range(1, 9)]])
@pytest.mark.parametrize("precision,rtol,atol", [("fp64", 1e-12, 1e-14), ("mixed", 0.0, 2e-6)])
def test_cycles_match_single_calls(L, nc, pairs, precision, rtol, atol):
    beta = {1: 1.0, 2: 2.3, 3: 6.0}[nc]
    prop = "exp" if nc == 3 else "reference"
    a = GaugeField(L, nc, precision, "hot", 31)
    b = GaugeField(L, nc, precision, "hot", 31)
    a.set_stream(31, 4)
    b.set_stream(31, 4)
    acc, plaq, w, ms = a.run_cycles(beta, 0.3, 3, 3, prop, 0.3, True, pairs)
    assert ms > 0
    for c in range(3):
        acc1 = b.metropolis(beta, 0.3, 3, 1, prop, 0.3)
        assert acc[c] == acc1[0]
        assert plaq[c] == pytest.approx(b.plaquette(), rel=rtol, abs=atol)
        np.testing.assert_allclose(w[c], b.wilson_loop_temporal(pairs), rtol=rtol, atol=atol)
    np.testing.assert_array_equal(a.download(), b.download())


@pytest.mark.parametrize("precision,rtol,atol", [("fp64", 1e-12, 1e-14), ("mixed", 0.0, 2e-6)])
def test_cycles_loops_without_plaquette_match_single_calls(precision, rtol, atol):
    """Loops measured and the plaquette not: the loop kernels of each cycle run
    beside the next cycle's sweep with nothing else on the second stream."""
    pairs = [(l, t) for l in range(1, 5) for t in range(1, 9)]
    a = GaugeField([4, 6, 4, 8], 3, precision, "hot", 77)
    b = GaugeField([4, 6, 4, 8], 3, precision, "hot", 77)
    a.set_stream(77, 2)
    b.set_stream(77, 2)
    acc, _, w, _ = a.run_cycles(6.0, 0.0, 4, 4, "exp", 0.3, False, pairs)
    for c in range(4):
        assert acc[c] == b.metropolis(6.0, 0.0, 4, 1, "exp", 0.3)[0]
        np.testing.assert_allclose(w[c], b.wilson_loop_temporal(pairs), rtol=rtol, atol=atol)
    np.testing.assert_array_equal(a.download(), b.download())


@pytest.mark.parametrize("L,nc,precision", [([8, 8, 8, 8], 1, "fp64"), ([4, 4, 6, 4], 3, "mixed"),
                                            ([6, 4, 8], 2, "fp64"), ([8, 6], 3, "fp64")])
# without planar loops the temporal loop kernel runs beside the following sweeps
@pytest.mark.parametrize("planar", [True, False])
def test_run_metropolis_fused_matches_single_calls(L, nc, precision, planar):
    """klft_run_metropolis (measurements every `interval` sweeps, step 0
    excluded, temporal and planar loops, all enqueued) against the same run
    through the single-call API, measurement by measurement, bit for bit."""
    beta = {1: 2.0, 2: 2.3, 3: 6.0}[nc]
    prop = "exp" if nc == 3 else "reference"
    nd = len(L)
    tp = [(1, 1), (2, 2), (2, 1)]
    planes = ([(0, 1), (1, 0)] + ([(1, 2), (2, 0)] if nd > 2 else [])) if planar else []
    pp = [(1, 1), (2, 2), (2, 1)] if planar else []
    a = GaugeField(L, nc, precision, "hot", 32091)
    b = GaugeField(L, nc, precision, "hot", 32091)
    a.set_stream(32091, 1)
    b.set_stream(32091, 1)
    nsweeps, interval = 23, 5
    acc, plaq, wt, wm, ms = a.run_metropolis_measured(beta, 0.1, 4, nsweeps, interval, prop, 0.25, True, tp, planes,
                                                      pp)
    assert ms > 0 and len(plaq) == (nsweeps - 1) // interval == wt.shape[0] == wm.shape[0]
    m = 0
    for step in range(nsweeps):
        assert acc[step] == b.metropolis(beta, 0.1, 4, 1, prop, 0.25)[0]
        if step % interval == 0 and step != 0:
            assert plaq[m] == b.plaquette()
            np.testing.assert_array_equal(wt[m], b.wilson_loop_temporal(tp))
            for q, (mu, nu) in enumerate(planes):
                np.testing.assert_array_equal(wm[m, q], b.wilson_loop_mu_nu(mu, nu, pp))
            m += 1
    np.testing.assert_array_equal(a.download(), b.download())
    a.close()
    b.close()
