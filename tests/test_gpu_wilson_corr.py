"""Column-correlation Wilson-loop kernel (every T in 1..8, FP32 and FP64
links) against the oracle: colour groups, tiles that do not divide the nu
axis, short axes, loops that wrap the lattice along mu, partial T lists, and
the tables that stay on the entry-per-origin kernel (T > 8, repeated pairs)."""
import numpy as np
import pytest

from klft_b200 import GaugeField
from oracle.oracle import Lat

pytestmark = pytest.mark.gpu

ATOL = 2e-6  # FP32 links: per-site traces in FP32, sums in FP64
TOL = {"mixed": dict(rtol=0, atol=ATOL), "fp64": dict(rtol=1e-12, atol=1e-14)}


def field(oracle, nc, L, seed, precision="mixed"):
    lat = Lat(nc, L)
    U = oracle.init(lat, True, seed)
    g = GaugeField(L, nc, precision)
    g.upload(U)
    return lat, U, g


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("nc", [1, 2, 3])
@pytest.mark.parametrize("L", [[4, 4, 4, 4], [6, 4, 2, 10], [4, 6, 4, 36], [6, 4, 20], [10, 6], [4, 2, 2, 70]])
def test_temporal_loops_match_oracle(oracle, nc, L, precision):
    lat, U, g = field(oracle, nc, L, 31 + nc, precision)
    pairs = [(l, t) for l in range(1, 10) for t in range(1, 9)]
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs),
                               **TOL[precision])
    g.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("nc", [2, 3])
def test_partial_t_lists_and_other_planes(oracle, nc, precision):
    L = [6, 4, 8, 12]
    lat, U, g = field(oracle, nc, L, 41, precision)
    tol = TOL[precision]
    pairs = [(3, 2), (1, 5), (7, 1), (2, 8), (5, 3)]  # tmax 8 with gaps; L in any order
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs), **tol)
    short = [(2, 1), (4, 3), (1, 2)]  # tmax 3
    np.testing.assert_allclose(g.wilson_loop_temporal(short), oracle.wilson_temporal(lat, U, short), **tol)
    for mu, nu in [(3, 0), (0, 2), (2, 1)]:
        np.testing.assert_allclose(g.wilson_loop_mu_nu(mu, nu, pairs), oracle.wilson_mu_nu(lat, U, mu, nu, pairs),
                                   **tol)
    g.close()


def test_tables_outside_the_correlation_form_agree(oracle):
    """T = 9 and a repeated pair keep the entry-per-origin kernel; the shared
    pairs agree with the correlation kernel to FP32 rounding."""
    L = [4, 4, 6, 16]
    lat, U, g = field(oracle, 3, L, 43)
    base = [(l, t) for l in (1, 2, 5) for t in (1, 4, 8)]
    w_corr = g.wilson_loop_temporal(base)
    w_long = g.wilson_loop_temporal(base + [(2, 9)])
    w_dup = g.wilson_loop_temporal(base + [(2, 4)])
    np.testing.assert_allclose(w_long[:-1], w_corr, rtol=0, atol=1e-6)
    np.testing.assert_allclose(w_dup[:-1], w_corr, rtol=0, atol=1e-6)
    np.testing.assert_allclose(w_dup[-1], w_dup[base.index((2, 4))], rtol=1e-12, atol=0)
    ref = oracle.wilson_temporal(lat, U, base + [(2, 9)])
    np.testing.assert_allclose(w_long, ref, rtol=0, atol=ATOL)
    g.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_largest_pair_table_over_three_planes(oracle, precision):
    """128 pairs (L up to 16, past the lattice) over the three spatial planes in
    one launch: the largest per-CTA accumulator block (128 x 3 sums)."""
    L = [6, 4, 4, 10]
    lat, U, g = field(oracle, 3, L, 47, precision)
    pairs = [(l, t) for l in range(1, 17) for t in range(1, 9)]
    assert len(pairs) == 128
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs),
                               **TOL[precision])
    g.close()
