"""Open boundaries (the intent of GaugeField.hpp:168-185 openBC<mu>): links across
the last slice of one direction are zero and never updated."""
import numpy as np
import pytest

from klft_b200 import GaugeField
from oracle.oracle import PROPOSAL_EXP, Lat

pytestmark = pytest.mark.gpu


def boundary(U, L, mu):
    """Links U_mu at x_mu = L_mu - 1 (host layout (V, Nd, Nc, Nc), x0 fastest)."""
    V = int(np.prod(L))
    x = np.arange(V)
    for d in range(mu):
        x //= L[d]
    xm = x % L[mu]
    return U[xm == L[mu] - 1, mu]


@pytest.fixture
def open_oracle(oracle):
    yield oracle
    oracle.set_open_boundary(-1)


@pytest.mark.parametrize("nc,L,mu,prop", [(1, [4, 6, 4, 4], 3, 0), (2, [4, 4, 6, 4], 1, 0), (3, [4, 4, 4, 6], 3, 0),
                                          (3, [4, 4, 6, 4], 0, PROPOSAL_EXP), (2, [6, 4, 4], 2, 0)])
def test_open_boundary_sweeps_match_oracle(open_oracle, nc, L, mu, prop):
    oracle = open_oracle
    lat = Lat(nc, L)
    g = GaugeField(L, nc, "fp64", "hot", 17)
    g.set_open_boundary(mu)
    U = g.download()
    assert np.all(boundary(U, L, mu) == 0)
    oracle.set_open_boundary(mu)
    g.set_stream(17, 2)
    pname = "exp" if prop == PROPOSAL_EXP else "reference"
    acc = g.metropolis(6.0 if nc == 3 else 2.3, 0.3, 3, 2, pname, 0.3)
    acc_o = oracle.metropolis(lat, U, 6.0 if nc == 3 else 2.3, 0.3, 3, 2, 17, chain=2, proposal=prop, eps=0.3)
    np.testing.assert_array_equal(acc, acc_o)
    U2 = g.download()
    np.testing.assert_allclose(U2, U, rtol=0, atol=1e-11)
    assert np.all(boundary(U2, L, mu) == 0)
    # observables through the zero links: plaquette and (gauge-fixed) Wilson loops
    assert g.plaquette() == pytest.approx(oracle.plaquette(lat, U2), rel=1e-12, abs=1e-14)
    pairs = [(1, 1), (2, 3), (1, L[-1] + 1)]
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U2, pairs),
                               rtol=1e-12, atol=1e-14)
    assert g.unitarity() < 1e-12


def test_open_boundary_hmc_and_mixed():
    L = [4, 4, 4, 6]
    g = GaugeField(L, 3, "mixed", "hot", 3)
    g.set_open_boundary(3)
    dH, acc = g.hmc(6.0, 1.0, 20, 3, "omelyan")
    assert np.all(np.isfinite(dH))
    U = g.download()
    assert np.all(boundary(U, L, 3) == 0)
    assert g.unitarity() < 1e-5
    g.metropolis(6.0, 0.0, 4, 2, "exp", 0.3)
    assert np.all(boundary(g.download(), L, 3) == 0)
    # uploads re-zero the boundary
    g.upload(np.broadcast_to(np.eye(3, dtype=complex), U.shape).copy())
    assert np.all(boundary(g.download(), L, 3) == 0)


def test_open_boundary_arguments_and_checkpoint(tmp_path):
    from klft_b200 import KlftError
    g = GaugeField([4, 4, 4, 4], 2, "fp64", "hot", 1)
    with pytest.raises(KlftError, match="EINVAL"):
        g.set_open_boundary(4)
    g.set_open_boundary(2)
    with pytest.raises(KlftError, match="EINVAL"):
        g.set_open_boundary(-1)
    with pytest.raises(KlftError, match="already open"):
        g.set_open_boundary(1)
    p = str(tmp_path / "o.ckpt")
    g.metropolis(2.3, 0.3, 2, 1)
    g.save(p)
    r = GaugeField.load(p)
    a = g.metropolis(2.3, 0.3, 2, 2)
    b = r.metropolis(2.3, 0.3, 2, 2)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(r.download(), g.download())
