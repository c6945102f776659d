"""PTBC: defect-weighted sweeps, defect sums and replica swaps.

CPU: the swap's action difference equals the change of the defect-weighted
action (the premise of the swap rule), computed by the oracle.
GPU: sweeps with a defect, defect sums and swap decisions against the oracle.
"""
import numpy as np
import pytest

from oracle.oracle import PROPOSAL_EXP, PROPOSAL_REFERENCE, Lat

DEFECT = [2, 1, 0, 3]  # len, pos1, pos2, pos3


@pytest.mark.parametrize("nc", [1, 2, 3])
def test_weighted_action_decomposes_into_defect_sums(oracle, nc):
    lat = Lat(nc, [4, 4, 4, 4])
    U = oracle.init(lat, True, 3)
    beta = 2.0
    A = oracle.defect_sums(lat, U, DEFECT, beta)
    S1 = oracle.defect_action(lat, U, DEFECT, 1.0, beta)
    for c in (0.0, 0.3, 0.8):
        Sc = oracle.defect_action(lat, U, DEFECT, c, beta)
        assert Sc - S1 == pytest.approx((c - 1) * A[0] + (c * c - 1) * A[1], abs=1e-10)


def test_swap_rule_is_detailed_balance_consistent(oracle):
    # swapping twice with the same uniforms restores labels only when both accepted; the
    # rule must accept every downhill move
    c = np.array([1.0, 0.5, 0.0])
    A = np.array([[-1.0, -0.5], [-3.0, -1.5], [-2.0, -0.1]])
    lab, acc = oracle.ptbc_swap(c, A, [0, 1, 2], 5, 0)
    assert sorted(lab.tolist()) == [0, 1, 2]
    assert acc.shape == (2,)


@pytest.mark.gpu
@pytest.mark.parametrize("nc,proposal", [(2, PROPOSAL_REFERENCE), (3, PROPOSAL_EXP), (1, PROPOSAL_REFERENCE)])
def test_defect_sweep_matches_oracle(oracle, nc, proposal):
    import klft_b200
    lat = Lat(nc, [4, 4, 4, 4])
    U = oracle.init(lat, True, 21)
    g = klft_b200.GaugeField(lat.L, nc, "fp64")
    g.upload(U)
    g.set_defect(DEFECT[0], DEFECT[1:], 0.4)
    g.set_stream(99, 1)
    delta = 0.0 if proposal == PROPOSAL_EXP else 0.3
    acc = g.metropolis(2.5, delta, 4, 3, proposal="exp" if proposal == PROPOSAL_EXP else "reference", eps=0.3)
    acc_o = oracle.metropolis(lat, U, 2.5, delta, 4, 3, 99, chain=1, proposal=proposal, eps=0.3, defect=DEFECT,
                              defect_c=0.4)
    np.testing.assert_array_equal(acc, acc_o)
    np.testing.assert_allclose(g.download(), U, rtol=0, atol=1e-11)
    np.testing.assert_allclose(g.defect_sums(2.5), oracle.defect_sums(lat, U, DEFECT, 2.5), rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_replica_swaps_match_oracle(oracle):
    import klft_b200
    nrep = 5
    c = np.linspace(1.0, 0.0, nrep)
    lat = Lat(2, [4, 4, 4, 4])
    fields, configs = [], []
    for r in range(nrep):
        U = oracle.init(lat, True, 100 + r)
        oracle.metropolis(lat, U, 2.2, 0.3, 3, 2, 100 + r, defect=DEFECT, defect_c=c[r])
        g = klft_b200.GaugeField(lat.L, 2, "fp64")
        g.upload(U)
        g.set_defect(DEFECT[0], DEFECT[1:], c[r])
        fields.append(g)
        configs.append(U)
    labels = np.arange(nrep)
    for cycle in range(3):
        A = np.array([oracle.defect_sums(lat, configs[r], DEFECT, 2.2) for r in range(nrep)])
        lab_o, acc_o = oracle.ptbc_swap(c, A, labels, 7, cycle)
        lab_g, acc_g = klft_b200.ptbc_swap(fields, c, labels, 2.2, 7, cycle)
        np.testing.assert_array_equal(lab_g, lab_o)
        np.testing.assert_array_equal(acc_g, acc_o)
        labels = lab_g
    # each replica now sweeps with its label's coefficient
    for r in range(nrep):
        fields[r].set_stream(500 + r, 0)
        a = fields[r].metropolis(2.2, 0.3, 2, 1)
        a_o = oracle.metropolis(lat, configs[r], 2.2, 0.3, 2, 1, 500 + r, defect=DEFECT, defect_c=c[labels[r]])
        np.testing.assert_array_equal(a, a_o)
