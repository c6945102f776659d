"""PTBC replicas over several ranks, host side: the swap decisions from gathered
defect sums (klft_ptbc_swap_sums) against the oracle, and the all-gather of
klft_b200.ptbc_dist on two gloo ranks giving every rank the labels a single
process computes."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SPLIT = {0: [0, 2, 3], 1: [1, 4]}  # replica ids held by each rank
NREP, NCYC, SEED = 5, 6, 4242


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def sums(cycle):
    """Defect sums of the five replicas at one cycle: magnitudes like a 16^4 SU(3) defect."""
    rng = np.random.default_rng(1000 + cycle)
    return np.stack([rng.normal(-30.0, 0.8, NREP), rng.normal(-1.2, 0.3, NREP)], axis=1)


def test_swap_sums_follow_the_oracle(oracle):
    import klft_b200
    c = np.linspace(1.0, 0.0, NREP)
    lab_k = lab_o = np.arange(NREP)
    nacc = 0
    for cyc in range(40):
        A = sums(cyc)
        lab_k, acc_k = klft_b200.ptbc_swap_sums(A, c, lab_k, SEED, cyc)
        lab_o, acc_o = oracle.ptbc_swap(c, A, lab_o, SEED, cyc)
        np.testing.assert_array_equal(lab_k, lab_o)
        np.testing.assert_array_equal(acc_k, acc_o)
        nacc += int(acc_k.sum())
        assert sorted(lab_k) == list(range(NREP))
    assert 0 < nacc < 40 * (NREP - 1)  # both outcomes occur


def test_swap_sums_reject_bad_labels():
    import klft_b200
    with pytest.raises(klft_b200.KlftError, match="EINVAL"):
        klft_b200.ptbc_swap_sums(sums(0), np.linspace(1, 0, NREP), [0, 0, 1, 2, 3], SEED, 0)


SPLITS = {"even": SPLIT, "empty_rank": {0: [0, 1, 2, 3, 4], 1: []}}


def _rank(rank, world, port, q, dup, split_name="even"):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import klft_b200
    from klft_b200.ptbc_dist import gather_defect_sums
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ids = [0] if dup else SPLITS[split_name][rank]
        c = np.linspace(1.0, 0.0, NREP)
        lab = np.arange(NREP)
        seq = []
        for cyc in range(NCYC):
            A_all = sums(cyc)
            A = gather_defect_sums([A_all[i] for i in ids], ids, NREP)
            lab, acc = klft_b200.ptbc_swap_sums(A, c, lab, SEED, cyc)
            seq.append((lab.tolist(), acc.tolist(), A.tolist()))
        q.put((rank, "ok", seq))
    except ValueError as e:
        q.put((rank, "ValueError", str(e)))
    finally:
        dist.destroy_process_group()


def _run(dup, split_name="even"):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q, dup, split_name)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    return sorted(q.get(timeout=10) for _ in range(2))


@pytest.mark.parametrize("split_name", ["even", "empty_rank"])
def test_gathered_swaps_agree_on_every_rank(split_name):
    import klft_b200
    got = _run(False, split_name)
    assert [g[1] for g in got] == ["ok", "ok"]
    assert got[0][2] == got[1][2]
    c = np.linspace(1.0, 0.0, NREP)
    lab = np.arange(NREP)
    for cyc, (lab_r, acc_r, A_r) in enumerate(got[0][2]):
        np.testing.assert_array_equal(A_r, sums(cyc))
        lab, acc = klft_b200.ptbc_swap_sums(sums(cyc), c, lab, SEED, cyc)
        assert lab_r == lab.tolist() and acc_r == acc.tolist()


def test_replica_held_twice_is_an_error_on_every_rank():
    got = _run(True)
    assert [g[1] for g in got] == ["ValueError", "ValueError"]
