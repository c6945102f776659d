"""PTBC replicas spread over processes (klft_b200.ptbc_dist): two ranks on one
GPU, gloo for the all-gather (two NCCL ranks cannot share a GPU), each sweeping
its own replicas, give the labels and links of the same ensemble run in one
process with klft_ptbc_swap.  A one-rank NCCL group covers the device-tensor
all-gather."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NREP, NCYC, BETA, SEED = 4, 4, 5.8, 77
SPLIT = {0: [0, 3], 1: [1, 2]}
L = [4, 4, 4, 4]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def replica(r):
    import klft_b200
    g = klft_b200.GaugeField(L, 3, "mixed", "hot", 500 + r)
    g.set_stream(500 + r, r)
    g.set_defect(2, (1, 0, 2), 1.0)
    return g


def _rank(rank, world, port, q, backend, split):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from klft_b200.ptbc_dist import DistributedPTBC
    if backend == "nccl":
        torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ids = split[rank]
        fields = [replica(r) for r in ids]
        ens = DistributedPTBC(fields, ids, np.linspace(1.0, 0.0, NREP), BETA, SEED)
        seq = []
        for cyc in range(NCYC):
            for f in fields:
                f.metropolis(BETA, 0.0, 3, 1, "exp", 0.3)
            lab, acc = ens.swap(cyc)
            seq.append(lab.tolist())
        q.put((rank, seq, {r: f.download() for r, f in zip(ids, fields)}))
    finally:
        dist.destroy_process_group()


def _run(world, backend, split):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q, backend, split)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    return sorted(out, key=lambda t: t[0])


def single_process():
    import klft_b200
    reps = [replica(r) for r in range(NREP)]
    c = np.linspace(1.0, 0.0, NREP)
    for r in range(NREP):
        reps[r].set_defect_c(c[r])
    lab = np.arange(NREP)
    seq = []
    for cyc in range(NCYC):
        for g in reps:
            g.metropolis(BETA, 0.0, 3, 1, "exp", 0.3)
        lab, _ = klft_b200.ptbc_swap(reps, c, lab, BETA, SEED, cyc)
        seq.append(lab.tolist())
    return seq, {r: g.download() for r, g in enumerate(reps)}


@pytest.mark.parametrize("world,backend,split", [(2, "gloo", SPLIT), (1, "nccl", {0: [0, 1, 2, 3]})])
def test_distributed_replicas_match_one_process(world, backend, split):
    seq, links = single_process()
    got = _run(world, backend, split)
    for rank, seq_r, links_r in got:
        assert seq_r == seq
        for r, a in links_r.items():
            np.testing.assert_array_equal(a, links[r])
