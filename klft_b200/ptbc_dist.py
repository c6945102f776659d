"""PTBC replicas spread over the ranks of a torch.distributed process group.

One process per GPU holds any subset of the replicas.  Per cycle every rank
sweeps its own replicas, computes their defect sums (`klft_ptbc_defect_sums`,
one FP64 pair per replica), the pairs are all-gathered -- the path's only
collective, 24 bytes per replica -- and every rank makes the same swap
decisions on the host (`klft_ptbc_swap_sums`), so the labels stay identical on
all ranks and no link moves.  The reference's PTBC field
(PTBCGaugeField.hpp:30-279) is single-process and never swaps.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch
import torch.distributed as dist

from . import GaugeField, ptbc_swap_sums


def _device(group) -> torch.device:
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_defect_sums(A_local: Sequence[Sequence[float]], ids_local: Sequence[int], nrep: int,
                       group=None) -> np.ndarray:
    """All-gather the (A_1, A_2) pairs of every rank's replicas; returns A[nrep, 2]
    in replica order, the same on every rank.  Each replica must be held by
    exactly one rank."""
    dev = _device(group)
    rows = torch.full((nrep, 3), -1.0, dtype=torch.float64, device=dev)
    for rid, a in zip(ids_local, A_local):
        if not 0 <= int(rid) < nrep:
            raise ValueError(f"replica id {rid} outside [0, {nrep})")
        rows[int(rid)] = torch.tensor([float(rid), float(a[0]), float(a[1])], dtype=torch.float64, device=dev)
    world = dist.get_world_size(group)
    out = [torch.empty_like(rows) for _ in range(world)]
    dist.all_gather(out, rows, group=group)
    A = np.zeros((nrep, 2))
    seen = np.zeros(nrep, dtype=np.int64)
    for t in out:
        t = t.cpu().numpy()
        held = t[:, 0] >= 0
        A[held] = t[held, 1:]
        seen += held
    if not np.all(seen == 1):
        raise ValueError(f"replicas held by no rank or by several: {np.nonzero(seen != 1)[0].tolist()}")
    return A


class DistributedPTBC:
    """The replicas `fields` (global ids `ids`) of this rank in an ensemble of
    len(c_of_label) PTBC replicas over the process group.  Replica r starts with
    label r; `swap(cycle)` runs one round of neighbour-label swaps (the decisions
    of `klft_ptbc_swap` for the whole ensemble) and gives every local replica its
    new label's coefficient."""

    def __init__(self, fields: Sequence[GaugeField], ids: Sequence[int], c_of_label, beta: float, seed: int,
                 group: Optional[dist.ProcessGroup] = None):
        if len(fields) != len(ids):
            raise ValueError("one global id per local field")
        self.fields = list(fields)
        self.ids = [int(i) for i in ids]
        self.c_of_label = np.ascontiguousarray(c_of_label, dtype=np.float64)
        self.nrep = len(self.c_of_label)
        self.beta = float(beta)
        self.seed = int(seed)
        self.group = group
        self.labels = np.arange(self.nrep, dtype=np.int32)
        for f, i in zip(self.fields, self.ids):
            f.set_defect_c(self.c_of_label[self.labels[i]])

    def swap(self, cycle: int):
        """One swap round; returns (label_of_rep, accepted[nrep - 1])."""
        A_local = [f.defect_sums(self.beta) for f in self.fields]
        A = gather_defect_sums(A_local, self.ids, self.nrep, self.group)
        self.labels, acc = ptbc_swap_sums(A, self.c_of_label, self.labels, self.seed, cycle)
        for f, i in zip(self.fields, self.ids):
            f.set_defect_c(self.c_of_label[self.labels[i]])
        return self.labels.copy(), acc
