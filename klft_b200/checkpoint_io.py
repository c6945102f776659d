"""Host-side reader and writer of klft_b200 checkpoint files (no GPU needed).

The format is the one klft_checkpoint_write produces (include/klft_b200.h):
a 128-byte little-endian header followed by the links in the host interchange
layout, complex128 (V, Nd, Nc, Nc) with site = x0 + L0 (x1 + L1 (x2 + L2 x3)).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

MAGIC = b"KLFTCKPT"
VERSION = 1
HEADER = 128
_FMT = "<8sII" + "7i" + "5i" + "QQ" + "4I" + "d" + "Q" + "Q"  # up to byte 120; then the header checksum
# the fourth u32 after the stream (byte 92) is the open-boundary direction + 1 (0: periodic)


def fnv1a64(data: bytes) -> int:
    """FNV-1a, 64-bit (Fowler/Noll/Vo), over raw bytes (sequential; meant for small files)."""
    h = 1469598103934665603
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


@dataclass
class Checkpoint:
    nc: int
    L: List[int]
    precision: int  # 0 = FP64, 1 = mixed
    seed: int
    chain: int
    counters: Tuple[int, int, int] = (0, 0, 0)
    open_mu: int = -1
    defect_len: int = 0
    defect_pos: Tuple[int, int, int] = (0, 0, 0)
    defect_c: float = 1.0
    links: np.ndarray = field(default=None)  # complex128 (V, Nd, Nc, Nc)

    @property
    def nd(self) -> int:
        return len(self.L)


def to_bytes(ck: Checkpoint) -> bytes:
    nd = ck.nd
    L4 = list(ck.L) + [1] * (4 - nd)
    payload = np.ascontiguousarray(ck.links, dtype=np.complex128).tobytes()
    head = struct.pack(_FMT, MAGIC, VERSION, HEADER, ck.nc, nd, *L4, ck.precision,
                       1 if ck.defect_len > 0 else 0, ck.defect_len, *ck.defect_pos, ck.seed, ck.chain,
                       *ck.counters, ck.open_mu + 1, ck.defect_c, len(payload), fnv1a64(payload))
    assert len(head) == 120
    head += struct.pack("<Q", fnv1a64(head))
    return head + payload


def write(path: str, ck: Checkpoint) -> None:
    with open(path, "wb") as f:
        f.write(to_bytes(ck))


def read(path: str) -> Checkpoint:
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < HEADER:
        raise ValueError("short header")
    vals = struct.unpack(_FMT, data[:120])
    (magic, ver, hb, nc, nd, l0, l1, l2, l3, prec, dact, dlen, p0, p1, p2, seed, chain, c0, c1, c2, open1, dc,
     nbytes, csum) = vals
    if magic != MAGIC:
        raise ValueError("not a checkpoint")
    if ver != VERSION or hb != HEADER:
        raise ValueError(f"unsupported format version {ver}")
    if struct.unpack("<Q", data[120:128])[0] != fnv1a64(data[:120]):
        raise ValueError("header checksum mismatch")
    payload = data[HEADER:HEADER + nbytes]
    if len(payload) != nbytes:
        raise ValueError("truncated payload")
    if fnv1a64(payload) != csum:
        raise ValueError("payload checksum mismatch")
    L = [l0, l1, l2, l3][:nd]
    V = int(np.prod(L))
    links = np.frombuffer(payload, dtype=np.complex128).reshape(V, nd, nc, nc).copy()
    return Checkpoint(nc=nc, L=L, precision=prec, seed=seed, chain=chain, counters=(c0, c1, c2),
                      open_mu=open1 - 1, defect_len=dlen if dact else 0, defect_pos=(p0, p1, p2), defect_c=dc,
                      links=links)
