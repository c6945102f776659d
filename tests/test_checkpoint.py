"""Checkpoint files: the host-side format checks need no GPU."""
import os

import numpy as np
import pytest

from klft_b200 import GaugeField, KlftError
from klft_b200 import checkpoint_io as cio

from conftest import has_gpu


def sample(nc=2, L=(4, 4, 2, 2), prec=1):
    rng = np.random.default_rng(3)
    V = int(np.prod(L))
    links = rng.normal(size=(V, len(L), nc, nc)) + 1j * rng.normal(size=(V, len(L), nc, nc))
    return cio.Checkpoint(nc=nc, L=list(L), precision=prec, seed=11, chain=4, counters=(7, 2, 1), open_mu=2,
                          defect_len=2, defect_pos=(1, 0, 1), defect_c=0.25, links=links)


def test_roundtrip_of_the_python_writer(tmp_path):
    ck = sample()
    p = str(tmp_path / "a.ckpt")
    cio.write(p, ck)
    assert os.path.getsize(p) == cio.HEADER + ck.links.nbytes
    back = cio.read(p)
    np.testing.assert_array_equal(back.links, ck.links)
    assert (back.nc, back.L, back.precision, back.seed, back.chain, back.counters) == \
        (ck.nc, ck.L, ck.precision, ck.seed, ck.chain, ck.counters)
    assert (back.defect_len, back.defect_pos, back.defect_c) == (2, (1, 0, 1), 0.25)
    assert back.open_mu == 2


def corrupt(data: bytes, off: int) -> bytes:
    b = bytearray(data)
    b[off] ^= 0x5A
    return bytes(b)


@pytest.mark.parametrize("case,msg", [
    ("magic", "not a checkpoint"),
    ("header", "header checksum"),
    ("payload", "payload checksum"),
    ("truncated", "truncated payload"),
    ("short", "short header"),
])
def test_library_rejects_bad_files_before_device_work(tmp_path, case, msg):
    data = cio.to_bytes(sample())
    if case == "magic":
        data = corrupt(data, 0)
    elif case == "header":
        data = corrupt(data, 30)
    elif case == "payload":
        data = corrupt(data, cio.HEADER + 100)
    elif case == "truncated":
        data = data[:-8]
    elif case == "short":
        data = data[:64]
    p = str(tmp_path / "bad.ckpt")
    with open(p, "wb") as f:
        f.write(data)
    with pytest.raises(KlftError, match=msg):
        GaugeField.load(p)
    with pytest.raises(ValueError):
        cio.read(p)


def test_missing_file(tmp_path):
    with pytest.raises(KlftError, match="EINVAL"):
        GaugeField.load(str(tmp_path / "nope.ckpt"))


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_valid_file_needs_a_device(tmp_path):
    p = str(tmp_path / "ok.ckpt")
    cio.write(p, sample())
    with pytest.raises(KlftError, match="ECUDA"):
        GaugeField.load(p)
