"""Checkpoint / resume on the GPU: a restored lattice continues bit for bit."""
import numpy as np
import pytest

from klft_b200 import GaugeField
from klft_b200 import checkpoint_io as cio

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nc,L,prec,prop", [(3, (4, 4, 4, 6), "mixed", "exp"), (2, (6, 4, 4, 4), "fp64", "reference"),
                                            (1, (4, 6, 8), "mixed", "reference")])
def test_metropolis_resume_is_exact(tmp_path, nc, L, prec, prop):
    beta = {1: 1.0, 2: 2.3, 3: 6.0}[nc]
    ref = GaugeField(L, nc, prec, "hot", 5)
    ref.set_stream(5, 3)
    ref.set_defect(2, (1, 0, 1), 0.5)
    a_ref = ref.metropolis(beta, 0.3, 4, 7, prop, 0.3)
    g = GaugeField(L, nc, prec, "hot", 5)
    g.set_stream(5, 3)
    g.set_defect(2, (1, 0, 1), 0.5)
    a1 = g.metropolis(beta, 0.3, 4, 3, prop, 0.3)
    p = str(tmp_path / "c.ckpt")
    g.save(p)
    g.close()
    r = GaugeField.load(p)
    assert (r.nc, r.L, r.precision) == (nc, list(L), prec)
    assert r.counters() == (3, 0)
    a2 = r.metropolis(beta, 0.3, 4, 4, prop, 0.3)
    np.testing.assert_array_equal(np.concatenate([a1, a2]), a_ref)
    np.testing.assert_array_equal(r.download(), ref.download())
    assert r.plaquette() == ref.plaquette()
    # the file is readable on the host and holds what download() gives
    ck = cio.read(p)
    assert ck.counters[0] == 3 and ck.seed == 5 and ck.chain == 3 and ck.defect_len == 2
    assert ck.links.shape == (int(np.prod(L)), len(L), nc, nc)


def test_hmc_resume_is_exact(tmp_path):
    ref = GaugeField((4, 4, 4, 4), 2, "mixed", "hot", 8)
    ref.set_stream(8, 1)
    dh_ref, acc_ref = ref.hmc(2.3, 1.0, 10, 4, "omelyan")
    g = GaugeField((4, 4, 4, 4), 2, "mixed", "hot", 8)
    g.set_stream(8, 1)
    dh1, acc1 = g.hmc(2.3, 1.0, 10, 2, "omelyan")
    p = str(tmp_path / "h.ckpt")
    g.save(p)
    r = GaugeField.load(p)
    assert r.counters() == (0, 2)
    dh2, acc2 = r.hmc(2.3, 1.0, 10, 2, "omelyan")
    np.testing.assert_array_equal(np.concatenate([dh1, dh2]), dh_ref)
    np.testing.assert_array_equal(r.download(), ref.download())


def test_host_written_checkpoint_loads(tmp_path):
    g = GaugeField((4, 4, 4, 4), 3, "fp64", "hot", 21)
    U = g.download()
    ck = cio.Checkpoint(nc=3, L=[4, 4, 4, 4], precision=0, seed=21, chain=0, counters=(5, 0, 0), links=U)
    p = str(tmp_path / "host.ckpt")
    cio.write(p, ck)
    r = GaugeField.load(p)
    np.testing.assert_array_equal(r.download(), U)
    assert r.counters() == (5, 0)
