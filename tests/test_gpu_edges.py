"""Edge cases across subsystems: batches of more than one chain table, open
boundaries inside a batch, serving jobs of every form, tiles that do not divide
the lattice, compact-storage checkpoints."""
import numpy as np
import pytest

from klft_b200 import Batch, GaugeField
from klft_b200.serve import JobSpec, Server
from oracle.oracle import Lat

pytestmark = pytest.mark.gpu


def make(L, nc, prec, seed, chain, start="hot"):
    g = GaugeField(L, nc, prec, start, seed)
    g.set_stream(seed, chain)
    return g


def test_batch_with_many_tables_and_open_boundary():
    """70 chains of one group (two 64-chain tables) plus an open-boundary chain."""
    specs = [([4, 4, 4, 4] if k % 2 else [4, 6, 4, 4], 2, "mixed", 2.3, 0.3, 2) for k in range(70)]
    b = Batch()
    batch, solo = [], []
    for k, (L, nc, prec, beta, delta, nh) in enumerate(specs):
        gb, gs = make(L, nc, prec, 500 + k, k), make(L, nc, prec, 500 + k, k)
        b.add(gb, beta, delta, nh)
        batch.append((gb, beta, delta, nh))
        solo.append(gs)
    ob, os_ = make([4, 4, 4, 6], 3, "fp64", 9, 1), make([4, 4, 4, 6], 3, "fp64", 9, 1)
    ob.set_open_boundary(3)
    os_.set_open_boundary(3)
    b.add(ob, 6.0, 0.0, 3, "exp", 0.3)
    acc, plaq, _, _ = b.run(2, True, True)
    for k, (gb, beta, delta, nh) in enumerate(batch):
        a = solo[k].metropolis(beta, delta, nh, 2)
        np.testing.assert_array_equal(acc[:, k], a)
        np.testing.assert_array_equal(gb.download(), solo[k].download())
    a = os_.metropolis(6.0, 0.0, 3, 2, "exp", 0.3)
    np.testing.assert_array_equal(acc[:, 70], a)
    np.testing.assert_array_equal(ob.download(), os_.download())
    assert plaq[-1, 70] == os_.plaquette()


def test_serving_jobs_of_every_form():
    jobs = [
        JobSpec(kind="metropolis", nc=3, extents=(6, 4, 4, 4), precision="fp64", proposal="reference", delta=0.2,
                nsweeps=5, nhits=3, seed=1, wilson_pairs=[(1, 1), (2, 2)]),
        JobSpec(kind="metropolis", nc=2, extents=(8, 6), precision="mixed", nsweeps=7, nhits=4, seed=2,
                wilson_pairs=[(3, 2)]),
        JobSpec(kind="metropolis", nc=1, extents=(6, 4), precision="fp64", nsweeps=3, seed=3),
        JobSpec(kind="hmc", nc=3, extents=(4, 4, 6), precision="fp64", ntraj=2, nsteps=8, integrator="reference",
                seed=4, wilson_pairs=[(1, 2)]),
        JobSpec(kind="hmc", nc=1, extents=(8, 8), precision="mixed", ntraj=3, nsteps=10, integrator="omelyan",
                seed=5),
        JobSpec(kind="metropolis", nc=2, extents=(4, 4, 4, 4), nsweeps=0, seed=6),
        JobSpec(kind="hmc", nc=2, extents=(4, 4, 4, 4), ntraj=0, seed=7),
    ]
    with Server() as s:
        ids = [s.submit(j) for j in jobs]
        res = s.wait(ids, 120)
    for j, jid in zip(jobs, ids):
        r = res[jid]
        assert r["status"] == 0, r["error"]
        g = make(list(j.extents), j.nc, j.precision, j.seed, j.chain, j.start)
        if j.kind == "metropolis":
            acc = g.metropolis(j.beta, j.delta, j.nhits, j.nsweeps, j.proposal, j.eps) if j.nsweeps else []
            if j.nsweeps:
                np.testing.assert_allclose(r["acceptance"], np.mean(acc), rtol=1e-12)
        else:
            if j.ntraj:
                dH, acc = g.hmc(j.beta, j.tau, j.nsteps, j.ntraj, j.integrator)
                np.testing.assert_allclose(r["mean_dH"], np.mean(dH), rtol=1e-12, atol=1e-300)
        assert r["plaquette"] == g.plaquette()
        if j.wilson_pairs:
            np.testing.assert_allclose(r["wilson"], g.wilson_loop_temporal(j.wilson_pairs), rtol=1e-13, atol=0)


@pytest.mark.parametrize("precision,rtol,atol", [("fp64", 1e-12, 1e-14), ("mixed", 0.0, 2e-6)])
def test_wilson_tiles_not_dividing_the_axis(oracle, precision, rtol, atol):
    """L_nu = 36: a 32-row tile plus a partial one; loops up to T = 10 and L = 9."""
    L = [4, 6, 4, 36]
    lat = Lat(3, L)
    U = oracle.init(lat, True, 5)
    g = GaugeField(L, 3, precision)
    g.upload(U)
    pairs = [(l, t) for l in (1, 3, 9) for t in (1, 4, 8, 10)]
    np.testing.assert_allclose(g.wilson_loop_temporal(pairs), oracle.wilson_temporal(lat, U, pairs), rtol=rtol,
                               atol=atol)


def test_compact_su2_checkpoint(tmp_path):
    g = make([4, 4, 6, 4], 2, "mixed", 12, 3)
    g.metropolis(2.3, 0.3, 3, 2)
    p = str(tmp_path / "su2.ckpt")
    g.save(p)
    r = GaugeField.load(p)
    np.testing.assert_array_equal(r.download(), g.download())
    np.testing.assert_array_equal(r.metropolis(2.3, 0.3, 3, 2), g.metropolis(2.3, 0.3, 3, 2))
    assert r.plaquette() == g.plaquette()
