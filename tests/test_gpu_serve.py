"""Serving: jobs admitted as they arrive, advanced together, results the same alone and in the mix.

The server has no reference counterpart (the reference runs one simulation per
process, Metropolis.hpp:113-223); the per-job results are checked against the
same job run through the lattice API, which the parity tests tie to the oracle.
"""
import time

import numpy as np
import pytest

from klft_b200 import GaugeField, KlftError
from klft_b200.serve import JobSpec, Server, footprint, latency_summary, poisson_jobs, run_stream

pytestmark = pytest.mark.gpu

FIELDS = ("plaquette", "wilson", "acceptance", "mean_exp_mdH", "mean_dH", "link_updates")


def small_stream(n, seed, rate=400.0):
    return poisson_jobs(n, rate, seed, extent_range=(4, 10), sweeps=(4, 24), trajectories=(2, 5))


def assert_same(a, b):
    assert a["status"] == 0 and b["status"] == 0, (a["error"], b["error"])
    for f in FIELDS:
        np.testing.assert_array_equal(np.asarray(a[f], dtype=float), np.asarray(b[f], dtype=float), err_msg=f)


def overlap(results):
    """Largest number of jobs admitted at the same time."""
    ev = sorted([(r["t_admit"], 1) for r in results] + [(r["t_finish"], -1) for r in results])
    cur = best = 0
    for _, d in ev:
        cur += d
        best = max(best, cur)
    return best


def test_results_same_alone_and_in_the_mix():
    jobs = small_stream(16, seed=11)
    with Server() as s:
        alone = []
        for _, j in jobs:
            jid = s.submit(j)
            alone.append(s.wait([jid], 120)[jid])
    # all at once
    with Server() as s:
        ids = [s.submit(j) for _, j in jobs]
        mix = s.wait(ids, 120)
        st = s.stats()
    for k, jid in enumerate(ids):
        assert_same(alone[k], mix[jid])
    assert overlap(list(mix.values())) > 1
    assert st["completed"] == len(jobs) and st["failed"] == 0 and st["active"] == 0 and st["bytes_in_use"] == 0
    # arriving while others run (Poisson arrivals at 400 jobs/s)
    with Server() as s:
        out = run_stream(s, jobs, 120)
    for k, jid in enumerate(out["ids"]):
        assert_same(alone[k], out["results"][jid])
    summ = latency_summary(list(out["results"].values()))
    assert summ["jobs"] == len(jobs) and summ["p99_s"] >= summ["p50_s"] > 0


@pytest.mark.parametrize("nc,ext,prop", [(1, (6, 4, 8), "reference"), (2, (4, 6, 4, 8), "reference"),
                                         (3, (4, 4, 6, 4), "exp")])
def test_metropolis_job_matches_lattice_api(nc, ext, prop):
    pairs = [(1, 1), (2, 3)]
    job = JobSpec(kind="metropolis", nc=nc, extents=ext, beta={1: 1.0, 2: 2.3, 3: 6.0}[nc], start="hot", seed=77,
                  chain=5, nsweeps=9, nhits=4, proposal=prop, delta=0.4, eps=0.3, wilson_pairs=pairs)
    with Server() as s:
        jid = s.submit(job)
        r = s.wait([jid], 60)[jid]
    assert r["status"] == 0, r["error"]
    g = GaugeField(ext, nc, "mixed", "hot", 77)
    g.set_stream(77, 5)
    acc = g.metropolis(job.beta, job.delta, job.nhits, job.nsweeps, prop, job.eps)
    assert r["plaquette"] == g.plaquette()
    np.testing.assert_allclose(r["wilson"], g.wilson_loop_temporal(pairs), rtol=1e-13, atol=0)
    np.testing.assert_allclose(r["acceptance"], np.mean(acc), rtol=1e-12)
    assert r["link_updates"] == job.link_updates
    assert np.isnan(r["mean_exp_mdH"])


@pytest.mark.parametrize("nc,integ", [(1, "leapfrog"), (2, "omelyan"), (3, "reference")])
def test_hmc_job_matches_lattice_api(nc, integ):
    ext = (4, 4, 4, 6)
    job = JobSpec(kind="hmc", nc=nc, extents=ext, beta={1: 1.0, 2: 2.3, 3: 6.0}[nc], start="hot", seed=91,
                  chain=2, ntraj=4, nsteps=10, tau=1.0, integrator=integ, wilson_pairs=[(1, 2)])
    with Server() as s:
        jid = s.submit(job)
        r = s.wait([jid], 60)[jid]
    assert r["status"] == 0, r["error"]
    g = GaugeField(ext, nc, "mixed", "hot", 91)
    g.set_stream(91, 2)
    dH, acc = g.hmc(job.beta, job.tau, job.nsteps, job.ntraj, integ)
    assert r["plaquette"] == g.plaquette()
    np.testing.assert_allclose(r["wilson"], g.wilson_loop_temporal([(1, 2)]), rtol=1e-13, atol=0)
    assert r["acceptance"] == np.mean(acc != 0)
    np.testing.assert_allclose(r["mean_exp_mdH"], np.mean(np.exp(-dH)), rtol=1e-12)
    np.testing.assert_allclose(r["mean_dH"], np.mean(dH), rtol=1e-12, atol=1e-300)


def test_admission_by_footprint_serialises_jobs():
    jobs = [JobSpec(kind="metropolis", nc=2, extents=(8, 8, 8, 8), seed=s, nsweeps=20) for s in (1, 2, 3)]
    fp = footprint(jobs[0])
    with Server(budget_bytes=fp + 1024) as s:
        ids = [s.submit(j) for j in jobs]
        res = s.wait(ids, 60)
    rs = [res[i] for i in ids]
    assert all(r["status"] == 0 for r in rs)
    for a, b in zip(rs, rs[1:]):
        assert b["t_admit"] >= a["t_finish"]


def wait_active(s, n, timeout=30.0):
    t_end = time.monotonic() + timeout
    while s.stats()["active"] < n:
        assert time.monotonic() < t_end
        time.sleep(0.005)


def test_rejections_and_cancellation():
    long_m = JobSpec(kind="metropolis", nc=3, extents=(16, 16, 16, 16), proposal="exp", nsweeps=200000, seed=3)
    with Server(budget_bytes=footprint(long_m) + 4096, max_queued=1) as s:
        bad = JobSpec(extents=(8, 7, 8, 8))
        with pytest.raises(KlftError, match="EINVAL"):
            s.submit(bad)
        with pytest.raises(KlftError, match="ENOMEM"):
            s.submit(JobSpec(nc=3, extents=(32, 32, 32, 32)))
        a = s.submit(long_m)
        wait_active(s, 1)
        b = s.submit(JobSpec(nsweeps=5, seed=4))  # waits: the budget is held by a
        with pytest.raises(KlftError, match="EBUSY"):
            s.submit(JobSpec(nsweeps=5, seed=5))
        s.cancel(b)
        s.cancel(a)
        with pytest.raises(KlftError, match="EINVAL"):
            s.cancel(987654)
        res = s.wait([a, b], 60)
        assert res[a]["status"] == 6 and res[b]["status"] == 6  # KLFT_ECANCELED
        st = s.stats()
        assert st["cancelled"] == 2 and st["rejected"] == 3 and st["active"] == 0 and st["bytes_in_use"] == 0
        # the server keeps serving
        c = s.submit(JobSpec(nsweeps=3, seed=6))
        assert s.wait([c], 60)[c]["status"] == 0


def test_cancel_running_hmc_job():
    job = JobSpec(kind="hmc", nc=2, extents=(12, 12, 12, 12), ntraj=100000, nsteps=10, seed=8)
    with Server() as s:
        a = s.submit(job)
        wait_active(s, 1)
        time.sleep(0.05)
        s.cancel(a)
        r = s.wait([a], 60)[a]
        assert r["status"] == 6


def test_worker_fault_fails_running_jobs_and_recovers():
    job = JobSpec(kind="metropolis", nc=2, extents=(16, 16, 16, 16), nsweeps=100000, seed=9)
    with Server() as s:
        a = s.submit(job)
        wait_active(s, 1)
        s.inject_fault(1)
        r = s.wait([a], 60)[a]
        assert r["status"] == 7 and "injected" in r["error"]  # KLFT_EINTERNAL
        jobs = small_stream(4, seed=12)
        ids = [s.submit(j) for _, j in jobs]
        res = s.wait(ids, 60)
        assert all(res[i]["status"] == 0 for i in ids)
        assert s.stats()["failed"] == 1
