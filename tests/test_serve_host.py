"""Host-side serving logic that needs no GPU: job streams, footprints, validation, summaries."""
import numpy as np
import pytest

from klft_b200 import KlftError
from klft_b200.serve import JobSpec, Server, footprint, latency_summary, poisson_jobs

from conftest import has_gpu


def test_poisson_stream_is_seeded_and_in_range():
    a = poisson_jobs(400, 20.0, seed=5)
    b = poisson_jobs(400, 20.0, seed=5)
    assert [(t, j) for t, j in a] == [(t, j) for t, j in b]
    t = np.array([x for x, _ in a])
    assert np.all(np.diff(t) > 0)
    rate = len(t) / t[-1]
    assert 16.0 < rate < 24.0
    groups = np.array([j.nc for _, j in a])
    for nc in (1, 2, 3):
        assert 0.25 < np.mean(groups == nc) < 0.42
    for _, j in a:
        assert len(j.extents) in (3, 4)
        assert all(8 <= x <= 32 and x % 2 == 0 for x in j.extents)
        lo, hi = {1: (0.9, 1.1), 2: (2.2, 2.6), 3: (5.7, 6.2)}[j.nc]
        assert lo <= j.beta <= hi
        if j.kind == "metropolis":
            assert 50 <= j.nsweeps <= 500
            assert j.proposal == ("exp" if j.nc == 3 else "reference")
        else:
            assert 10 <= j.ntraj <= 50
        assert len(j.wilson_pairs) <= 3
        assert j.plaquette or j.wilson_pairs
    assert poisson_jobs(10, 20.0, seed=6) != poisson_jobs(10, 20.0, seed=5)


def test_footprint_counts_what_a_job_holds():
    m = JobSpec(kind="metropolis", nc=3, extents=(16, 16, 16, 16), precision="mixed", plaquette=True)
    links = 16 ** 4 * 4 * 6 * 8  # mixed-form SU(3) links keep two rows (12 reals)
    fm = footprint(m)
    assert links < fm < links + (1 << 20)
    h = JobSpec(kind="hmc", nc=3, extents=(16, 16, 16, 16), precision="mixed", ntraj=10)
    # HMC keeps momenta (8 reals per link) and a saved copy of the links
    assert footprint(h) - fm >= links + 16 ** 4 * 4 * 8 * 4
    w = JobSpec(kind="metropolis", nc=3, extents=(16, 16, 16, 16), precision="mixed", wilson_pairs=[(2, 2)])
    assert footprint(w) > fm
    d = JobSpec(kind="metropolis", nc=3, extents=(16, 16, 16, 16), precision="fp64")
    assert footprint(d) > 16 ** 4 * 4 * 9 * 16


@pytest.mark.parametrize("bad", [
    dict(extents=(8, 7, 8, 8)),
    dict(extents=(8,)),
    dict(nc=4),
    dict(kind="hmc", nsteps=0),
    dict(nsweeps=-1),
    dict(nc=3, proposal="reference", delta=0.0),
    dict(beta=float("nan")),
    dict(wilson_pairs=[(-1, 2)]),
])
def test_malformed_jobs_are_rejected(bad):
    with pytest.raises(KlftError, match="EINVAL"):
        footprint(JobSpec(**bad))


def test_too_many_wilson_pairs():
    with pytest.raises(ValueError):
        JobSpec(wilson_pairs=[(1, 1)] * 17).to_c()


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_server_needs_a_device():
    with pytest.raises(KlftError, match="ECUDA"):
        Server()


def test_latency_summary():
    res = [{"status": 0, "latency": x, "t_submit": i * 0.1, "t_finish": i * 0.1 + x, "link_updates": 1000}
           for i, x in enumerate(np.linspace(0.1, 1.0, 100))]
    res.append({"status": 6, "latency": 50.0, "t_submit": 0.0, "t_finish": 50.0, "link_updates": 0})
    s = latency_summary(res)
    assert s["jobs"] == 100
    assert abs(s["p50_s"] - 0.55) < 1e-9
    assert s["p99_s"] < 1.0 + 1e-9
    assert s["link_updates"] == 100000
