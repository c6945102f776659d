"""Job server over device-resident lattices (klft_server_* in include/klft_b200.h).

The reference runs one simulation per process (Metropolis.hpp:113-223,
HMC.hpp:20-117).  Here a server on one GPU admits jobs as they arrive, keeps
their lattices resident, advances all running Metropolis jobs together in
multi-chain sweep launches and runs HMC jobs beside them on their own streams.
A job's result depends only on its description, so it is the same alone and
in any mix of other jobs.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from ._lib import JOB_MAX_WILSON, Job, JobResult, KlftError, ServerStats, check, lib

KIND = {"metropolis": 0, "hmc": 1}
_PREC = {"fp64": 0, "mixed": 1}
_START = {"cold": 0, "hot": 1}
_PROP = {"reference": 0, "exp": 1}
_INTEG = {"reference": 0, "leapfrog": 1, "omelyan": 2}


@dataclass
class JobSpec:
    """One simulation job: lattice, update algorithm, measurements of the final configuration."""
    kind: str = "metropolis"
    nc: int = 2
    extents: Tuple[int, ...] = (8, 8, 8, 8)
    beta: float = 2.3
    precision: str = "mixed"
    start: str = "cold"
    seed: int = 1234
    chain: int = 0
    # Metropolis
    nsweeps: int = 100
    nhits: int = 10
    proposal: str = "reference"
    delta: float = 0.3
    eps: float = 0.25
    # HMC
    ntraj: int = 10
    nsteps: int = 20
    tau: float = 1.0
    integrator: str = "leapfrog"
    # measurements
    plaquette: bool = True
    wilson_pairs: Sequence[Tuple[int, int]] = field(default_factory=list)

    def to_c(self) -> Job:
        j = Job()
        j.kind = KIND[self.kind]
        j.nc = self.nc
        j.ndims = len(self.extents)
        for d in range(4):
            j.L[d] = self.extents[d] if d < len(self.extents) else 1
        j.precision = _PREC[self.precision]
        j.start = _START[self.start]
        j.seed = self.seed
        j.chain = self.chain
        j.beta = self.beta
        j.nsweeps = self.nsweeps
        j.nhits = self.nhits
        j.proposal = _PROP[self.proposal]
        j.delta = self.delta
        j.eps = self.eps
        j.ntraj = self.ntraj
        j.nsteps = self.nsteps
        j.tau = self.tau
        j.integrator = _INTEG[self.integrator]
        j.measure_plaquette = int(self.plaquette)
        pairs = list(self.wilson_pairs)
        if len(pairs) > JOB_MAX_WILSON:
            raise ValueError(f"at most {JOB_MAX_WILSON} Wilson loop pairs per job")
        j.n_wilson = len(pairs)
        for k, (l, t) in enumerate(pairs):
            j.wilson_pairs[2 * k] = l
            j.wilson_pairs[2 * k + 1] = t
        return j

    @property
    def volume(self) -> int:
        return int(np.prod(self.extents))

    @property
    def link_updates(self) -> int:
        links = self.volume * len(self.extents)
        if self.kind == "metropolis":
            return links * self.nsweeps
        per = {"reference": self.nsteps + 1, "leapfrog": self.nsteps, "omelyan": 2 * self.nsteps}[self.integrator]
        return links * self.ntraj * per


def footprint(job: JobSpec) -> int:
    """Device bytes the job holds while admitted (klft_job_footprint)."""
    b = C.c_uint64()
    j = job.to_c()
    check(lib().klft_job_footprint(C.byref(j), C.byref(b)))
    return b.value


def _result(r: JobResult, nw: int) -> Dict:
    return {
        "id": r.id, "status": r.status, "kind": "metropolis" if r.kind == 0 else "hmc",
        "plaquette": r.plaquette, "wilson": [r.wilson[k] for k in range(nw)],
        "acceptance": r.acceptance, "mean_exp_mdH": r.mean_exp_mdH, "mean_dH": r.mean_dH,
        "link_updates": r.link_updates, "t_submit": r.t_submit, "t_admit": r.t_admit,
        "t_finish": r.t_finish, "latency": r.t_finish - r.t_submit, "error": r.error.decode(errors="replace"),
    }


class Server:
    """A job server on one GPU with a device-memory budget for the admitted jobs."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, max_active: int = 0, max_queued: int = 0):
        h = C.c_void_p()
        check(lib().klft_server_create(device, budget_bytes, max_active, max_queued, C.byref(h)))
        self._h = h
        self._nw: Dict[int, int] = {}

    def submit(self, job: JobSpec) -> int:
        j = job.to_c()
        jid = C.c_uint64()
        check(lib().klft_server_submit(self._h, C.byref(j), C.byref(jid)))
        self._nw[jid.value] = j.n_wilson
        return jid.value

    def cancel(self, job_id: int) -> None:
        check(lib().klft_server_cancel(self._h, job_id))

    def poll(self, max_results: int = 64, timeout_ms: int = 0) -> List[Dict]:
        buf = (JobResult * max_results)()
        n = C.c_int()
        check(lib().klft_server_poll(self._h, buf, max_results, timeout_ms, C.byref(n)))
        return [_result(buf[i], self._nw.pop(buf[i].id, 0)) for i in range(n.value)]

    def wait(self, ids: Sequence[int], timeout_s: float = 600.0) -> Dict[int, Dict]:
        """Poll until every id in ids has a result; returns {id: result}."""
        import time
        want = set(ids)
        out: Dict[int, Dict] = {}
        t_end = time.monotonic() + timeout_s
        while want - set(out):
            if time.monotonic() > t_end:
                raise TimeoutError(f"jobs {sorted(want - set(out))} did not finish in {timeout_s} s")
            for r in self.poll(64, 100):
                out[r["id"]] = r
        return out

    def stats(self) -> Dict:
        s = ServerStats()
        check(lib().klft_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def inject_fault(self, what: int = 1) -> None:
        check(lib().klft_server_inject_fault(self._h, what))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().klft_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ synthetic job streams
BETA_RANGE = {1: (0.9, 1.1), 2: (2.2, 2.6), 3: (5.7, 6.2)}
WILSON_CHOICES = [(1, 1), (1, 2), (2, 1), (2, 2), (2, 4), (4, 2), (3, 3), (4, 4)]


def poisson_jobs(n: int, rate: float, seed: int, extent_range: Tuple[int, int] = (8, 32),
                 sweeps: Tuple[int, int] = (50, 500), trajectories: Tuple[int, int] = (10, 50),
                 precision: str = "mixed") -> List[Tuple[float, JobSpec]]:
    """n jobs with Poisson arrival times (mean rate jobs/s), from one seed.

    Group uniform over U(1), SU(2), SU(3); 3 or 4 dims; every extent uniform over
    the even numbers in extent_range; beta uniform in the group's usual range;
    Metropolis (sweeps, nHits = 10; the exp(i eps H) proposal for SU(3)) or HMC
    (trajectories, tau = 1, 20 leapfrog steps) with equal odds; the plaquette
    and a random subset of temporal Wilson loops measured at the end."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    evens = np.arange(extent_range[0], extent_range[1] + 1, 2)
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        nc = int(rng.integers(1, 4))
        nd = int(rng.integers(3, 5))
        ext = tuple(int(x) for x in rng.choice(evens, size=nd))
        lo, hi = BETA_RANGE[nc]
        beta = float(rng.uniform(lo, hi))
        kind = "metropolis" if rng.random() < 0.5 else "hmc"
        nw = int(rng.integers(0, 4))
        pairs = [WILSON_CHOICES[k] for k in sorted(rng.choice(len(WILSON_CHOICES), size=nw, replace=False))]
        job = JobSpec(kind=kind, nc=nc, extents=ext, beta=beta, precision=precision,
                      start="hot" if rng.random() < 0.5 else "cold", seed=int(rng.integers(1, 2**62)), chain=i,
                      plaquette=bool(rng.random() < 0.75) or nw == 0, wilson_pairs=pairs)
        if kind == "metropolis":
            job.nsweeps = int(rng.integers(sweeps[0], sweeps[1] + 1))
            job.nhits = 10
            job.proposal = "exp" if nc == 3 else "reference"
            job.delta = 0.3
            job.eps = 0.25
        else:
            job.ntraj = int(rng.integers(trajectories[0], trajectories[1] + 1))
            job.nsteps = 20
            job.tau = 1.0
            job.integrator = "leapfrog"
        out.append((t, job))
    return out


def run_stream(server: Server, jobs: List[Tuple[float, JobSpec]], timeout_s: float = 600.0) -> Dict:
    """Submit each job at its arrival time (seconds after the call) and collect
    every result.  Returns {"results": {id: result}, "ids": [...], "wall_s": ...}."""
    import time
    t0 = time.monotonic()
    ids = []
    results: Dict[int, Dict] = {}
    for t_arr, job in jobs:
        while True:
            now = time.monotonic() - t0
            if now >= t_arr:
                break
            for r in server.poll(64, max(0, min(20, int((t_arr - now) * 1000)))):
                results[r["id"]] = r
        ids.append(server.submit(job))
    rest = server.wait([i for i in ids if i not in results], timeout_s)
    results.update(rest)
    return {"results": results, "ids": ids, "wall_s": time.monotonic() - t0}


def latency_summary(results: Sequence[Dict]) -> Dict:
    lat = np.array([r["latency"] for r in results if r["status"] == 0])
    ok = [r for r in results if r["status"] == 0]
    if len(ok) == 0:
        return {"jobs": 0}
    t_first = min(r["t_submit"] for r in ok)
    t_last = max(r["t_finish"] for r in ok)
    lu = sum(r["link_updates"] for r in ok)
    return {
        "jobs": len(ok),
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
        "mean_s": float(lat.mean()),
        "max_s": float(lat.max()),
        "makespan_s": t_last - t_first,
        "link_updates": int(lu),
        "link_updates_per_s": lu / (t_last - t_first) if t_last > t_first else math.nan,
    }
