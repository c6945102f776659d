#!/usr/bin/env python
"""Update-and-measure throughput of SU(3) 32^4 Metropolis on B200.

Workload (one step = one cycle of run_metropolis, Metropolis.hpp:204-218):
one Metropolis sweep of SU(3) 32^4 (beta = 6, nHits = 10, proposals
X = exp(i eps H), eps tuned to ~50% acceptance during 200 thermalisation
sweeps from a cold start), then GaugePlaquette and WilsonLoop_temporal for all
(L, T) in 1..8 (64 pairs, averaged over the 3 spatial directions).

Metric: link updates/s (a link update = one link visited by the sweep, Nd*V per
step), for the mixed form (FP32 links, FP64 reductions; `value`) and the plain
FP64 form (`fp64`).  Inputs are synthetic (seeded cold start).

At N = 1 the same line also carries the other workloads: `batched_ptbc` (12
PTBC SU(3) 16^4 replicas + 48 SU(2) chains per captured cycle), `hmc` (SU(2)
24^4, 500 trajectories, mixed vs FP64), `serving` (a seeded Poisson stream of
mixed jobs at 20 jobs/s through the job server: p50/p99 latency and aggregate
link updates/s) and `plaquettes_per_s`.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica (the path does
not shard); `value` sums the ranks' link updates over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L_DEFAULT = 32
BETA, NHITS = 6.0, 10
PAIRS = [(l, t) for l in range(1, 9) for t in range(1, 9)]
METRIC = "Link updates/s (SU(3) 32^4), mixed vs FP64 form; serving p50/p99 job latency"
REF_WARMUP_S, REF_TIMED_S = 30.0, 120.0  # time bounds of the reference arm (host cycles of seconds each)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=L_DEFAULT)
    ap.add_argument("--therm", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-PTBC, HMC and serving legs (they run at N=1 only)")
    ap.add_argument("--batch-cycles", type=int, default=40)
    ap.add_argument("--hmc-traj", type=int, default=500)
    ap.add_argument("--serve-jobs", type=int, default=100)
    ap.add_argument("--serve-rate", type=float, default=20.0)
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
class Dist:
    """One process per GPU (torchrun env).  NCCL carries only the barrier and the
    max-over-ranks timing; KLFT_DIST_BACKEND=gloo runs the same steps on CPU."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = os.environ.get("KLFT_DIST_BACKEND", "nccl")
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if self.backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def set_device(self):
        if self.world > 1:
            import klft_b200
            klft_b200.set_device(self.local)

    def barrier(self):
        if self.pg:
            import torch
            if self.backend == "nccl":
                self.pg.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int = 0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # start the timed region only once the sampler is running; keep only
            # the samples taken inside it
            t_end = time.monotonic() + 3.0
            while not self.rows and time.monotonic() < t_end and self.proc.poll() is None:
                time.sleep(0.005)
            self.rows.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ our arm
def thermalise(g, nsweeps: int, eps0: float = 0.25):
    """Cold start -> nsweeps sweeps, tuning eps towards 50% acceptance (then frozen)."""
    eps = eps0
    done = 0
    while done < nsweeps:
        n = min(20, nsweeps - done)
        acc = g.metropolis(BETA, 0.0, NHITS, n, proposal="exp", eps=eps)
        a = float(acc[-1])
        if a > 0.55:
            eps *= 1.15
        elif a < 0.45:
            eps /= 1.15
        done += n
    return eps


def time_cycles(g, eps, steps, warmup, clocks=None):
    g.run_cycles(BETA, 0.0, NHITS, warmup, "exp", eps, True, PAIRS)
    if clocks:
        with clocks:
            acc, plaq, w, ms = g.run_cycles(BETA, 0.0, NHITS, steps, "exp", eps, True, PAIRS)
    else:
        acc, plaq, w, ms = g.run_cycles(BETA, 0.0, NHITS, steps, "exp", eps, True, PAIRS)
    return acc, plaq, w, ms


def kernel_split(g, eps, reps=3):
    """Device time of the sweep alone and of the measurement alone (ms per cycle)."""
    _, _, _, ms_sweep = g.run_cycles(BETA, 0.0, NHITS, reps, "exp", eps, False, [])
    _, _, _, ms_all = g.run_cycles(BETA, 0.0, NHITS, reps, "exp", eps, True, PAIRS)
    return ms_sweep / reps, max(ms_all - ms_sweep, 0.0) / reps


def e2e_public_api(g, eps, steps, per_call=False):
    """Per step through the public API with host buffers: one klft_run_cycles
    call (sweep, plaquette, W_temp; the pair list goes up and the step's
    acceptance, plaquette and loops come back to the host), or with per_call
    the three single calls sweep, plaquette, W_temp (each a host round trip)."""
    pairs = np.array(PAIRS, dtype=np.int32)
    t0 = time.perf_counter()
    for _ in range(steps):
        if per_call:
            g.metropolis(BETA, 0.0, NHITS, 1, proposal="exp", eps=eps)
            g.plaquette()
            g.wilson_loop_temporal(pairs)
        else:
            g.run_cycles(BETA, 0.0, NHITS, 1, "exp", eps, True, pairs)
    dt = time.perf_counter() - t0
    if per_call:
        h2d = pairs.nbytes * 3  # the pair list goes up once per spatial direction
        d2h = 8 + 8 + 8 * len(PAIRS) * 3
    else:
        # up: the pair list (kernel parameters); down: one copy of the step's
        # accept count, plaquette sum and the loop sums of the 3 spatial planes
        h2d = pairs.nbytes
        d2h = 8 + 8 + 8 * len(PAIRS) * 3
    return dt, h2d, d2h


def host_buffer(shape, pinned):
    """A complex128 host array: page-locked (through torch) or ordinary numpy."""
    if pinned:
        import torch
        n = int(np.prod(shape))
        return torch.empty(n, dtype=torch.complex128, pin_memory=True).numpy().reshape(shape)
    a = np.empty(shape, dtype=np.complex128)
    a.fill(0)  # touch the pages before timing
    return a


def e2e_host_lattice(g, eps, steps, pinned=False):
    """Per step: upload links from host, cycle, download links (users keeping
    configurations on the host), with one reused host buffer."""
    U = host_buffer(g.shape(), pinned)
    g.download(U)
    g.upload(U)  # warm-up: staging buffers and pages
    t0 = time.perf_counter()
    for _ in range(steps):
        g.upload(U)
        g.run_cycles(BETA, 0.0, NHITS, 1, "exp", eps, True, PAIRS)
        g.download(U)
    dt = time.perf_counter() - t0
    return dt, U.nbytes, U.nbytes


def host_io_rates(g, reps=3):
    """klft_lattice_upload / klft_lattice_download rates (GB/s of the FP64
    interchange array), from ordinary and from page-locked host memory."""
    out = {"bytes": int(np.prod(g.shape())) * 16}
    for pinned in (False, True):
        U = host_buffer(g.shape(), pinned)
        g.download(U)
        g.upload(U)
        up, down = [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            g.upload(U)
            t1 = time.perf_counter()
            g.download(U)
            t2 = time.perf_counter()
            up.append(t1 - t0)
            down.append(t2 - t1)
        key = "pinned" if pinned else "pageable"
        out[f"upload_gbs_{key}"] = out["bytes"] / min(up) / 1e9
        out[f"download_gbs_{key}"] = out["bytes"] / min(down) / 1e9
    return out


def peak(dtype):
    import ctypes
    from klft_b200._lib import lib
    v = ctypes.c_double()
    return v.value if lib().klft_peak_flops(dtype, ctypes.byref(v)) == 0 else None


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def cpu_baseline_reference(L: int):
    """klft's own code (oracle/_ref shim) on the host cores: one cycle of the same workload."""
    from oracle.oracle import REF_SO, Lat, RefShim
    if not os.path.exists(REF_SO):
        return None
    r = RefShim()
    cores = r.set_threads(os.cpu_count() or 1)
    lat = Lat(3, [L] * 4)
    U = lat.field()
    U[:, :, 0, 0] = U[:, :, 1, 1] = U[:, :, 2, 2] = 1.0
    t0 = time.perf_counter()
    r.cycles(lat, U, BETA, 0.1, NHITS, 1, 1234, PAIRS)
    dt = time.perf_counter() - t0
    t0 = time.perf_counter()
    r.plaquette(lat, U)
    dtp = time.perf_counter() - t0
    return {"value": lat.V * 4 / dt, "unit": "link updates/s", "cores": cores, "kind": "reference",
            "sample": f"1 cycle of SU(3) {L}^4 (sweep + plaquette + 64 temporal Wilson loops), klft's headers on "
                      f"the project's Kokkos-API OpenMP shim, reference SU(3) proposal, {cores} threads, "
                      f"{dt:.2f} s",
            "plaquettes_per_s": lat.V * 6 / dtp,
            "note": "klft's code and this library share the cycle's structure, but klft's SU(3) proposal is its "
                    "Gram-Schmidt generator (an exp(i eps H) proposal does not exist there) and this cycle starts "
                    "cold, not from the GPU arm's thermalised configuration"}


# DRAM traffic of one link pass (dram__bytes_read.sum + dram__bytes_write.sum of one
# metropolis_exp_kernel launch in the ncu capture summarised in the profile below).
TRAFFIC_PASS_BYTES = 204658944 + 19519744
TRAFFIC_SOURCE = "profiles/metropolis_exp_su3_32x4_mixed.md"


def sweep_flops_per_link_update(nhits: int, acceptance: float) -> float:
    """Flops of one SU(3) exp(i eps H) link update of the mixed form as the
    kernel forms it (6 per complex multiply, 2 per complex add, 198 per 3x3
    product, 132 for two rows of one, 42 to complete a third row from the first
    two; an FMA counts 2): the two-row staple 2574 (per forward term: B's third
    row 42, C B on two rows 132 and completed 42, A (C B)^+ on two rows 132 and
    completed 42, the sum 18; per backward term the same with D's and G's third
    rows), M0 = U0 S 240, per hit the proposal (8 Box-Muller normals 32, the
    Gell-Mann coefficients 8, c1 and c0 = det Q 47, the 12-term coefficient
    series 99, Q^2 from the coefficients 35, X = f0 + f1 Q + f2 Q^2 with its
    hermitian pairs 75) and Re Tr(X A M0) 36, the product X A on every hit but
    the first (A is the identity there) 198; then the link A U0 240 and one
    reunitarisation (~100).  The accept rate does not enter: the one product
    per hit is also the accepted A."""
    del acceptance
    proposal = 32 + 8 + 47 + 99 + 35 + 75
    return 2574 + 240 + nhits * (proposal + 36) + (nhits - 1) * 198 + 240 + 100


def mixed_errors(g, L):
    """Error of the mixed form per observable: the final mixed-form configuration
    evaluated by both forms on identical links (its FP32 values are exact in FP64),
    plus the unitarity drift max ||U^+ U - 1|| of the mixed links."""
    import klft_b200
    U = g.download()
    g64 = klft_b200.GaugeField(L, 3, "fp64", "cold", 0)
    g64.upload(U)
    p32, p64 = g.plaquette(), g64.plaquette()
    w32, w64 = g.wilson_loop_temporal(PAIRS), g64.wilson_loop_temporal(PAIRS)
    out = {"plaquette_abs": abs(p32 - p64), "wilson_temporal_max_abs": float(np.max(np.abs(w32 - w64))),
           "wilson_temporal_max_rel": float(np.max(np.abs(w32 - w64) / np.abs(w64))),
           "unitarity_mixed": g.unitarity(),
           "note": "same configuration, FP32 link arithmetic vs FP64; sums in FP64 in both"}
    g64.close()
    return out


def plaquette_ms(g, eps, reps=5):
    """Device time of one GaugePlaquette (ms) from cycles with and without it."""
    _, _, _, ms_sweep = g.run_cycles(BETA, 0.0, NHITS, reps, "exp", eps, False, [])
    _, _, _, ms_plaq = g.run_cycles(BETA, 0.0, NHITS, reps, "exp", eps, True, [])
    return max(ms_plaq - ms_sweep, 1e-6) / reps


def bench_batched_ptbc(cycles: int, warmup: int = 3):
    """12 PTBC replicas of SU(3) 16^4 (4^3 defect, c_r = 1 - r/11, beta = 6) plus
    48 SU(2) chains with extents drawn from {8,12,16,20,24}^4 and beta in
    [2.2, 2.6]: one sweep of every chain, replica swaps, every chain's
    plaquette per cycle, one captured graph per cycle; FP32 links, FP64 sums."""
    import klft_b200
    rng = np.random.default_rng(2718)
    b = klft_b200.Batch()
    fields = []
    links = 0
    for r in range(12):
        g = klft_b200.GaugeField([16] * 4, 3, "mixed", "hot", 5000 + r)
        g.set_stream(5000, r)
        g.set_defect(4, (0, 0, 0), 1.0)
        b.add(g, 6.0, 0.0, NHITS, "exp", 0.25)
        fields.append(g)
        links += 4 * 16 ** 4
    c_of_label = [1.0 - r / 11.0 for r in range(12)]
    b.set_ptbc(list(range(12)), c_of_label, 6.0, 99)
    su2_beta = []
    for k in range(48):
        L = [int(x) for x in rng.choice([8, 12, 16, 20, 24], size=4)]
        g = klft_b200.GaugeField(L, 2, "mixed", "hot", 7000 + k)
        g.set_stream(7000, k)
        su2_beta.append(float(rng.uniform(2.2, 2.6)))
        b.add(g, su2_beta[-1], 0.3, NHITS, "reference", 0.0)
        fields.append(g)
        links += 4 * int(np.prod(L))
    b.run(warmup, True, True)
    acc, plaq, lab, ms = b.run(cycles, True, True)
    _, _, _, ms_ng = b.run(max(cycles // 4, 2), True, False)
    swaps = b.swap_stats()
    # the two groups alone (their launches overlap on forked streams in the full cycle)
    parts = {}
    for name, sel in (("replicas_only", fields[:12]), ("su2_chains_only", fields[12:])):
        bp = klft_b200.Batch()
        for k, g in enumerate(sel):
            if name == "replicas_only":
                bp.add(g, 6.0, 0.0, NHITS, "exp", 0.25)
            else:
                bp.add(g, su2_beta[k], 0.3, NHITS, "reference", 0.0)
        bp.run(2, True, True)
        _, _, _, msp = bp.run(max(cycles // 4, 4), True, True)
        parts[name] = msp / max(cycles // 4, 4)
        bp.close()
    out = {"workload": "12 PTBC SU(3) 16^4 replicas (L_d=4, c_r=1-r/11, beta=6) + 48 SU(2) chains "
                       "extents {8..24}^4, beta U[2.2,2.6]; per cycle 1 sweep + swaps + plaquettes, CUDA graph",
           "chains": len(fields), "cycles": cycles, "ms_per_cycle": ms / cycles,
           "ms_per_cycle_without_graph": ms_ng / max(cycles // 4, 2),
           "ms_per_cycle_groups_alone": parts,
           "link_updates_per_s": links * cycles / (ms * 1e-3),
           "cycles_per_s": cycles / (ms * 1e-3),
           "replica_acceptance": float(np.mean(acc[:, :12])), "su2_acceptance": float(np.mean(acc[:, 12:])),
           "swaps_accepted_per_pair": [int(x) for x in swaps]}
    b.close()
    for g in fields:
        g.close()
    return out


def bench_hmc(ntraj: int, cpu: bool = True):
    """SU(2) 24^4 HMC, beta = 2.3, tau = 1, 20 steps, hot start, mixed vs FP64.

    as_given: klft's Pauli generators and the 20-step leapfrog, the workload as
    stated; its effective step is twice that of the t_a/2 normalisation and at
    this volume it accepts almost nothing.  accepting: t_a/2 generators and the
    20-step Omelyan integrator from the same kind of hot start, thermalised by
    HMC itself (100 trajectories), then ntraj measured trajectories with the
    acceptance, <exp(-dH)> with its standard error, <dH> and the mean
    plaquette.  cpu_oracle: one as-given trajectory of the FP64 oracle on the
    host threads (OpenMP force and updates)."""
    import klft_b200
    out = {"workload": f"SU(2) 4D 24^4 HMC beta=2.3 tau=1 20 steps, {ntraj} trajectories from a hot start"}

    def run(prec, generators, integrator, ntherm, seed):
        g = klft_b200.GaugeField([24] * 4, 2, prec, "hot", seed)
        g.set_stream(seed, 0)
        g.set_hmc_generators(generators)
        g.hmc(2.3, 1.0, 20, max(ntherm, 2), integrator)  # warm-up / thermalisation, same stream continues
        dHs, accs, plaqs = [], [], []
        t_dev = 0.0
        nblk = 5
        for b in range(nblk):
            n = ntraj // nblk + (1 if b < ntraj % nblk else 0)
            t0 = time.perf_counter()
            dH, acc = g.hmc(2.3, 1.0, 20, n, integrator)
            t_dev += time.perf_counter() - t0
            dHs.append(dH)
            accs.append(acc)
            plaqs.append(g.plaquette())
        dH = np.concatenate(dHs)
        acc = np.concatenate(accs)
        # <exp(-dH)> and <dH> over the second half (the first trajectories of the
        # as-given chain start far from equilibrium with dH of either sign in the
        # hundreds)
        h = dH[ntraj // 2:]
        e = np.exp(-h)
        r = {"trajectories_per_s": ntraj / t_dev, "ms_per_trajectory": t_dev * 1e3 / ntraj,
             "acceptance": float(np.mean(acc != 0)),
             "acceptance_last_half": float(np.mean(acc[ntraj // 2:] != 0)),
             "mean_exp_mdH_last_half": float(np.mean(e)),
             "mean_exp_mdH_last_half_err": float(np.std(e, ddof=1) / np.sqrt(len(e))),
             "mean_dH_last_half": float(np.mean(h)), "mean_plaquette": float(np.mean(plaqs)),
             "final_plaquette": plaqs[-1], "unitarity": g.unitarity()}
        g.close()
        return r

    def hbm(r, integrator, prec):
        # algorithmic bytes of one trajectory: each force update reads U and P and
        # writes P, each gauge update reads U and P and writes U, plus momenta,
        # two energy evaluations (U and P read), the saved copy of U
        n = 24 ** 4 * 4
        ub = n * (16 if prec == "mixed" else 64)
        pb = n * 3 * (4 if prec == "mixed" else 8)
        nf, nu = (3 * 20, 2 * 20) if integrator == "omelyan" else (21, 20)
        byt = nf * (ub + 2 * pb) + nu * (2 * ub + pb) + pb + 2 * (ub + pb) + 2 * ub
        gbs = byt * r["trajectories_per_s"] / 1e9
        pk = measured_peaks().get("hbm_gbs")
        r["hbm"] = {"algorithmic_bytes_per_trajectory": byt, "achieved_gbs": gbs,
                    "frac": gbs / pk if pk else None,
                    "note": "links and momenta (37 MB mixed) stay in the 126 MB L2 between kernels"}

    out["as_given"] = {"generators": "reference (Pauli)", "integrator": "leapfrog, 20 steps"}
    out["accepting"] = {"generators": "half (t_a/2)", "integrator": "omelyan, 20 steps", "thermalisation": 100}
    for prec in ("mixed", "fp64"):
        out["as_given"][prec] = run(prec, "reference", "leapfrog", 2, 4242)
        out["accepting"][prec] = run(prec, "half", "omelyan", 100, 4343)
        hbm(out["as_given"][prec], "leapfrog", prec)
        hbm(out["accepting"][prec], "omelyan", prec)
    for k in ("as_given", "accepting"):
        out[k]["speedup_mixed_vs_fp64"] = (out[k]["mixed"]["trajectories_per_s"] /
                                           out[k]["fp64"]["trajectories_per_s"])
    if cpu:
        from oracle.oracle import INTEGRATOR_LEAPFROG, Lat, Oracle
        o = Oracle()
        lat = Lat(2, [24] * 4)
        U = o.init(lat, True, 4242)
        t0 = time.perf_counter()
        o.hmc(lat, U, 2.3, 1.0, 20, INTEGRATOR_LEAPFROG, 4242, 0, 0, 1)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"trajectories_per_s": 1.0 / dt, "kind": "port", "cores": os.cpu_count(),
                             "sample": "1 as-given FP64 trajectory of the oracle (SU(2) 24^4, 20 leapfrog steps)"}
    return out


C1_TEMPORAL = [(2, 2), (3, 4), (4, 3), (4, 4)]
C1_PLANES = [(0, 1), (1, 2), (3, 2)]
C1_PLANAR = [(2, 2), (3, 3), (4, 3)]


def bench_c1(cpu: bool = True):
    """The small plain-method workload: U(1) 4D 8^4, hot start (phases uniform in
    [-pi, pi) from seed 32091), Metropolis beta 2, delta 0.1, nHits 10, 1000
    sweeps, plaquette and the listed temporal and planar Wilson loops every 10
    sweeps (step 0 excluded).  The GPU runs the FP64 form through the public
    API (wall clock, host results every measurement); klft's own code runs the
    same chain on the host cores, on one thread and on all of them.  Both
    follow the same random stream, so their final plaquettes agree to
    rounding."""
    import klft_b200
    L = [8, 8, 8, 8]
    V = 8 ** 4
    g = klft_b200.GaugeField(L, 1, "fp64", "hot", 32091)
    U0 = g.download()
    g.set_stream(32091, 0)

    # run_metropolis: sweep `step` then measure when step % 10 == 0 and step != 0,
    # i.e. after sweeps 11, 21, ..., 991 (99 measurements) of 1000
    def run_gpu():
        g.metropolis(2.0, 0.1, 10, 1)
        for _ in range(99):
            g.metropolis(2.0, 0.1, 10, 10)
            g.plaquette()
            g.wilson_loop_temporal(C1_TEMPORAL)
            for m, n in C1_PLANES:
                g.wilson_loop_mu_nu(m, n, C1_PLANAR)
        g.metropolis(2.0, 0.1, 10, 9)

    def run_fused():
        return g.run_metropolis_measured(2.0, 0.1, 10, 1000, 10, "reference", 0.0, True, C1_TEMPORAL, C1_PLANES,
                                         C1_PLANAR)

    run_gpu()  # warm-up on a copy of the chain
    g.upload(U0)
    g.set_counters(0, 0)
    t0 = time.perf_counter()
    run_gpu()
    dt = time.perf_counter() - t0
    p_calls = g.plaquette()
    run_fused()  # warm-up
    g.upload(U0)
    g.set_counters(0, 0)
    t0 = time.perf_counter()
    _, plaq, _, _, dev_ms = run_fused()
    dt_f = time.perf_counter() - t0
    p_fused = g.plaquette()
    out = {"workload": "U(1) 4D 8^4, hot start seed 32091, beta 2, delta 0.1, nHits 10, 1000 sweeps, plaquette + "
                       "W_temp (2,2),(3,4),(4,3),(4,4) + W_mu_nu (0,1),(1,2),(3,2) x (2,2),(3,3),(4,3) every 10",
           "gpu_per_call": {"seconds": dt, "link_updates_per_s": 1000 * V * 4 / dt, "plaquette": p_calls,
                            "path": "GaugeField.metropolis / plaquette / wilson_loop_* per measurement (C ABI), "
                                    "FP64, wall clock"},
           "gpu": {"seconds": dt_f, "device_ms": dev_ms, "link_updates_per_s": 1000 * V * 4 / dt_f,
                   "plaquette": p_fused, "measurements": len(plaq),
                   "path": "klft_run_metropolis (the run_metropolis loop with its 100 measurements enqueued), "
                           "FP64, wall clock"}}
    g.close()
    if cpu:
        from oracle.oracle import REF_SO, Lat, RefShim
        if os.path.exists(REF_SO):
            r = RefShim()
            lat = Lat(1, L)
            for nt in (1, os.cpu_count() or 1):
                cores = r.set_threads(nt)
                U = U0.copy()
                t0 = time.perf_counter()
                r.metropolis(lat, U, 2.0, 0.1, 10, 1, 32091, sweep0=0)
                for k in range(99):
                    r.metropolis(lat, U, 2.0, 0.1, 10, 10, 32091, sweep0=1 + 10 * k)
                    r.plaquette(lat, U)
                    r.wilson_temporal(lat, U, C1_TEMPORAL)
                    for m, n in C1_PLANES:
                        r.wilson_mu_nu(lat, U, m, n, C1_PLANAR)
                r.metropolis(lat, U, 2.0, 0.1, 10, 9, 32091, sweep0=991)
                dt = time.perf_counter() - t0
                out[f"cpu_reference_{cores}_threads"] = {
                    "seconds": dt, "link_updates_per_s": 1000 * V * 4 / dt, "plaquette": r.plaquette(lat, U),
                    "kind": "reference", "cores": cores,
                    "sample": "the whole workload, klft's headers on the project's Kokkos-API OpenMP shim"}
    return out


def bench_serving(njobs: int, rate: float):
    """A seeded Poisson stream of mixed jobs through the job server."""
    from klft_b200.serve import Server, latency_summary, poisson_jobs, run_stream
    jobs = poisson_jobs(njobs, rate, seed=2024)
    with Server() as s:
        out = run_stream(s, jobs, timeout_s=600)
        st = s.stats()
    res = [out["results"][i] for i in out["ids"]]
    summ = latency_summary(res)
    summ.update({
        "workload": f"{njobs} jobs, Poisson arrivals at {rate} jobs/s (seed 2024): U(1)/SU(2)/SU(3), 3-4 dims, "
                    "even extents 8..32, 50-500 Metropolis sweeps or 10-50 HMC trajectories, final plaquette and "
                    "temporal Wilson loops; FP32 links / FP64 sums",
        "offered_rate_jobs_per_s": rate, "failed": sum(1 for r in res if r["status"] != 0),
        "metropolis_p99_s": float(np.percentile([r["latency"] for r in res if r["kind"] == "metropolis"], 99)),
        "hmc_p99_s": float(np.percentile([r["latency"] for r in res if r["kind"] == "hmc"], 99)),
        "queue_wait_p99_s": float(np.percentile([r["t_admit"] - r["t_submit"] for r in res], 99)),
        "server": {k: st[k] for k in ("rounds", "launches", "busy_s", "completed")},
    })
    return summ


def run_ours(a, dist: Dist):
    import klft_b200
    dist.set_device()
    L = [a.L] * 4
    V = a.L ** 4
    links_per_step = 4 * V
    g = klft_b200.GaugeField(L, 3, "mixed", "cold", 1234 + dist.rank)
    g.set_stream(1234, dist.rank)
    eps = thermalise(g, a.therm)
    # mixed form, timed
    dist.barrier()
    clocks = Clocks(dist.local)
    acc, plaq, w, ms = time_cycles(g, eps, a.steps, a.warmup, clocks)
    dist.barrier()
    ms_max = dist.max(ms)
    value = links_per_step * a.steps * dist.world / (ms_max * 1e-3)
    # breakdown and roofline of the dominant kernel
    ms_sweep, ms_meas = kernel_split(g, eps)
    pk = measured_peaks()
    hbm = pk.get("hbm_gbs")
    fp32 = peak(1)
    fp64 = peak(0)
    # read + write one FP32 SU(3) link, stored as two rows (12 reals); a sweep
    # of the exp proposal is 8 link passes of V/2 links each
    bytes_link_mixed = 2 * 6 * 8
    npass = 2 * 4
    pass_ms = ms_sweep / npass
    units_per_launch = V // 2
    achieved = units_per_launch * bytes_link_mixed / (pass_ms * 1e-3) / 1e9
    flop_lu = sweep_flops_per_link_update(NHITS, float(np.mean(acc)))
    tflops = units_per_launch * flop_lu / (pass_ms * 1e-3) / 1e12
    roofline = {"bound": "hbm", "kernel": "metropolis_exp_kernel<4,float,false>", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": (achieved / hbm) if hbm else None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm else "fallback 6650",
                "traffic": TRAFFIC_PASS_BYTES, "traffic_source": TRAFFIC_SOURCE,
                "algorithmic_bytes_per_launch": units_per_launch * bytes_link_mixed,
                "units_per_launch": units_per_launch, "avg_launch_ms": pass_ms,
                "cuda_core": {"achieved_tflops": tflops, "peak_tflops": fp32, "frac": (tflops / fp32) if fp32 else None,
                              "flop_per_link_update": flop_lu,
                              "peak_source": "klft_peak_flops (measured FP32 FMA throughput)",
                              "note": "the binding roof: ~86 flop per algorithmic byte, above the FP32 ridge of ~11"},
                "cuda_core_peak_tflops": {"fp32": fp32, "fp64": fp64}}
    # whole-job end-to-end rates: every rank's steps over the slowest rank's wall clock
    e2e_steps = max(2, a.steps // 2)
    dist.barrier()
    e2e_dt, h2d, d2h = e2e_public_api(g, eps, e2e_steps)
    e2e_dt = dist.max(e2e_dt)
    dist.barrier()
    pc_dt, _, _ = e2e_public_api(g, eps, e2e_steps, per_call=True)
    pc_dt = dist.max(pc_dt)
    e2e = {"value": links_per_step * e2e_steps * dist.world / e2e_dt, "unit": "link updates/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "path": "klft_run_cycles per step (sweep + plaquette + W_temp, results to the host), host wall clock",
           "value_per_call": links_per_step * e2e_steps * dist.world / pc_dt,
           "path_per_call": "klft_metropolis_sweeps + klft_plaquette + klft_wilson_loop_temporal per step"}
    dist.barrier()
    hl_dt, hb, db = e2e_host_lattice(g, eps, 3)
    hl_dt = dist.max(hl_dt)
    dist.barrier()
    hp_dt, _, _ = e2e_host_lattice(g, eps, 3, pinned=True)
    hp_dt = dist.max(hp_dt)
    e2e_host = {"value": links_per_step * 3 * dist.world / hl_dt, "unit": "link updates/s",
                "h2d_bytes_per_step": hb, "d2h_bytes_per_step": db,
                "path": "upload links + cycle + download links per step, one reused ordinary (pageable) host array",
                "pcie_bytes_per_step": 2 * V * 4 * 12 * 4,
                "note": "the host array is klft's FP64 interchange layout; the library rounds / completes links on "
                        "host threads so that only the two stored FP32 rows of each SU(3) link cross PCIe",
                "value_pinned_host": links_per_step * 3 * dist.world / hp_dt,
                "host_io": host_io_rates(g)}
    # FP64 form from the same thermalised configuration
    fp64_line = None
    if not a.no_fp64:
        U = g.download()
        g64 = klft_b200.GaugeField(L, 3, "fp64", "cold", 0)
        g64.upload(U)
        g64.set_stream(1234, dist.rank)
        _, plaq64, _, ms64 = time_cycles(g64, eps, a.steps, a.warmup)
        ms64 = dist.max(ms64)
        s64, m64 = kernel_split(g64, eps, 2)
        fp64_line = {"value": links_per_step * a.steps * dist.world / (ms64 * 1e-3), "ms_per_step": ms64 / a.steps,
                     "ms_sweep": s64, "ms_measure": m64, "mean_plaquette": float(np.mean(plaq64))}
        g64.close()
    mixed_err = mixed_errors(g, L)
    # like for like with the reference arm: klft's own SU(3) proposal (delta 0.1)
    # from a cold start, the same cycle (sweep + plaquette + 64 W_temp), FP64
    # and mixed, on this GPU
    same_chain = {}
    for prec in ("fp64", "mixed"):
        gr = klft_b200.GaugeField(L, 3, prec, "cold", 1234)
        gr.set_stream(1234, dist.rank)
        gr.run_cycles(BETA, 0.1, NHITS, 2, "reference", 0.0, True, PAIRS)
        _, _, _, msr = gr.run_cycles(BETA, 0.1, NHITS, 5, "reference", 0.0, True, PAIRS)
        msr = dist.max(msr)
        same_chain[prec] = {"value": links_per_step * 5 * dist.world / (msr * 1e-3), "ms_per_step": msr / 5}
        gr.close()
    same_chain["note"] = ("klft's SU(3) Gram-Schmidt proposal (SUN.hpp:192-251) and a cold start, the chain the "
                          "reference arm runs; link updates/s, CUDA events")
    # 8 link passes + counter advance + plaquette and its reduction + the axial-gauge
    # transform (once, shared by the spatial planes) + 3 x U' + one loop kernel over
    # the three planes + one reduction of the three planes' loop sums
    launches_per_step = npass + 1 + 2 + 1 + 3 + 1 + 1
    line = {
        "metric": METRIC, "value": value, "unit": "link updates/s", "n_gpus": dist.world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 links / f64 reductions", "data": "synthetic (seeded cold start, "
        f"{a.therm} thermalisation sweeps)",
        "config": {"workload": f"SU(3) 4D {a.L}^4 Metropolis beta=6 nHits=10 exp(i eps H) proposals "
                               f"(eps={eps:.4f}), per step 1 sweep + plaquette + W_temp(L,T in 1..8)",
                   "parallelism": f"replicas x{dist.world}",
                   "l2": f"inputs larger than L2 ({V * 4 * 6 * 8 / 1e6:.0f} MB of FP32 links, two rows stored)"},
        "breakdown_ms": {"sweep": ms_sweep, "measure": ms_meas},
        "acceptance": float(np.mean(acc)), "mean_plaquette": float(np.mean(plaq)),
        "fp64": fp64_line, "mixed_error": mixed_err, "reference_proposal": same_chain,
        "roofline": roofline, "e2e": e2e, "e2e_host_lattice": e2e_host,
        "clocks": clocks.summary(), "gpu_launches": launches_per_step * a.steps,
    }
    pl_ms = plaquette_ms(g, eps)
    pl_bytes = V * 4 * 6 * 8  # every two-row FP32 link read once
    line["plaquettes_per_s"] = {"value": V * 6 / (pl_ms * 1e-3), "ms": pl_ms,
                                "hbm": {"algorithmic_bytes": pl_bytes, "achieved_gbs": pl_bytes / (pl_ms * 1e-3) / 1e9,
                                        "frac": (pl_bytes / (pl_ms * 1e-3) / 1e9 / hbm) if hbm else None},
                                "note": "V*Nd(Nd-1)/2 plaquettes per GaugePlaquette, device time; issue-bound "
                                        "(profiles/plaquette_hmc_streams_batch_pass.md)"}
    if dist.world == 1 and not a.no_extras:
        for key, fn in (("c1_u1_8x4", lambda: bench_c1(not a.no_cpu_baseline)),
                        ("batched_ptbc", lambda: bench_batched_ptbc(a.batch_cycles)),
                        ("hmc", lambda: bench_hmc(a.hmc_traj, not a.no_cpu_baseline)),
                        ("serving", lambda: bench_serving(a.serve_jobs, a.serve_rate))):
            try:
                line[key] = fn()
            except Exception as ex:  # reported, not fatal for the headline
                line[key] = {"error": f"{type(ex).__name__}: {ex}"}
    if dist.rank == 0 and dist.world == 1 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_reference(a.L)
        except Exception as ex:  # reported, not fatal
            line["cpu_baseline"] = {"error": str(ex)}
    g.close()
    return line


def run_reference(a, dist: Dist):
    """klft's own code (headers compiled unchanged on the project's OpenMP shim) on the host cores."""
    if dist.rank != 0:
        return None
    from oracle.oracle import REF_SO, Lat, RefShim
    if not os.path.exists(REF_SO):
        return {"impl": "reference", "unavailable": "oracle/_ref/libklft_ref.so not built (reference sources absent at "
                                                    "build time)"}
    r = RefShim()
    cores = r.set_threads(os.cpu_count() or 1)
    lat = Lat(3, [a.L] * 4)
    U = lat.field()
    for c in range(3):
        U[:, :, c, c] = 1.0
    # A step is one whole cycle (seconds on the host), so the run is bounded by
    # time: at most REF_WARMUP_S of warm-up cycles (at least one) and the timed
    # cycles stop once REF_TIMED_S have passed (at least one is timed).
    nwarm = 0
    tw = time.perf_counter()
    while nwarm < max(1, a.warmup) and (nwarm == 0 or time.perf_counter() - tw < REF_WARMUP_S):
        r.cycles(lat, U, BETA, 0.1, NHITS, 1, 1234, PAIRS, sweep0=nwarm)
        nwarm += 1
    t0 = time.perf_counter()
    steps = 0
    while steps < a.steps and (steps == 0 or time.perf_counter() - t0 < REF_TIMED_S):
        r.cycles(lat, U, BETA, 0.1, NHITS, 1, 1234, PAIRS, sweep0=nwarm + steps)
        steps += 1
    dt = time.perf_counter() - t0
    v = lat.V * 4 * steps / dt
    return {"metric": METRIC, "value": v, "unit": "link updates/s", "n_gpus": dist.world, "steps": steps,
            "steps_requested": a.steps, "warmup": nwarm, "warmup_requested": a.warmup,
            "ms_per_step": dt * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (cold start)", "impl": "reference",
            "config": {"workload": f"SU(3) 4D {a.L}^4 Metropolis beta=6 nHits=10 (reference SU(3) proposal), per "
                                   f"step 1 sweep + plaquette + W_temp(L,T in 1..8)", "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": v, "unit": "link updates/s", "cores": cores, "kind": "reference",
                             "sample": f"{steps} full cycles of SU(3) {a.L}^4 on {cores} host threads (time-bounded: "
                                       f"{REF_WARMUP_S:.0f} s of warm-up, {REF_TIMED_S:.0f} s timed at most)"},
            "e2e": {"value": v, "unit": "link updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    a = parse()
    dist = Dist() if a.impl == "ours" else None
    if a.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0

        class _D:
            rank, world = 0, 1
        line = run_reference(a, _D())
    else:
        line = run_ours(a, dist)
    if line is not None and (dist is None or dist.rank == 0):
        print(json.dumps(line))
    if dist:
        dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
