"""Ensemble comparison of the mixed form (FP32 links, FP64 sums) with the FP64
form.

Per form, `chains` independent chains of one lattice (seeds seed + c, hot
starts) advance together in one batch (one CUDA graph per cycle); after `therm`
unmeasured cycles every cycle measures each chain's plaquette.  A chain's mean
over the measured cycles is one sample; the ensemble mean is the mean over
chains and its error the standard error of the chain means, which needs no
autocorrelation model because the chains are independent (each chain's mean
already averages over its own correlated cycles).

    python -m klft_b200.ensemble --L 8 8 8 8 --nc 3 --chains 128 --therm 500 --cycles 20000

`--dS-error` measures instead, on thermalised FP64 SU(3) configurations, the
error of the mixed form's action change against FP64 hit by hit with
identical proposals (klft_exp_proposal_dS_error): its mean, spread, largest
value, its slope against dS (a relative error of beta) and the fraction of hits
the FP32 accept test decides differently.  These bound the bias of the mixed
form's stationary plaquette: a relative error k of every dS is a shift of beta
by beta k, so the plaquette moves by beta k d<P>/d(beta).

    python -m klft_b200.ensemble --dS-error --L 16 16 16 16 --therm 300 --configs 8
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import Batch, GaugeField


def run_form(precision: str, L, nc: int, beta: float, nhits: int, proposal: str, eps: float, delta: float,
             chains: int, therm: int, cycles: int, seed: int, chunk: int = 500):
    """Per-chain mean plaquette over `cycles` measured cycles; returns (means, device_ms)."""
    b = Batch()
    fields = []
    try:
        for c in range(chains):
            g = GaugeField(L, nc, precision, "hot", seed + c)
            g.set_stream(seed + c, c)
            b.add(g, beta, delta, nhits, proposal, eps)
            fields.append(g)
        left = therm
        while left > 0:
            k = min(chunk, left)
            b.run(k, False, True)
            left -= k
        sums = np.zeros(chains)
        ms = 0.0
        left = cycles
        while left > 0:
            k = min(chunk, left)
            _, plaq, _, dms = b.run(k, True, True)
            sums += plaq.sum(axis=0)
            ms += dms
            left -= k
        return sums / cycles, ms
    finally:
        b.close()
        for g in fields:
            g.close()


def summary(means: np.ndarray):
    """(ensemble mean, standard error) of independent chain means."""
    return float(np.mean(means)), float(np.std(means, ddof=1) / math.sqrt(len(means)))


def compare(L=(8, 8, 8, 8), nc=3, beta=6.0, nhits=10, proposal="exp", eps=0.25, delta=0.0, chains=128, therm=500,
            cycles=20000, seed=9000):
    out = {"lattice": list(L), "nc": nc, "beta": beta, "nhits": nhits, "proposal": proposal, "eps": eps,
           "chains": chains, "therm_cycles": therm, "measured_cycles": cycles}
    for form in ("mixed", "fp64"):
        t0 = time.perf_counter()
        means, ms = run_form(form, list(L), nc, beta, nhits, proposal, eps, delta, chains, therm, cycles, seed)
        m, e = summary(means)
        out[form] = {"plaquette": m, "error": e, "device_s_measured": ms * 1e-3,
                     "wall_s": time.perf_counter() - t0}
    d = out["mixed"]["plaquette"] - out["fp64"]["plaquette"]
    ed = math.hypot(out["mixed"]["error"], out["fp64"]["error"])
    out["difference"] = {"mixed_minus_fp64": d, "error": ed, "sigmas": d / ed if ed > 0 else None}
    return out


def dS_error(L=(16, 16, 16, 16), beta=6.0, nhits=10, eps=0.25, therm=300, configs=8, seed=9100):
    """Per-hit FP32 vs FP64 action-change error on `configs` configurations of
    one FP64 chain (hot start, `therm` sweeps, 20 sweeps between configurations)."""
    g = GaugeField(list(L), 3, "fp64", "hot", seed)
    g.set_stream(seed, 0)
    try:
        g.metropolis(beta, 0.0, nhits, therm, "exp", eps)
        rows = []
        for _ in range(configs):
            g.metropolis(beta, 0.0, nhits, 20, "exp", eps)
            r = g.exp_dS_error(beta, eps, nhits)
            r["plaquette"] = g.plaquette()
            rows.append(r)
        n = sum(r["hits"] for r in rows)
        out = {"lattice": list(L), "beta": beta, "eps": eps, "nhits": nhits, "configs": configs, "hits": n,
               "mean": sum(r["mean"] * r["hits"] for r in rows) / n,
               "rms": math.sqrt(sum(r["rms"] ** 2 * r["hits"] for r in rows) / n),
               "max_abs": max(r["max_abs"] for r in rows),
               "slope": sum(r["slope"] for r in rows) / configs,
               "slope_spread": float(np.std([r["slope"] for r in rows], ddof=1)) if configs > 1 else None,
               "decision_flip_fraction": sum(r["decision_flip_fraction"] * r["hits"] for r in rows) / n,
               "plaquette": float(np.mean([r["plaquette"] for r in rows])), "per_config": rows}
        return out
    finally:
        g.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--L", type=int, nargs="+", default=[8, 8, 8, 8])
    ap.add_argument("--nc", type=int, default=3)
    ap.add_argument("--beta", type=float, default=6.0)
    ap.add_argument("--nhits", type=int, default=10)
    ap.add_argument("--proposal", default="exp")
    ap.add_argument("--eps", type=float, default=0.25)
    ap.add_argument("--delta", type=float, default=0.0)
    ap.add_argument("--chains", type=int, default=128)
    ap.add_argument("--therm", type=int, default=500)
    ap.add_argument("--cycles", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=9000)
    ap.add_argument("--dS-error", action="store_true")
    ap.add_argument("--configs", type=int, default=8)
    a = ap.parse_args(argv)
    if a.dS_error:
        print(json.dumps(dS_error(tuple(a.L), a.beta, a.nhits, a.eps, a.therm, a.configs, a.seed)))
        return
    print(json.dumps(compare(tuple(a.L), a.nc, a.beta, a.nhits, a.proposal, a.eps, a.delta, a.chains, a.therm,
                             a.cycles, a.seed)))


if __name__ == "__main__":
    main()
