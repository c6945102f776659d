"""klft_b200 -- B200-native lattice-gauge update-and-measure (klft's API).

Python mirror of the reference's operator interface, over the C ABI of
libklft_b200.so (include/klft_b200.h).  Names follow klft:

* ``GaugeField``            deviceGaugeField{,3D,2D}<Nd,Nc> (GaugeField.hpp)
* ``MetropolisParams``      Metropolis_Params.hpp:28-99
* ``GaugeObservableParams`` GaugeObservable.hpp:31-61
* ``sweep_Metropolis``      Metropolis.hpp:118-178
* ``run_metropolis``        Metropolis.hpp:180-223
* ``GaugePlaquette``        GaugePlaquette.hpp:89-135
* ``WilsonLoop_mu_nu``      WilsonLoop.hpp:170-245
* ``WilsonLoop_temporal``   WilsonLoop.hpp:250-304
* ``measureGaugeObservables`` / ``flushAllGaugeObservables``  GaugeObservable.hpp:64-230
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, List, Sequence, Tuple

import numpy as np

from ._lib import KlftError, check, lib

PRECISION = {"fp64": 0, "mixed": 1}
START = {"cold": 0, "hot": 1}
PROPOSAL = {"reference": 0, "exp": 1}
INTEGRATOR = {"reference": 0, "leapfrog": 1, "omelyan": 2}
GENERATORS = {"reference": 0, "half": 1}

__all__ = [
    "GaugeField", "MetropolisParams", "GaugeObservableParams", "KlftError", "sweep_Metropolis",
    "run_metropolis", "GaugePlaquette", "WilsonLoop_mu_nu", "WilsonLoop_temporal",
    "measureGaugeObservables", "flushAllGaugeObservables", "device_count", "Server", "JobSpec",
]


def device_count() -> int:
    n = C.c_int(0)
    lib().klft_device_count(C.byref(n))
    return n.value


def set_device(device: int) -> None:
    """Make `device` current for this thread in the library's CUDA runtime."""
    check(lib().klft_set_device(device))


def _pairs(pairs) -> np.ndarray:
    return np.ascontiguousarray(np.array(pairs, dtype=np.int32).reshape(-1, 2))


class GaugeField:
    """A device-resident SU(Nc) (Nc = 1: U(1)) gauge field on a periodic lattice."""

    def __init__(self, L: Sequence[int], nc: int, precision: str = "fp64", start: str = "cold", seed: int = 0):
        self.L = [int(x) for x in L]
        self.nd = len(self.L)
        self.nc = int(nc)
        self.precision = precision
        self.V = int(np.prod(self.L))
        Lc = (C.c_int * 4)(*(self.L + [1] * (4 - self.nd)))
        h = C.c_void_p()
        check(lib().klft_lattice_create(self.nc, self.nd, Lc, PRECISION[precision], START[start], seed, C.byref(h)))
        self._h = h

    @classmethod
    def load(cls, path: str) -> "GaugeField":
        """A lattice restored from a checkpoint (klft_checkpoint_read)."""
        h = C.c_void_p()
        check(lib().klft_checkpoint_read(os.fsencode(path), C.byref(h)))
        g = cls.__new__(cls)
        g._h = h
        nc, nd, prec = C.c_int(), C.c_int(), C.c_int()
        Lc = (C.c_int * 4)()
        V = C.c_longlong()
        check(lib().klft_lattice_info(h, C.byref(nc), C.byref(nd), Lc, C.byref(prec), C.byref(V)))
        g.nc, g.nd = nc.value, nd.value
        g.L = [Lc[d] for d in range(g.nd)]
        g.precision = {v: k for k, v in PRECISION.items()}[prec.value]
        g.V = V.value
        return g

    def save(self, path: str) -> None:
        """Write a checkpoint: links, Philox stream, counters, defect (klft_checkpoint_write)."""
        check(lib().klft_checkpoint_write(self._h, os.fsencode(path)))

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().klft_lattice_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- state
    def shape(self):
        return (self.V, self.nd, self.nc, self.nc)

    def upload(self, U: np.ndarray) -> None:
        a = np.ascontiguousarray(U, dtype=np.complex128)
        assert a.size == self.V * self.nd * self.nc * self.nc
        check(lib().klft_lattice_upload(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))

    def download(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The links in the host interchange layout; into `out` (a C-contiguous
        complex128 array of shape()) when given, e.g. a reused or page-locked buffer."""
        if out is None:
            out = np.empty(self.shape(), dtype=np.complex128)
        assert out.dtype == np.complex128 and out.flags.c_contiguous and out.size == int(np.prod(self.shape()))
        check(lib().klft_lattice_download(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def set_stream(self, seed: int, chain: int = 0) -> None:
        check(lib().klft_lattice_set_stream(self._h, seed, chain))

    def counters(self) -> Tuple[int, int]:
        s, t = C.c_uint32(), C.c_uint32()
        check(lib().klft_lattice_get_counters(self._h, C.byref(s), C.byref(t)))
        return s.value, t.value

    def set_counters(self, sweep: int, trajectory: int = 0) -> None:
        check(lib().klft_lattice_set_counters(self._h, sweep, trajectory))

    # -- update
    def metropolis(self, beta: float, delta: float, nhits: int, nsweeps: int = 1, proposal: str = "reference",
                   eps: float = 0.0) -> np.ndarray:
        acc = np.zeros(max(nsweeps, 1))
        check(lib().klft_metropolis_sweeps(self._h, beta, delta, nhits, PROPOSAL[proposal], eps, nsweeps,
                                           acc.ctypes.data_as(C.POINTER(C.c_double))))
        return acc[:nsweeps]

    # -- measure
    def plaquette(self) -> float:
        o = C.c_double()
        check(lib().klft_plaquette(self._h, C.byref(o)))
        return o.value

    def wilson_loop_mu_nu(self, mu: int, nu: int, pairs) -> np.ndarray:
        p = _pairs(pairs)
        o = np.zeros(len(p))
        check(lib().klft_wilson_loop_mu_nu(self._h, mu, nu, p.ctypes.data_as(C.POINTER(C.c_int)), len(p),
                                           o.ctypes.data_as(C.POINTER(C.c_double))))
        return o

    def wilson_loop(self, mu: int, nu: int, Lmu: int, Lnu: int, normalize: bool = True) -> float:
        """One Lmu x Lnu loop in the (mu, nu) plane: klft's legacy get_W_loop_mu_nu
        (GaugeVector.hpp:237-262); normalize=False gives the Re Tr sum over sites."""
        w = float(self.wilson_loop_mu_nu(mu, nu, [(Lmu, Lnu)])[0])
        return w if normalize else w * self.V * self.nc

    def wilson_loop_temporal(self, pairs) -> np.ndarray:
        p = _pairs(pairs)
        o = np.zeros(len(p))
        check(lib().klft_wilson_loop_temporal(self._h, p.ctypes.data_as(C.POINTER(C.c_int)), len(p),
                                              o.ctypes.data_as(C.POINTER(C.c_double))))
        return o

    def staple_field(self) -> np.ndarray:
        a = np.zeros(self.shape(), dtype=np.complex128)
        check(lib().klft_staple_field(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))
        return a

    def run_cycles(self, beta: float, delta: float, nhits: int, ncycles: int, proposal: str = "reference",
                   eps: float = 0.0, measure_plaquette: bool = True, temporal_pairs=()):
        """ncycles sweep+measure cycles back to back; returns (acc, plaq, W, device_ms)."""
        p = _pairs(temporal_pairs) if len(temporal_pairs) else np.zeros((0, 2), dtype=np.int32)
        acc = np.zeros(max(ncycles, 1))
        plaq = np.zeros(max(ncycles, 1))
        w = np.zeros((max(ncycles, 1), max(len(p), 1)))
        ms = C.c_double()
        dp = C.POINTER(C.c_double)
        check(lib().klft_run_cycles(self._h, beta, delta, nhits, PROPOSAL[proposal], eps, ncycles,
                                    int(measure_plaquette), p.ctypes.data_as(C.POINTER(C.c_int)), len(p),
                                    acc.ctypes.data_as(dp), plaq.ctypes.data_as(dp), w.ctypes.data_as(dp),
                                    C.byref(ms)))
        return acc[:ncycles], plaq[:ncycles], w[:ncycles, :len(p)], ms.value

    def run_metropolis_measured(self, beta: float, delta: float, nhits: int, nsweeps: int, interval: int,
                                proposal: str = "reference", eps: float = 0.0, measure_plaquette: bool = True,
                                temporal_pairs=(), planes=(), planar_pairs=()):
        """klft_run_metropolis: nsweeps sweeps with measurements after sweeps
        interval, 2 interval, ... < nsweeps, all enqueued without host round
        trips.  Returns (acc[nsweeps], plaq[nmeas], W_temp[nmeas, ntemporal],
        W_mu_nu[nmeas, nplanes, nplanar], device_ms)."""
        tp = _pairs(temporal_pairs) if len(temporal_pairs) else np.zeros((0, 2), dtype=np.int32)
        pl = _pairs(planes) if len(planes) else np.zeros((0, 2), dtype=np.int32)
        pp = _pairs(planar_pairs) if len(planar_pairs) else np.zeros((0, 2), dtype=np.int32)
        nmeas = (nsweeps - 1) // interval if interval > 0 and nsweeps > 0 else 0
        acc = np.zeros(max(nsweeps, 1))
        plaq = np.zeros(max(nmeas, 1))
        wt = np.zeros((max(nmeas, 1), max(len(tp), 1)))
        wm = np.zeros((max(nmeas, 1), max(len(pl), 1), max(len(pp), 1)))
        ms = C.c_double()
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        check(lib().klft_run_metropolis(self._h, beta, delta, nhits, PROPOSAL[proposal], eps, nsweeps, interval,
                                        int(measure_plaquette), tp.ctypes.data_as(ip), len(tp), pl.ctypes.data_as(ip),
                                        len(pl), pp.ctypes.data_as(ip), len(pp), acc.ctypes.data_as(dp),
                                        plaq.ctypes.data_as(dp), wt.ctypes.data_as(dp), wm.ctypes.data_as(dp),
                                        C.byref(ms)))
        wt = wt[:nmeas, :len(tp)]
        wm = wm.reshape(max(nmeas, 1), -1)[:nmeas, :len(pl) * len(pp)].reshape(nmeas, len(pl), len(pp))
        return acc[:nsweeps], plaq[:nmeas], wt, wm, ms.value

    # -- HMC
    def ncomp(self) -> int:
        return {1: 1, 2: 3, 3: 8}[self.nc]

    def _pshape(self):
        return (self.V, self.nd, self.ncomp())

    def hmc(self, beta: float, tau: float, n_steps: int, ntraj: int = 1, integrator: str = "leapfrog"):
        """ntraj HMC trajectories; returns (dH, accepted)."""
        dH = np.zeros(max(ntraj, 1))
        acc = np.zeros(max(ntraj, 1), dtype=np.int32)
        check(lib().klft_hmc_trajectories(self._h, beta, tau, n_steps, INTEGRATOR[integrator], ntraj,
                                          dH.ctypes.data_as(C.POINTER(C.c_double)),
                                          acc.ctypes.data_as(C.POINTER(C.c_int))))
        return dH[:ntraj], acc[:ntraj]

    def hmc_integrate(self, beta: float, tau: float, n_steps: int, integrator: str = "leapfrog") -> None:
        check(lib().klft_hmc_integrate(self._h, beta, tau, n_steps, INTEGRATOR[integrator]))

    def refresh_momenta(self) -> None:
        check(lib().klft_hmc_refresh_momenta(self._h))

    def set_momenta(self, P: np.ndarray) -> None:
        a = np.ascontiguousarray(P, dtype=np.float64)
        assert a.size == int(np.prod(self._pshape()))
        check(lib().klft_hmc_set_momenta(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))

    def momenta(self) -> np.ndarray:
        a = np.zeros(self._pshape())
        check(lib().klft_hmc_get_momenta(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))
        return a

    def gauge_force(self, beta: float) -> np.ndarray:
        a = np.zeros(self._pshape())
        check(lib().klft_gauge_force(self._h, beta, a.ctypes.data_as(C.POINTER(C.c_double))))
        return a

    def hmc_energies(self, beta: float):
        k, s = C.c_double(), C.c_double()
        check(lib().klft_hmc_energies(self._h, beta, C.byref(k), C.byref(s)))
        return k.value, s.value

    def set_hmc_generators(self, generators: str) -> None:
        """"reference" (klft's Pauli / Gell-Mann generators, the default) or
        "half" (t_a / 2: a trajectory of length tau equals the reference one of
        length tau / 2)."""
        check(lib().klft_hmc_set_generators(self._h, GENERATORS[generators]))

    # -- PTBC
    def set_open_boundary(self, mu: int) -> None:
        """Open boundary in direction mu: links across the last slice are zero and never updated."""
        check(lib().klft_lattice_set_open_boundary(self._h, mu))

    def set_defect(self, length: int, pos=(0, 0, 0), c: float = 1.0) -> None:
        p = (C.c_int * 3)(*(list(pos) + [0, 0, 0])[:3])
        check(lib().klft_lattice_set_defect(self._h, length, p, c))

    def set_defect_c(self, c: float) -> None:
        """Coefficient of the existing defect (a PTBC replica's new label)."""
        check(lib().klft_lattice_set_defect_c(self._h, c))

    def defect_sums(self, beta: float) -> np.ndarray:
        o = np.zeros(2)
        check(lib().klft_ptbc_defect_sums(self._h, beta, o.ctypes.data_as(C.POINTER(C.c_double))))
        return o

    def unitarity(self) -> float:
        o = C.c_double()
        check(lib().klft_unitarity(self._h, C.byref(o)))
        return o.value

    def exp_dS_error(self, beta: float, eps: float, nhits: int) -> dict:
        """FP32 (mixed form) against FP64 action changes of the current sweep's
        exp(i eps H) proposals on this FP64 SU(3) configuration."""
        o = np.zeros(6)
        check(lib().klft_exp_proposal_dS_error(self._h, beta, eps, nhits, o.ctypes.data_as(C.POINTER(C.c_double))))
        return {"hits": int(o[0]), "mean": o[1], "rms": o[2], "max_abs": o[3], "slope": o[4],
                "decision_flip_fraction": o[5]}

    def reunitarize(self) -> None:
        check(lib().klft_reunitarize(self._h))


def ptbc_swap(fields: Sequence[GaugeField], c_of_label, label_of_rep, beta: float, seed: int, cycle: int):
    """Neighbour-label swap attempts over PTBC replicas; returns (labels, accepted)."""
    n = len(fields)
    reps = (C.c_void_p * n)(*[f.handle.value for f in fields])
    c = np.ascontiguousarray(c_of_label, dtype=np.float64)
    lab = np.ascontiguousarray(label_of_rep, dtype=np.int32).copy()
    acc = np.zeros(max(n - 1, 1), dtype=np.int32)
    check(lib().klft_ptbc_swap(reps, n, c.ctypes.data_as(C.POINTER(C.c_double)),
                               lab.ctypes.data_as(C.POINTER(C.c_int)), beta, seed, cycle,
                               acc.ctypes.data_as(C.POINTER(C.c_int))))
    return lab, acc[: n - 1]


def ptbc_swap_sums(A, c_of_label, label_of_rep, seed: int, cycle: int):
    """Swap decisions from defect sums A[r] = (A_1, A_2) of replica r, on the host
    (klft_ptbc_swap_sums); returns (labels, accepted)."""
    a = np.ascontiguousarray(A, dtype=np.float64).reshape(-1)
    n = a.size // 2
    c = np.ascontiguousarray(c_of_label, dtype=np.float64)
    lab = np.ascontiguousarray(label_of_rep, dtype=np.int32).copy()
    acc = np.zeros(max(n - 1, 1), dtype=np.int32)
    check(lib().klft_ptbc_swap_sums(a.ctypes.data_as(C.POINTER(C.c_double)), n, c.ctypes.data_as(C.POINTER(C.c_double)),
                                    lab.ctypes.data_as(C.POINTER(C.c_int)), seed, cycle,
                                    acc.ctypes.data_as(C.POINTER(C.c_int))))
    return lab, acc[: n - 1]


class Batch:
    """Chains (and PTBC replicas) advanced together; one cycle per graph replay."""

    def __init__(self):
        h = C.c_void_p()
        check(lib().klft_batch_create(C.byref(h)))
        self._h = h
        self.fields: List[GaugeField] = []
        self.nrep = 0

    def add(self, field: GaugeField, beta: float, delta: float, nhits: int, proposal: str = "reference",
            eps: float = 0.0) -> int:
        cid = C.c_int()
        check(lib().klft_batch_add_chain(self._h, field.handle, beta, delta, nhits, PROPOSAL[proposal], eps,
                                         C.byref(cid)))
        self.fields.append(field)
        return cid.value

    def set_ptbc(self, chain_ids, c_of_label, beta: float, swap_seed: int) -> None:
        ids = np.ascontiguousarray(chain_ids, dtype=np.int32)
        c = np.ascontiguousarray(c_of_label, dtype=np.float64)
        check(lib().klft_batch_set_ptbc(self._h, ids.ctypes.data_as(C.POINTER(C.c_int)), len(ids),
                                        c.ctypes.data_as(C.POINTER(C.c_double)), beta, swap_seed))
        self.nrep = len(ids)

    def run(self, ncycles: int, measure_plaquette: bool = True, use_graph: bool = True):
        """Returns (acc[ncycles, nchains], plaq[ncycles, nchains], labels[ncycles, nrep], device_ms)."""
        n = len(self.fields)
        acc = np.zeros((ncycles, n))
        plaq = np.zeros((ncycles, n))
        lab = np.zeros((ncycles, max(self.nrep, 1)), dtype=np.int32)
        ms = C.c_double()
        dp = C.POINTER(C.c_double)
        check(lib().klft_batch_run(self._h, ncycles, int(measure_plaquette), int(use_graph), acc.ctypes.data_as(dp),
                                   plaq.ctypes.data_as(dp), lab.ctypes.data_as(C.POINTER(C.c_int)), C.byref(ms)))
        return acc, plaq, lab[:, : self.nrep], ms.value

    def swap_stats(self) -> np.ndarray:
        a = np.zeros(max(self.nrep - 1, 1), dtype=np.uint64)
        check(lib().klft_batch_swap_stats(self._h, a.ctypes.data_as(C.POINTER(C.c_ulonglong))))
        return a[: max(self.nrep - 1, 0)]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().klft_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ reference-style API
@dataclass
class MetropolisParams:
    """Metropolis_Params.hpp:28-99 (struct defaults); YAML defaults differ (InputParser.hpp:41-54)."""
    Ndims: int = 4
    L0: int = 4
    L1: int = 4
    L2: int = 4
    L3: int = 4
    nHits: int = 10
    nSweep: int = 1000
    seed: int = 1234
    Nd: int = 4
    Nc: int = 2
    beta: float = 1.0
    delta: float = 0.1
    # additions (ignored by the reference parser): SU(3) proposal and precision
    proposal: str = "reference"
    eps: float = 0.0
    precision: str = "fp64"
    start: str = "cold"

    def dims(self) -> List[int]:
        return [self.L0, self.L1, self.L2, self.L3][: self.Ndims]


@dataclass
class GaugeObservableParams:
    """GaugeObservable.hpp:31-61."""
    measurement_interval: int = 0
    measure_plaquette: bool = False
    measure_wilson_loop_temporal: bool = False
    measure_wilson_loop_mu_nu: bool = False
    W_temp_L_T_pairs: List[Tuple[int, int]] = field(default_factory=list)
    W_mu_nu_pairs: List[Tuple[int, int]] = field(default_factory=list)
    W_Lmu_Lnu_pairs: List[Tuple[int, int]] = field(default_factory=list)
    measurement_steps: List[int] = field(default_factory=list)
    plaquette_measurements: List[float] = field(default_factory=list)
    W_temp_measurements: List[list] = field(default_factory=list)
    W_mu_nu_measurements: List[list] = field(default_factory=list)
    plaquette_filename: str = ""
    W_temp_filename: str = ""
    W_mu_nu_filename: str = ""
    write_to_file: bool = False


def sweep_Metropolis(g: GaugeField, params: MetropolisParams) -> float:
    return float(g.metropolis(params.beta, params.delta, params.nHits, 1, params.proposal, params.eps)[0])


def GaugePlaquette(g: GaugeField) -> float:
    return g.plaquette()


def WilsonLoop_mu_nu(g: GaugeField, mu: int, nu: int, pairs) -> List[Tuple[float, float, float, float, float]]:
    w = g.wilson_loop_mu_nu(mu, nu, pairs)
    return [(float(mu), float(nu), float(p[0]), float(p[1]), float(x)) for p, x in zip(_pairs(pairs), w)]


def WilsonLoop_temporal(g: GaugeField, pairs) -> List[Tuple[float, float, float]]:
    w = g.wilson_loop_temporal(pairs)
    return [(float(p[0]), float(p[1]), float(x)) for p, x in zip(_pairs(pairs), w)]


def measureGaugeObservables(g: GaugeField, params: GaugeObservableParams, step: int) -> None:
    """GaugeObservable.hpp:64-127: measures at nonzero multiples of the interval."""
    if params.measurement_interval == 0 or step % params.measurement_interval != 0 or step == 0:
        return
    if params.measure_plaquette:
        params.plaquette_measurements.append(GaugePlaquette(g))
    if params.measure_wilson_loop_temporal:
        params.W_temp_measurements.append(WilsonLoop_temporal(g, params.W_temp_L_T_pairs))
    if params.measure_wilson_loop_mu_nu:
        rows = []
        for mu, nu in params.W_mu_nu_pairs:
            rows += WilsonLoop_mu_nu(g, mu, nu, params.W_Lmu_Lnu_pairs)
        params.W_mu_nu_measurements.append(rows)
    params.measurement_steps.append(step)


def _fmt(x: float) -> str:
    """Default std::ostream formatting of a double (6 significant digits, %g)."""
    return "%g" % x


def flushAllGaugeObservables(params: GaugeObservableParams, header: bool = True) -> None:
    """GaugeObservable.hpp:130-230: append the measurements to their files."""
    if not params.write_to_file:
        print("write_to_file is not enabled")
        return
    if params.plaquette_filename:
        with open(params.plaquette_filename, "a") as f:
            if not params.measure_plaquette:
                print("Error: no plaquette measurements available")
            else:
                if header:
                    f.write("# step, plaquette\n")
                for s, p in zip(params.measurement_steps, params.plaquette_measurements):
                    f.write(f"{s}, {_fmt(p)}\n")
    if params.W_temp_filename:
        with open(params.W_temp_filename, "a") as f:
            if not params.measure_wilson_loop_temporal:
                print("Error: no temporal Wilson loop measurements available")
            else:
                if header:
                    f.write("# step, L, T, W_temp\n")
                for s, rows in zip(params.measurement_steps, params.W_temp_measurements):
                    for r in rows:
                        f.write(f"{s}, {_fmt(r[0])}, {_fmt(r[1])}, {_fmt(r[2])}\n")
    if params.W_mu_nu_filename:
        with open(params.W_mu_nu_filename, "a") as f:
            if not params.measure_wilson_loop_mu_nu:
                print("Error: no mu-nu Wilson loop measurements available")
            else:
                if header:
                    f.write("# step, mu, nu, Lmu, Lnu, W_mu_nu\n")
                for s, rows in zip(params.measurement_steps, params.W_mu_nu_measurements):
                    for r in rows:
                        f.write(f"{s}, " + ", ".join(_fmt(v) for v in r) + "\n")


def run_metropolis(g: GaugeField, mp: MetropolisParams, op: GaugeObservableParams, verbosity: int = 0) -> int:
    """Metropolis.hpp:180-223.  Without per-step output (verbosity 0) the whole
    run is one klft_run_metropolis call; the measurements are the same."""
    import time
    if verbosity == 0:
        tp = op.W_temp_L_T_pairs if op.measure_wilson_loop_temporal else []
        pl = op.W_mu_nu_pairs if op.measure_wilson_loop_mu_nu else []
        pp = op.W_Lmu_Lnu_pairs if op.measure_wilson_loop_mu_nu else []
        _, plaq, wt, wm, _ = g.run_metropolis_measured(mp.beta, mp.delta, mp.nHits, mp.nSweep,
                                                       op.measurement_interval, mp.proposal, mp.eps,
                                                       op.measure_plaquette, tp, pl, pp)
        for i in range(len(plaq) if op.measurement_interval else 0):
            step = (i + 1) * op.measurement_interval
            if op.measure_plaquette:
                op.plaquette_measurements.append(float(plaq[i]))
            if op.measure_wilson_loop_temporal:
                op.W_temp_measurements.append([(float(p[0]), float(p[1]), float(x))
                                               for p, x in zip(_pairs(tp), wt[i])])
            if op.measure_wilson_loop_mu_nu:
                rows = []
                for q, (mu, nu) in enumerate(_pairs(pl)):
                    rows += [(float(mu), float(nu), float(p[0]), float(p[1]), float(x))
                             for p, x in zip(_pairs(pp), wm[i, q])]
                op.W_mu_nu_measurements.append(rows)
            op.measurement_steps.append(step)
        flushAllGaugeObservables(op)
        return 0
    for step in range(mp.nSweep):
        t0 = time.perf_counter()
        acc = sweep_Metropolis(g, mp)
        if verbosity > 0:
            print("Step: %d, Acceptance rate: %f, Time: %f" % (step, acc, time.perf_counter() - t0))
        measureGaugeObservables(g, op, step)
    flushAllGaugeObservables(op)
    return 0


from .serve import JobSpec, Server  # noqa: E402
