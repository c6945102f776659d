"""ctypes loader for the CPU checker libraries.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py.  The product package
(klft_b200) never imports this module.

* ``Oracle``   -- the FP64 restatement in oracle.cpp (built to _build/liboracle.so)
* ``RefShim``  -- klft's own headers compiled against the project's Kokkos-API
                  host shim (built to _ref/libklft_ref.so when the reference
                  sources were available at build time)

Arrays use the host interchange layout: complex128 of shape
(V, Nd, Nc, Nc) with site = x0 + L0*(x1 + L1*(x2 + L2*x3)).
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libklft_ref.so")

KIND_METROPOLIS, KIND_INIT, KIND_MOMENTUM, KIND_HMC_ACCEPT, KIND_SWAP = 1, 2, 3, 4, 5
PROPOSAL_REFERENCE, PROPOSAL_EXP = 0, 1
INTEGRATOR_REFERENCE_LEAPFROG, INTEGRATOR_LEAPFROG, INTEGRATOR_OMELYAN = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint32)


def build(force: bool = False) -> None:
    """Compile liboracle.so, and libklft_ref.so from the klft source tree that
    the environment variable KLFT_REF_DIR names.

    Without KLFT_REF_DIR an existing libklft_ref.so is kept as built; when there
    is none, the reference-code checks are skipped and this says so on stderr.
    """
    if force or _stale(ORACLE_SO, [os.path.join(HERE, "oracle.cpp")]):
        subprocess.run(["make", "-C", HERE, "all"], check=True, capture_output=True)
    ref_dir = os.environ.get("KLFT_REF_DIR", "")
    if ref_dir:
        if not os.path.isdir(os.path.join(ref_dir, "include")):
            raise FileNotFoundError(f"KLFT_REF_DIR={ref_dir} has no include/ directory")
        deps = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "ref_adjoint.cpp")]
        deps += glob.glob(os.path.join(HERE, "ref_shim", "*.hpp"))
        if force or _stale(REF_SO, deps) or _stale(os.path.join(HERE, "_ref", "libklft_ref_adjoint.so"), deps):
            subprocess.run(["make", "-C", HERE, "ref", "KLFT_REF_DIR=" + ref_dir], check=True, capture_output=True)
    elif not os.path.exists(REF_SO):
        sys.stderr.write("oracle: KLFT_REF_DIR is not set and oracle/_ref/libklft_ref.so does not exist; "
                         "the checks against klft's own code are skipped\n")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def ncomp(nc: int) -> int:
    return {1: 1, 2: 3, 3: 8}[nc]


class Lat:
    """Geometry + helpers shared by the oracle and the reference shim."""

    def __init__(self, nc: int, L):
        self.nc = nc
        self.L = [int(x) for x in L]
        self.nd = len(self.L)
        self.V = int(np.prod(self.L))
        self.Lc = np.array(self.L + [1] * (4 - self.nd), dtype=np.int32)

    def field(self):
        return np.zeros((self.V, self.nd, self.nc, self.nc), dtype=np.complex128)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        L.oracle_philox.argtypes = [_up, _up, _up]
        L.oracle_uniforms.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                      C.c_int, _dp]
        L.oracle_init.argtypes = [C.c_int, C.c_int, _ip, C.c_int, C.c_uint64, C.c_uint64, _dp]
        L.oracle_staple_field.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp]
        L.oracle_plaquette.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int, _dp]
        L.oracle_wilson_mu_nu.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int, C.c_int, _ip, C.c_int, _dp]
        L.oracle_wilson_legacy.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           _dp]
        L.oracle_wilson_temporal.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, C.c_int, _dp]
        L.oracle_metropolis.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, C.c_double, C.c_int, C.c_int,
                                        C.c_double, C.c_uint64, C.c_uint64, C.c_uint32, C.c_int, _ip, C.c_double,
                                        _dp]
        L.oracle_expi_su3.argtypes = [_dp, _dp]
        L.oracle_set_open_boundary.argtypes = [C.c_int]
        L.oracle_set_open_boundary.restype = None
        L.oracle_set_generators.argtypes = [C.c_int]
        L.oracle_set_generators.restype = None
        L.oracle_adjoint.argtypes = [C.c_int, _dp, _dp]
        L.oracle_expmap.argtypes = [C.c_int, _dp, C.c_double, _dp]
        L.oracle_gauge_force.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, _dp]
        L.oracle_momenta.argtypes = [C.c_int, C.c_int, _ip, C.c_uint64, C.c_uint64, C.c_uint32, _dp]
        L.oracle_gauge_action.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, _dp]
        L.oracle_integrate.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int]
        L.oracle_hmc.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_uint64,
                                 C.c_uint64, C.c_uint32, C.c_int, _dp, _ip]
        L.oracle_defect_sums.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, C.c_double, _dp]
        L.oracle_defect_action.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, C.c_double, C.c_double, _dp]
        L.oracle_unitarity.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp]
        L.oracle_ptbc_swap.argtypes = [C.c_int, _dp, _dp, _ip, C.c_uint64, C.c_uint32, _ip]

    def ptbc_swap(self, c, A, label_of_rep, seed, cycle):
        """Sequential neighbour-label swap attempts; returns (new labels, accepted per pair)."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        A = np.ascontiguousarray(A, dtype=np.float64).reshape(-1)
        lab = np.ascontiguousarray(label_of_rep, dtype=np.int32).copy()
        acc = np.zeros(max(len(c) - 1, 1), dtype=np.int32)
        self.lib.oracle_ptbc_swap(len(c), _d(c), _d(A), _i(lab), seed, cycle, _i(acc))
        return lab, acc[: len(c) - 1]

    # -- random stream
    def philox(self, ctr, key):
        c = np.array(ctr, dtype=np.uint32)
        k = np.array(key, dtype=np.uint32)
        o = np.zeros(4, dtype=np.uint32)
        self.lib.oracle_philox(c.ctypes.data_as(_up), k.ctypes.data_as(_up), o.ctypes.data_as(_up))
        return o

    def uniforms(self, seed, chain, site, step, kind, sub, n):
        o = np.zeros(n)
        self.lib.oracle_uniforms(seed, chain, site, step, kind, sub, n, _d(o))
        return o

    # -- fields
    def init(self, lat: Lat, hot: bool, seed: int = 0, chain: int = 0):
        U = lat.field()
        self.lib.oracle_init(lat.nc, lat.nd, _i(lat.Lc), int(hot), seed, chain, _d(U))
        return U

    def staple_field(self, lat: Lat, U):
        out = lat.field()
        self.lib.oracle_staple_field(lat.nc, lat.nd, _i(lat.Lc), _d(U), _d(out))
        return out

    def plaquette(self, lat: Lat, U, normalize=True):
        o = np.zeros(1)
        self.lib.oracle_plaquette(lat.nc, lat.nd, _i(lat.Lc), _d(U), int(normalize), _d(o))
        return float(o[0])

    def wilson_mu_nu(self, lat: Lat, U, mu, nu, pairs):
        p = np.ascontiguousarray(np.array(pairs, dtype=np.int32).reshape(-1, 2))
        o = np.zeros(len(p))
        self.lib.oracle_wilson_mu_nu(lat.nc, lat.nd, _i(lat.Lc), _d(U), mu, nu, _i(p), len(p), _d(o))
        return o

    def wilson_legacy(self, lat: Lat, U, mu, nu, Lmu, Lnu, normalize=True):
        """GaugeVector.hpp:237-262 get_W_loop_mu_nu, step by step over whole fields."""
        o = np.zeros(1)
        self.lib.oracle_wilson_legacy(lat.nc, lat.nd, _i(lat.Lc), _d(U), mu, nu, Lmu, Lnu, int(normalize), _d(o))
        return float(o[0])

    def wilson_temporal(self, lat: Lat, U, pairs):
        p = np.ascontiguousarray(np.array(pairs, dtype=np.int32).reshape(-1, 2))
        o = np.zeros(len(p))
        self.lib.oracle_wilson_temporal(lat.nc, lat.nd, _i(lat.Lc), _d(U), _i(p), len(p), _d(o))
        return o

    def set_open_boundary(self, mu: int) -> None:
        """Open boundary in direction mu for the following calls (-1: periodic)."""
        self.lib.oracle_set_open_boundary(mu)

    def metropolis(self, lat: Lat, U, beta, delta, nhits, nsweeps, seed, chain=0, sweep0=0,
                   proposal=PROPOSAL_REFERENCE, eps=0.0, defect=None, defect_c=1.0):
        """Run nsweeps sweeps in place on U; returns per-sweep acceptance."""
        acc = np.zeros(nsweeps)
        dp = None
        if defect is not None:
            dpa = np.array(defect, dtype=np.int32)
            dp = _i(dpa)
        self.lib.oracle_metropolis(lat.nc, lat.nd, _i(lat.Lc), _d(U), beta, delta, nhits, proposal, eps, seed,
                                   chain, sweep0, nsweeps, dp, defect_c, _d(acc))
        return acc

    def expi_su3(self, Q):
        q = np.ascontiguousarray(np.asarray(Q, dtype=np.complex128))
        o = np.zeros((3, 3), dtype=np.complex128)
        self.lib.oracle_expi_su3(_d(q), _d(o))
        return o

    def set_generators(self, half: bool) -> None:
        """HMC generators for the following calls: the reference's, or t_a / 2."""
        self.lib.oracle_set_generators(int(half))

    def adjoint(self, M):
        """Adj(M) of one Nc x Nc complex matrix (reference normalisation)."""
        m = np.ascontiguousarray(M, dtype=np.complex128)
        v = np.zeros(ncomp(m.shape[0]))
        self.lib.oracle_adjoint(m.shape[0], _d(m), _d(v))
        return v

    def expmap(self, nc, p, t):
        """exp(i t sum_a p_a t_a) in the reference normalisation."""
        pa = np.ascontiguousarray(p, dtype=np.float64)
        m = np.zeros((nc, nc), dtype=np.complex128)
        self.lib.oracle_expmap(nc, _d(pa), t, _d(m))
        return m

    def gauge_force(self, lat: Lat, U, beta):
        f = np.zeros((lat.V, lat.nd, ncomp(lat.nc)))
        self.lib.oracle_gauge_force(lat.nc, lat.nd, _i(lat.Lc), _d(U), beta, _d(f))
        return f

    def momenta(self, lat: Lat, seed, chain, traj):
        p = np.zeros((lat.V, lat.nd, ncomp(lat.nc)))
        self.lib.oracle_momenta(lat.nc, lat.nd, _i(lat.Lc), seed, chain, traj, _d(p))
        return p

    def gauge_action(self, lat: Lat, U, beta):
        o = np.zeros(1)
        self.lib.oracle_gauge_action(lat.nc, lat.nd, _i(lat.Lc), _d(U), beta, _d(o))
        return float(o[0])

    def integrate(self, lat: Lat, U, P, beta, tau, nsteps, integrator):
        self.lib.oracle_integrate(lat.nc, lat.nd, _i(lat.Lc), _d(U), _d(P), beta, tau, nsteps, integrator)

    def hmc(self, lat: Lat, U, beta, tau, nsteps, integrator, seed, chain, traj0, ntraj):
        dH = np.zeros(ntraj)
        acc = np.zeros(ntraj, dtype=np.int32)
        self.lib.oracle_hmc(lat.nc, lat.nd, _i(lat.Lc), _d(U), beta, tau, nsteps, integrator, seed, chain, traj0,
                            ntraj, _d(dH), _i(acc))
        return dH, acc

    def defect_sums(self, lat: Lat, U, defect, beta):
        d = np.array(defect, dtype=np.int32)
        o = np.zeros(2)
        self.lib.oracle_defect_sums(lat.nc, lat.nd, _i(lat.Lc), _d(U), _i(d), beta, _d(o))
        return o

    def defect_action(self, lat: Lat, U, defect, c, beta):
        d = np.array(defect, dtype=np.int32)
        o = np.zeros(1)
        self.lib.oracle_defect_action(lat.nc, lat.nd, _i(lat.Lc), _d(U), _i(d), c, beta, _d(o))
        return float(o[0])

    def unitarity(self, lat: Lat, U):
        o = np.zeros(1)
        self.lib.oracle_unitarity(lat.nc, lat.nd, _i(lat.Lc), _d(U), _d(o))
        return float(o[0])


REF_ADJ_SO = os.path.join(HERE, "_ref", "libklft_ref_adjoint.so")


class RefAdjoint:
    """klft's HMC Lie-algebra maps (AdjointGroup.hpp on the SU2 / U1 structs of
    GaugeGroup.hpp), compiled unchanged on the shim (oracle/_ref)."""

    def __init__(self, path: str = REF_ADJ_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_su2_adjoint.argtypes = [_dp, _dp]
        L.ref_su2_exp.argtypes = [_dp, C.c_double, _dp]
        L.ref_su2_mul.argtypes = [_dp, _dp, _dp]
        L.ref_u1_adjoint.argtypes = [_dp, _dp]
        L.ref_u1_exp.argtypes = [C.c_double, C.c_double, _dp]

    def adjoint(self, M):
        m = np.ascontiguousarray(M, dtype=np.complex128)
        v = np.zeros(3 if m.shape[0] == 2 else 1)
        (self.lib.ref_su2_adjoint if m.shape[0] == 2 else self.lib.ref_u1_adjoint)(_d(m), _d(v))
        return v

    def expmap(self, nc, p, t):
        m = np.zeros((nc, nc), dtype=np.complex128)
        if nc == 2:
            pa = np.ascontiguousarray(p, dtype=np.float64)
            self.lib.ref_su2_exp(_d(pa), t, _d(m))
        else:
            self.lib.ref_u1_exp(float(np.asarray(p).reshape(-1)[0]), t, _d(m))
        return m

    def su2_mul(self, A, B):
        a = np.ascontiguousarray(A, dtype=np.complex128)
        b = np.ascontiguousarray(B, dtype=np.complex128)
        c = np.zeros((2, 2), dtype=np.complex128)
        self.lib.ref_su2_mul(_d(a), _d(b), _d(c))
        return c


class RefShim:
    """klft's own headers on the project's Kokkos-API host shim (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_plaquette.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp]
        L.ref_wilson_temporal.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, C.c_int, _dp]
        L.ref_wilson_mu_nu.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int, C.c_int, _ip, C.c_int, _dp]
        L.ref_staple_field.argtypes = [C.c_int, _ip, _dp, _dp]
        L.ref_metropolis.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_uint32, C.c_int, _dp]
        L.ref_cycles.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_uint32,
                                 C.c_int, _ip, C.c_int, _dp, _dp, _dp]

    def set_threads(self, n: int) -> int:
        return int(self.lib.ref_set_threads(n))

    def plaquette(self, lat: Lat, U):
        o = np.zeros(1)
        self.lib.ref_plaquette(lat.nc, lat.nd, _i(lat.Lc), _d(U), _d(o))
        return float(o[0])

    def wilson_temporal(self, lat: Lat, U, pairs):
        p = np.ascontiguousarray(np.array(pairs, dtype=np.int32).reshape(-1, 2))
        o = np.zeros(len(p))
        self.lib.ref_wilson_temporal(lat.nc, lat.nd, _i(lat.Lc), _d(U), _i(p), len(p), _d(o))
        return o

    def wilson_mu_nu(self, lat: Lat, U, mu, nu, pairs):
        p = np.ascontiguousarray(np.array(pairs, dtype=np.int32).reshape(-1, 2))
        o = np.zeros(len(p))
        self.lib.ref_wilson_mu_nu(lat.nc, lat.nd, _i(lat.Lc), _d(U), mu, nu, _i(p), len(p), _d(o))
        return o

    def staple_field(self, lat: Lat, U):
        assert lat.nd == 4
        out = lat.field()
        self.lib.ref_staple_field(lat.nc, _i(lat.Lc), _d(U), _d(out))
        return out

    def metropolis(self, lat: Lat, U, beta, delta, nhits, nsweeps, seed, sweep0=0):
        acc = np.zeros(nsweeps)
        self.lib.ref_metropolis(lat.nc, lat.nd, _i(lat.Lc), _d(U), beta, delta, nhits, seed, sweep0, nsweeps,
                                _d(acc))
        return acc

    def cycles(self, lat: Lat, U, beta, delta, nhits, nsweeps, seed, pairs, sweep0=0):
        p = np.ascontiguousarray(np.array(pairs, dtype=np.int32).reshape(-1, 2))
        acc = np.zeros(nsweeps)
        plaq = np.zeros(nsweeps)
        w = np.zeros((nsweeps, max(len(p), 1)))
        self.lib.ref_cycles(lat.nc, lat.nd, _i(lat.Lc), _d(U), beta, delta, nhits, seed, sweep0, nsweeps, _i(p),
                            len(p), _d(acc), _d(plaq), _d(w))
        return acc, plaq, w
