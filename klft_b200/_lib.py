"""ctypes binding of libklft_b200.so (the C ABI in include/klft_b200.h).

The shared library is built in-tree (python -m klft_b200.build).  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libklft_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u32p = C.POINTER(C.c_uint32)
_llp = C.POINTER(C.c_longlong)
_vp = C.c_void_p

JOB_MAX_WILSON = 16


class Job(C.Structure):
    """struct klft_job (include/klft_b200.h)."""
    _fields_ = [("kind", C.c_int), ("nc", C.c_int), ("ndims", C.c_int), ("L", C.c_int * 4),
                ("precision", C.c_int), ("start", C.c_int), ("seed", C.c_uint64), ("chain", C.c_uint64),
                ("beta", C.c_double), ("nsweeps", C.c_int), ("nhits", C.c_int), ("proposal", C.c_int),
                ("delta", C.c_double), ("eps", C.c_double), ("ntraj", C.c_int), ("nsteps", C.c_int),
                ("integrator", C.c_int), ("tau", C.c_double), ("measure_plaquette", C.c_int),
                ("n_wilson", C.c_int), ("wilson_pairs", C.c_int * (2 * JOB_MAX_WILSON))]


class JobResult(C.Structure):
    """struct klft_job_result."""
    _fields_ = [("id", C.c_uint64), ("status", C.c_int), ("kind", C.c_int), ("plaquette", C.c_double),
                ("wilson", C.c_double * JOB_MAX_WILSON), ("acceptance", C.c_double),
                ("mean_exp_mdH", C.c_double), ("mean_dH", C.c_double), ("link_updates", C.c_ulonglong),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_finish", C.c_double),
                ("error", C.c_char * 160)]


class ServerStats(C.Structure):
    """struct klft_server_stats."""
    _fields_ = [("submitted", C.c_ulonglong), ("completed", C.c_ulonglong), ("failed", C.c_ulonglong),
                ("cancelled", C.c_ulonglong), ("rejected", C.c_ulonglong), ("queued", C.c_int),
                ("active", C.c_int), ("bytes_in_use", C.c_uint64), ("bytes_budget", C.c_uint64),
                ("link_updates", C.c_ulonglong), ("rounds", C.c_ulonglong), ("launches", C.c_ulonglong),
                ("busy_s", C.c_double)]


# name -> (restype, argtypes); every symbol declared in include/klft_b200.h
SIGNATURES = {
    "klft_last_error": (C.c_char_p, []),
    "klft_version": (C.c_int, []),
    "klft_device_count": (C.c_int, [_ip]),
    "klft_set_device": (C.c_int, [C.c_int]),
    "klft_lattice_create": (C.c_int, [C.c_int, C.c_int, _ip, C.c_int, C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "klft_lattice_destroy": (C.c_int, [_vp]),
    "klft_lattice_info": (C.c_int, [_vp, _ip, _ip, _ip, _ip, _llp]),
    "klft_lattice_set_stream": (C.c_int, [_vp, C.c_uint64, C.c_uint64]),
    "klft_lattice_get_counters": (C.c_int, [_vp, _u32p, _u32p]),
    "klft_lattice_set_counters": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "klft_lattice_upload": (C.c_int, [_vp, _dp]),
    "klft_lattice_download": (C.c_int, [_vp, _dp]),
    "klft_lattice_set_open_boundary": (C.c_int, [_vp, C.c_int]),
    "klft_metropolis_sweeps": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, _dp]),
    "klft_plaquette": (C.c_int, [_vp, _dp]),
    "klft_wilson_loop_mu_nu": (C.c_int, [_vp, C.c_int, C.c_int, _ip, C.c_int, _dp]),
    "klft_wilson_loop_temporal": (C.c_int, [_vp, _ip, C.c_int, _dp]),
    "klft_staple_field": (C.c_int, [_vp, _dp]),
    "klft_unitarity": (C.c_int, [_vp, _dp]),
    "klft_reunitarize": (C.c_int, [_vp]),
    "klft_run_cycles": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, _ip,
                                  C.c_int, _dp, _dp, _dp, _dp]),
    "klft_peak_flops": (C.c_int, [C.c_int, _dp]),
    "klft_run_metropolis": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                      C.c_int, _ip, C.c_int, _ip, C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    "klft_exp_proposal_dS_error": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, _dp]),
    "klft_hmc_trajectories": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _ip]),
    "klft_hmc_integrate": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int]),
    "klft_hmc_refresh_momenta": (C.c_int, [_vp]),
    "klft_hmc_set_momenta": (C.c_int, [_vp, _dp]),
    "klft_hmc_get_momenta": (C.c_int, [_vp, _dp]),
    "klft_gauge_force": (C.c_int, [_vp, C.c_double, _dp]),
    "klft_hmc_energies": (C.c_int, [_vp, C.c_double, _dp, _dp]),
    "klft_hmc_set_generators": (C.c_int, [_vp, C.c_int]),
    "klft_lattice_set_defect": (C.c_int, [_vp, C.c_int, _ip, C.c_double]),
    "klft_batch_create": (C.c_int, [C.POINTER(_vp)]),
    "klft_batch_destroy": (C.c_int, [_vp]),
    "klft_batch_add_chain": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _ip]),
    "klft_batch_set_ptbc": (C.c_int, [_vp, _ip, C.c_int, _dp, C.c_double, C.c_uint64]),
    "klft_batch_run": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _ip, _dp]),
    "klft_batch_swap_stats": (C.c_int, [_vp, C.POINTER(C.c_ulonglong)]),
    "klft_tuner_configure": (C.c_int, [C.c_int, C.c_int]),
    "klft_tuner_read_cache": (C.c_int, [C.c_char_p]),
    "klft_tuner_write_cache": (C.c_int, [C.c_char_p]),
    "klft_tuner_lookup": (C.c_int, [C.c_char_p, _ip, _ip]),
    "klft_tuner_clear": (C.c_int, []),
    "klft_ptbc_defect_sums": (C.c_int, [_vp, C.c_double, _dp]),
    "klft_ptbc_swap": (C.c_int, [C.POINTER(_vp), C.c_int, _dp, _ip, C.c_double, C.c_uint64, C.c_uint32, _ip]),
    "klft_ptbc_swap_sums": (C.c_int, [_dp, C.c_int, _dp, _ip, C.c_uint64, C.c_uint32, _ip]),
    "klft_lattice_set_defect_c": (C.c_int, [_vp, C.c_double]),
    "klft_checkpoint_write": (C.c_int, [_vp, C.c_char_p]),
    "klft_checkpoint_read": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "klft_job_footprint": (C.c_int, [C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "klft_server_create": (C.c_int, [C.c_int, C.c_uint64, C.c_int, C.c_int, C.POINTER(_vp)]),
    "klft_server_destroy": (C.c_int, [_vp]),
    "klft_server_submit": (C.c_int, [_vp, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "klft_server_cancel": (C.c_int, [_vp, C.c_uint64]),
    "klft_server_poll": (C.c_int, [_vp, C.POINTER(JobResult), C.c_int, C.c_int, _ip]),
    "klft_server_stats_get": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "klft_server_inject_fault": (C.c_int, [_vp, C.c_int]),
    "klft_metropolis_sweeps_noalloc": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                                 _dp]),
}

STATUS = {0: "KLFT_OK", 1: "KLFT_EINVAL", 2: "KLFT_ENOMEM", 3: "KLFT_ECUDA", 4: "KLFT_ETIMEOUT", 5: "KLFT_ENOTSUP",
          6: "KLFT_ECANCELED", 7: "KLFT_EINTERNAL", 8: "KLFT_EBUSY"}


class KlftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libklft_b200.so once; raise if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libklft_b200.so not built at {LIB_PATH}; run `python -m klft_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != 0:
        raise KlftError(code, lib().klft_last_error().decode())
