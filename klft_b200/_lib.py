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

# name -> (restype, argtypes); every symbol declared in include/klft_b200.h
SIGNATURES = {
    "klft_last_error": (C.c_char_p, []),
    "klft_version": (C.c_int, []),
    "klft_device_count": (C.c_int, [_ip]),
    "klft_lattice_create": (C.c_int, [C.c_int, C.c_int, _ip, C.c_int, C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "klft_lattice_destroy": (C.c_int, [_vp]),
    "klft_lattice_info": (C.c_int, [_vp, _ip, _ip, _ip, _ip, _llp]),
    "klft_lattice_set_stream": (C.c_int, [_vp, C.c_uint64, C.c_uint64]),
    "klft_lattice_get_counters": (C.c_int, [_vp, _u32p, _u32p]),
    "klft_lattice_set_counters": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "klft_lattice_upload": (C.c_int, [_vp, _dp]),
    "klft_lattice_download": (C.c_int, [_vp, _dp]),
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
    "klft_hmc_trajectories": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _ip]),
    "klft_hmc_integrate": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int]),
    "klft_hmc_refresh_momenta": (C.c_int, [_vp]),
    "klft_hmc_set_momenta": (C.c_int, [_vp, _dp]),
    "klft_hmc_get_momenta": (C.c_int, [_vp, _dp]),
    "klft_gauge_force": (C.c_int, [_vp, C.c_double, _dp]),
    "klft_hmc_energies": (C.c_int, [_vp, C.c_double, _dp, _dp]),
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
    "klft_metropolis_sweeps_noalloc": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                                 _dp]),
}

STATUS = {0: "KLFT_OK", 1: "KLFT_EINVAL", 2: "KLFT_ENOMEM", 3: "KLFT_ECUDA", 4: "KLFT_ETIMEOUT", 5: "KLFT_ENOTSUP"}


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
