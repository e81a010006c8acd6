"""ctypes binding of the in-tree native library ``libhyowon_pm.so``.

The library is the product: every compute call below goes to sm_100a kernels.
There is no CPU fallback -- if the library is missing or cannot be loaded,
``lib()`` raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libhyowon_pm.so")

_lock = threading.Lock()
_lib = None

c_double = ctypes.c_double
c_u64 = ctypes.c_uint64
c_int = ctypes.c_int
c_void_p = ctypes.c_void_p
P_double = ctypes.POINTER(ctypes.c_double)
P_i64 = ctypes.POINTER(ctypes.c_int64)
P_u64 = ctypes.POINTER(ctypes.c_uint64)

# hyowon_status (include/hyowon_pm.h)
OK, EINVAL, ELOGIC, EOVERFLOW, EUNDERFLOW, ERUNTIME, ECUDA, ENOMEM = range(8)


class HyowonLogicError(RuntimeError):
    """std::logic_error counterpart (state / cell-assignment escape)."""


class HyowonUnderflowError(ArithmeticError):
    """std::underflow_error counterpart."""


class HyowonCudaError(RuntimeError):
    """CUDA / cuFFT failure."""


_EXC = {
    EINVAL: ValueError,
    ELOGIC: HyowonLogicError,
    EOVERFLOW: OverflowError,
    EUNDERFLOW: HyowonUnderflowError,
    ERUNTIME: RuntimeError,
    ECUDA: HyowonCudaError,
    ENOMEM: MemoryError,
}

class Diagnostics(ctypes.Structure):
    """hyowon_pm_diagnostics_t (include/hyowon_pm.h)."""
    _fields_ = [("potential_energy_comoving", c_double), ("kinetic_energy", c_double),
                ("momentum", c_double * 3), ("mass_weighted_force", c_double * 3),
                ("force_norm_sum", c_double), ("force_balance", c_double),
                ("momentum_force_contraction", c_double),
                ("directional_potential_energy_comoving", c_double)]


class PkBin(ctypes.Structure):
    """hyowon_pk_bin_t (include/hyowon_pm.h)."""
    _fields_ = [("k_low", c_double), ("k_mean", c_double), ("k_high", c_double),
                ("p_raw", c_double), ("p_corrected", c_double),
                ("mean_cic_power_deconvolution_factor", c_double),
                ("shot_noise_reference", c_double), ("mode_count", c_u64)]


class ICParams(ctypes.Structure):
    """hyowon_ic_params_t (include/hyowon_ic.h)."""
    _fields_ = [("particles_per_dimension", c_u64), ("mesh_per_dimension", c_u64),
                ("box_size", c_double), ("seed", c_u64), ("max_mode_per_axis", ctypes.c_int64),
                ("amplitude_mode", c_int), ("phase_pairing", c_int), ("lpt_order", c_int),
                ("momentum_factor_1", c_double), ("position_factor_2", c_double),
                ("momentum_factor_2", c_double)]


# name -> (restype, argtypes)
_SIGS = {
    "hyowon_pm_create": (c_int, [c_double, c_u64, c_int, c_int, c_double, c_int,
                                 ctypes.POINTER(c_void_p)]),
    "hyowon_pm_destroy": (c_int, [c_void_p]),
    "hyowon_pm_last_error": (ctypes.c_char_p, [c_void_p]),
    "hyowon_pm_upload": (c_int, [c_void_p, c_u64] + [P_double] * 7 + [c_double]),
    "hyowon_pm_download": (c_int, [c_void_p] + [P_double] * 9),
    "hyowon_pm_snapshot_payload": (c_int, [c_void_p, c_double, P_double, P_double]),
    "hyowon_pm_lpt_ics": (c_int, [c_void_p, c_u64, P_double, c_u64, P_double, P_double,
                                  P_double, c_double, c_double]),
    "hyowon_pm_compute_forces": (c_int, [c_void_p] + [P_double] * 3),
    "hyowon_pm_forces_host": (c_int, [c_void_p, c_u64] + [P_double] * 4 + [c_double]
                              + [P_double] * 3),
    "hyowon_pm_kdk_step": (c_int, [c_void_p, c_double, c_double, c_double, P_double]),
    "hyowon_pm_run": (c_int, [c_void_p, c_u64, P_double, P_double, P_double, P_double]),
    "hyowon_pm_info": (c_int, [c_void_p, P_u64, P_u64, ctypes.POINTER(c_int),
                               ctypes.POINTER(c_int)]),
    "hyowon_pm_download_potential": (c_int, [c_void_p, P_double]),
    "hyowon_pm_download_mass_mesh": (c_int, [c_void_p, P_double]),
    "hyowon_pm_cell_coords": (c_int, [c_void_p, P_i64, P_double]),
    "hyowon_pm_set_timing": (c_int, [c_void_p, c_int]),
    "hyowon_pm_set_sort_interval": (c_int, [c_void_p, c_int]),
    "hyowon_pm_last_timing": (c_int, [c_void_p, P_double]),
    "hyowon_pm_diagnostics": (c_int, [c_void_p, c_double, ctypes.POINTER(Diagnostics)]),
    "hyowon_pm_power_spectrum": (c_int, [c_void_p, c_u64, c_int, c_double, c_int, c_int,
                                         ctypes.POINTER(PkBin)]),
    "hyowon_vjp_1lpt_pm": (c_int, [c_void_p, P_double, P_double, P_double, P_double,
                                   P_double, P_double]),
    "hyowon_vjp_last_error": (ctypes.c_char_p, []),
    "hyowon_pm_vjp": (c_int, [c_void_p, c_void_p, P_double, P_double, P_double, P_double,
                              P_double, P_double]),
    "hyowon_treepm_short_forces": (c_int, [c_void_p, c_u64, P_double, P_double, P_double, c_u64,
                                           ctypes.POINTER(ctypes.c_uint32), P_double, P_double,
                                           P_double, P_double]),
    "hyowon_treepm_last_error": (ctypes.c_char_p, []),
    "hyowon_pm_set_treepm_short_range": (c_int, [c_void_p, c_double, c_double, c_double]),
    "hyowon_pm_debug_set_wait_limit": (c_int, [c_void_p, ctypes.c_uint]),
    "hyowon_pm_debug_offset_mass_target": (c_int, [c_void_p, c_double]),
    "hyowon_pm_treepm_short_forces": (c_int, [c_void_p, c_double, c_double, c_double]
                                      + [P_double] * 4),
    "hyowon_cic_deposit_noalloc": (c_int, [c_double, c_u64, c_u64, c_void_p, c_void_p,
                                           c_void_p, c_void_p, c_double, c_void_p, c_void_p]),
    "hyowon_noalloc_last_error": (ctypes.c_char_p, []),
    "hyowon_hubble": (c_int, [c_double, c_double, c_u64, P_double, P_double]),
    "hyowon_drift_factor": (c_int, [c_double, c_double, c_double, c_double, P_double]),
    "hyowon_kick_factor": (c_int, [c_double, c_double, c_double, c_double, P_double]),
    "hyowon_geometric_mean": (c_int, [c_double, c_double, P_double]),
    "hyowon_schedule": (c_int, [c_double, c_double, c_double, c_double, c_double, c_u64,
                                P_double, P_u64]),
    "hyowon_growth": (c_int, [c_double, c_double, c_u64, P_double, P_double, P_double]),
    "hyowon_growth2": (c_int, [c_double, c_double, c_u64] + [P_double] * 5),
    "hyowon_ic_resolve": (c_int, [ctypes.POINTER(ICParams), P_u64, P_u64]),
    "hyowon_ic_mode_amplitudes": (c_int, [c_u64, c_double, c_u64, P_double, P_double]),
    "hyowon_ic_field": (c_int, [ctypes.POINTER(ICParams), c_u64, P_double, P_double]),
    "hyowon_ic_generate": (c_int, [ctypes.POINTER(ICParams), c_u64, P_double] + [P_double] * 6),
    "hyowon_pm_generate_ics": (c_int, [c_void_p, ctypes.POINTER(ICParams), c_u64, P_double,
                                       c_double]),
    "hyowon_ic_last_error": (ctypes.c_char_p, []),
}


def lib():
    """Load libhyowon_pm.so (raises if it is missing: no fallback exists)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is not built; run `python -m hyowon_b200.build` "
                    "(the PM path has no CPU fallback)")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def dptr(a):
    """double* of a C-contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(P_double)


def raise_for(code: int, handle=None, where: str = ""):
    if code == OK:
        return
    msg = ""
    if handle is not None:
        msg = lib().hyowon_pm_last_error(handle).decode(errors="replace")
    exc = _EXC.get(code, RuntimeError)
    raise exc(f"{where}: {msg}" if where else msg)
