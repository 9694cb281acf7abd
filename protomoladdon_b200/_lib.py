"""ctypes binding of libpmb200.so (the C ABI in include/pmb200.h).

The library is built in-tree (``python -m protomoladdon_b200.build`` or
``__graft_entry__.build()``).  There is no CPU fallback: loading fails with
an error when the shared library is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmb200.so")

PMB200_OK = 0
PMB200_EINVAL = 1
PMB200_ECUDA = 2
PMB200_ESTATE = 3
PMB200_EUNSUPPORTED = 4
PMB200_EDEVICE = 5
PMB200_ENOMEM = 6

PMB200_MIXED = 0
PMB200_FP64 = 1

PMB200_ENERGY = 1
PMB200_VIRIAL = 2
PMB200_MOLVIRIAL = 4

PMB200_SW_NONE = 0
PMB200_SW_C1 = 1
PMB200_SW_C2 = 2
PMB200_SW_CN = 3
PMB200_SW_CMPCNCN = 4
PMB200_SW_TABLE = 16  # flag on the LJ switch: LennardJonesTableForce

PMB200_KERNEL_SEARCH = 0
PMB200_KERNEL_TILES = 1
PMB200_KERNEL_CLUSTERS = 2

PMB200_ERFC_POLY5 = 0
PMB200_ERFC_EXACT = 1

# Every symbol include/pmb200.h declares.
EXPORTED = (
    "pmb200_create", "pmb200_destroy", "pmb200_last_error", "pmb200_set_topology",
    "pmb200_set_box", "pmb200_eval", "pmb200_eval_device", "pmb200_sync",
    "pmb200_leapfrog_device", "pmb200_last_pair_count", "pmb200_grid",
    "pmb200_step_device", "pmb200_set_kernel_timing", "pmb200_last_kernel_ms",
    "pmb200_measure_fp32_peak", "pmb200_set_rigid_waters", "pmb200_host_kick_drift",
    "pmb200_autotune", "pmb200_set_pair_kernel",
    "pmb200_eval_noalloc", "pmb200_create_ewald_real", "pmb200_ewald_info",
    "pmb200_param_grad_device", "pmb200_hvp_device", "pmb200_update_params",
    "pmb200_update_params_device",
    "pmb200_batch_create", "pmb200_batch_destroy", "pmb200_batch_last_error",
    "pmb200_batch_eval_device", "pmb200_batch_set_schedule", "pmb200_batch_get_schedule",
    "pmb200_batch_autotune", "pmb200_batch_set_kernel_timing", "pmb200_batch_last_kernel_ms",
    "pmb200_batch_pair_counts", "pmb200_create_pair", "pmb200_set_vacuum_domain",
    "pmb200_batch_sync", "pmb200_shard_eval_device", "pmb200_shard_finalize",
    "pmb200_eval_cells",
)

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int


class Params(ctypes.Structure):
    _fields_ = [("precision", _I), ("device", _I), ("switchon", _D), ("cutoff_lj", _D),
                ("cutoff_coul", _D), ("cutoff_alg", _D), ("cellsize", _D)]


class EwaldParams(ctypes.Structure):
    _fields_ = [("precision", _I), ("device", _I), ("erfc", _I), ("alpha", _D),
                ("accuracy", _D), ("cellsize", _D)]


class PairParams(ctypes.Structure):
    _fields_ = [("precision", _I), ("device", _I), ("lj_switch", _I), ("lj", _D * 4),
                ("coulomb_switch", _I), ("coulomb", _D * 4), ("cutoff_alg", _D),
                ("cellsize", _D)]


class PmbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pmb200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Loads libpmb200.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libpmb200.so not found at {LIB_PATH}; build it with "
            "`python -m protomoladdon_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.pmb200_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(_P)]
    L.pmb200_destroy.argtypes = [_P]
    L.pmb200_last_error.argtypes = [_P]
    L.pmb200_last_error.restype = ctypes.c_char_p
    L.pmb200_set_topology.argtypes = [_P, _I, _P, _P, _P, _P, _I, _P, _I, _P, _D]
    L.pmb200_set_box.argtypes = [_P, _P, _P, _P, _P]
    L.pmb200_eval.argtypes = [_P, _P, _P, _P, _P, _P, ctypes.c_uint]
    L.pmb200_eval_device.argtypes = [_P, _P, _P, _P, ctypes.c_uint, _P]
    L.pmb200_shard_eval_device.argtypes = [_P, _P, _I, _I, _P, _P, ctypes.c_uint, _P]
    L.pmb200_shard_finalize.argtypes = [_P, _P, _P, _P]
    L.pmb200_sync.argtypes = [_P]
    L.pmb200_leapfrog_device.argtypes = [_P, _P, _P, _P, _P, _D, _I, ctypes.c_uint, _P]
    L.pmb200_last_pair_count.argtypes = [_P, ctypes.POINTER(ctypes.c_longlong)]
    L.pmb200_grid.argtypes = [_P, ctypes.POINTER(_I), ctypes.POINTER(_D)]
    L.pmb200_step_device.argtypes = [_P, _P, _P, _P, _P, _D, ctypes.c_uint, _P]
    L.pmb200_set_kernel_timing.argtypes = [_P, _I]
    L.pmb200_last_kernel_ms.argtypes = [_P, ctypes.POINTER(ctypes.c_float)]
    L.pmb200_measure_fp32_peak.argtypes = [_I, ctypes.POINTER(_D)]
    L.pmb200_set_rigid_waters.argtypes = [_P, _I, _P, _D, _D]
    L.pmb200_host_kick_drift.argtypes = [_I, _P, _P, _P, _P, _D, _D, _I, _P, _D, _D, _I]
    L.pmb200_autotune.argtypes = [_P, _P, _P, _I, _P]
    L.pmb200_set_pair_kernel.argtypes = [_P, _I]
    L.pmb200_eval_noalloc.argtypes = [ctypes.POINTER(Params), _I, _P, _P, _P, _P, _P, _P, _I, _P,
                                      _D, _P, _P, _P, _P, _P, _P]
    L.pmb200_create_ewald_real.argtypes = [ctypes.POINTER(EwaldParams), ctypes.POINTER(_P)]
    L.pmb200_ewald_info.argtypes = [_P, ctypes.POINTER(_D), ctypes.POINTER(_D)]
    L.pmb200_param_grad_device.argtypes = [_P, _P, _P, _P, _P]
    L.pmb200_hvp_device.argtypes = [_P, _P, _P, _P, _P, _P, _P]
    L.pmb200_update_params.argtypes = [_P, _P, _P]
    L.pmb200_update_params_device.argtypes = [_P, _P, _P, _P]
    L.pmb200_set_vacuum_domain.argtypes = [_P, _P, _P]
    L.pmb200_eval_cells.argtypes = [_P, _P, _P, _P, _P, _P, ctypes.c_uint, _I, _I]
    L.pmb200_create_pair.argtypes = [ctypes.POINTER(PairParams), ctypes.POINTER(_P)]
    L.pmb200_batch_create.argtypes = [ctypes.POINTER(_P), _I, ctypes.POINTER(_P)]
    L.pmb200_batch_destroy.argtypes = [_P]
    L.pmb200_batch_last_error.argtypes = [_P]
    L.pmb200_batch_last_error.restype = ctypes.c_char_p
    L.pmb200_batch_eval_device.argtypes = [_P, _P, _P, _P, ctypes.c_uint, _P]
    L.pmb200_batch_set_schedule.argtypes = [_P, _I, _I, _I]
    L.pmb200_batch_get_schedule.argtypes = [_P, ctypes.POINTER(_I)]
    L.pmb200_batch_autotune.argtypes = [_P, _P, _P, _I, ctypes.POINTER(_I),
                                        ctypes.POINTER(ctypes.c_float)]
    L.pmb200_batch_set_kernel_timing.argtypes = [_P, _I]
    L.pmb200_batch_last_kernel_ms.argtypes = [_P, ctypes.POINTER(ctypes.c_float)]
    L.pmb200_batch_sync.argtypes = [_P, _P]
    L.pmb200_batch_pair_counts.argtypes = [_P, ctypes.POINTER(ctypes.c_longlong)]
    for name in EXPORTED:
        getattr(L, name).restype = getattr(L, name).restype or _I
    L.pmb200_last_error.restype = ctypes.c_char_p
    L.pmb200_batch_last_error.restype = ctypes.c_char_p
    _lib = L
    return L
