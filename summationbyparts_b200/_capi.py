"""ctypes binding of libsbp_b200.so (the C ABI declared in include/sbp_b200.h).

The library is loaded from summationbyparts_b200/_lib/ on first use (so the package can be
imported to build it).  There is no fallback: if the shared library is missing or fails to
load, the first call raises, so a run can never silently compute on the CPU.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsbp_b200.so")

SBP_OK = 0
STATUS_NAMES = {0: "SBP_OK", 1: "SBP_ERR_INVALID_ARGUMENT", 2: "SBP_ERR_SHAPE", 3: "SBP_ERR_UNSUPPORTED",
                4: "SBP_ERR_CUDA", 5: "SBP_ERR_NONPHYSICAL", 6: "SBP_ERR_NO_DEVICE", 7: "SBP_ERR_OUT_OF_MEMORY"}

F64, F32 = 0, 1
PRECISION_F64, PRECISION_F32_COMPENSATED = 0, 1
BC_THIS, BC_GRID, BC_VORTEX, BC_INTERPOLATE, BC_MULTIGRID, BC_EVAL = 0, 1, 2, 3, 4, 5
EVAL_CONSERVATION, EVAL_PRESSURE = 0, 1
INTERP4, INTERP8, INTERP9, INTERP9H2 = 0, 1, 2, 3
TABLEAUS = {"rk4": 0, "rk4_38": 1, "euler": 2, "midpoint": 3, "rk6": 4, "fehlberg": 5, "bogacki_shampine": 6}
NORTH, SOUTH, EAST, WEST = 0, 1, 2, 3


class SbpError(RuntimeError):
    """A C-ABI call returned a status other than SBP_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class VortexParams(ctypes.Structure):
    _fields_ = [("nvortices", ctypes.c_int), ("x0", ctypes.c_double * 5), ("y0", ctypes.c_double * 5),
                ("rstar", ctypes.c_double * 5), ("eps", ctypes.c_double * 5), ("mach", ctypes.c_double)]


class BlockDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("op_xi", ctypes.c_int), ("op_eta", ctypes.c_int),
                ("x", ctypes.POINTER(ctypes.c_double)), ("y", ctypes.POINTER(ctypes.c_double)),
                ("bc_kind", ctypes.c_int * 4), ("bc_neighbour", ctypes.c_int * 4), ("instance", ctypes.c_int),
                ("bc_interp_op", ctypes.c_int * 4), ("bc_multigrid_count", ctypes.c_int * 4),
                ("bc_multigrid", ctypes.POINTER(ctypes.c_int) * 4)]


_i, _i64, _d, _vp = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)

# name: (restype, argtypes)
SIGNATURES = {
    "sbp_last_error": (ctypes.c_char_p, []),
    "sbp_version": (ctypes.c_char_p, []),
    "sbp_operator_h": (_i, [_i, _dp, _i]),
    "sbp_operator_is_h2": (_i, [_i]),
    "sbp_operator_is_upwind": (_i, [_i]),
    "sbp_operator_table": (_i, [_i, _i, _i, _dp, _i]),
    "sbp_diffxi": (_i, [_i, _i, _vp, _vp, _i64, _i64, _i64, _i64, _vp]),
    "sbp_diffeta": (_i, [_i, _i, _vp, _vp, _i64, _i64, _i64, _i64, _vp]),
    "sbp_dissxi": (_i, [_i, _i, _vp, _vp, _i64, _i64, _i64, _i64, _vp]),
    "sbp_interpolate": (_i, [_i, _i, _i, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp]),
    "sbp_disseta": (_i, [_i, _i, _vp, _vp, _i64, _i64, _i64, _i64, _vp]),
    "sbp_metrics": (_i, [_i, _i, _vp, _vp, _i64, _i64, _vp, _vp]),
    "sbp_metrics_noalloc": (_i, [_i, _i, _vp, _vp, _i64, _i64, _vp, _vp]),
    "sbp_system_create": (_i, [_i, ctypes.POINTER(BlockDesc), _i, _i, _i, _d, ctypes.POINTER(_vp)]),
    "sbp_system_destroy": (_i, [_vp]),
    "sbp_system_set_force_trad": (_i, [_vp, _i]),
    "sbp_system_set_vortex": (_i, [_vp, _i, ctypes.POINTER(VortexParams)]),
    "sbp_system_init_vortex": (_i, [_vp, _i, _d]),
    "sbp_system_set_state": (_i, [_vp, _i, _dp]),
    "sbp_system_get_state": (_i, [_vp, _i, _dp]),
    "sbp_system_set_state_all": (_i, [_vp, _i, _vp]),
    "sbp_system_get_state_all": (_i, [_vp, _i, _vp]),
    "sbp_system_get_state_all_device": (_i, [_vp, _i, _vp]),
    "sbp_system_advance_host": (_i, [_vp, _i, _vp, _vp, _i64, _i]),
    "sbp_system_set_eval": (_i, [_vp, _i, ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(ctypes.c_int32), _dp, _i]),
    "sbp_system_advance_host_chunks": (_i, [_vp]),
    "sbp_system_state_count": (_i64, [_vp, _i]),
    "sbp_system_set_dt": (_i, [_vp, _i, _d]),
    "sbp_system_set_time": (_i, [_vp, _i, _d]),
    "sbp_system_get_time": (_i, [_vp, _i, _dp]),
    "sbp_system_max_dt": (_i, [_vp, _i, _dp]),
    "sbp_system_advance": (_i, [_vp, _i64]),
    "sbp_system_advance_instances": (_i, [_vp, ctypes.POINTER(_i64)]),
    "sbp_system_error": (_i, [_vp, _dp]),
    "sbp_system_h2_err": (_i, [_vp, _i, _dp, _dp]),
    "sbp_system_set_tiles": (_i, [_vp, _i, _i, _i]),
    "sbp_system_autotune": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sbp_system_group_tiles": (_i, [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sbp_system_set_stream": (_i, [_vp, _vp]),
    "sbp_system_device_state": (_i, [_vp, _i, ctypes.POINTER(_vp)]),
    "sbp_system_launches_per_step": (_i, [_vp]),
    "sbp_system_advance_tableau": (_i, [_vp, _i, _i64]),
    "sbp_system_advance_adaptive": (_i, [_vp, _d, _dp, _d]),
    "sbp_system_group_count": (_i, [_vp]),
    "sbp_system_group_info": (_i, [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i64)]),
    "sbp_system_launch_stage": (_i, [_vp, _i, _i, _i]),
    "sbp_cnn_create": (_i, [_i, _i, ctypes.c_ulonglong, ctypes.POINTER(_vp)]),
    "sbp_cnn_destroy": (_i, [_vp]),
    "sbp_cnn_set_stream": (_i, [_vp, _vp]),
    "sbp_cnn_synchronize": (_i, [_vp]),
    "sbp_cnn_param_count": (_i64, [_vp]),
    "sbp_cnn_get_params": (_i, [_vp, _vp]),
    "sbp_cnn_set_params": (_i, [_vp, _vp]),
    "sbp_cnn_set_normalisation": (_i, [_vp, _vp, _vp, _vp]),
    "sbp_cnn_forward": (_i, [_vp, _i, _vp, _i, _i64]),
    "sbp_cnn_output": (_i, [_vp, _i, _vp]),
    "sbp_cnn_gradients": (_i, [_vp, _i, _vp, _i, _i64, _vp, ctypes.POINTER(ctypes.c_float), _vp]),
    "sbp_cnn_train_step": (_i, [_vp, _i, _vp, _i, _i64, _vp, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
    "sbp_cnn_apply": (_i, [_vp, _i, _vp, _i, _i64, _vp]),
    "sbp_restrict_linspace": (_i, [_i, _i, _i, _vp, _vp, _vp]),
    "sbp_rel_l2_images": (_i, [_i, _i64, _vp, _i, _i64, _vp, _i, _i64, _vp, _vp]),
}


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m summationbyparts_b200.build` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


class _Library:
    """Loads libsbp_b200.so on first attribute access."""

    _handle = None

    def __getattr__(self, name):
        if _Library._handle is None:
            _Library._handle = _load()
        return getattr(_Library._handle, name)


lib = _Library()


def check(status: int) -> None:
    if status != SBP_OK:
        raise SbpError(status, lib.sbp_last_error().decode(errors="replace"))


def version() -> str:
    return lib.sbp_version().decode()
