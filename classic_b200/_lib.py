"""ctypes binding of the C ABI in include/claw_b200.h.

The CUDA library (``libclawb200.so``) is built in-tree by
``classic_b200.build.build_library`` and loaded from this package directory.
There is no fallback: if the library is missing or fails to load, importing a
solver raises immediately.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclawb200.so")

CLAW_MAX_WAVES = 8

SOLVER_IDS = {
    "acoustics_2d": 1,
    "vc_advection_2d": 2,
    "euler_roe_2d": 3,
    "acoustics_1d": 11,
    "vc_acoustics_1d": 12,
    "advection_1d": 13,
    "euler_roe_1d": 14,
    "vc_acoustics_3d": 21,
}

PRECISIONS = {"fp64": 0, "fp64_fma": 1, "fp32": 2}

ERRORS = {-1: "CLAW_E_INVALID", -2: "CLAW_E_CUDA", -3: "CLAW_E_UNSUPPORTED",
          -4: "CLAW_E_DEVICE", -5: "CLAW_E_NAN"}


class ClawConfig(ctypes.Structure):
    _fields_ = [
        ("num_dim", ctypes.c_int),
        ("num_cells", ctypes.c_int * 3),
        ("lower", ctypes.c_double * 3),
        ("upper", ctypes.c_double * 3),
        ("num_eqn", ctypes.c_int),
        ("num_waves", ctypes.c_int),
        ("num_aux", ctypes.c_int),
        ("capa_index", ctypes.c_int),
        ("dt_variable", ctypes.c_int),
        ("order", ctypes.c_int),
        ("transverse_waves", ctypes.c_int),
        ("dimensional_split", ctypes.c_int),
        ("verbosity", ctypes.c_int),
        ("source_split", ctypes.c_int),
        ("use_fwaves", ctypes.c_int),
        ("limiter", ctypes.c_int * CLAW_MAX_WAVES),
        ("num_ghost", ctypes.c_int),
        ("bc_lower", ctypes.c_int * 3),
        ("bc_upper", ctypes.c_int * 3),
        ("dt_initial", ctypes.c_double),
        ("dt_max", ctypes.c_double),
        ("cfl_max", ctypes.c_double),
        ("cfl_desired", ctypes.c_double),
        ("steps_max", ctypes.c_int),
        ("solver_id", ctypes.c_int),
        ("solver_params", ctypes.c_double * 8),
        ("precision", ctypes.c_int),
        ("source_id", ctypes.c_int),
        ("source_ndim", ctypes.c_int),
        ("b4step_id", ctypes.c_int),
        ("reserved", ctypes.c_int * 2),
        ("b4step_param", ctypes.c_double),
    ]


class ClawStats(ctypes.Structure):
    _fields_ = [
        ("t_reached", ctypes.c_double),
        ("dt_min", ctypes.c_double),
        ("dt_max_taken", ctypes.c_double),
        ("dt_next", ctypes.c_double),
        ("cfl_max_seen", ctypes.c_double),
        ("cfl_last", ctypes.c_double),
        ("steps_taken", ctypes.c_int),
        ("steps_rejected", ctypes.c_int),
        ("info", ctypes.c_int),
        ("device_error", ctypes.c_int),
        ("device_ms", ctypes.c_double),
        ("launches", ctypes.c_longlong),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# Every symbol declared in include/claw_b200.h, with its ctypes signature.
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "claw_create": (ctypes.c_int, [ctypes.POINTER(ClawConfig), ctypes.POINTER(_P)]),
    "claw_destroy": (ctypes.c_int, [_P]),
    "claw_set_q": (ctypes.c_int, [_P, _D]),
    "claw_get_q": (ctypes.c_int, [_P, _D]),
    "claw_set_aux": (ctypes.c_int, [_P, _D]),
    "claw_step": (ctypes.c_int, [_P, ctypes.c_double, _D]),
    "claw_advance": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.POINTER(ClawStats)]),
    "claw_advance_host": (ctypes.c_int, [_P, _D, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.POINTER(ClawStats)]),
    "claw_q_device": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_longlong),
                                     ctypes.POINTER(ctypes.c_longlong)]),
    "claw_launch_count": (ctypes.c_longlong, [_P]),
    "claw_debug_fault": (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.c_int]),
    "claw_set_steps_max": (ctypes.c_int, [_P, ctypes.c_int]),
    "claw_totals": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double)]),
    "claw_step2d_noalloc": (ctypes.c_int, [ctypes.POINTER(ClawConfig), _P, _P, ctypes.c_longlong,
                                           _P, ctypes.c_longlong, ctypes.c_double, _D, _P]),
    "claw_batch_create": (ctypes.c_int, [ctypes.POINTER(ClawConfig), ctypes.c_int,
                                         ctypes.POINTER(_P)]),
    "claw_batch_destroy": (ctypes.c_int, [_P]),
    "claw_batch_set_q": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "claw_batch_get_q": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "claw_batch_autotune": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_double)]),
    "claw_batch_set_shape": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "claw_batch_advance": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _D,
                                          ctypes.POINTER(ClawStats)]),
    "claw_last_error": (ctypes.c_char_p, []),
    "claw_probe_fp64": (ctypes.c_int, [_D, _D]),
    "claw_check_newton": (ctypes.c_int, [_D, ctypes.c_int, _D, _D]),
    # learned corrector kernels (include/claw_nn.h)
    "nn_conv3x3_forward": (ctypes.c_int, [_P, _P, _P, _P, _P] + [ctypes.c_int] * 7 + [_P]),
    "nn_conv3x3_wgrad": (ctypes.c_int, [_P] * 6 + [ctypes.c_int] * 5 + [_P]),
    "nn_device_error": (ctypes.c_int, [ctypes.c_int]),
    "nn_flip_weights": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, _P]),
    "nn_gelu_backward": (ctypes.c_int, [_P, _P, _P, ctypes.c_longlong, _P]),
    "nn_mse_grad": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_float, _P]),
    "nn_adam": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_longlong] + [ctypes.c_float] * 4 +
                [ctypes.c_int, _P]),
    "nn_block_average": (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.c_longlong, _P,
                                        ctypes.c_longlong, ctypes.c_longlong] + [ctypes.c_int] * 4 +
                         [_P]),
    "nn_features": (ctypes.c_int, [_P, _P, ctypes.c_longlong, ctypes.c_longlong] +
                    [ctypes.c_int] * 3 + [_P, _P, _P]),
    "nn_residual_target": (ctypes.c_int, [_P, _P, ctypes.c_longlong, ctypes.c_longlong] +
                           [ctypes.c_int] * 3 + [_P, _P, _P]),
    "nn_apply_correction": (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int,
                                           ctypes.c_int, _P, ctypes.c_int, _P, ctypes.c_double,
                                           ctypes.c_double, _P, _P]),
    "claw_build_info": (ctypes.c_char_p, []),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libclawb200.so (once) and attach the C signatures.  Raises
    OSError when the library is absent: there is no CPU path."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(
            f"{path} is missing: build it with classic_b200.build.build_library() "
            "(nvcc, sm_100a); there is no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class ClawError(RuntimeError):
    def __init__(self, code: int, where: str):
        lib = _lib
        msg = lib.claw_last_error().decode() if lib is not None else ""
        name = ERRORS.get(code, f"info={code}")
        super().__init__(f"{where}: {name} ({code}) {msg}")
        self.code = code


def check(code: int, where: str):
    if code < 0:
        raise ClawError(code, where)
    return code
