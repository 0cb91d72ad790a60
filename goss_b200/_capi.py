"""ctypes binding of the C ABI in ``include/goss_b200.h``.

The runtime library ``goss_b200/_lib/libgoss_b200.so`` is required: there is
no CPU implementation behind this package, so a missing or unloadable
library raises :class:`ExtensionMissingError` instead of falling back.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
RUNTIME_SO = PKG / "_lib" / "libgoss_b200.so"

ABI_VERSION = 4

(GOSS_EXPLICIT_EULER, GOSS_RK4, GOSS_GRL1, GOSS_GRL2, GOSS_THETA, GOSS_ESDIRK23A, GOSS_RL1, GOSS_RL2, GOSS_RK2,
 GOSS_IMPLICIT_EULER) = range(10)
GOSS_FP64, GOSS_FP32, GOSS_FP64_PRINTED = 0, 1, 2
GOSS_OK, GOSS_ERR_ARGUMENT, GOSS_ERR_CUDA, GOSS_ERR_NEWTON, GOSS_ERR_UNSUPPORTED, GOSS_ERR_TIMEOUT = range(6)
GOSS_FLAG_NONFINITE, GOSS_FLAG_NEWTON_FAILED, GOSS_FLAG_ITERATION_CAP = 1, 2, 4

SOLVER_KINDS = {
    "ExplicitEuler": GOSS_EXPLICIT_EULER,
    "RK4": GOSS_RK4,
    "GRL1": GOSS_GRL1,
    "GRL2": GOSS_GRL2,
    "ThetaSolver": GOSS_THETA,
    "ESDIRK23a": GOSS_ESDIRK23A,
    "RL1": GOSS_RL1,
    "RL2": GOSS_RL2,
    "RK2": GOSS_RK2,
    "ImplicitEuler": GOSS_IMPLICIT_EULER,
}


class ExtensionMissingError(RuntimeError):
    """The compiled goss_b200 CUDA library is not available."""


class GossError(RuntimeError):
    """An error status returned by the goss_b200 runtime."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class SolverParams(C.Structure):
    _fields_ = [
        ("ldt", C.c_double),
        ("delta", C.c_double),
        ("eta_0", C.c_double),
        ("kappa", C.c_double),
        ("relative_tolerance", C.c_double),
        ("max_relative_previous_residual", C.c_double),
        ("max_iterations", C.c_int32),
        ("always_recompute_jacobian", C.c_int32),
        ("num_refinements_without_always_recomputing_jacobian", C.c_int32),
        ("min_dt", C.c_double),
        ("theta", C.c_double),
    ]


class ModelDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("name", C.c_char_p),
        ("num_states", C.c_uint32),
        ("num_parameters", C.c_uint32),
        ("num_field_parameters", C.c_uint32),
        ("num_monitored", C.c_uint32),
        ("state_names", C.POINTER(C.c_char_p)),
        ("parameter_names", C.POINTER(C.c_char_p)),
        ("field_parameter_names", C.POINTER(C.c_char_p)),
        ("field_parameter_indices", C.POINTER(C.c_uint32)),
        ("initial_conditions", C.POINTER(C.c_double)),
        ("default_parameters", C.POINTER(C.c_double)),
        ("linear_terms", C.POINTER(C.c_uint8)),
        ("supported_solvers", C.c_uint32),
        ("launch", C.c_void_p),
        ("eval", C.c_void_p),
        ("solver_state_rows", C.CFUNCTYPE(C.c_uint32, C.c_int32)),
        ("op_census_linearized", C.POINTER(C.c_uint32)),
        ("op_census_rhs", C.POINTER(C.c_uint32)),
        ("adjoint", C.c_void_p),
        ("has_jacobian", C.c_uint32),
        ("lu_nnz", C.c_uint32),
    ]


class AdjointLaunch(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("solver", C.c_int32),
        ("precision", C.c_int32),
        ("num_nodes", C.c_uint32),
        ("block", C.c_uint32),
        ("ld", C.c_uint64),
        ("states", C.c_void_p),
        ("field_params", C.c_void_p),
        ("params", C.POINTER(C.c_double)),
        ("t0", C.c_double),
        ("interval", C.c_double),
        ("num_intervals", C.c_uint32),
        ("steps_per_interval", C.c_uint32),
        ("checkpoint_every", C.c_uint32),
        ("trace_state", C.c_uint32),
        ("checkpoints", C.c_void_p),
        ("trace", C.c_void_p),
        ("trace_bar", C.c_void_p),
        ("scratch", C.c_void_p),
        ("field_params_bar", C.c_void_p),
        ("states_bar", C.c_void_p),
        ("flags", C.c_void_p),
        ("stream", C.c_void_p),
        ("tape", C.c_void_p),
        ("taped_segments", C.c_uint32),
        ("reverse_precision", C.c_int32),
    ]


class BatchDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("name", C.c_char_p),
        ("num_kinds", C.c_uint32),
        ("kind_variants", C.POINTER(C.c_char_p)),
        ("kind_solvers", C.POINTER(C.c_int32)),
        ("kind_num_states", C.POINTER(C.c_uint32)),
        ("launch", C.c_void_p),
    ]


_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)
_sys = C.c_void_p
_desc = C.POINTER(ModelDesc)

_PROTOS = {
    "goss_abi_version": (C.c_uint32, []),
    "goss_measure_peaks": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "goss_measure_fp64_peak": (C.c_int, [C.c_int32, C.POINTER(C.c_double)]),
    "goss_last_error": (C.c_char_p, []),
    "goss_system_last_error": (C.c_char_p, [_sys]),
    "goss_solver_default_params": (C.c_int, [C.c_int32, C.POINTER(SolverParams)]),
    "goss_system_create": (C.c_int, [_desc, C.c_int32, C.POINTER(SolverParams), C.c_uint32, C.c_int32, C.c_int32,
                                     C.POINTER(C.c_void_p)]),
    "goss_system_destroy": (C.c_int, [_sys]),
    "goss_system_set_solver_params": (C.c_int, [_sys, C.POINTER(SolverParams)]),
    "goss_system_get_solver_params": (C.c_int, [_sys, C.POINTER(SolverParams)]),
    "goss_system_forward": (C.c_int, [_sys, C.c_double, C.c_double]),
    "goss_system_forward_async": (C.c_int, [_sys, C.c_double, C.c_double]),
    "goss_system_synchronize": (C.c_int, [_sys]),
    "goss_system_solve": (C.c_int, [_sys, _dp, _dp, C.c_uint64, C.c_int32]),
    "goss_system_set_field_state_indices": (C.c_int, [_sys, _u32p, C.c_uint32]),
    "goss_system_get_field_states": (C.c_int, [_sys, _dp, C.c_int32]),
    "goss_system_set_field_states": (C.c_int, [_sys, _dp, C.c_int32]),
    "goss_system_get_field_state_components": (C.c_int, [_sys, _dp, C.c_uint32, _u32p, C.c_int32]),
    "goss_system_set_field_state_components": (C.c_int, [_sys, _dp, C.c_uint32, _u32p, C.c_int32]),
    "goss_system_get_field_parameters": (C.c_int, [_sys, _dp, C.c_int32]),
    "goss_system_set_field_parameters": (C.c_int, [_sys, _dp, C.c_int32]),
    "goss_system_get_states": (C.c_int, [_sys, _dp]),
    "goss_system_set_states": (C.c_int, [_sys, _dp]),
    "goss_system_set_parameter": (C.c_int, [_sys, C.c_uint32, C.c_double]),
    "goss_system_get_parameter": (C.c_int, [_sys, C.c_uint32, _dp]),
    "goss_system_reset_default": (C.c_int, [_sys]),
    "goss_system_set_num_threads": (C.c_int, [_sys, C.c_uint32]),
    "goss_system_get_num_threads": (C.c_uint32, [_sys]),
    "goss_system_num_nodes": (C.c_uint32, [_sys]),
    "goss_system_set_block_size": (C.c_int, [_sys, C.c_uint32]),
    "goss_system_status": (C.c_int, [_sys, _u32p, C.c_int32]),
    "goss_system_node_status": (C.c_int, [_sys, C.POINTER(C.c_uint8)]),
    "goss_system_counters": (C.c_int, [_sys, _i64p, _i64p, _i64p]),
    "goss_system_device_states": (C.c_int, [_sys, C.POINTER(_dp), C.POINTER(C.c_uint64)]),
    "goss_system_device_field_params": (C.c_int, [_sys, C.POINTER(_dp), C.POINTER(C.c_uint64)]),
    "goss_system_set_stream": (C.c_int, [_sys, C.c_void_p]),
    "goss_system_capture": (C.c_int, [_sys, C.c_double, C.c_double, C.c_uint32]),
    "goss_system_replay": (C.c_int, [_sys]),
    "goss_batch_create": (C.c_int, [C.POINTER(BatchDesc), C.POINTER(C.c_void_p), C.POINTER(C.c_int32), C.c_uint32,
                                    C.c_int32, C.POINTER(C.c_void_p)]),
    "goss_batch_destroy": (C.c_int, [C.c_void_p]),
    "goss_batch_set_config": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, _u32p]),
    "goss_batch_set_forwards_per_launch": (C.c_int, [C.c_void_p, C.c_uint32]),
    "goss_batch_forward": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "goss_batch_capture": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_uint32]),
    "goss_batch_replay": (C.c_int, [C.c_void_p]),
    "goss_batch_time": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_uint32, C.c_int32,
                                  C.POINTER(C.c_float)]),
    "goss_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "goss_model_eval_noalloc":(C.c_int, [_desc, C.c_int32, C.c_int32, _dp, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_uint64, C.c_void_p, C.c_void_p]),
    "goss_model_eval_noalloc_capacity": (C.c_uint64, []),
    "goss_lu_factorize": (C.c_int, [C.c_uint32, _dp]),
    "goss_forward_backward_subst": (C.c_int, [C.c_uint32, _dp, _dp, _dp]),
    "goss_model_eval": (C.c_int, [_desc, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp, C.c_uint64, _dp, C.c_int32]),
}

#: every function the header declares (checked by the tests)
EXPORTED = sorted(_PROTOS)

_lib = None


def lib():
    """Load the runtime library once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not RUNTIME_SO.exists():
            raise ExtensionMissingError(
                f"{RUNTIME_SO} is missing; build it with goss_b200.build.build_runtime() "
                "(python -c 'import __graft_entry__ as g; g.build()')")
        try:
            handle = C.CDLL(str(RUNTIME_SO))
        except OSError as exc:
            raise ExtensionMissingError(f"cannot load {RUNTIME_SO}: {exc}") from exc
        for name, (res, args) in _PROTOS.items():
            f = getattr(handle, name)
            f.restype = res
            f.argtypes = args
        if handle.goss_abi_version() != ABI_VERSION:
            raise ExtensionMissingError("libgoss_b200.so was built for another ABI version")
        _lib = handle
    return _lib


def check(rc: int, sys_handle=None) -> None:
    """Raise the exception that corresponds to a status code."""
    if rc == GOSS_OK:
        return
    L = lib()
    msg = L.goss_system_last_error(sys_handle).decode() if sys_handle else ""
    if not msg:
        msg = L.goss_last_error().decode()
    if rc == GOSS_ERR_ARGUMENT:
        raise ValueError(msg)
    raise GossError(rc, msg)


def ptr(a):
    """double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(_dp)
