"""ctypes binding of the C ABI in include/orchard_b200.h.

The library is built in-tree (``solver_b200/liborchard_b200.so``, see
``solver_b200/Makefile``).  There is no CPU fallback: if the library or a GPU
is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborchard_b200.so")

OF_OK, OF_INVALID_ARGUMENT, OF_RUNTIME_ERROR, OF_NOT_CONVERGED, OF_NONFINITE, OF_CUDA_ERROR, \
    OF_TIMEOUT = range(7)
OF_FP64, OF_MIXED = 0, 1
OF_CORRECTION_TAYLOR_GREEN, OF_CORRECTION_CAVITY = 0, 1

EXPORTED_SYMBOLS = (
    "of_abi_version", "of_last_error", "of_create", "of_destroy", "of_set_precision",
    "of_device_bytes", "of_compute_advection_term", "of_solve_predictor_adi",
    "of_solve_pressure_poisson", "of_project_velocity", "of_state_upload", "of_state_download",
    "of_tg_init", "of_run_steps", "of_stream", "of_kernel_class_count", "of_kernel_class_name",
    "of_profile_enable", "of_profile_reset", "of_profile_read", "of_tangent_linear",
    "of_adjoint_gradient", "of_pressure_rhs_noalloc", "of_step_host",
    "of_adjoint_gradient_binomial", "of_adjoint_schedule_cost", "of_profile_coarse_chain",
)


class OfGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class OfFaceBC(C.Structure):
    _fields_ = [("type", C.c_int), ("velocity", C.c_double * 3), ("pressure", C.c_double),
                ("pressure_gradient", C.c_double)]


class OfBC(C.Structure):
    _fields_ = [("faces", OfFaceBC * 6)]


class OfPFaceBC(C.Structure):
    _fields_ = [("type", C.c_int), ("value", C.c_double), ("gradient", C.c_double)]


class OfPBC(C.Structure):
    _fields_ = [("faces", OfPFaceBC * 6)]


class OfPoissonDiag(C.Structure):
    _fields_ = [("iterations", C.c_int), ("initial_residual_l2", C.c_double),
                ("final_residual_l2", C.c_double), ("relative_residual", C.c_double),
                ("removed_rhs_mean", C.c_double), ("multigrid_levels", C.c_int),
                ("coarse_unknowns", C.c_int), ("pre_smoothing_steps", C.c_int),
                ("post_smoothing_steps", C.c_int), ("converged", C.c_int),
                ("zero_mean_enforced", C.c_int)]


class OfProjectionDiag(C.Structure):
    _fields_ = [("rhs_l2", C.c_double), ("divergence_l2_before", C.c_double),
                ("divergence_l2_after", C.c_double), ("pressure_mean", C.c_double),
                ("pressure_solve", OfPoissonDiag)]


class OfStepMetrics(C.Structure):
    _fields_ = [("step", C.c_int), ("time", C.c_double), ("dt", C.c_double),
                ("max_cfl", C.c_double), ("max_velocity_change", C.c_double),
                ("divergence_l2", C.c_double), ("max_divergence_l2", C.c_double),
                ("pressure_iterations", C.c_int), ("pressure_relative_residual", C.c_double)]


class OfStepParams(C.Structure):
    _fields_ = [("viscosity", C.c_double), ("dt", C.c_double), ("density", C.c_double),
                ("poisson_max_iterations", C.c_int), ("poisson_tolerance", C.c_double),
                ("correction_variant", C.c_int), ("track_max_divergence", C.c_int),
                ("solver_name", C.c_char_p)]


class OfAdjointInfo(C.Structure):
    _fields_ = [("loss", C.c_double), ("grad_viscosity", C.c_double), ("forward_steps", C.c_int),
                ("forward_ms", C.c_double), ("backward_ms", C.c_double),
                ("device_bytes", C.c_size_t), ("snapshots", C.c_int),
                ("device_bytes_in_use", C.c_size_t)]


DP = C.POINTER(C.c_double)

_lib = None


def load():
    """Loads the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C solver_b200` "
                "(the B200 path has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        lib.of_last_error.restype = C.c_char_p
        lib.of_create.argtypes = [C.POINTER(OfGrid), C.POINTER(OfBC), C.c_int, C.POINTER(C.c_void_p)]
        lib.of_destroy.argtypes = [C.c_void_p]
        lib.of_set_precision.argtypes = [C.c_void_p, C.c_int]
        lib.of_device_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
        lib.of_compute_advection_term.argtypes = [C.c_void_p] + [DP] * 6
        lib.of_solve_predictor_adi.argtypes = [C.c_void_p, C.c_double] + [DP] * 6 + [C.POINTER(C.c_int)]
        lib.of_solve_pressure_poisson.argtypes = [C.c_void_p, C.POINTER(OfPBC), C.c_int, C.c_double,
                                                  DP, DP, C.POINTER(OfPoissonDiag), DP, C.c_int]
        lib.of_project_velocity.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int,
                                            C.c_double] + [DP] * 8 + [C.POINTER(OfProjectionDiag)]
        lib.of_state_upload.argtypes = [C.c_void_p] + [DP] * 7 + [C.c_int, C.POINTER(OfStepMetrics)]
        lib.of_state_download.argtypes = [C.c_void_p] + [DP] * 7 + [C.POINTER(C.c_int),
                                                                     C.POINTER(OfStepMetrics)]
        lib.of_tg_init.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        lib.of_run_steps.argtypes = [C.c_void_p, C.POINTER(OfStepParams), C.c_int,
                                     C.POINTER(OfStepMetrics)]
        lib.of_step_host.argtypes = [C.c_void_p, C.POINTER(OfStepParams)] + [DP] * 7 + \
            [C.POINTER(C.c_int), C.POINTER(OfStepMetrics)]
        lib.of_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        # device pointers (u, v, w, pressure_rhs, stream) as c_void_p
        lib.of_pressure_rhs_noalloc.argtypes = [C.POINTER(OfGrid), C.c_double, C.c_double] + \
            [C.c_void_p] * 4 + [DP, C.c_void_p]
        lib.of_tangent_linear.argtypes = [C.c_void_p, C.POINTER(OfStepParams), C.c_int] + [DP] * 6
        lib.of_adjoint_gradient.argtypes = [C.c_void_p, C.POINTER(OfStepParams), C.c_int,
                                            C.c_int] + [DP] * 6 + [C.POINTER(OfAdjointInfo)]
        lib.of_adjoint_gradient_binomial.argtypes = lib.of_adjoint_gradient.argtypes
        lib.of_adjoint_schedule_cost.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_longlong),
                                                 C.POINTER(C.c_longlong)]
        lib.of_kernel_class_name.restype = C.c_char_p
        lib.of_profile_enable.argtypes = [C.c_int]
        lib.of_profile_read.argtypes = [C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                        C.POINTER(C.c_double)]
        lib.of_profile_coarse_chain.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                                C.POINTER(C.c_int)]
        _lib = lib
    return _lib


class OfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class NotConvergedError(OfError):
    pass


class NonFiniteError(OfError):
    pass


def check(status):
    """Turns a status code into the exception type the reference would raise."""
    if status == OF_OK:
        return
    msg = load().of_last_error().decode()
    if status == OF_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == OF_NOT_CONVERGED:
        raise NotConvergedError(status, msg)
    if status == OF_NONFINITE:
        raise NonFiniteError(status, msg)
    raise OfError(status, msg)
