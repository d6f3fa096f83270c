"""ctypes binding of the sonium-b200 C ABI (include/sonium_b200.h).

The shared library is built in-tree by ``python -m sonium_b200.build``. If it is missing, or the
CUDA runtime cannot be used, calls raise: there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsonium_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "sonium_b200.h")

SB_OK = 0
SB_ERR_INVALID_ARGUMENT = 1
SB_ERR_UNSUPPORTED_ELEMENT = 2
SB_ERR_OUT_OF_MEMORY = 3
SB_ERR_CUDA = 4
SB_ERR_DEVICE_CHECK = 5
SB_ERR_INJECTED = 6
SB_ERR_NOT_FINITE = 7

SB_PRECISION_FP64 = 0
SB_PRECISION_FP64_FP32 = 1
SB_PRECISION_FP32 = 2
SB_PRECISION_FP32_HALF = 3
SB_INNER_FP32 = 0
SB_INNER_FP16 = 1
SB_INNER_PRECOND_NONE = 0
SB_INNER_PRECOND_BLOCK_JACOBI = 1
SB_OP_N, SB_OP_T, SB_OP_C = 0, 1, 2
SB_PRECOND_IDENTITY, SB_PRECOND_JACOBI, SB_PRECOND_BLOCK_JACOBI = 0, 1, 2
SB_BC_VELOCITY, SB_BC_PRESSURE = 0, 1
SB_INJECT_NONE, SB_INJECT_ALLOC, SB_INJECT_LAUNCH = 0, 1, 2
SB_SOLVER_CONVERGED, SB_SOLVER_MAX_ITERATIONS, SB_SOLVER_BREAKDOWN, SB_SOLVER_NUMERICAL_ERROR = 0, 1, 2, 3
SB_BATCH_ASM_AUTO, SB_BATCH_ASM_PERSISTENT, SB_BATCH_ASM_STREAMS = 0, 1, 2
SB_BASIS_CONSTANT, SB_BASIS_LINEAR, SB_BASIS_QUADRATIC = 0, 1, 2

_ERROR_NAMES = {
    SB_ERR_INVALID_ARGUMENT: "InvalidInput",
    SB_ERR_UNSUPPORTED_ELEMENT: "UnsupportedElement",
    SB_ERR_OUT_OF_MEMORY: "OutOfMemory",
    SB_ERR_CUDA: "Backend",
    SB_ERR_DEVICE_CHECK: "DeviceCheck",
    SB_ERR_INJECTED: "Injected",
    SB_ERR_NOT_FINITE: "NotFinite",
}


class SoniumError(RuntimeError):
    """A failed sonium-b200 call (the CudaTbemAssemblyError / SolverError analogue)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_ERROR_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class SbComplex(ct.Structure):
    _fields_ = [("re", ct.c_double), ("im", ct.c_double)]


class SbPhysics(ct.Structure):
    _fields_ = [(n, ct.c_double) for n in (
        "frequency", "speed_of_sound", "density", "wave_number", "omega", "wave_length",
        "harmonic_factor", "pressure_factor", "tau")]


class SbMeshInfo(ct.Structure):
    _fields_ = [("n_nodes", ct.c_int64), ("n_elements", ct.c_int64),
                ("n_near_pairs", ct.c_int64), ("device", ct.c_int32), ("reserved", ct.c_int32)]


class SbOperatorInfo(ct.Structure):
    _fields_ = [("n", ct.c_int64), ("precision", ct.c_int32), ("device", ct.c_int32),
                ("assembly_ms", ct.c_double), ("bytes_fp64", ct.c_uint64),
                ("bytes_fp32", ct.c_uint64)]


class SbGmresConfig(ct.Structure):
    _fields_ = [("max_iterations", ct.c_int64), ("restart", ct.c_int64),
                ("tolerance", ct.c_double), ("convergence_check_interval", ct.c_int64)]


class SbGmresStats(ct.Structure):
    _fields_ = [("iterations", ct.c_int64), ("restarts", ct.c_int64), ("matvecs", ct.c_int64),
                ("matvecs_fp32", ct.c_int64), ("refinements", ct.c_int64),
                ("residual", ct.c_double), ("estimated_residual", ct.c_double),
                ("backward_error", ct.c_double), ("device_ms", ct.c_double),
                ("converged", ct.c_int32), ("status", ct.c_int32)]


(SB_PROF_FAR, SB_PROF_NEAR, SB_PROF_SELF, SB_PROF_GEMV64, SB_PROF_GEMV32, SB_PROF_ARNOLDI, SB_PROF_OTHER,
 SB_PROF_TENSOR, SB_PROF_GEMV16, SB_PROF_RESIDUAL) = range(10)
SB_PROF_KINDS = 10
PROF_NAMES = ["far", "near", "self", "gemv64", "gemv32", "arnoldi", "other", "tensor", "gemv16", "residual"]


class SbProfile(ct.Structure):
    _fields_ = [("ms", ct.c_double * SB_PROF_KINDS), ("launches", ct.c_int64 * SB_PROF_KINDS),
                ("kernels", ct.c_int64)]


class SbIrConfig(ct.Structure):
    _fields_ = [("max_refinements", ct.c_int64), ("tolerance", ct.c_double),
                ("inner_restart", ct.c_int64), ("inner_max_iterations", ct.c_int64),
                ("inner_tolerance", ct.c_double)]


P = ct.c_void_p
_SIGNATURES = {
    "sb_last_error": ([ct.c_char_p, ct.c_size_t], ct.c_int),
    "sb_version": ([P, P, P], ct.c_int),
    "sb_device_count": ([ct.POINTER(ct.c_int)], ct.c_int),
    "sb_physics_new": ([ct.c_double, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(SbPhysics)], ct.c_int),
    "sb_physics_validate": ([ct.POINTER(SbPhysics)], ct.c_int),
    "sb_burton_miller_beta": ([ct.POINTER(SbPhysics), ct.c_double, ct.POINTER(SbComplex)], ct.c_int),
    "sb_icosphere_counts": ([ct.c_int, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)], ct.c_int),
    "sb_icosphere": ([ct.c_double, ct.c_int, P, P, P], ct.c_int),
    "sb_mesh_create": ([P, ct.c_int64, P, ct.c_int64, ct.c_int, ct.POINTER(P)], ct.c_int),
    "sb_mesh_create_quad4": ([P, ct.c_int64, P, ct.c_int64, ct.c_int, ct.POINTER(P)], ct.c_int),
    "sb_mesh_destroy": ([P], ct.c_int),
    "sb_mesh_info_get": ([P, ct.POINTER(SbMeshInfo)], ct.c_int),
    "sb_mesh_element_geometry": ([P, P, P, P], ct.c_int),
    "sb_mesh_set_bc": ([P, P, P, P, P], ct.c_int),
    "sb_assemble": ([P, ct.POINTER(SbPhysics), SbComplex, ct.c_int, ct.POINTER(P)], ct.c_int),
    "sb_assemble_into": ([P, ct.POINTER(SbPhysics), SbComplex], ct.c_int),
    "sb_operator_from_dense": ([ct.c_int, ct.c_int64, P, ct.c_int, ct.POINTER(P)], ct.c_int),
    "sb_assemble_linear": ([P, ct.POINTER(SbPhysics), SbComplex, ct.POINTER(P)], ct.c_int),
    "sb_mesh_collocation": ([P, ct.c_int, P, P], ct.c_int),
    "sb_assemble_discontinuous": ([P, ct.POINTER(SbPhysics), SbComplex, ct.c_int, ct.c_double, ct.POINTER(P)],
                                  ct.c_int),
    "sb_rhs_plane_wave_points": ([ct.c_int, ct.c_int64, P, P, ct.POINTER(SbPhysics), SbComplex, P, P, ct.c_int64, P],
                                 ct.c_int),
    "sb_operator_destroy": ([P], ct.c_int),
    "sb_operator_info_get": ([P, ct.POINTER(SbOperatorInfo)], ct.c_int),
    "sb_operator_copy_to_host": ([P, P, P], ct.c_int),
    "sb_operator_copy_rows_to_host": ([P, ct.c_int64, ct.c_int64, P], ct.c_int),
    "sb_operator_copy_to_host_c64": ([P, P], ct.c_int),
    "sb_operator_apply": ([P, ct.c_int, P, P], ct.c_int),
    "sb_operator_apply_block": ([P, P, P, ct.c_int64], ct.c_int),
    "sb_operator_apply_device": ([P, ct.c_int, P, P], ct.c_int),
    "sb_operator_apply_device_noalloc": ([P, ct.c_int, P, P], ct.c_int),
    "sb_preconditioner_apply": ([P, ct.c_int, P, P], ct.c_int),
    "sb_operator_set_block_jacobi_size": ([P, ct.c_int], ct.c_int),
    "sb_measure_fp32_rate": ([ct.c_int, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)], ct.c_int),
    "sb_rhs_plane_wave": ([P, ct.POINTER(SbPhysics), SbComplex, P, P, ct.c_int64, P], ct.c_int),
    "sb_gmres": ([P, P, P, ct.POINTER(SbGmresConfig), ct.c_int, P, ct.POINTER(SbGmresStats)], ct.c_int),
    "sb_gmres_device": ([P, P, P, ct.c_int, ct.POINTER(SbGmresConfig), ct.c_int, ct.POINTER(SbGmresStats)], ct.c_int),
    "sb_gmres_mixed": ([P, P, P, ct.POINTER(SbIrConfig), P, ct.POINTER(SbGmresStats)], ct.c_int),
    "sb_gmres_mixed_device": ([P, P, P, ct.c_int, ct.POINTER(SbIrConfig), ct.POINTER(SbGmresStats)], ct.c_int),
    "sb_operator_set_inner_precision": ([P, ct.c_int], ct.c_int),
    "sb_operator_set_inner_preconditioner": ([P, ct.c_int, ct.c_int], ct.c_int),
    "sb_rhs_plane_wave_device": ([P, P, P, ct.c_int64, P], ct.c_int),
    "sb_gcro_subspace_create": ([ct.c_int, ct.c_int64, ct.POINTER(P)], ct.c_int),
    "sb_gcro_subspace_destroy": ([P], ct.c_int),
    "sb_gcro_subspace_reset": ([P], ct.c_int),
    "sb_gcro_subspace_info": ([P, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)], ct.c_int),
    "sb_gcro_subspace_get_vectors": ([P, P], ct.c_int),
    "sb_gcro_subspace_set_vectors": ([P, ct.c_int64, ct.c_int64, P], ct.c_int),
    "sb_gcro_dr": ([P, P, P, P, ct.POINTER(SbGmresConfig), ct.c_int, P, ct.POINTER(SbGmresStats)], ct.c_int),
    "sb_gcro_dr_device": ([P, P, P, ct.c_int, P, ct.POINTER(SbGmresConfig), ct.c_int, ct.POINTER(SbGmresStats)],
                          ct.c_int),
    "sb_field_eval": ([P, ct.POINTER(SbPhysics), P, P, P, ct.c_int64, P], ct.c_int),
    "sb_operator_prepare_block_tensor": ([P], ct.c_int),
    "sb_operator_apply_block_tensor": ([P, P, P, ct.c_int64], ct.c_int),
    "sb_operator_apply_block_tensor_device": ([P, P, P, ct.c_int64], ct.c_int),
    "sb_operator_block_residual": ([P, P, P, ct.c_int64, P], ct.c_int),
    "sb_operator_block_residual_device": ([P, P, P, ct.c_int64, P], ct.c_int),
    "sb_gmres_multi": ([P, P, ct.c_int64, ct.POINTER(SbIrConfig), P, P], ct.c_int),
    "sb_gmres_multi_device": ([P, P, ct.c_int64, ct.POINTER(SbIrConfig), P, P], ct.c_int),
    "sb_batch_create": ([ct.c_int64, P, P, P, ct.POINTER(P)], ct.c_int),
    "sb_batch_destroy": ([P], ct.c_int),
    "sb_batch_assemble": ([P], ct.c_int),
    "sb_batch_set_rhs_plane_wave": ([P, P], ct.c_int),
    "sb_batch_set_rhs": ([P, ct.c_int64, P], ct.c_int),
    "sb_batch_solve": ([P, ct.POINTER(SbIrConfig), P], ct.c_int),
    "sb_batch_set_inner_precision": ([P, ct.c_int], ct.c_int),
    "sb_batch_set_inner_preconditioner": ([P, ct.c_int, ct.c_int], ct.c_int),
    "sb_batch_solution": ([P, ct.c_int64, P], ct.c_int),
    "sb_batch_matrix_c64": ([P, ct.c_int64, P], ct.c_int),
    "sb_batch_timings": ([P, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)], ct.c_int),
    "sb_batch_set_assembly_mode": ([P, ct.c_int], ct.c_int),
    "sb_batch_assembly_tuning": ([P, ct.POINTER(ct.c_int), ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)],
                                 ct.c_int),
    "sb_batch_assembly_split": ([P, ct.POINTER(ct.c_int), P], ct.c_int),
    "sb_memory_trim": ([ct.c_int], ct.c_int),
    "sb_memory_stats": ([ct.c_int, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)], ct.c_int),
    "sb_profile_enable": ([ct.c_int], ct.c_int),
    "sb_profile_enable_classes": ([ct.c_uint], ct.c_int),
    "sb_profile_read": ([ct.POINTER(SbProfile), ct.c_int], ct.c_int),
    "sb_event_create": ([ct.POINTER(P)], ct.c_int),
    "sb_event_destroy": ([P], ct.c_int),
    "sb_event_record": ([P, P], ct.c_int),
    "sb_event_elapsed_ms": ([P, P, ct.POINTER(ct.c_float)], ct.c_int),
    "sb_math_sincos": ([ct.c_int, P, ct.c_int64, P, P], ct.c_int),
    "sb_inject_failure": ([ct.c_int], ct.c_int),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the C-ABI library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SoniumError(SB_ERR_CUDA, f"{path} is missing: build it with `python -m sonium_b200.build`")
    lib = ct.CDLL(path)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error() -> str:
    buf = ct.create_string_buffer(1024)
    load().sb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != SB_OK:
        raise SoniumError(status, last_error())


def header_symbols(path: str = HEADER_PATH):
    """Names of every SB_API function declared in the public header."""
    import re

    text = open(path).read()
    return sorted(set(re.findall(r"SB_API\s+\w+\s+(sb_\w+)\s*\(", text)))
