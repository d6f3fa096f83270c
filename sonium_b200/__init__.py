"""sonium-b200: dense Burton-Miller TBEM (assembly, matvec, GMRES) on NVIDIA B200 (sm_100a).

The compute path is the CUDA shared library built from ``sonium_b200/csrc`` (C ABI in
``include/sonium_b200.h``); this package is its Python binding. There is no CPU fallback.
"""
from ._lib import (SB_INNER_FP16, SB_INNER_FP32, SB_INNER_PRECOND_BLOCK_JACOBI, SB_INNER_PRECOND_NONE,
                   SB_BASIS_CONSTANT, SB_BASIS_LINEAR, SB_BASIS_QUADRATIC, SB_BC_PRESSURE, SB_BC_VELOCITY, SB_INJECT_ALLOC, SB_INJECT_LAUNCH, SB_INJECT_NONE,
                   SB_OP_C, SB_OP_N, SB_OP_T, SB_PRECISION_FP32, SB_PRECISION_FP32_HALF, SB_PRECISION_FP64,
                   SB_PRECISION_FP64_FP32, SB_PRECOND_BLOCK_JACOBI, SB_PRECOND_IDENTITY, SB_PRECOND_JACOBI,
                   SoniumError)
from .tbem import (BlockJacobiPreconditioner, DenseMatrixOperator, GcroDrConfig, GcroDrSubspace, build_tbem_system_linear, gcro_dr,
                   build_tbem_system_discontinuous_stabilized, build_tbem_system_quadratic_stabilized,
                   rhs_plane_wave_at,
                   GmresConfig, GmresSolution, IrConfig, JacobiPreconditioner, LinearOperator, Mesh,
                   PhysicsParams, TbemOperator, build_tbem_system, build_tbem_system_with_beta,
                   compute_scattered_field, compute_total_field, device_count,
                   block_residual, fibonacci_sphere_directions, gmres, gmres_mixed, gmres_multi, icosphere,
                   inject_failure, rhs_plane_wave)
from .sweep import (FrequencySweepConfig, FrequencySweepResult, SweepBatch, frequency_sweep,
                    frequency_sweep_batched)

__all__ = [
    "GmresConfig", "GmresSolution", "IrConfig", "JacobiPreconditioner", "LinearOperator", "Mesh",
    "PhysicsParams", "TbemOperator", "build_tbem_system", "build_tbem_system_with_beta", "device_count",
    "gmres", "gmres_mixed", "icosphere", "inject_failure", "rhs_plane_wave", "SoniumError",
    "FrequencySweepConfig", "FrequencySweepResult", "SweepBatch", "frequency_sweep", "frequency_sweep_batched", "gmres_multi", "block_residual", "fibonacci_sphere_directions",
    "compute_scattered_field", "compute_total_field",
    "DenseMatrixOperator", "GcroDrConfig", "GcroDrSubspace", "gcro_dr", "build_tbem_system_linear",
    "rhs_plane_wave_at", "SB_BASIS_CONSTANT", "SB_BASIS_LINEAR", "SB_BASIS_QUADRATIC",
    "build_tbem_system_discontinuous_stabilized", "build_tbem_system_quadratic_stabilized",
    "SB_BC_PRESSURE", "SB_BC_VELOCITY", "SB_INJECT_ALLOC", "SB_INJECT_LAUNCH", "SB_INJECT_NONE",
    "SB_OP_C", "SB_OP_N", "SB_OP_T", "SB_PRECISION_FP32", "SB_PRECISION_FP64", "SB_PRECISION_FP64_FP32",
    "SB_PRECOND_IDENTITY", "SB_PRECOND_JACOBI", "SB_PRECOND_BLOCK_JACOBI", "BlockJacobiPreconditioner",
    "SB_INNER_FP16", "SB_INNER_FP32",
    "SB_INNER_PRECOND_BLOCK_JACOBI", "SB_INNER_PRECOND_NONE", "SB_PRECISION_FP32_HALF",
]
