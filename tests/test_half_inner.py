"""Complex-half inner matrix of the mixed solver (sb_operator_set_inner_precision, SB_INNER_FP16).

The inner GMRES of iterative refinement (crates/sonium-solvers/crates/sonium-solvers-iterative/src/
gmres_ir.rs:1-80) runs on a power-of-two-scaled FP16 copy of the complex64 matrix; the outer
residual stays on the complex64 matrix with FP64 vectors, so the converged solution is the one of
the complex64 system. GPU: the solution equals the FP32-inner solution and the FP64 solution to
the solver tolerance on TBEM systems (sphere, ellipsoid, re-assembly at a new wavenumber); on
matrices whose entries are exact in FP16 after the scale (at magnitudes 2^-24 to 2^22: the scale
is a power of two) the FP16-inner solve takes the FP32-inner solve's iterations; odd sizes exercise the
column tail; operators without a complex64 matrix are rejected.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
@pytest.mark.parametrize("level,k,scale", [(3, 4.0, (1.0, 1.0, 1.0)), (4, 10.0, (1.0, 0.6, 0.4))])
def test_half_inner_tbem_matches_fp32_inner(gpu, level, k, scale):
    nodes, tris = gpu.icosphere(1.0, level, scale)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    op64 = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    x64 = gpu.gmres(op64, b, gpu.GmresConfig(max_iterations=200, restart=50, tolerance=1e-10)).x
    op64.close()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32)
    s32 = gpu.gmres_mixed(op, b, gpu.IrConfig(20, 1e-8, 50, 50, 1e-5))
    op.set_inner_precision(gpu.SB_INNER_FP16)
    s16 = gpu.gmres_mixed(op, b, gpu.IrConfig(20, 1e-8, 50, 50, 1e-3))
    assert s32.converged and s16.converged
    assert s16.residual < 1e-8
    assert _rel(s16.x, s32.x) < 1e-6
    assert _rel(s16.x, x64) < 1e-5
    assert s16.matvecs_fp32 > 0 and s16.refinements >= 2
    # Re-assembly at another wavenumber rebuilds the half copy on the next solve.
    ph2 = gpu.PhysicsParams.for_wavenumber(0.8 * k)
    beta2 = ph2.burton_miller_beta()
    b2 = gpu.rhs_plane_wave(mesh, ph2, beta2, [1.0, 0.0, 0.0])[:, 0]
    op.reassemble(ph2, beta2)
    s16b = gpu.gmres_mixed(op, b2, gpu.IrConfig(20, 1e-8, 50, 50, 1e-3))
    op.set_inner_precision(gpu.SB_INNER_FP32)
    s32b = gpu.gmres_mixed(op, b2, gpu.IrConfig(20, 1e-8, 50, 50, 1e-5))
    assert s16b.converged and s32b.converged
    assert _rel(s16b.x, s32b.x) < 1e-6
    op.close()
    mesh.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,mag", [(1001, 1.0), (1024, 2.0 ** -24), (515, 2.0 ** 22)])
def test_half_inner_exact_entries(gpu, n, mag):
    # Off-diagonal parts j / 16 (|j| <= 8) and diagonal 32 + j / 16, times a power of two: every
    # part needs at most 10 significant bits, so the half copy equals the complex64 matrix times
    # the device's power-of-two scale exactly, at any magnitude.
    rng = np.random.default_rng(n)
    A = (rng.integers(-8, 9, (n, n)) + 1j * rng.integers(-8, 9, (n, n))) / 16.0
    A += np.diag(np.full(n, 32.0))
    A *= mag
    x_true = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = A @ x_true
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP32)
    assert np.array_equal(op.matrix_c64(), A.astype(np.complex64))
    cfg = gpu.IrConfig(20, 1e-9, 50, 50, 1e-6)
    s32 = gpu.gmres_mixed(op, b, cfg)
    op.set_inner_precision(gpu.SB_INNER_FP16)
    s16 = gpu.gmres_mixed(op, b, cfg)
    assert s32.converged and s16.converged
    # Same operator to FP32 accumulation order: the same iterations up to rounding noise.
    assert abs(s16.iterations - s32.iterations) <= 2
    assert _rel(s16.x, x_true) < 1e-7
    # Inner restarts every 6 steps: the inner solve forms explicit residuals on the half copy.
    cfg = gpu.IrConfig(20, 1e-9, 6, 60, 1e-6)
    r16 = gpu.gmres_mixed(op, b, cfg)
    op.set_inner_precision(gpu.SB_INNER_FP32)
    r32 = gpu.gmres_mixed(op, b, cfg)
    assert r16.converged and r32.converged and r16.restarts > 0
    assert abs(r16.iterations - r32.iterations) <= 3
    assert _rel(r16.x, x_true) < 1e-7
    op.close()


@pytest.mark.gpu
def test_half_inner_rejections(gpu):
    A = np.eye(8, dtype=complex) * 3.0
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    with pytest.raises(gpu.SoniumError):
        op.set_inner_precision(gpu.SB_INNER_FP16)
    op.set_inner_precision(gpu.SB_INNER_FP32)
    op.close()
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64_FP32)
    with pytest.raises(gpu.SoniumError):
        op.set_inner_precision(7)
    op.set_inner_precision(gpu.SB_INNER_FP16)
    s = gpu.gmres_mixed(op, np.ones(8, complex), gpu.IrConfig(20, 1e-10, 50, 50, 1e-3))
    assert s.converged and np.allclose(s.x, 1.0 / 3.0, rtol=1e-9)
    op.close()


@pytest.mark.gpu
def test_half_copy_from_assembly_matches_rebuilt_copy(gpu):
    # After a re-assembly with SB_INNER_FP16 set, the FP32 assembly writes the complex-half copy
    # itself (row scales from each row's near and diagonal entries); a dense operator over the
    # same complex64 matrix builds its copy from full-row scans. Both inner operators carry the
    # same complex64 matrix to FP16 rounding, so the solves agree to the solver tolerance.
    nodes, tris = gpu.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(5.0)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32)
    dense = gpu.DenseMatrixOperator(op.matrix_c64().astype(complex), gpu.SB_PRECISION_FP32)
    cfg = gpu.IrConfig(20, 1e-8, 50, 50, 1e-3)
    for o in (op, dense):
        o.set_inner_precision(gpu.SB_INNER_FP16)
    op.reassemble(ph, beta)  # the assembly writes the copy
    assert np.array_equal(op.matrix_c64(), dense.matrix_c64())
    s1 = gpu.gmres_mixed(op, b, cfg)
    s2 = gpu.gmres_mixed(dense, b, cfg)
    assert s1.converged and s2.converged
    assert abs(s1.iterations - s2.iterations) <= 2
    assert _rel(s1.x, s2.x) < 1e-6
    # the copy written by the assembly and a rebuilt one give the same solve
    op.set_inner_precision(gpu.SB_INNER_FP32)
    op.set_inner_precision(gpu.SB_INNER_FP16)  # no copy now: the next solve rebuilds it
    s3 = gpu.gmres_mixed(op, b, cfg)
    assert abs(s1.iterations - s3.iterations) <= 2 and _rel(s1.x, s3.x) < 1e-6
    op.close()
    dense.close()
    mesh.close()


@pytest.mark.gpu
def test_precision_fp32_half_writes_copy_at_first_assembly(gpu):
    # SB_PRECISION_FP32_HALF: the first assembly writes the complex-half copy; the operator is an
    # SB_PRECISION_FP32 one with SB_INNER_FP16 set, and solves as one that switched later.
    nodes, tris = gpu.icosphere(1.0, 3)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(4.0)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    cfg = gpu.IrConfig(20, 1e-8, 50, 50, 1e-3)
    oh = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32_HALF)
    assert oh.info().precision == gpu.SB_PRECISION_FP32
    o32 = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32)
    assert np.array_equal(oh.matrix_c64(), o32.matrix_c64())
    o32.set_inner_precision(gpu.SB_INNER_FP16)
    s1 = gpu.gmres_mixed(oh, b, cfg)
    s2 = gpu.gmres_mixed(o32, b, cfg)
    assert s1.converged and s2.converged
    assert abs(s1.iterations - s2.iterations) <= 2 and _rel(s1.x, s2.x) < 1e-6
    oh.close()
    o32.close()
    mesh.close()
