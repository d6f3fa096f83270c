"""Block-Jacobi right preconditioner of the mixed solver's inner GMRES
(sb_operator_set_inner_preconditioner, SB_INNER_PRECOND_BLOCK_JACOBI).

GPU: on TBEM systems the preconditioned solve (FP32 or complex-half inner products) reaches the
unpreconditioned solution to the solver tolerance with fewer inner iterations; on a dense
block-diagonal matrix (index-order blocks, rows needing pivoting, a partial last block) the
preconditioner is the exact inverse, so every inner solve converges in one step; a singular
diagonal block falls back to the identity and the solve still converges; re-assembly rebuilds
the block inverses; invalid arguments are rejected. The same block-Jacobi preconditioner on the
right of the FP64 GMRES (SB_PRECOND_BLOCK_JACOBI): fewer iterations to the same solution and
residual, an initial guess, re-assembly, the apply entry point against numpy's block inverses.
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
@pytest.mark.parametrize("inner,bs", [(0, 128), (1, 64), (1, 96), (1, 128), (0, 32)])
def test_block_jacobi_tbem(gpu, inner, bs):
    nodes, tris = gpu.icosphere(1.0, 4, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(12.0)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32)
    op.set_inner_precision(inner)
    cfg = gpu.IrConfig(20, 1e-8, 50, 50, 1e-3 if inner else 1e-5)
    s0 = gpu.gmres_mixed(op, b, cfg)
    op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, bs)
    s1 = gpu.gmres_mixed(op, b, cfg)
    assert s0.converged and s1.converged and s1.residual < 1e-8
    assert _rel(s1.x, s0.x) < 1e-6
    assert s1.iterations < s0.iterations, (s1.iterations, s0.iterations)
    # re-assembly at another wavenumber: the block inverses follow the new matrix
    ph2 = gpu.PhysicsParams.for_wavenumber(9.0)
    beta2 = ph2.burton_miller_beta()
    b2 = gpu.rhs_plane_wave(mesh, ph2, beta2, [0.0, 1.0, 0.0])[:, 0]
    op.reassemble(ph2, beta2)
    s2 = gpu.gmres_mixed(op, b2, cfg)
    op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_NONE, 0)
    s3 = gpu.gmres_mixed(op, b2, cfg)
    assert s2.converged and s3.converged
    assert _rel(s2.x, s3.x) < 1e-6
    assert s2.iterations < s3.iterations
    op.close()
    mesh.close()


def _block_diag(rng, n, bs, zero_diag=True):
    A = np.zeros((n, n), complex)
    for s in range(0, n, bs):
        e = min(n, s + bs)
        m = e - s
        B = (rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))) / np.sqrt(m)
        # a shifted permutation part keeps the block well conditioned while its diagonal is zero
        P = np.roll(np.eye(m), 1, axis=1) * 4.0
        B = B + P
        if zero_diag and m > 1:
            np.fill_diagonal(B, 0.0)
        A[s:e, s:e] = B
    return A


@pytest.mark.gpu
@pytest.mark.parametrize("n,bs", [(300, 64), (256, 128), (97, 32), (200, 96)])
def test_block_jacobi_exact_on_block_diagonal(gpu, n, bs):
    rng = np.random.default_rng(n + bs)
    A = _block_diag(rng, n, bs)
    x_true = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = A @ x_true
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP32)
    op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, bs)
    s = gpu.gmres_mixed(op, b, gpu.IrConfig(20, 1e-10, 50, 50, 1e-5))
    assert s.converged
    assert s.iterations <= 2 * s.refinements, (s.iterations, s.refinements)
    # the solution of the complex64 system the mixed solver refines on
    x32 = np.linalg.solve(A.astype(np.complex64).astype(complex), b)
    assert _rel(s.x, x32) < 1e-8
    op.close()


@pytest.mark.gpu
def test_block_jacobi_singular_block_falls_back(gpu):
    # [[0, I], [I, 0]] blocks of 32: every diagonal block is zero (singular), the matrix is not
    n, bs = 128, 32
    A = np.zeros((n, n), complex)
    for s in range(0, n, 2 * bs):
        A[s:s + bs, s + bs:s + 2 * bs] = np.eye(bs) * 2.0
        A[s + bs:s + 2 * bs, s:s + bs] = np.eye(bs) * 2.0
    rng = np.random.default_rng(7)
    x_true = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = A @ x_true
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP32)
    op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, bs)
    s = gpu.gmres_mixed(op, b, gpu.IrConfig(20, 1e-10, 50, 50, 1e-6))
    assert s.converged and _rel(s.x, x_true) < 1e-8  # entries 2.0: the complex64 matrix is exact
    op.close()


@pytest.mark.gpu
def test_block_jacobi_rejections(gpu):
    A = np.eye(8, dtype=complex) * 3.0
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    with pytest.raises(gpu.SoniumError):
        op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, 64)
    op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_NONE, 0)
    op.close()
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP32)
    for kind, bs in ((gpu.SB_INNER_PRECOND_BLOCK_JACOBI, 48), (gpu.SB_INNER_PRECOND_BLOCK_JACOBI, 256), (9, 64)):
        with pytest.raises(gpu.SoniumError):
            op.set_inner_preconditioner(kind, bs)
    op.close()


# ---- the FP64 solver's block-Jacobi right preconditioner (SB_PRECOND_BLOCK_JACOBI) ----

@pytest.mark.gpu
@pytest.mark.parametrize("bs", [64, 128])
def test_fp64_block_jacobi_tbem(gpu, bs):
    """FP64 GMRES(50) to 1e-8 with the block-Jacobi right preconditioner reaches the unpreconditioned
    FP64 solution in fewer iterations; with an initial guess it returns the same solution."""
    nodes, tris = gpu.icosphere(1.0, 4, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(12.0)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP64)
    cfg = gpu.GmresConfig(100, 50, 1e-8)
    s0 = gpu.gmres(op, b, cfg)
    pre = gpu.BlockJacobiPreconditioner(op, bs)
    s1 = gpu.gmres(op, b, cfg, preconditioner=pre)
    assert s0.converged and s1.converged and s1.residual < 1e-8
    A = op.matrix
    assert np.linalg.norm(b - A @ s1.x) / np.linalg.norm(b) < 1e-8  # the reported residual is b - A x
    assert _rel(s1.x, s0.x) < 1e-6
    assert s1.iterations < s0.iterations, (s1.iterations, s0.iterations)
    # an initial guess: the tolerance stays relative to ||b||
    s2 = gpu.gmres(op, b, cfg, x0=0.5 * s0.x, preconditioner=pre)
    assert s2.converged and s2.residual < 1e-8 and _rel(s2.x, s0.x) < 1e-6
    # an initial guess that already meets it: no iteration, x returned unchanged
    s5 = gpu.gmres(op, b, cfg, x0=s1.x, preconditioner=pre)
    assert s5.converged and s5.iterations == 0 and np.array_equal(s5.x, s1.x)
    # re-assembly: the block inverses follow the new matrix
    ph2 = gpu.PhysicsParams.for_wavenumber(9.0)
    beta2 = ph2.burton_miller_beta()
    b2 = gpu.rhs_plane_wave(mesh, ph2, beta2, [0.0, 1.0, 0.0])[:, 0]
    op.reassemble(ph2, beta2)
    s3 = gpu.gmres(op, b2, cfg, preconditioner=pre)
    s4 = gpu.gmres(op, b2, cfg)
    assert s3.converged and s4.converged and _rel(s3.x, s4.x) < 1e-6
    assert s3.iterations < s4.iterations
    op.close()
    mesh.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,bs", [(300, 64), (97, 32), (200, 96)])
def test_fp64_block_jacobi_apply_and_exact(gpu, n, bs):
    """sb_preconditioner_apply(SB_PRECOND_BLOCK_JACOBI) is the inverse of the (complex64-rounded)
    diagonal blocks; on a block-diagonal matrix the preconditioned FP64 GMRES converges at once."""
    rng = np.random.default_rng(3 * n + bs)
    A = _block_diag(rng, n, bs)
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    pre = gpu.BlockJacobiPreconditioner(op, bs)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = np.zeros(n, complex)
    pre.apply_into(x, y)
    A32 = A.astype(np.complex64).astype(complex)
    y_ref = np.zeros(n, complex)
    for s in range(0, n, bs):
        e = min(n, s + bs)
        y_ref[s:e] = np.linalg.solve(A32[s:e, s:e], x[s:e])
    assert _rel(y, y_ref) < 1e-4  # FP32 Gauss-Jordan inverse
    x_true = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = A @ x_true
    s = gpu.gmres(op, b, gpu.GmresConfig(20, 50, 1e-12), preconditioner=pre)
    assert s.converged and s.iterations <= 4, s.iterations
    assert _rel(s.x, x_true) < 1e-10
    op.close()


@pytest.mark.gpu
def test_fp64_block_jacobi_rejections(gpu):
    A = np.eye(8, dtype=complex) * 3.0
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP32)  # no complex128 matrix
    with pytest.raises(gpu.SoniumError):
        gpu.gmres(op, np.ones(8, complex), gpu.GmresConfig(10, 8, 1e-8),
                  preconditioner=gpu.BlockJacobiPreconditioner(op, 32))
    op.close()
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    for bs in (48, 256):
        with pytest.raises(gpu.SoniumError):
            gpu.BlockJacobiPreconditioner(op, bs)
    op.close()
