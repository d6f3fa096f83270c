"""Tensor-core block product (sb_operator_apply_block_tensor): Y = A X for many complex64 vectors
as BF16 hi/lo split products on tcgen05, against the exact complex128 product.

Bar: each result vector within 3e-5 (relative 2-norm) of A x computed in complex128 from the
assembled matrix. The split keeps 16 significant bits of every operand (relative 2^-17), the
dropped lo*lo term is ~2^-16 of each product, and FP32 accumulation adds ~1e-7: the per-vector
error of a diagonally dominant BEM matrix is expected near 1e-5.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _apply_tensor(op, X):
    from sonium_b200 import _lib as L

    X = np.ascontiguousarray(X, np.complex64)
    Y = np.zeros_like(X)
    L.check(L.load().sb_operator_apply_block_tensor(op.handle, X.ctypes.data, Y.ctypes.data, X.shape[0]))
    return Y


def _rel_errors(Y, A, X):
    ref = (A @ X.astype(np.complex128).T).T
    return np.linalg.norm(Y - ref, axis=1) / np.linalg.norm(ref, axis=1)


@pytest.mark.parametrize("level,k,r,drop", [(2, 2.0, 128, 0), (2, 3.0, 200, 1), (3, 6.0, 256, 0), (1, 1.0, 5, 3)])
def test_block_product_matches_complex128(gpu, oracle, level, k, r, drop):
    from sonium_b200 import _lib as L

    nodes, tris = oracle.icosphere(1.0, level, (1.0, 0.6, 0.4))
    if drop:
        tris = tris[:-drop]  # n not a multiple of 64: padded K and rows
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(k)
    op = gpu.build_tbem_system(mesh, ph)
    A = op.matrix
    n = A.shape[0]
    L.check(L.load().sb_operator_prepare_block_tensor(op.handle))
    rng = np.random.default_rng(0x5EED + level)
    X = (rng.standard_normal((r, n)) + 1j * rng.standard_normal((r, n))).astype(np.complex64)
    Y = _apply_tensor(op, X)
    err = _rel_errors(Y, A, X)
    assert err.max() < 3e-5, (err.max(), np.argmax(err))
    # a second product through the same planes, and a smaller block (fewer vectors than the tile)
    Y2 = _apply_tensor(op, X[:3])
    assert np.array_equal(Y2, Y[:3])
    op.close()


def test_block_product_plane_wave_rhs_block(gpu, oracle):
    """The right-hand sides of a multi-direction incident field (the shape of the 256-direction
    multi-right-hand-side workload, smaller)."""
    from sonium_b200 import _lib as L

    nodes, tris = oracle.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(4.0)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    A = op.matrix
    rng = np.random.default_rng(7)
    d = rng.standard_normal((64, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    B = gpu.rhs_plane_wave(mesh, ph, beta, d)  # n x 64
    L.check(L.load().sb_operator_prepare_block_tensor(op.handle))
    X = B.T.astype(np.complex64)
    Y = _apply_tensor(op, X)
    assert _rel_errors(Y, A, X).max() < 3e-5
    # re-assembly drops the planes: the product must be prepared again
    op.reassemble(ph, beta)
    with pytest.raises(gpu.SoniumError):
        _apply_tensor(op, X)
    op.close()


def test_multi_rhs_solve_matches_fp64_solves(gpu, oracle):
    """sb_gmres_multi: 64 plane-wave right-hand sides (Fibonacci directions) on an ellipsoid, each
    within 1e-6 of its own FP64 GMRES solve, every one converged to its FP64 residual target."""
    nodes, tris = oracle.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(4.0)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    dirs = gpu.fibonacci_sphere_directions(64)
    B = gpu.rhs_plane_wave(mesh, ph, beta, dirs)
    cfg = gpu.IrConfig(tolerance=1e-9)
    X, st = gpu.gmres_multi(op, B, cfg)
    A = op.matrix
    for c in (0, 17, 40, 63):
        ref = gpu.gmres(op, B[:, c], gpu.GmresConfig(max_iterations=100, restart=50, tolerance=1e-11)).x
        assert np.linalg.norm(X[:, c] - ref) / np.linalg.norm(ref) < 1e-6, c
    assert all(s.converged and s.residual < 1e-9 for s in st)
    res = np.linalg.norm(B - A @ X, axis=0) / np.linalg.norm(B, axis=0)
    assert res.max() < 1e-9
    assert np.allclose([s.residual for s in st], res, rtol=1e-3, atol=1e-14)
    assert all(s.matvecs_fp32 > 0 and s.refinements >= 1 for s in st)
    op.close()


def test_multi_rhs_partial_block_zero_rhs_and_rejections(gpu, oracle):
    """Fewer right-hand sides than a tile, one of them zero (done at once, x = 0), a second solve
    reusing the workspace, and an operator without the complex128 matrix rejected."""
    nodes, tris = oracle.icosphere(1.0, 2)
    mesh = gpu.Mesh(nodes, tris[:-1])  # odd n
    ph = gpu.PhysicsParams.for_wavenumber(2.0)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP64_FP32)
    B = gpu.rhs_plane_wave(mesh, ph, beta, gpu.fibonacci_sphere_directions(5))
    B[:, 2] = 0
    X, st = gpu.gmres_multi(op, B, gpu.IrConfig(tolerance=1e-10))
    assert st[2].iterations == 0 and st[2].converged and np.all(X[:, 2] == 0)
    A = op.matrix
    for c in (0, 1, 3, 4):
        assert st[c].converged
        assert np.linalg.norm(B[:, c] - A @ X[:, c]) / np.linalg.norm(B[:, c]) < 1e-10
    X2, _ = gpu.gmres_multi(op, B, gpu.IrConfig(tolerance=1e-10))
    assert np.array_equal(X2, X)
    op32 = gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32)
    with pytest.raises(gpu.SoniumError) as e:
        gpu.gmres_multi(op32, B, gpu.IrConfig())
    assert "complex128" in str(e.value)
    op.close()
    op32.close()
