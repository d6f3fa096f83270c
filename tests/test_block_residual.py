"""The integer-slice FP64 block residual (sb_operator_block_residual, ozaki.cu) against an
extended-precision residual.

R = B - A X is the block residual of block GMRES (crates/sonium-solvers/crates/
sonium-solvers-iterative/src/block_gmres.rs:829, block_true_metrics :571-620), an FP64 complex
GEMM there. Here it is computed from 8 signed 8-bit slices of every row of A and every vector
(power-of-two scales sigma_i, tau_c) with exact INT32 products, the 36 slice products of
diagonals 2..9 kept. Checks, against numpy's complex long double (64-bit significand) residual:

* every entry within the analytic bound: 2n terms of at most 9.05 * 2^-56 * sigma_i * tau_c each
  (dropped diagonals and slice remainders), plus 16 FP64 roundings of sum |a||x| + |b| (the FP64
  epilogue, the K-range partials and the subtraction);
* FP64-grade: the largest error over sum |a||x| + |b| below 1e-14 for random and TBEM matrices;
* ragged sizes (n not a multiple of the 64-byte K block, 2n not of the 128-row tile, r across two
  128-vector tiles), one vector, a zero vector (R = B exactly), duplicated vectors (identical
  columns), a power-of-two scaled vector (the A X part scaled exactly), a non-finite vector (its
  column NaN, the others unaffected);
* the many-right-hand-side solver's final residuals agree with numpy's.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps
SLICE_TERM = 9.05 * 2.0 ** -56


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _scale(v, axis):
    """2^e with e the frexp exponent of the largest |Re|, |Im| along `axis` (0 for a zero run)."""
    m = np.max(np.maximum(np.abs(v.real), np.abs(v.imag)), axis=axis)
    _, e = np.frexp(m)
    return np.where(m > 0, np.ldexp(1.0, e), 0.0)


def _exact(A, B, X):
    return B.astype(np.clongdouble) - A.astype(np.clongdouble) @ X.astype(np.clongdouble)


def _check(A, B, X, R):
    n = A.shape[0]
    ref = _exact(A, B, X)
    err = np.maximum(np.abs((R.real - ref.real).astype(np.float64)), np.abs((R.imag - ref.imag).astype(np.float64)))
    mag = (np.abs(A.real) + np.abs(A.imag)) @ (np.abs(X.real) + np.abs(X.imag)) + np.abs(B.real) + np.abs(B.imag)
    sigma = _scale(A, 1)[:, None]
    tau = _scale(X, 0)[None, :]
    bound = SLICE_TERM * sigma * tau * 2 * n + 16 * EPS * mag
    assert np.all(err <= bound), float(np.max(err / bound))
    return float(np.max(err / np.maximum(mag, 1e-300)))


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("n,r", [(700, 130), (64, 1), (257, 3)])
def test_random_matrix_within_bound(gpu, n, r):
    rng = np.random.default_rng(n + r)
    # rows of very different magnitudes and a few tiny entries: the per-row scales matter
    A = _rand(rng, n, n) * np.exp(rng.uniform(-8, 8, n))[:, None]
    A[rng.integers(0, n, 20), rng.integers(0, n, 20)] *= 1e-12
    X = _rand(rng, n, r) * np.exp(rng.uniform(-5, 5, r))[None, :]
    B = A @ X + 1e-3 * _rand(rng, n, r) * np.abs(A @ X)
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    R = gpu.block_residual(op, B, X)
    rel = _check(A, B, X, R)
    assert rel < 1e-14, rel
    op.close()


def test_edge_vectors(gpu):
    rng = np.random.default_rng(5)
    n = 300
    A = _rand(rng, n, n)
    x = _rand(rng, n, 1)[:, 0]
    X = np.stack([x, np.zeros(n), x, 2.0 ** 20 * x], axis=1)
    B = np.zeros((n, 4), complex)
    B[:, 1] = _rand(rng, n, 1)[:, 0]
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    R = gpu.block_residual(op, B, X)
    _check(A, B, X, R)
    assert np.array_equal(R[:, 1], B[:, 1])                  # zero vector: R = B exactly
    assert np.array_equal(R[:, 0], R[:, 2])                  # the same vector, the same residual
    assert np.array_equal(R[:, 3], 2.0 ** 20 * R[:, 0])     # power-of-two scaling is exact
    Xn = X.copy()
    Xn[7, 2] = np.nan
    Rn = gpu.block_residual(op, B, Xn)
    assert np.all(np.isnan(Rn[:, 2]))
    for c in (0, 1, 3):
        assert np.array_equal(Rn[:, c], R[:, c])
    op.close()


def test_duplicate_vectors_identical(gpu):
    rng = np.random.default_rng(9)
    n = 500
    A = _rand(rng, n, n)
    x = _rand(rng, n, 1)[:, 0]
    b = _rand(rng, n, 1)[:, 0]
    X = np.stack([x] * 4 + [_rand(rng, n, 1)[:, 0]], axis=1)
    B = np.stack([b] * 5, axis=1)
    op = gpu.DenseMatrixOperator(A, gpu.SB_PRECISION_FP64)
    R = gpu.block_residual(op, B, X)
    for c in range(1, 4):
        assert np.array_equal(R[:, c], R[:, 0])
    op.close()


def test_tbem_operator(gpu, oracle):
    k = 6.0
    nodes, tris = oracle.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    A = op.matrix
    B = gpu.rhs_plane_wave(mesh, ph, beta, gpu.fibonacci_sphere_directions(160))
    X = np.linalg.solve(A, B) * (1 + 1e-9)  # near-solutions: the residual cancels ~9 digits
    R = gpu.block_residual(op, B, X)
    rel = _check(A, B, X, R)
    assert rel < 1e-14, rel
    op.close()
    mesh.close()


def test_multi_solver_final_residuals(gpu, oracle):
    tol = 1e-10
    nodes, tris = oracle.icosphere(1.0, 3)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(4.0)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    A = op.matrix
    B = gpu.rhs_plane_wave(mesh, ph, beta, gpu.fibonacci_sphere_directions(12))
    X, stats = gpu.gmres_multi(op, B, gpu.IrConfig(20, tol, 50, 20, 1e-5))
    for j, st in enumerate(stats):
        true_rel = np.linalg.norm(B[:, j] - A @ X[:, j]) / np.linalg.norm(B[:, j])
        assert st.converged and true_rel <= tol
        assert abs(st.residual - true_rel) <= 1e-3 * true_rel + 1e-15, (j, st.residual, true_rel)
    op.close()
    mesh.close()
