"""The block GMRES restatement (oracle/block_gmres_oracle.py) against the reference's own block
GMRES tests (crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:1269-1950),
on the same 1-D Laplacian problems and bars, on the CPU."""
import numpy as np

from oracle import block_gmres_oracle as BG
from oracle import gcro_oracle


def laplacian_1d(n):
    A = 2.0 * np.eye(n)
    A -= np.eye(n, k=1)
    A -= np.eye(n, k=-1)
    return A


def check_residual(A, X, B, j):
    return np.linalg.norm(B[:, j] - A @ X[:, j]) / np.linalg.norm(B[:, j])


def test_single_rhs():  # block_gmres.rs:1269
    n = 50
    A = laplacian_1d(n)
    B = (np.arange(n) + 1.0)[:, None]
    r = BG.block_gmres(A, B, 50, 30, 1e-10)
    assert r.converged


def test_multiple_rhs():  # block_gmres.rs:1348
    n = 50
    A = laplacian_1d(n)
    i = np.arange(n)
    B = np.stack([np.ones(n), np.sin(i), np.where(i < n // 2, 1.0, -1.0)], axis=1)
    r = BG.block_gmres(A, B, 50, 40, 1e-8)
    assert r.converged and r.x.shape == (n, 3)
    for j in range(3):
        assert check_residual(A, r.x, B, j) < 1e-7


def test_matches_individual():  # block_gmres.rs:1412
    n = 30
    A = laplacian_1d(n)
    B = np.stack([np.ones(n), 2.0 * np.ones(n)], axis=1)
    rb = BG.block_gmres(A, B, 100, 30, 1e-10)
    assert rb.converged
    for j in range(2):
        x = np.linalg.solve(A, B[:, j])
        assert np.max(np.abs(rb.x[:, j] - x)) < 1e-6


def test_rank_deficient_block():  # block_gmres.rs:1517
    n = 40
    A = laplacian_1d(n)
    i = np.arange(n)
    b0 = np.sqrt(i + 1.0)
    B = np.stack([b0, b0, np.cos(i * 0.2)], axis=1)
    r = BG.block_gmres(A, B, 50, 30, 1e-10)
    assert r.converged
    assert np.max(np.abs(r.x[:, 0] - r.x[:, 1])) < 1e-8
    for j in range(3):
        assert check_residual(A, r.x, B, j) < 1e-9


def test_zero_rhs_column():  # block_gmres.rs:1559
    n = 32
    A = laplacian_1d(n)
    i = np.arange(n)
    B = np.stack([np.zeros(n), np.sin(i * 0.31) + 0.25], axis=1)
    r = BG.block_gmres(A, B, 50, 24, 1e-10)
    assert r.converged
    assert np.all(r.x[:, 0] == 0.0)
    assert r.true_residuals[0] < 1e-12
    assert check_residual(A, r.x, B, 1) < 1e-9


def test_scaled_dependent_rhs_columns():  # block_gmres.rs:1600
    n = 36
    A = laplacian_1d(n)
    i = np.arange(n)
    base = np.cos(i * 0.23) + 0.4
    B = np.stack([base, 2.0 * base, np.sin(i * 0.47) - 0.1], axis=1)
    r = BG.block_gmres(A, B, 50, 24, 1e-10)
    assert r.converged
    assert np.max(np.abs(r.x[:, 1] - 2.0 * r.x[:, 0])) < 1e-8
    for j in range(3):
        assert check_residual(A, r.x, B, j) < 1e-9


def test_complex_laplacian():  # block_gmres.rs:1638 (complex shift)
    n = 40
    A = laplacian_1d(n).astype(complex) + 0.3j * np.eye(n)
    i = np.arange(n)
    B = np.stack([np.exp(0.2j * i), np.cos(0.1 * i) + 0.5j], axis=1)
    r = BG.block_gmres(A, B, 50, 30, 1e-10)
    assert r.converged
    for j in range(2):
        assert check_residual(A, r.x, B, j) < 1e-9


def test_true_residuals_match_direct_computation():  # block_gmres.rs:1818
    n = 40
    A = laplacian_1d(n)
    i = np.arange(n)
    B = np.stack([np.ones(n), np.sin(i), np.where(i < n // 2, 1.0, -1.0)], axis=1)
    r = BG.block_gmres(A, B, 50, 40, 1e-10)
    assert r.converged
    for j in range(3):
        direct = check_residual(A, r.x, B, j)
        assert abs(r.true_residuals[j] - direct) < 1e-14
        assert r.true_residuals[j] <= r.residuals[j] * 10.0 + 1e-12
        assert np.isfinite(r.backward_errors[j])


def test_converged_gates_on_configured_residual():  # block_gmres.rs:1866
    n = 40
    A = laplacian_1d(n)
    i = np.arange(n)
    B = np.stack([np.ones(n), np.cos(i * 0.2)], axis=1)
    tol = 1e-10
    for trc in (True, False):
        r = BG.block_gmres(A, B, 50, 40, tol, true_residual_check=trc)
        gated = r.true_residuals if trc else r.residuals
        assert r.converged == bool(np.all(gated <= tol))
        assert r.converged
    r = BG.block_gmres(A, B, 0, 40, tol, true_residual_check=False)
    assert not r.converged and np.all(r.true_residuals > tol)


def test_with_guess_reduces_iterations():  # block_gmres.rs:1756
    n = 50
    A = 6.0 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)
    i = np.arange(n)
    B = np.stack([np.ones(n), np.sin(i)], axis=1)
    cold = BG.block_gmres(A, B, 50, 40, 1e-8)
    assert cold.converged and cold.iterations > 0
    exact = BG.block_gmres(A, B, 50, 40, 1e-8, x0=cold.x)
    assert exact.converged and exact.iterations == 0 and np.all(exact.true_residuals <= 1e-8)
    warm = BG.block_gmres(A, B, 50, 40, 1e-8, x0=cold.x * 1.001)
    assert warm.converged and warm.iterations < cold.iterations
    for j in range(2):
        assert check_residual(A, warm.x, B, j) < 1e-7


def test_single_column_matches_scalar_gmres_oracle():
    """One right-hand side: the block method is scalar GMRES; same solution as the GCRO-DR
    oracle's plain GMRES path (empty subspace) to the tolerance."""
    rng = np.random.default_rng(3)
    n = 60
    A = laplacian_1d(n) + 0.5 * np.eye(n) + 0.05 * rng.standard_normal((n, n))
    b = rng.standard_normal(n) + 0j
    r = BG.block_gmres(A, b[:, None], 20, 30, 1e-10)
    x = np.linalg.solve(A, b)
    assert r.converged and np.linalg.norm(r.x[:, 0] - x) / np.linalg.norm(x) < 1e-8
    assert hasattr(gcro_oracle, "gcro_dr")
