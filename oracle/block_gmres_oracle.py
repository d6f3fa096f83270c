"""Block GMRES with a shared block Krylov basis -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's block GMRES (crates/sonium-solvers/crates/
sonium-solvers-iterative/src/block_gmres.rs: block_gmres_inner :706-1120, solve_block_ls
:635-705, block_true_metrics :570-620, apply_block_update :548-568; givens_rotation and
solve_upper_triangular of gmres_common.rs:91-127), unpreconditioned, with an optional block
initial guess. It is the checker of the many-right-hand-side solver's semantics: per-RHS
relative tolerance, convergence gated on the recomputed true residuals ||b_j - A x_j|| / ||b_j||,
rank-deficient blocks deflated instead of breaking down, a zero right-hand side giving x = 0.
Pinned on the CPU by the reference's own block GMRES tests (tests/test_block_gmres_oracle.py).
Only the tests import it.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

TINY = 1e-30


@dataclass
class BlockResult:
    x: np.ndarray                 # n x s
    iterations: int               # block Arnoldi steps
    residuals: np.ndarray         # projected relative residual per RHS
    true_residuals: np.ndarray    # ||b_j - A x_j|| / ||b_j|| (absolute for ||b_j|| ~ 0)
    backward_errors: np.ndarray
    converged: bool


def _givens(a: complex, b: complex):
    """givens_rotation (gmres_common.rs:91-106)."""
    if abs(b) < TINY:
        return 1.0 + 0j, 0j
    if abs(a) < TINY:
        return 0j, 1.0 + 0j
    r = np.sqrt(abs(a) ** 2 + abs(b) ** 2)
    return a / r, b / r


def _upper_solve(R: np.ndarray, g: np.ndarray, k: int) -> np.ndarray:
    """solve_upper_triangular (gmres_common.rs:109-127): a zero pivot leaves y_i = 0."""
    y = np.zeros(k, complex)
    for i in range(k - 1, -1, -1):
        s = g[i] - R[i, i + 1:k] @ y[i + 1:k]
        if abs(R[i, i]) > TINY:
            y[i] = s / R[i, i]
    return y


def solve_block_ls(h: np.ndarray, rows: int, cols: int, c0: np.ndarray, s1: int, s: int):
    """solve_block_ls (block_gmres.rs:635-705): Givens QR of the rows x cols block Hessenberg
    applied to all s right-hand sides; returns (y cols x s, tail norms per RHS)."""
    hw = h[:rows, :cols].astype(complex).copy()
    gw = np.zeros((rows, s), complex)
    gw[:min(s1, rows)] = c0[:min(s1, rows)]
    for col in range(cols):
        for row in range(col + 1, rows):
            if abs(hw[row, col]) < TINY:
                continue
            c, sn = _givens(hw[col, col], hw[row, col])
            a, b = hw[col, col:].copy(), hw[row, col:].copy()
            hw[col, col:] = np.conj(c) * a + np.conj(sn) * b
            hw[row, col:] = -sn * a + c * b
            a, b = gw[col].copy(), gw[row].copy()
            gw[col] = np.conj(c) * a + np.conj(sn) * b
            gw[row] = -sn * a + c * b
    y = np.zeros((cols, s), complex)
    for j in range(s):
        y[:, j] = _upper_solve(hw, gw[:cols, j], cols)
    tail = np.sqrt(np.sum(np.abs(gw[cols:rows]) ** 2, axis=0)) if rows > cols else np.zeros(s)
    return y, tail


def _true_metrics(A, x, b, b_true_norms):
    """block_true_metrics (block_gmres.rs:570-620)."""
    ax = A @ x
    res = np.linalg.norm(b - ax, axis=0)
    true_res = np.where(b_true_norms <= TINY, res, res / np.maximum(b_true_norms, TINY))
    denom = np.maximum(np.linalg.norm(ax, axis=0) + np.linalg.norm(b, axis=0), np.finfo(float).tiny)
    return true_res, res / denom


def block_gmres(A: np.ndarray, B: np.ndarray, max_iterations: int = 100, restart: int = 30,
                tolerance: float = 1e-6, true_residual_check: bool = True, x0=None) -> BlockResult:
    """block_gmres(_with_guess) (block_gmres.rs:148-197 -> block_gmres_inner :706-1120), no
    preconditioner, exact_residual_check_interval = 0."""
    A = np.asarray(A, complex)
    B = np.asarray(B, complex)
    n, s = B.shape
    defl_tol = np.sqrt(np.finfo(float).eps)
    dgks = 0.707
    b_norms = np.linalg.norm(B, axis=0)
    b_true_norms = b_norms.copy()
    x = np.zeros((n, s), complex) if x0 is None else np.asarray(x0, complex).copy()
    total = 0
    projected = np.full(s, np.inf)
    max_steps = max(restart, 1)
    max_basis = (max_steps + 1) * s
    for _cycle in range(max_iterations):
        R = B - A @ x
        col_norms = np.linalg.norm(R, axis=0)
        projected = np.where(b_norms >= TINY, col_norms / np.maximum(b_norms, TINY), 0.0)
        if all(not (b_norms[j] >= TINY and projected[j] > tolerance) for j in range(s)):
            break
        # initial block QR with rank-drop deflation (CGS2 per column)
        V = []
        for j in range(s):
            w = R[:, j].copy()
            for _ in range(2):
                if not V:
                    break
                Q = np.stack(V, axis=1)
                w = w - Q @ (Q.conj().T @ w)
            wn = np.linalg.norm(w)
            if wn > defl_tol * max(col_norms[j], TINY):
                V.append(w / wn)
        p = len(V)
        if p == 0:
            break
        s1 = p
        c0 = np.stack(V, axis=1).conj().T @ R  # s1 x s
        h = np.zeros((max_basis + s, max_basis), complex)
        converged_cycle = False
        next_cycle = False  # an optimistic projected convergence: the candidate is the next base
        sj = s1
        y = None
        for _step in range(max_steps):
            if p >= max_basis:
                break
            p_start = p - sj
            W = A @ np.stack(V[p_start:p], axis=1)
            frob_before = np.linalg.norm(W)
            Q = np.stack(V[:p], axis=1)
            for pas in range(2):
                G = Q.conj().T @ W
                h[:p, p_start:p_start + sj] += G
                W = W - Q @ G
                if pas == 0 and np.linalg.norm(W) >= dgks * frob_before:
                    break
            budget = max_basis - p
            s_next = 0
            for c in range(sj):
                w = W[:, c].copy()
                orig = np.linalg.norm(w)
                for _ in range(2):
                    for a_ in range(s_next):
                        d = np.vdot(V[p + a_], w)
                        h[p + a_, p_start + c] += d
                        w = w - d * V[p + a_]
                wn = np.linalg.norm(w)
                if wn > defl_tol * max(orig, TINY) and s_next < budget:
                    h[p + s_next, p_start + c] = wn
                    V.append(w / wn)
                    s_next += 1
            total += 1
            y, tail = solve_block_ls(h, p + s_next, p, c0, s1, s)
            projected = np.where(b_norms >= TINY, tail / np.maximum(b_norms, TINY), 0.0)
            cycle_done = bool(np.all(projected <= tolerance))
            if s_next > 0 and cycle_done and true_residual_check:
                cand = x + np.stack(V[:p], axis=1) @ y
                tr, _ = _true_metrics(A, cand, B, b_true_norms)
                if np.all(tr <= tolerance):
                    x = cand
                    converged_cycle = True
                    break
                x = cand
                next_cycle = True
                break
            if cycle_done or s_next == 0:
                x = x + np.stack(V[:p], axis=1) @ y
                converged_cycle = cycle_done
                break
            p += s_next
            sj = s_next
        if next_cycle:
            continue
        if not converged_cycle and p > s1:
            # block-step budget exhausted: least squares over the whole (square) basis, then restart
            y, tail = solve_block_ls(h, p, p, c0, s1, s)
            projected = np.where(b_norms >= TINY, tail / np.maximum(b_norms, TINY), 0.0)
            x = x + np.stack(V[:p], axis=1) @ y
        if converged_cycle:
            break
    tr, be = _true_metrics(A, x, B, b_true_norms)
    conv = bool(np.all(tr <= tolerance)) if true_residual_check else bool(np.all(projected <= tolerance))
    return BlockResult(x=x, iterations=total, residuals=projected, true_residuals=tr, backward_errors=be,
                       converged=conv)
