"""GCRO-DR restated in numpy -- TEST INFRASTRUCTURE ONLY (the checker of the device solver).

Follows the reference's gcro_dr_core (crates/sonium-solvers/crates/sonium-solvers-iterative/src/
gcro_dr.rs:339-760) step by step: build_c_r (:769-850), the per-cycle U correction (:438-452),
Arnoldi with two unconditional C projections before CGS + DGKS (0.707) against V (:510-580), Givens
(gmres_common.rs:91-106), the V and U corrections and the exact-residual acceptance (:636-720),
update_recycled_subspace (:922-1050) with the G_top^H solve (:1057-1090).

One deliberate difference: the harmonic-Ritz eigenproblem is solved with numpy's eig (LAPACK).
The reference reduces the matrix with Householder reflectors whose alpha is real
(gmres_dr.rs:1857-1950); for complex data those reflectors do not zero the column, and the
entries left below the subdiagonal are then discarded, so its eigenvalues are not exactly those
of the augmented matrix. This oracle (and the device solver) use the exact eigenpairs.

Only the tests import this module.
"""
from __future__ import annotations

import numpy as np


class Subspace:
    """GcroDrSubspace (gcro_dr.rs:65-110): the recycled vectors U and the target size k."""

    def __init__(self, k: int):
        self.k = int(k)
        self.u: list[np.ndarray] = []

    def is_populated(self) -> bool:
        return len(self.u) > 0


def _givens(a: complex, b: complex):
    """givens_rotation (gmres_common.rs:91-106)."""
    if abs(b) < 1e-30:
        return 1.0 + 0j, 0j
    if abs(a) < 1e-30:
        return 0j, 1.0 + 0j
    r = np.sqrt(abs(a) ** 2 + abs(b) ** 2)
    return a / r, b / r


def _upper_solve(R: np.ndarray, g: np.ndarray, k: int) -> np.ndarray:
    """solve_upper_triangular(_dense) (gmres_common.rs:108-127, gcro_dr.rs:853-870)."""
    y = np.zeros(k, np.complex128)
    for i in range(k - 1, -1, -1):
        s = g[i] - (R[i, i + 1:k] @ y[i + 1:k] if i + 1 < k else 0.0)
        if abs(R[i, i]) > 1e-30:
            y[i] = s / R[i, i]
    return y


def build_c_r(apply, u):
    """build_c_r (gcro_dr.rs:769-850): C orthonormal, R upper triangular, M^-1 A U = C R."""
    k_in = len(u)
    C = []
    R = np.zeros((k_in, k_in), np.complex128)
    matvecs = 0
    for j in range(k_in):
        z = apply(u[j])
        matvecs += 1
        if C:
            Cm = np.array(C)
            c1 = Cm.conj() @ z
            R[: len(C), j] = c1
            z = z - Cm.T @ c1
            c2 = Cm.conj() @ z
            R[: len(C), j] += c2
            z = z - Cm.T @ c2
        nz = np.linalg.norm(z)
        if nz < 1e-12:
            break
        R[j, j] = nz
        C.append(z / nz)
    return C, R, matvecs


def _unapply_givens(h: np.ndarray, cs, sn, steps: int) -> np.ndarray:
    """unapply_givens_local (gcro_dr.rs:874-900)."""
    h = h.copy()
    for j in range(steps - 1, -1, -1):
        if j >= len(cs):
            continue
        c, s = cs[j], sn[j]
        for col in range(j, steps):
            hj, hj1 = h[j, col], h[j + 1, col]
            h[j, col] = c * hj - np.conj(s) * hj1
            h[j + 1, col] = np.conj(s) * hj + np.conj(c) * hj1
    return h


def update_recycled_subspace(sub: Subspace, R, B, h_rot, cs, sn, V, steps: int, k_in: int):
    """update_recycled_subspace (gcro_dr.rs:922-1050)."""
    if sub.k == 0 or steps == 0:
        return
    total = k_in + steps
    h_raw = _unapply_givens(h_rot, cs, sn, steps)
    rho = h_raw[steps, steps - 1]
    G = np.zeros((total, total), np.complex128)
    G[:k_in, :k_in] = R[:k_in, :k_in]
    G[:k_in, k_in:] = B[:k_in, :steps]
    G[k_in:, k_in:] = h_raw[:steps, :steps]
    e = np.zeros(total, np.complex128)
    e[-1] = 1.0
    Gh = G.conj().T
    try:
        w = np.linalg.solve(Gh, e)
    except np.linalg.LinAlgError:
        try:
            w = np.linalg.solve(Gh + 1e-12 * np.eye(total), e)
        except np.linalg.LinAlgError:
            w = e.copy()
    M = G.copy()
    M[:, total - 1] += abs(rho) ** 2 * w
    lam, Y = np.linalg.eig(M)
    order = sorted(range(total), key=lambda i: abs(lam[i]))  # stable, ascending |theta|
    take = min(sub.k, total)
    new_u = []
    for idx in order[:take]:
        psi = np.zeros(V.shape[1], np.complex128)
        for i in range(k_in):
            psi += Y[i, idx] * sub.u[i]
        for j in range(steps):
            psi += Y[k_in + j, idx] * V[j]
        for prev in new_u:
            psi = psi - np.vdot(prev, psi) * prev
        nrm = np.linalg.norm(psi)
        if nrm > 1e-12:
            new_u.append(psi / nrm)
    if new_u:
        sub.u = new_u


def gcro_dr(A, b, sub: Subspace, max_iterations: int = 100, restart: int = 30, tol: float = 1e-6, x0=None,
            jacobi: bool = False):
    """gcro_dr_core (gcro_dr.rs:339-760) for a dense matrix A (identity or Jacobi left
    preconditioner). Returns a dict with x, iterations, restarts, residual, estimated, converged,
    status and matvecs; `sub` is updated in place."""
    A = np.asarray(A, np.complex128)
    b = np.asarray(b, np.complex128)
    n = b.shape[0]
    m = restart
    dinv = 1.0 / np.diag(A) if jacobi else None
    mv = [0]

    def prec(v):
        return dinv * v if jacobi else v

    def apply(v):
        mv[0] += 1
        return prec(A @ v)

    def exact(x):
        mv[0] += 1
        return np.linalg.norm(b - A @ x) / public_b

    x = np.zeros(n, np.complex128) if x0 is None else np.array(x0, np.complex128)
    if any(len(v) != n for v in sub.u):
        return dict(x=x, iterations=0, restarts=0, residual=np.inf, estimated=np.inf, converged=False,
                    status="NumericalError", matvecs=0)
    pb = prec(b)
    b_norm = np.linalg.norm(pb)
    true_b = np.linalg.norm(b)
    public_b = 1.0 if true_b < 1e-15 else true_b
    if b_norm < 1e-15:
        return dict(x=x, iterations=0, restarts=0, residual=0.0, estimated=0.0, converged=True,
                    status="Converged", matvecs=0)
    k = 0
    C, R = [], np.zeros((0, 0), np.complex128)
    if sub.is_populated():
        C, R, _ = build_c_r(apply, sub.u)  # its products are counted by apply
        if not C:
            sub.u = []
        k = len(C)
        sub.u = sub.u[:k]
    Cm = np.array(C) if k else None
    total_it = 0
    restarts = 0
    V = np.zeros((m + 1, n), np.complex128)
    h = np.zeros((m + 1, m), np.complex128)
    Bb = np.zeros((max(k, 1), m), np.complex128)
    cs, sn = [], []
    last_steps = 0

    def result(status, conv, res, est):
        return dict(x=x, iterations=total_it, restarts=restarts, residual=res, estimated=est, converged=conv,
                    status=status, matvecs=mv[0])

    for _outer in range(max_iterations):
        mv[0] += 1
        w = prec(b - A @ x)
        if k:
            alpha = Cm.conj() @ w
            w = w - Cm.T @ alpha
            zu = _upper_solve(R, alpha, k)
            for i in range(k):
                x = x + zu[i] * sub.u[i]
        beta = np.linalg.norm(w)
        rel0 = beta / b_norm
        if rel0 < tol:
            tr = exact(x)
            if tr < tol or tr < 1e-20:
                return result("Converged", True, tr, rel0)
        V[0] = w / beta
        h[:] = 0
        Bb[:] = 0
        cs, sn = [], []
        g = np.zeros(m + 1, np.complex128)
        g[0] = beta
        inner = False
        converged_at = None
        for j in range(m):
            total_it += 1
            w = apply(V[j])
            if k:
                c1 = Cm.conj() @ w
                Bb[:k, j] = c1
                w = w - Cm.T @ c1
                c2 = Cm.conj() @ w
                Bb[:k, j] += c2
                w = w - Cm.T @ c2
            wb = np.linalg.norm(w)
            hc = V[: j + 1].conj() @ w
            h[: j + 1, j] = hc
            w = w - V[: j + 1].T @ hc
            wn = np.linalg.norm(w)
            if wn < 0.707 * wb:
                hc2 = V[: j + 1].conj() @ w
                h[: j + 1, j] += hc2
                w = w - V[: j + 1].T @ hc2
                wn = np.linalg.norm(w)
            h[j + 1, j] = wn
            if wn < 1e-20:
                inner = True
            else:
                V[j + 1] = w / wn
            for i in range(j):
                t = np.conj(cs[i]) * h[i, j] + np.conj(sn[i]) * h[i + 1, j]
                h[i + 1, j] = -sn[i] * h[i, j] + cs[i] * h[i + 1, j]
                h[i, j] = t
            c, s = _givens(h[j, j], h[j + 1, j])
            cs.append(c)
            sn.append(s)
            h[j, j] = np.conj(c) * h[j, j] + np.conj(s) * h[j + 1, j]
            h[j + 1, j] = 0
            t = np.conj(c) * g[j] + np.conj(s) * g[j + 1]
            g[j + 1] = -s * g[j] + c * g[j + 1]
            g[j] = t
            absr = abs(g[j + 1])
            if absr / b_norm < tol or absr < 1e-20 or inner:
                converged_at = j
                break
        steps = m if converged_at is None else converged_at + 1
        last_steps = steps
        yv = _upper_solve(h, g, steps)
        x = x + V[:steps].T @ yv
        if k:
            by = -(Bb[:k, :steps] @ yv)
            zu = _upper_solve(R, by, k)
            for i in range(k):
                x = x + zu[i] * sub.u[i]
        rel_after = abs(g[steps]) / b_norm if steps else 0.0
        if converged_at is not None or rel_after < tol:
            tr = exact(x)
            if tr < tol or tr < 1e-20:
                update_recycled_subspace(sub, R, Bb, h, cs, sn, V, steps, k)
                return result("Converged", True, tr, rel_after)
            if inner:
                return result("Breakdown", False, tr, rel_after)
        restarts += 1
    update_recycled_subspace(sub, R, Bb, h, cs[:last_steps], sn[:last_steps], V, m, k)
    tr = exact(x)
    return result("MaxIterationsReached", False, tr, tr)


def helmholtz_like(n: int, freq: float) -> np.ndarray:
    """build_helmholtz_like of the reference's GCRO-DR tests (gcro_dr.rs:1096-1111): tridiagonal,
    diagonal 4 - 0.05 f^2 + 0.01 f i, off-diagonals -1."""
    k2 = freq * freq * 0.05
    A = np.zeros((n, n), np.complex128)
    i = np.arange(n)
    A[i, i] = 4.0 - k2 + 0.01j * freq
    A[i[1:], i[:-1]] = -1.0
    A[i[:-1], i[1:]] = -1.0
    return A
