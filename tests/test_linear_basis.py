"""Discontinuous linear and quadratic Tri3 bases (sb_assemble_linear, sb_assemble_discontinuous;
build_tbem_system_linear and build_tbem_system_discontinuous_stabilized,
crates/sonium-bem/src/core/assembly/tbem.rs:1490-1620, 2810-2990).

CPU: the oracle's restatement pinned by identities the reference's formulas imply (the basis
functions sum to one and their gradients to zero, so the summed basis channels equal the
constant-basis channels of the same source point, the self term when that point is the
centroid), by convergence of the solved linear-basis rigid sphere to the Mie series, and for the
quadratic basis by the reference's own Mie bound. GPU: the device
matrix against the oracle's entry by entry (1e-10 relative to the entry, floor 1e-8 of the
largest), the collocation points and incident right-hand side, re-assembly at another
frequency, the GMRES solution against the oracle's dense solve.
"""
import numpy as np
import pytest


def _coords(nodes, tris, e):
    return nodes[tris[e]].copy()


# ---- CPU: the oracle ----

@pytest.mark.parametrize("nbas", [3, 6])
@pytest.mark.parametrize("k", [0.5, 2.0, 9.0])
def test_oracle_basis_channels_sum_to_constant(oracle, k, nbas):
    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    c, nrm, ar = oracle.element_geometry(nodes, tris)
    pts, pn = oracle.disc_collocation(nodes, tris, nbas)
    ph = oracle.physics_for_k(k)
    rng = np.random.default_rng(3)
    for r in rng.choice(pts.shape[0], 12, replace=False):
        i = r // nbas
        for j in (i + 1, (i + 7) % tris.shape[0], int(rng.integers(tris.shape[0]))):
            if j == i or j >= tris.shape[0]:
                continue
            lin = oracle.regular_pair_disc(pts[r], pn[r], _coords(nodes, tris, j), ar[j], ph, nbas).sum(axis=0)
            con = oracle.regular_pair(pts[r], pn[r], _coords(nodes, tris, j), ar[j], ph)
            assert np.max(np.abs(lin - con)) <= 1e-12 * np.max(np.abs(con)), (r, j)
    for e in (0, 5, 77):
        lin = oracle.singular_pair_disc(c[e], nrm[e], _coords(nodes, tris, e), ph, nbas).sum(axis=0)
        con = oracle.singular_pair(c[e], nrm[e], _coords(nodes, tris, e), ph)
        assert np.max(np.abs(lin - con)) <= 1e-11 * np.max(np.abs(con)), e


def test_oracle_quadratic_sign_and_sphere(oracle):
    nodes, tris = oracle.icosphere(1.0, 1)
    ph = oracle.physics_for_k(2.0)
    beta = oracle.bm_beta(ph)
    Ap, _ = oracle.assemble_discontinuous(nodes, tris, ph, beta, 6, 1.0)
    Am, _ = oracle.assemble_discontinuous(nodes, tris, ph, beta, 6, -1.0)
    assert np.array_equal(Am, -Ap)
    # The unknowns are the quadratic Lagrange coefficients (vertex and edge-midpoint values), so
    # the surface pressure at collocation point c is sum_b x_b N_b(point c). The reference bounds
    # its own quadratic-panel Mie error at 0.80 (tests/higher_order_formulation_reference.rs:
    # 264-283): the free term sits on the diagonal as if the basis were cardinal at the
    # collocation points, which the quadratic one is not.
    a, b_, c, d = 0.8168475729804585, 0.0915762135097715, 0.108103018168070, 0.445948490915965
    coll = [(b_, b_), (a, b_), (b_, a), (d, d), (d, c), (c, d)]

    def p2(s, t):
        l0 = 1 - s - t
        return [l0 * (2 * l0 - 1), s * (2 * s - 1), t * (2 * t - 1), 4 * l0 * s, 4 * s * t, 4 * t * l0]

    N = np.array([p2(s, t) for s, t in coll])
    for level in (1, 2):
        nodes, tris = oracle.icosphere(1.0, level)
        A, _ = oracle.assemble_discontinuous(nodes, tris, ph, beta, 6)
        pts, pn = oracle.disc_collocation(nodes, tris, 6)
        b = oracle.rhs_plane_wave(pts, pn, ph, beta, [[0.0, 0.0, 1.0]])[:, 0]
        x = np.linalg.solve(A, b)
        p = (N @ x.reshape(-1, 6).T).T.reshape(-1)
        _, _, ar = oracle.element_geometry(nodes, tris)
        err = oracle.rigid_sphere_surface_error(p, pts, np.repeat(ar / 6, 6), 2.0, 1.0)
        assert np.isfinite(err) and err < 0.8, (level, err)


def test_oracle_linear_collocation_points(oracle):
    nodes, tris = oracle.icosphere(1.0, 1)
    pts, pn = oracle.linear_collocation(nodes, tris)
    for e in (0, 13):
        v = nodes[tris[e]]
        for q, (s, t) in enumerate([(1 / 6, 1 / 6), (2 / 3, 1 / 6), (1 / 6, 2 / 3)]):
            assert np.allclose(pts[3 * e + q], (1 - s - t) * v[0] + s * v[1] + t * v[2], atol=1e-15)
    c, nrm, _ = oracle.element_geometry(nodes, tris)
    assert np.array_equal(pn[::3], nrm)


def test_oracle_linear_sphere_converges_to_mie(oracle):
    errs = []
    for level in (1, 2, 3):
        nodes, tris = oracle.icosphere(1.0, level)
        ph = oracle.physics_for_k(2.0)
        beta = oracle.bm_beta(ph)
        A, rhs = oracle.assemble_linear(nodes, tris, ph, beta)
        assert np.all(rhs == 0)
        pts, pn = oracle.linear_collocation(nodes, tris)
        b = oracle.rhs_plane_wave(pts, pn, ph, beta, [[0.0, 0.0, 1.0]])[:, 0]
        x = np.linalg.solve(A, b)
        _, _, ar = oracle.element_geometry(nodes, tris)
        errs.append(oracle.rigid_sphere_surface_error(x, pts, np.repeat(ar / 3, 3), 2.0, 1.0))
    assert errs[0] > errs[1] > errs[2] and errs[2] < 0.03, errs


# ---- GPU: the device assembly against the oracle ----

@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _entry_err(A, R):
    floor = 1e-8 * np.abs(R).max()
    return float(np.max(np.abs(A - R) / np.maximum(np.abs(R), floor)))


@pytest.mark.gpu
@pytest.mark.parametrize("level,k,scale", [(1, 2.0, (1.0, 1.0, 1.0)), (2, 0.4, (1.0, 0.6, 0.4)),
                                           (2, 7.0, (1.0, 1.0, 1.0)), (2, 15.0, (1.0, 0.6, 0.4))])
def test_linear_matrix_matches_oracle(gpu, oracle, level, k, scale):
    nodes, tris = oracle.icosphere(1.0, level, scale)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_linear(mesh, ph, beta)
    A = op.matrix
    R, _ = oracle.assemble_linear(nodes, tris, oracle.physics_for_k(k), beta)
    assert A.shape == (3 * tris.shape[0],) * 2
    assert _entry_err(A, R) < 1e-10
    assert np.all(op.rhs == 0)
    op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("level,k,sign", [(1, 2.0, 1.0), (2, 7.0, -1.0)])
def test_quadratic_matrix_matches_oracle(gpu, oracle, level, k, sign):
    nodes, tris = oracle.icosphere(1.0, level, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(k)
    op = gpu.build_tbem_system_quadratic_stabilized(mesh, ph, sign=sign, beta_scale=4.0)
    R, _ = oracle.assemble_discontinuous(nodes, tris, oracle.physics_for_k(k), ph.burton_miller_beta(4.0), 6, sign)
    assert op.n == 6 * tris.shape[0]
    assert _entry_err(op.matrix, R) < 1e-10
    pts, pn = mesh.collocation(gpu.SB_BASIS_QUADRATIC)
    opts, _ = oracle.disc_collocation(nodes, tris, 6)
    assert np.max(np.abs(pts - opts)) <= 1e-15
    # (the quadratic system is poorly conditioned for restarted GMRES: its free term treats the
    # non-cardinal basis as cardinal; the product is what a solver sees)
    x = gpu.rhs_plane_wave_at(pts, pn, ph, op.beta, [0.0, 0.0, 1.0])[:, 0]
    assert np.linalg.norm(op.apply(x) - R @ x) <= 1e-13 * np.linalg.norm(R @ x)
    op.close()


@pytest.mark.gpu
def test_linear_admittance_and_reassembly(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2)
    m = tris.shape[0]
    mesh = gpu.Mesh(nodes, tris)
    adm = np.full(m, np.nan, complex)
    adm[::5] = 0.02 - 0.01j
    mesh.set_boundary_conditions(admittance=adm)
    ph1, ph2 = gpu.PhysicsParams.for_wavenumber(2.0), gpu.PhysicsParams.for_wavenumber(3.3)
    b1, b2 = ph1.burton_miller_beta(), ph2.burton_miller_beta()
    op = gpu.build_tbem_system_linear(mesh, ph1, b1)
    op.reassemble(ph2, b2)
    R, _ = oracle.assemble_linear(nodes, tris, oracle.physics_for_k(3.3), b2, admittance=adm)
    assert _entry_err(op.matrix, R) < 1e-10
    op.close()
    # prescribed values are not part of the linear path
    mesh.set_boundary_conditions(value=np.ones(m, complex))
    with pytest.raises(gpu.SoniumError):
        gpu.build_tbem_system_linear(mesh, ph1, b1)


@pytest.mark.gpu
def test_linear_collocation_rhs_and_solve(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2)
    mesh = gpu.Mesh(nodes, tris)
    pts, pn = mesh.collocation(gpu.SB_BASIS_LINEAR)
    opts, opn = oracle.linear_collocation(nodes, tris)
    assert np.max(np.abs(pts - opts)) <= 1e-15 and np.array_equal(pn, opn)
    cpts, cpn = mesh.collocation(gpu.SB_BASIS_CONSTANT)
    c, nrm, _ = oracle.element_geometry(nodes, tris)
    assert np.max(np.abs(cpts - c)) <= 1e-15 and np.max(np.abs(cpn - nrm)) <= 1e-15
    ph = gpu.PhysicsParams.for_wavenumber(2.0)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave_at(pts, pn, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    b_ref = oracle.rhs_plane_wave(opts, opn, oracle.physics_for_k(2.0), beta, [[0.0, 0.0, 1.0]])[:, 0]
    assert np.max(np.abs(b - b_ref)) <= 1e-13 * np.max(np.abs(b_ref))
    op = gpu.build_tbem_system_linear(mesh, ph, beta)
    sol = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=100, restart=50, tolerance=1e-10))
    A_ref, _ = oracle.assemble_linear(nodes, tris, oracle.physics_for_k(2.0), beta)
    x_ref = np.linalg.solve(A_ref, b_ref)
    assert sol.converged and np.linalg.norm(sol.x - x_ref) / np.linalg.norm(x_ref) < 1e-8
    _, _, ar = oracle.element_geometry(nodes, tris)
    e_dev = oracle.rigid_sphere_surface_error(sol.x, pts, np.repeat(ar / 3, 3), 2.0, 1.0)
    e_ref = oracle.rigid_sphere_surface_error(x_ref, opts, np.repeat(ar / 3, 3), 2.0, 1.0)
    assert abs(e_dev - e_ref) < 1e-8
    op.close()
