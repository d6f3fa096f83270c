"""Discontinuous linear Tri3 basis (sb_assemble_linear; build_tbem_system_linear,
crates/sonium-bem/src/core/assembly/tbem.rs:1490-1620).

CPU: the oracle's restatement pinned by identities the reference's formulas imply (the three
basis functions sum to one and their gradients to zero, so the summed linear channels equal the
constant-basis channels of the same source point, the self term when that point is the
centroid), and by convergence of the solved rigid sphere to the Mie series. GPU: the device
matrix against the oracle's entry by entry (1e-10 relative to the entry, floor 1e-8 of the
largest), the collocation points and incident right-hand side, re-assembly at another
frequency, the GMRES solution against the oracle's dense solve.
"""
import numpy as np
import pytest


def _coords(nodes, tris, e):
    return nodes[tris[e]].copy()


# ---- CPU: the oracle ----

@pytest.mark.parametrize("k", [0.5, 2.0, 9.0])
def test_oracle_linear_channels_sum_to_constant(oracle, k):
    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    c, nrm, ar = oracle.element_geometry(nodes, tris)
    pts, pn = oracle.linear_collocation(nodes, tris)
    ph = oracle.physics_for_k(k)
    rng = np.random.default_rng(3)
    for r in rng.choice(pts.shape[0], 12, replace=False):
        i = r // 3
        for j in (i + 1, (i + 7) % tris.shape[0], int(rng.integers(tris.shape[0]))):
            if j == i:
                continue
            lin = oracle.regular_pair_linear(pts[r], pn[r], _coords(nodes, tris, j), ar[j], ph).sum(axis=0)
            con = oracle.regular_pair(pts[r], pn[r], _coords(nodes, tris, j), ar[j], ph)
            assert np.max(np.abs(lin - con)) <= 1e-12 * np.max(np.abs(con)), (r, j)
    for e in (0, 5, 77):
        lin = oracle.singular_pair_linear(c[e], nrm[e], _coords(nodes, tris, e), ph).sum(axis=0)
        con = oracle.singular_pair(c[e], nrm[e], _coords(nodes, tris, e), ph)
        assert np.max(np.abs(lin - con)) <= 1e-11 * np.max(np.abs(con)), e


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
