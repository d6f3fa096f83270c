"""Quad4 constant panels (sb_mesh_create_quad4 + sb_assemble: the ElementType::Quad4 branches of
crates/sonium-bem/src/core/integration/{regular,singular,gauss}.rs and mesh/generators.rs).

CPU: the oracle's Quad4 restatement on a cubed sphere converges to the Mie series, and its
geometry follows the reference's conventions (centre = node average, diagonal normal, mean-split
area). GPU: the device matrix against the oracle entry by entry (1e-10 of the entry, floor 1e-8
of the largest) on spheres and ellipsoids across the self-term ka brackets, with admittance; the
GMRES solution and the Mie error equal the oracle's; Tri3-only entry points reject Quad4 meshes.
"""
import numpy as np
import pytest


def test_oracle_quad_geometry_and_mie(oracle):
    nodes, quads = oracle.cubed_sphere(1.0, 4)
    c, nrm, ar = oracle.quad_geometry(nodes, quads)
    p = nodes[quads]
    assert np.allclose(c, p.mean(axis=1), atol=1e-15)
    d = np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 1])
    assert np.allclose(nrm, d / np.linalg.norm(d, axis=1, keepdims=True), atol=1e-15)
    assert np.all(np.sum(c * nrm, axis=1) > 0)  # outward on the test mesh
    errs = []
    for n in (3, 6, 10):
        nodes, quads = oracle.cubed_sphere(1.0, n)
        c, nrm, ar = oracle.quad_geometry(nodes, quads)
        ph = oracle.physics_for_k(2.0)
        beta = oracle.bm_beta(ph)
        A, rhs = oracle.assemble_quad(nodes, quads, ph, beta)
        assert np.all(rhs == 0)
        b = oracle.rhs_plane_wave(c, nrm, ph, beta, [[0.0, 0.0, 1.0]])[:, 0]
        errs.append(oracle.rigid_sphere_surface_error(np.linalg.solve(A, b), c, ar, 2.0, 1.0))
    assert errs[0] > errs[1] > errs[2] and errs[2] < 0.02, errs


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _entry_err(A, R):
    floor = 1e-8 * np.abs(R).max()
    return float(np.max(np.abs(A - R) / np.maximum(np.abs(R), floor)))


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,scale", [(3, 2.0, (1.0, 1.0, 1.0)), (6, 0.5, (1.0, 0.6, 0.4)),
                                       (6, 6.0, (1.0, 1.0, 1.0)), (8, 14.0, (1.0, 0.6, 0.4))])
def test_quad_matrix_matches_oracle(gpu, oracle, n, k, scale):
    nodes, quads = oracle.cubed_sphere(1.0, n, scale)
    mesh = gpu.Mesh.quad4(nodes, quads)
    c, nrm, ar = oracle.quad_geometry(nodes, quads)
    dc, dn = mesh.collocation(gpu.SB_BASIS_CONSTANT)
    assert np.max(np.abs(dc - c)) <= 1e-15 and np.max(np.abs(dn - nrm)) <= 1e-15
    ph = gpu.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    R, _ = oracle.assemble_quad(nodes, quads, oracle.physics_for_k(k), beta)
    assert _entry_err(op.matrix, R) < 1e-10
    op.close()


@pytest.mark.gpu
def test_quad_admittance_solve_and_rejections(gpu, oracle):
    nodes, quads = oracle.cubed_sphere(1.0, 6)
    m = quads.shape[0]
    mesh = gpu.Mesh.quad4(nodes, quads)
    adm = np.full(m, np.nan, complex)
    adm[::4] = 0.01 + 0.02j
    mesh.set_boundary_conditions(admittance=adm)
    ph = gpu.PhysicsParams.for_wavenumber(2.0)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    R, _ = oracle.assemble_quad(nodes, quads, oracle.physics_for_k(2.0), beta, admittance=adm)
    assert _entry_err(op.matrix, R) < 1e-10
    op.close()
    mesh.set_boundary_conditions()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    sol = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=100, restart=50, tolerance=1e-10))
    A_ref, _ = oracle.assemble_quad(nodes, quads, oracle.physics_for_k(2.0), beta)
    x_ref = np.linalg.solve(A_ref, b)
    assert sol.converged and np.linalg.norm(sol.x - x_ref) / np.linalg.norm(x_ref) < 1e-8
    c, _, ar = oracle.quad_geometry(nodes, quads)
    e_dev = oracle.rigid_sphere_surface_error(sol.x, c, ar, 2.0, 1.0)
    e_ref = oracle.rigid_sphere_surface_error(x_ref, c, ar, 2.0, 1.0)
    assert abs(e_dev - e_ref) < 1e-8
    op.close()
    with pytest.raises(gpu.SoniumError):
        gpu.build_tbem_system_with_beta(mesh, ph, beta, gpu.SB_PRECISION_FP32)
    with pytest.raises(gpu.SoniumError):
        gpu.build_tbem_system_linear(mesh, ph, beta)
    with pytest.raises(gpu.SoniumError):
        gpu.compute_scattered_field(mesh, ph, np.ones(m, complex), np.array([[0.0, 0.0, 3.0]]))
    with pytest.raises(gpu.SoniumError):
        gpu.Mesh.quad4(nodes, np.array([[0, 1, 2, nodes.shape[0]]], np.uint32))
