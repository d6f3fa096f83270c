"""GPU parity of the CUDA path against the CPU oracle, through the C ABI.

Bars (written into each test):
  * matrix / RHS entries: relative 1e-10 per entry (entries below 1e-8 of the matrix maximum are
    held to 1e-10 of that maximum instead), plus the reference's own 1e-9 Frobenius bound
    (crates/sonium-bem/src/core/assembly/tbem.rs:6533-6625),
  * matvec products (N, T, C): relative 1e-12 against numpy on the same matrix,
  * GMRES: same Krylov iteration count as the oracle and a solution within 1e-7,
  * mixed precision: surface pressure within 1e-5 of the FP64 solution.
"""
import json
from decimal import Decimal

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


def entry_error(A, R):
    """Max relative per-entry error with a floor of 1e-8 * max|R|."""
    floor = 1e-8 * np.abs(R).max()
    return float(np.max(np.abs(A - R) / np.maximum(np.abs(R), floor)))


def frob(A, R):
    return float(np.linalg.norm(A - R) / np.linalg.norm(R))


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def test_device_sincos_matches_golden(gpu):
    from sonium_b200 import _lib as L

    g = json.load(open(golden_path("sincos_golden.json")))
    xs, ss, cs = [], [], []
    for c in g["cases"]:
        xv = float(Decimal(c["x"]))
        xs.append(xv)
        if Decimal(xv) == Decimal(c["x"]):
            ss.append(float(Decimal(c["sin"])))
            cs.append(float(Decimal(c["cos"])))
        else:
            # golden taken at a decimal that is not a binary64 value (exact pi, or the midpoint
            # between two doubles next to k pi/2): the device evaluates the rounded double, whose
            # correctly rounded sin / cos the host libm supplies
            ss.append(float(np.sin(xv)))
            cs.append(float(np.cos(xv)))
    x = np.array(xs)
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    L.check(L.load().sb_math_sincos(0, x.ctypes.data, len(x), s.ctypes.data, c.ctypes.data))
    # The reference's fastmath contract is a few ulp (crates/sonium-fastmath/src/lib.rs:59-62);
    # hold the device sin/cos to 4 ulp of the correctly rounded golden value.
    ss, cs = np.array(ss), np.array(cs)
    es = np.abs(s - ss) / np.maximum(np.spacing(np.abs(ss)), 5e-324)
    ec = np.abs(c - cs) / np.maximum(np.spacing(np.abs(cs)), 5e-324)
    bad = [(x[i], es[i], ec[i]) for i in range(len(x)) if es[i] > 4 or ec[i] > 4]
    assert not bad, bad
    # a dense sweep over the assembly's argument range against numpy (libm)
    x = np.linspace(-700.0, 700.0, 200_001)
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    L.check(L.load().sb_math_sincos(0, x.ctypes.data, len(x), s.ctypes.data, c.ctypes.data))
    assert np.max(np.abs(s - np.sin(x))) < 4e-16 and np.max(np.abs(c - np.cos(x))) < 4e-16


def assemble_both(sb, oracle, nodes, tris, k, beta_scale=1.0, bc=None, precision=0, rows=None):
    nodes = np.ascontiguousarray(nodes)
    ph_o = oracle.physics_for_k(k)
    beta = oracle.bm_beta(ph_o, beta_scale)
    kw = {} if bc is None else bc
    A_o, r_o = oracle.assemble(nodes, tris, ph_o, beta, rows=rows, **kw)
    mesh = sb.Mesh(nodes, tris)
    if bc is not None:
        mesh.set_boundary_conditions(bc.get("bc_kind"), bc.get("bc_value"), bc.get("admittance"))
    ph = sb.PhysicsParams.for_wavenumber(k)
    assert ph.wave_number == ph_o.wave_number
    op = sb.build_tbem_system_with_beta(mesh, ph, beta, precision)
    return op, A_o, r_o, mesh, ph, beta


def test_assembly_parity_reference_fixture(gpu, oracle):
    """The reference's own CUDA parity case: icosphere level 2, k = 1, element 0 velocity 1."""
    nodes, tris = oracle.icosphere(1.0, 2)
    m = tris.shape[0]
    val = np.zeros(m, complex)
    val[0] = 1.0
    op, A_o, r_o, *_ = assemble_both(gpu, oracle, nodes, tris, 1.0, bc={"bc_value": val})
    A = op.matrix
    assert entry_error(A, A_o) < 1e-10
    assert frob(A, A_o) < 1e-9
    r = op.rhs
    assert np.abs(r_o).max() > 0
    assert entry_error(r[:, None], r_o[:, None]) < 1e-10
    assert frob(r, r_o) < 1e-9


def test_assembly_parity_sphere_level3_k2(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 3)
    op, A_o, r_o, *_ = assemble_both(gpu, oracle, nodes, tris, 2.0)
    assert entry_error(op.matrix, A_o) < 1e-10


def test_assembly_parity_fp32_copy(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2)
    op, A_o, *_ = assemble_both(gpu, oracle, nodes, tris, 3.0, precision=gpu.SB_PRECISION_FP64_FP32)
    A32 = op.matrix_c64()
    assert entry_error(op.matrix, A_o) < 1e-10
    assert np.array_equal(A32, op.matrix.astype(np.complex64))


@pytest.mark.parametrize("k", [4.0, 12.0, 40.0, 90.0])
def test_assembly_parity_self_rule_brackets(gpu, oracle, k):
    """Level 1 (sqrt(area) ~ 0.21) spans every QuadratureParams::for_ka bracket (singular.rs:51-85)."""
    nodes, tris = oracle.icosphere(1.0, 1)
    op, A_o, *_ = assemble_both(gpu, oracle, nodes, tris, k)
    assert entry_error(op.matrix, A_o) < 1e-10


def test_assembly_parity_ellipsoid_mixed_bcs(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    m = tris.shape[0]
    kind = np.zeros(m, np.int32)
    kind[::3] = 1
    val = np.linspace(0.1, 1.0, m) * (1 + 0.5j)
    val[5::7] = 0
    adm = np.full(m, np.nan + 0j)
    adm[1::4] = 0.01 - 0.002j
    bc = {"bc_kind": kind, "bc_value": val, "admittance": adm}
    op, A_o, r_o, *_ = assemble_both(gpu, oracle, nodes, tris, 5.0, beta_scale=0.2, bc=bc)
    assert entry_error(op.matrix, A_o) < 1e-10
    assert entry_error(op.rhs[:, None], r_o[:, None]) < 1e-10


def test_near_pair_deep_subdivision(gpu, oracle):
    """A source point 1e-4 above a large panel: the tree hits the 15-split / 110-leaf limits."""
    nodes = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0],
                      [0.29, 0.29, 1e-4], [0.31, 0.30, 1e-4], [0.30, 0.31, 1e-4],
                      [0.6, 0.1, 0.02], [0.62, 0.1, 0.02], [0.6, 0.13, 0.03]])
    tris = np.array([[0, 1, 2], [3, 4, 5], [6, 7, 8]], np.uint32)
    leaves = oracle.subelements(oracle.element_geometry(nodes, tris)[0][1], nodes[:3], 0.5)
    assert len(leaves) == 110
    op, A_o, *_ = assemble_both(gpu, oracle, nodes, tris, 3.0)
    assert entry_error(op.matrix, A_o) < 1e-10


def test_full_size_rows_match_oracle(gpu, oracle):
    """Level-5 sphere (N = 20480), k = 10: sampled rows against the oracle's row assembly."""
    nodes, tris = oracle.icosphere(1.0, 5)
    ph_o = oracle.physics_for_k(10.0)
    beta = oracle.bm_beta(ph_o)
    mesh = gpu.Mesh(nodes, tris)
    op = gpu.build_tbem_system_with_beta(mesh, gpu.PhysicsParams.for_wavenumber(10.0), beta)
    n = tris.shape[0]
    for r in (0, 1, 4097, n // 2 + 3, n - 1):
        A_o, _ = oracle.assemble(nodes, tris, ph_o, beta, rows=(r, r + 1))
        assert entry_error(op.rows(r, r + 1), A_o) < 1e-10, r


def test_rhs_plane_wave_parity(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    ph_o = oracle.physics_for_k(7.0)
    beta = oracle.bm_beta(ph_o)
    c, nrm, a = oracle.element_geometry(nodes, tris)
    rng = np.random.default_rng(0x5EED)
    dirs = rng.standard_normal((5, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    amps = rng.standard_normal(5) + 1j * rng.standard_normal(5)
    ref = oracle.rhs_plane_wave(c, nrm, ph_o, beta, dirs, amps)
    mesh = gpu.Mesh(nodes, tris)
    got = gpu.rhs_plane_wave(mesh, gpu.PhysicsParams.for_wavenumber(7.0), beta, dirs, amps)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.abs(ref).max()
    gc, gn, ga = mesh.element_geometry()
    assert np.array_equal(gc, c) and np.array_equal(gn, nrm) and np.array_equal(ga, a)


def test_matvec_parity(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 3)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(2.0)
    op = gpu.build_tbem_system(mesh, ph)
    A = op.matrix
    n = A.shape[0]
    probe = 0.25 + np.arange(n) * 0.003 + 1j * (-0.1 + np.arange(n) * 0.002)  # tbem.rs:6640-6642
    for fn, ref in ((op.apply_into, A @ probe), (op.apply_transpose_into, A.T @ probe),
                    (op.apply_hermitian_into, A.conj().T @ probe)):
        y = np.zeros(n, complex)
        fn(probe, y)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12
    X = np.stack([probe, probe[::-1] * 1j, np.ones(n)], axis=1)
    assert np.linalg.norm(op.apply_block(X) - A @ X) / np.linalg.norm(A @ X) < 1e-12
    y = np.zeros(n, complex)
    bad = probe.copy()
    bad[3] = np.nan
    with pytest.raises(gpu.SoniumError):
        op.apply_into(bad, y)


def test_gmres_parity_config1(gpu, oracle):
    """Sphere level 3, k = 2, beta = i/k, GMRES(30) to 1e-8: iterations and solution vs the oracle."""
    nodes, tris = oracle.icosphere(1.0, 3)
    ph_o = oracle.physics_for_k(2.0)
    beta = oracle.bm_beta(ph_o)
    A_o, r_o = oracle.assemble(nodes, tris, ph_o, beta)
    c, nrm, a = oracle.element_geometry(nodes, tris)
    b = r_o + oracle.rhs_plane_wave(c, nrm, ph_o, beta, [0, 0, 1])[:, 0]
    x_o, res_o = oracle.gmres(A_o, b, restart=30, max_iterations=100, tol=1e-8)
    mesh = gpu.Mesh(nodes, tris)
    op = gpu.build_tbem_system_with_beta(mesh, gpu.PhysicsParams.for_wavenumber(2.0), beta)
    sol = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=100, restart=30, tolerance=1e-8))
    assert sol.converged and sol.status == "Converged"
    assert abs(sol.iterations - res_o.iterations) <= 1
    assert np.linalg.norm(sol.x - x_o) / np.linalg.norm(x_o) < 1e-7
    assert sol.residual < 1e-8
    e_gpu = oracle.rigid_sphere_surface_error(sol.x, c, a, ph_o.wave_number, 1.0)
    e_cpu = oracle.rigid_sphere_surface_error(x_o, c, a, ph_o.wave_number, 1.0)
    assert abs(e_gpu - e_cpu) < 1e-6 and e_gpu < 0.01


def test_gmres_jacobi_and_restart(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(6.0)
    op = gpu.build_tbem_system(mesh, ph)
    b = gpu.rhs_plane_wave(mesh, ph, ph.burton_miller_beta(), [0, 0, 1])[:, 0]
    A = op.matrix
    xr = np.linalg.solve(A, b)
    s1 = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=200, restart=5, tolerance=1e-10))
    s2 = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=200, restart=40, tolerance=1e-10),
                   preconditioner=gpu.JacobiPreconditioner(op))
    for s in (s1, s2):
        assert s.converged and np.linalg.norm(s.x - xr) / np.linalg.norm(xr) < 1e-8
    assert s1.restarts > 0
    s3 = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=1, restart=2, tolerance=1e-14))
    assert not s3.converged and s3.status == "MaxIterationsReached"


def test_mixed_precision_solution_within_1e5(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 3)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(2.0)
    op = gpu.build_tbem_system(mesh, ph, precision=gpu.SB_PRECISION_FP64_FP32)
    b = gpu.rhs_plane_wave(mesh, ph, ph.burton_miller_beta(), [0, 0, 1])[:, 0]
    x64 = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=100, restart=30, tolerance=1e-10)).x
    mix = gpu.gmres_mixed(op, b, gpu.IrConfig(tolerance=1e-10))
    assert mix.converged and mix.refinements >= 2 and mix.matvecs_fp32 > 0
    assert np.linalg.norm(mix.x - x64) / np.linalg.norm(x64) < 1e-5
    assert mix.residual < 1e-10


def test_fault_injection_and_recovery(gpu, oracle):
    """tbem.rs:6740-6794: an injected failure is a typed error and the backend recovers."""
    nodes, tris = oracle.icosphere(1.0, 1)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(1.0)
    gpu.inject_failure(gpu.SB_INJECT_LAUNCH)
    with pytest.raises(gpu.SoniumError) as e:
        gpu.build_tbem_system(mesh, ph)
    assert "injected" in str(e.value)
    gpu.inject_failure(gpu.SB_INJECT_ALLOC)
    with pytest.raises(gpu.SoniumError):
        gpu.build_tbem_system(mesh, ph)
    op = gpu.build_tbem_system(mesh, ph)
    A_o, _ = oracle.assemble(nodes, tris, oracle.physics_for_k(1.0), ph.burton_miller_beta())
    assert entry_error(op.matrix, A_o) < 1e-10


def test_reassemble_in_place(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2)
    mesh = gpu.Mesh(nodes, tris)
    op = gpu.build_tbem_system(mesh, gpu.PhysicsParams.for_wavenumber(1.0))
    ph2 = gpu.PhysicsParams.for_wavenumber(3.0)
    op.reassemble(ph2, ph2.burton_miller_beta())
    A_o, _ = oracle.assemble(nodes, tris, oracle.physics_for_k(3.0), ph2.burton_miller_beta())
    assert entry_error(op.matrix, A_o) < 1e-10


@pytest.mark.parametrize("level,k,scale", [(3, 2.0, None), (3, 6.0, (1.0, 0.6, 0.4)), (3, 12.0, None)])
def test_mixed_assembly_entries_within_fp32_tolerance(gpu, oracle, level, k, scale):
    """SB_PRECISION_FP32: far pairs in FP32 with the FP64 phase argument; near/self pairs FP64.

    Bar: every entry within 3e-5 relative of the FP64 oracle (floor 1e-6 of the matrix maximum;
    FP32 sums of the 13 leaf points with cancellation next to the near threshold reach ~1e-5 on
    meshes with 5 elements per wavelength), the median entry within 1e-6; near and self entries
    are the FP64 values rounded to complex64. The solution bar (1e-5) is tested below."""
    nodes, tris = oracle.icosphere(1.0, level, scale or (1.0, 1.0, 1.0))
    op, A_o, *_ = assemble_both(gpu, oracle, nodes, tris, k, precision=gpu.SB_PRECISION_FP32)
    A = op.matrix
    floor = 1e-6 * np.abs(A_o).max()
    err = np.abs(A - A_o) / np.maximum(np.abs(A_o), floor)
    assert err.max() < 3e-5, err.max()
    assert np.median(err) < 1e-6, np.median(err)
    d = np.diag_indices(A.shape[0])
    assert np.array_equal(A[d], A_o[d].astype(np.complex64).astype(np.complex128))


def test_mixed_assembly_solution_within_1e5(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 4)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(6.0)
    beta = ph.burton_miller_beta()
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0, 0, 1])[:, 0]
    op64 = gpu.build_tbem_system(mesh, ph)
    x64 = gpu.gmres(op64, b, gpu.GmresConfig(max_iterations=100, restart=50, tolerance=1e-10)).x
    op32 = gpu.build_tbem_system(mesh, ph, precision=gpu.SB_PRECISION_FP32)
    mix = gpu.gmres_mixed(op32, b, gpu.IrConfig(tolerance=1e-8))
    assert mix.converged
    assert np.linalg.norm(mix.x - x64) / np.linalg.norm(x64) < 1e-5
    c, nrm, a = mesh.element_geometry()
    e64 = oracle.rigid_sphere_surface_error(x64, c, a, ph.wave_number, 1.0)
    e32 = oracle.rigid_sphere_surface_error(mix.x, c, a, ph.wave_number, 1.0)
    assert abs(e32 - e64) < 1e-5
