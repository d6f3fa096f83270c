"""GCRO-DR subspace recycling (sb_gcro_dr, crates/sonium-solvers/crates/sonium-solvers-iterative/src/
gcro_dr.rs:339-1090) and the recycling frequency sweep (frequency_sweep.rs:592-850).

CPU: the oracle's restatement (oracle/gcro_oracle.py) against the reference's own GCRO-DR tests
(gcro_dr.rs:1113-1330: first solve, recycled second solve, equality with GMRES, the 100-frequency
sweep win, the diagonal smoke case). GPU: the device solver against the oracle on the reference's
test operators and on assembled TBEM systems of consecutive frequencies (solutions within 1e-8
relative, iteration counts within one), subspace bookkeeping and input rejection.
"""
import numpy as np
import pytest

from oracle import gcro_oracle as G


# ---- CPU: the oracle pinned by the reference's GCRO-DR tests ----

def test_oracle_first_solve_with_empty_subspace_converges():
    A = G.helmholtz_like(40, 1.0)
    b = np.sin(np.arange(40)).astype(complex)
    sub = G.Subspace(8)
    r = G.gcro_dr(A, b, sub, max_iterations=100, restart=30, tol=1e-10)
    err = np.linalg.norm(A @ r["x"] - b)
    assert r["converged"]
    assert abs(r["residual"] - err / np.linalg.norm(b)) < 1e-12
    assert err < 1e-7
    assert sub.is_populated()


def test_oracle_sequential_solves_use_recycled_subspace():
    n = 60
    b = np.cos(np.arange(n)) + 0.5j
    sub = G.Subspace(10)
    s0 = G.gcro_dr(G.helmholtz_like(n, 1.0), b, sub, 100, 30, 1e-9)
    s1 = G.gcro_dr(G.helmholtz_like(n, 1.05), b, sub, 100, 30, 1e-9)
    assert s0["converged"] and s1["converged"]
    assert s1["iterations"] <= s0["iterations"]


def test_oracle_matches_plain_gmres(oracle):
    A = G.helmholtz_like(32, 0.5)
    b = 0.1 * np.arange(32).astype(complex)
    r = G.gcro_dr(A, b, G.Subspace(6), 100, 30, 1e-12)
    xg, res = oracle.gmres(A, b, restart=30, max_iterations=100, tol=1e-12)
    assert r["converged"] and res.converged
    assert np.linalg.norm(xg - r["x"]) < 1e-7


def test_oracle_sweep_recycling_beats_independent_solves(oracle):
    n, b = 800, np.cos(np.arange(800)) + 0.5j
    sub = G.Subspace(20)
    indep = recycled = 0
    for i in range(100):
        A = G.helmholtz_like(n, 1.0 + 0.05 * i)
        _, res = oracle.gmres(A, b, restart=40, max_iterations=200, tol=1e-8)
        r = G.gcro_dr(A, b, sub, 200, 40, 1e-8)
        assert res.converged and r["converged"]
        assert np.linalg.norm(A @ r["x"] - b) / np.linalg.norm(b) < 1e-4
        indep += res.iterations
        recycled += r["iterations"]
    assert indep / recycled >= 2.0


def test_oracle_small_diagonal():
    r = G.gcro_dr(np.diag([2.0, 3.0]).astype(complex), np.array([2.0, 6.0], complex), G.Subspace(2), 10, 5, 1e-12)
    assert r["converged"] and abs(r["x"][0] - 1) < 1e-9 and abs(r["x"][1] - 2) < 1e-9


def test_oracle_rejects_mismatched_subspace():
    sub = G.Subspace(2)
    sub.u = [np.ones(5, complex) / np.sqrt(5)]
    r = G.gcro_dr(G.helmholtz_like(6, 1.0), np.ones(6, complex), sub, 10, 5, 1e-8)
    assert r["status"] == "NumericalError" and not r["converged"]


def test_sweep_config_recycle_validation(sb):
    cfg = sb.FrequencySweepConfig(frequencies=[100.0, 200.0], max_recycle_relative_frequency_delta=-1.0)
    with pytest.raises(sb.SoniumError):
        cfg.validate()
    cfg = sb.FrequencySweepConfig(frequencies=[100.0, 200.0], recycle_subspace_size=-2)
    with pytest.raises(sb.SoniumError):
        cfg.validate()


# ---- GPU: the device solver against the oracle ----

@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
@pytest.mark.parametrize("jacobi", [False, True])
def test_device_matches_oracle_on_reference_operators(gpu, jacobi):
    n = 60
    b = np.cos(np.arange(n)) + 0.5j
    sub_d, sub_o = gpu.GcroDrSubspace(10), G.Subspace(10)
    cfg = gpu.GcroDrConfig(max_iterations=100, restart=30, tolerance=1e-9)
    for f in (1.0, 1.05, 1.1, 1.15):
        A = G.helmholtz_like(n, f)
        op = gpu.DenseMatrixOperator(A)
        pre = gpu.JacobiPreconditioner(op) if jacobi else None
        d = gpu.gcro_dr(op, b, sub_d, cfg, preconditioner=pre)
        o = G.gcro_dr(A, b, sub_o, 100, 30, 1e-9, jacobi=jacobi)
        assert d.converged and o["converged"], f
        assert abs(d.iterations - o["iterations"]) <= 1, (f, d.iterations, o["iterations"])
        assert _rel(d.x, o["x"]) < 1e-8, f
        assert abs(d.residual - np.linalg.norm(b - A @ d.x) / np.linalg.norm(b)) < 1e-12
        assert sub_d.num_vectors() == len(sub_o.u)
        op.close()
    U = sub_d.vectors()
    assert np.allclose(U.conj() @ U.T, np.eye(U.shape[0]), atol=1e-10)
    sub_d.close()


@pytest.mark.gpu
def test_empty_subspace_is_gmres_with_every_step_checked(gpu):
    nodes, tris = gpu.icosphere(1.0, 2)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(3.0)
    beta = ph.burton_miller_beta()
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    g = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=50, restart=20, tolerance=1e-9))
    sub = gpu.GcroDrSubspace(0)
    r = gpu.gcro_dr(op, b, sub, gpu.GcroDrConfig(50, 20, 1e-9))
    assert r.converged and g.converged
    assert r.iterations == g.iterations
    assert _rel(r.x, g.x) < 1e-9
    assert not sub.is_populated()  # k = 0 never keeps vectors
    op.close()


@pytest.mark.gpu
def test_tbem_frequency_sequence_matches_oracle(gpu):
    nodes, tris = gpu.icosphere(1.0, 3)
    mesh = gpu.Mesh(nodes, tris)
    sub_d, sub_o = gpu.GcroDrSubspace(12), G.Subspace(12)
    cfg = gpu.GcroDrConfig(max_iterations=50, restart=30, tolerance=1e-9)
    op = None
    for k in (3.0, 3.1, 3.2, 3.3, 3.4):
        ph = gpu.PhysicsParams.for_wavenumber(k)
        beta = ph.burton_miller_beta(4.0)
        if op is None:
            op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
        else:
            op.reassemble(ph, beta)
        b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
        A = op.matrix
        d = gpu.gcro_dr(op, b, sub_d, cfg)
        o = G.gcro_dr(A, b, sub_o, 50, 30, 1e-9)
        g = gpu.gmres(op, b, gpu.GmresConfig(50, 30, 1e-9))
        assert d.converged and o["converged"]
        assert abs(d.iterations - o["iterations"]) <= 1, (k, d.iterations, o["iterations"])
        assert _rel(d.x, o["x"]) < 1e-8
        assert _rel(d.x, g.x) < 1e-7
    op.close()


@pytest.mark.gpu
def test_device_sweep_recycling_beats_independent_solves(gpu):
    """frequency_sweep_recycling_beats_independent_solves (gcro_dr.rs:1222-1302) on the device:
    100 consecutive Helmholtz-like systems (n = 800), recycled total Krylov steps at least 2x
    fewer than independent GMRES solves."""
    n, b = 800, np.cos(np.arange(800)) + 0.5j
    sub = gpu.GcroDrSubspace(20)
    cfg = gpu.GcroDrConfig(max_iterations=200, restart=40, tolerance=1e-8)
    indep = recycled = 0
    for i in range(100):
        A = G.helmholtz_like(n, 1.0 + 0.05 * i)
        op = gpu.DenseMatrixOperator(A)
        g = gpu.gmres(op, b, gpu.GmresConfig(200, 40, 1e-8))
        r = gpu.gcro_dr(op, b, sub, cfg)
        assert g.converged and r.converged, i
        assert np.linalg.norm(A @ r.x - b) / np.linalg.norm(b) < 1e-4
        indep += g.iterations
        recycled += r.iterations
        op.close()
    assert indep / recycled >= 2.0, (indep, recycled)


@pytest.mark.gpu
def test_subspace_bookkeeping_and_rejections(gpu):
    A = G.helmholtz_like(40, 1.0)
    op = gpu.DenseMatrixOperator(A)
    b = np.sin(np.arange(40)).astype(complex)
    sub = gpu.GcroDrSubspace(8)
    assert sub.target_size() == 8 and not sub.is_populated()
    # non-finite right-hand side: rejected before any device work, subspace untouched
    bad = b.copy()
    bad[3] = np.nan
    with pytest.raises(gpu.SoniumError):
        gpu.gcro_dr(op, bad, sub)
    assert not sub.is_populated()
    r = gpu.gcro_dr(op, b, sub, gpu.GcroDrConfig(100, 30, 1e-10))
    assert r.converged and sub.num_vectors() == 8
    # checkpoint round trip
    U = sub.vectors()
    sub.reset()
    assert not sub.is_populated()
    sub.replace_vectors(U)
    assert np.array_equal(sub.vectors(), U)
    with pytest.raises(gpu.SoniumError):
        sub.replace_vectors(np.ones((9, 40), complex))  # more than the target
    # vectors of another length: NumericalError, x = x0, subspace kept
    op2 = gpu.DenseMatrixOperator(G.helmholtz_like(30, 1.0))
    r2 = gpu.gcro_dr(op2, np.ones(30, complex), sub)
    assert r2.status == "NumericalError" and not r2.converged and np.all(r2.x == 0)
    assert sub.num_vectors() == 8
    with pytest.raises(gpu.SoniumError):
        gpu.GcroDrSubspace(101)
    op.close()
    op2.close()
    sub.close()


@pytest.mark.gpu
def test_dense_operator_matches_its_matrix(gpu):
    rng = np.random.default_rng(5)
    n = 97
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 40 * np.eye(n)  # spectrum in |z - 40| < 15
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for prec in (gpu.SB_PRECISION_FP64, gpu.SB_PRECISION_FP64_FP32):
        op = gpu.DenseMatrixOperator(A, prec)
        assert _rel(op.apply(x), A @ x) < 1e-14
        assert np.array_equal(op.matrix, A)
        if prec == gpu.SB_PRECISION_FP64_FP32:
            assert np.array_equal(op.matrix_c64(), A.astype(np.complex64))
            s = gpu.gmres_mixed(op, A @ x, gpu.IrConfig(tolerance=1e-10))
            assert s.converged and _rel(s.x, x) < 1e-8
        with pytest.raises(gpu.SoniumError):
            op.reassemble(gpu.PhysicsParams.for_wavenumber(1.0), 0.5j)
        op.close()
    with pytest.raises(gpu.SoniumError):
        gpu.DenseMatrixOperator(np.full((3, 3), np.inf))


@pytest.mark.gpu
def test_recycling_sweep_matches_warm_start_sweep(gpu):
    """test_frequency_sweep_gcro_dr_matches_legacy and the recycle-bound bookkeeping of
    frequency_sweep_records_and_enforces_recycle_frequency_bound (frequency_sweep.rs:1549-1640)."""
    mesh = gpu.Mesh(*gpu.icosphere(0.1, 2))
    freqs = [300.0, 320.0, 340.0, 500.0, 520.0]
    legacy = gpu.frequency_sweep(mesh, gpu.FrequencySweepConfig(frequencies=freqs, tolerance=1e-9))
    cfg = gpu.FrequencySweepConfig(frequencies=freqs, tolerance=1e-9, recycle_subspace_size=6)
    rec = gpu.frequency_sweep(mesh, cfg)
    assert rec.recycled_subspace_eligible == [False, True, True, False, True]
    assert rec.num_converged() == len(freqs)
    for a, b in zip(legacy.solutions, rec.solutions):
        assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-5
    with pytest.raises(gpu.SoniumError):
        gpu.frequency_sweep(mesh, cfg, mixed=True)
