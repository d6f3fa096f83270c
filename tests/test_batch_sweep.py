"""Batched frequency sweep (sb_batch_*): the batched assembly of many instances (one persistent
launch, or per-instance kernels on two streams, chosen by the autotuner) and the batched
mixed-precision GMRES with per-instance convergence masks.

Bars (written into each test):
  * each instance's complex64 matrix meets the mixed-assembly bar against the FP64 oracle (3e-5
    per entry, median 1e-6) and matches the single-instance SB_PRECISION_FP32 assembly of the same
    mesh and wavenumber to 1e-6 of the largest entry (the same device functions compiled into
    another kernel may contract or order FP32 operations differently),
  * each batched solution is within 1e-6 (relative) of the single-instance sb_gmres_mixed
    solution and within 1e-5 of the FP64 solve (the metric's tolerance); every instance
    converges to its own tolerance with its own iteration count,
  * per-instance masks: a converged or already-solved instance stops costing iterations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _instances(gpu, oracle, spec):
    """spec: [(level, k, scale)] -> meshes (one per (level, scale)), physics, betas."""
    cache, meshes, phys, betas = {}, [], [], []
    for level, k, scale in spec:
        key = (level, scale)
        if key not in cache:
            nodes, tris = oracle.icosphere(1.0, level, scale)
            cache[key] = gpu.Mesh(nodes, tris)
        ph = gpu.PhysicsParams.for_wavenumber(k)
        meshes.append(cache[key])
        phys.append(ph)
        betas.append(ph.burton_miller_beta())
    return meshes, phys, betas


SPEC = [(1, 0.7, (1.0, 1.0, 1.0)), (2, 2.0, (1.0, 0.6, 0.4)), (2, 3.5, (1.0, 0.6, 0.4)),
        (3, 2.0, (1.0, 1.0, 1.0)), (3, 6.0, (1.0, 0.6, 0.4)), (1, 1.3, (1.0, 0.6, 0.4))]


def test_batch_matrices_match_single_instance_assembly(gpu, oracle):
    from sonium_b200.sweep import SweepBatch

    meshes, phys, betas = _instances(gpu, oracle, SPEC)
    oracle_nodes = [oracle.icosphere(1.0, lv, sc)[0] for lv, _, sc in SPEC]
    oracle_tris = [oracle.icosphere(1.0, lv, sc)[1] for lv, _, sc in SPEC]
    batch = SweepBatch(meshes, phys, betas)
    batch.assemble()
    for i, (m, ph, be) in enumerate(zip(meshes, phys, betas)):
        op = gpu.build_tbem_system_with_beta(m, ph, be, precision=gpu.SB_PRECISION_FP32)
        A1 = op.matrix_c64()
        Ab = batch.matrix_c64(i)
        # the FP32 bar of the single-instance mixed assembly against the FP64 oracle
        A_o, _ = oracle.assemble(oracle_nodes[i], oracle_tris[i], oracle.physics_for_k(SPEC[i][1]), be)
        floor = 1e-6 * np.abs(A_o).max()
        err = np.abs(Ab - A_o) / np.maximum(np.abs(A_o), floor)
        assert err.max() < 3e-5 and np.median(err) < 1e-6, (i, err.max(), np.median(err))
        # and the two kernels agree to FP32 rounding of the largest entries
        assert np.abs(Ab - A1).max() <= 1e-6 * np.abs(A1).max(), (i, float(np.abs(Ab - A1).max()))
        op.close()
    batch.close()


def test_batch_assembly_forms_agree_and_autotune(gpu, oracle):
    """The persistent single launch and the per-instance two-stream form write the same matrices;
    the autotuner measures both on the first assembly of a new batch shape and keeps the faster."""
    from sonium_b200._lib import SB_BATCH_ASM_AUTO, SB_BATCH_ASM_PERSISTENT, SB_BATCH_ASM_STREAMS
    from sonium_b200.sweep import SweepBatch

    spec = [(2, 1.7, (1.0, 0.6, 0.4)), (3, 3.1, (1.0, 0.6, 0.4)), (1, 0.9, (1.0, 1.0, 1.0))]  # a shape no other test uses
    meshes, phys, betas = _instances(gpu, oracle, spec)
    batch = SweepBatch(meshes, phys, betas)
    batch.set_assembly_mode(SB_BATCH_ASM_PERSISTENT)
    batch.assemble()
    assert batch.assembly_tuning()[0] == SB_BATCH_ASM_PERSISTENT
    Ap = [batch.matrix_c64(i) for i in range(len(batch))]
    batch.set_assembly_mode(SB_BATCH_ASM_STREAMS)
    batch.assemble()
    assert batch.assembly_tuning()[0] == SB_BATCH_ASM_STREAMS
    for i in range(len(batch)):
        As = batch.matrix_c64(i)
        assert np.abs(As - Ap[i]).max() <= 1e-6 * np.abs(Ap[i]).max(), i
    batch.set_assembly_mode(SB_BATCH_ASM_AUTO)
    batch.assemble()
    chosen, t_p, t_s = batch.assembly_tuning()
    assert t_p > 0 and t_s > 0
    assert chosen == (SB_BATCH_ASM_STREAMS if t_s < t_p else SB_BATCH_ASM_PERSISTENT)
    batch.assemble()  # remembered: no second tuning run
    assert batch.assembly_tuning()[0] == chosen
    with pytest.raises(gpu.SoniumError):
        batch.set_assembly_mode(7)
    batch.close()


def test_batch_odd_size_mesh(gpu, oracle):
    """n odd (open surface): padded leading dimensions, the odd last column of the products."""
    from sonium_b200.sweep import SweepBatch

    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    mesh_odd = gpu.Mesh(nodes, tris[:-1])
    nodes3, tris3 = oracle.icosphere(1.0, 1)
    mesh_even = gpu.Mesh(nodes3, tris3)
    ph1, ph2 = gpu.PhysicsParams.for_wavenumber(1.5), gpu.PhysicsParams.for_wavenumber(0.9)
    batch = SweepBatch([mesh_even, mesh_odd], [ph1, ph2], [ph1.burton_miller_beta(), ph2.burton_miller_beta()])
    batch.assemble()
    op = gpu.build_tbem_system_with_beta(mesh_odd, ph2, ph2.burton_miller_beta(), precision=gpu.SB_PRECISION_FP32)
    A1 = op.matrix_c64()
    assert np.abs(batch.matrix_c64(1) - A1).max() <= 1e-6 * np.abs(A1).max()
    b = gpu.rhs_plane_wave(mesh_odd, ph2, ph2.burton_miller_beta(), [0, 0, 1])[:, 0]
    batch.set_rhs_plane_wave([0, 0, 1])
    st = batch.solve(gpu.IrConfig(tolerance=1e-9))
    assert all(s.converged for s in st)
    ref = gpu.gmres_mixed(op, b, gpu.IrConfig(tolerance=1e-9))
    x = batch.solution(1)
    assert np.linalg.norm(x - ref.x) / np.linalg.norm(ref.x) < 1e-6


def test_batch_solutions_match_single_instance_and_fp64(gpu, oracle):
    from sonium_b200.sweep import SweepBatch

    meshes, phys, betas = _instances(gpu, oracle, SPEC)
    cfg = gpu.IrConfig(tolerance=1e-8)
    batch = SweepBatch(meshes, phys, betas)
    batch.assemble()
    batch.set_rhs_plane_wave([0.0, 0.0, 1.0])
    stats = batch.solve(cfg)
    for i, (m, ph, be) in enumerate(zip(meshes, phys, betas)):
        b = gpu.rhs_plane_wave(m, ph, be, [0, 0, 1])[:, 0]
        op32 = gpu.build_tbem_system_with_beta(m, ph, be, precision=gpu.SB_PRECISION_FP32)
        single = gpu.gmres_mixed(op32, b, cfg)
        op64 = gpu.build_tbem_system_with_beta(m, ph, be)
        x64 = gpu.gmres(op64, b, gpu.GmresConfig(max_iterations=100, restart=50, tolerance=1e-10)).x
        x = batch.solution(i)
        st = stats[i]
        assert st.converged and st.residual < cfg.tolerance, (i, st)
        assert np.linalg.norm(x - single.x) / np.linalg.norm(single.x) < 1e-6, i
        assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-5, i
        # same algorithm per instance: the Krylov work matches the single-instance solve closely
        assert abs(st.iterations - single.iterations) <= max(2, single.iterations // 10), (i, st, single)
        assert abs(st.refinements - single.refinements) <= 1, (i, st.refinements, single.refinements)
        # the residual reported is the FP64 residual of the batch's own (complex64) matrix
        A32 = batch.matrix_c64(i).astype(np.complex128)
        r = b - A32 @ x
        assert abs(np.linalg.norm(r) / np.linalg.norm(b) - st.residual) < 1e-3 * st.residual + 1e-14
        op32.close()
        op64.close()
    batch.close()


def test_batch_instances_converge_independently(gpu, oracle):
    """Masks: an instance with a zero right-hand side is done at once (no Krylov steps), the
    others proceed; solving twice gives identical results (state fully reset per solve)."""
    from sonium_b200.sweep import SweepBatch

    meshes, phys, betas = _instances(gpu, oracle, SPEC[:3])
    batch = SweepBatch(meshes, phys, betas)
    batch.assemble()
    batch.set_rhs_plane_wave([1.0, 0.0, 0.0])
    batch.set_rhs(1, np.zeros(meshes[1].num_elements, np.complex128))
    cfg = gpu.IrConfig(tolerance=1e-9)
    st = batch.solve(cfg)
    assert st[1].iterations == 0 and st[1].converged and np.all(batch.solution(1) == 0)
    assert st[0].iterations > 0 and st[2].iterations > 0
    x0, x2 = batch.solution(0), batch.solution(2)
    st2 = batch.solve(cfg)
    assert np.array_equal(batch.solution(0), x0) and np.array_equal(batch.solution(2), x2)
    assert [s.iterations for s in st2] == [s.iterations for s in st]
    # a different restart re-sizes the workspace and still converges
    st3 = batch.solve(gpu.IrConfig(tolerance=1e-9, inner_restart=20))
    assert all(s.converged for s in st3)
    assert np.linalg.norm(batch.solution(2) - x2) / np.linalg.norm(x2) < 1e-7
    batch.close()


def test_batch_rejects_bc_values_and_bad_config(gpu, oracle):
    from sonium_b200.sweep import SweepBatch

    nodes, tris = oracle.icosphere(1.0, 1)
    mesh = gpu.Mesh(nodes, tris)
    ph = gpu.PhysicsParams.for_wavenumber(1.0)
    mesh_bc = gpu.Mesh(nodes, tris)
    mesh_bc.set_boundary_conditions(kind=gpu.SB_BC_VELOCITY, value=1.0)
    with pytest.raises(gpu.SoniumError) as e:
        SweepBatch([mesh, mesh_bc], [ph, ph], [ph.burton_miller_beta()] * 2)
    assert "boundary values" in str(e.value)
    batch = SweepBatch([mesh], [ph], [ph.burton_miller_beta()])
    with pytest.raises(gpu.SoniumError):
        batch.solve(gpu.IrConfig())  # not assembled
    with pytest.raises(gpu.SoniumError):
        batch.solution(0)
    batch.assemble()
    with pytest.raises(gpu.SoniumError):
        batch.solve(gpu.IrConfig(inner_restart=500))
    with pytest.raises(gpu.SoniumError):
        batch.set_rhs(0, np.full(mesh.num_elements, np.nan, np.complex128))
    batch.close()



def test_sequential_sweep_warm_start(gpu, oracle):
    """frequency_sweep (frequency_sweep.rs:592-850, dense branch): re-assembly into one operator
    per frequency, warm start from the previous solution. Recycling gives the same solutions (to
    the tolerance) with fewer GMRES iterations on a closely spaced grid; every point passes the
    exact-residual acceptance check; the mixed solver gives the FP64 solutions within 1e-5."""
    from sonium_b200.sweep import FrequencySweepConfig, frequency_sweep

    nodes, tris = oracle.icosphere(1.0, 2)
    mesh = gpu.Mesh(nodes, tris)
    c = 343.0
    freqs = list(np.linspace(2.0, 2.4, 6) * c / (2 * np.pi))  # k = 2.0 .. 2.4
    warm = frequency_sweep(mesh, FrequencySweepConfig(frequencies=freqs, tolerance=1e-9), speed_of_sound=c)
    cold = frequency_sweep(mesh, FrequencySweepConfig(frequencies=freqs, tolerance=1e-9, recycle_solution=False),
                           speed_of_sound=c)
    assert warm.num_converged() == len(freqs) == cold.num_converged()
    assert warm.total_iterations() < cold.total_iterations()
    for xw, xc in zip(warm.solutions, cold.solutions):
        assert np.linalg.norm(xw - xc) / np.linalg.norm(xc) < 1e-7
    assert max(warm.exact_relative_residuals) < 1e-9
    mixed = frequency_sweep(mesh, FrequencySweepConfig(frequencies=freqs, tolerance=1e-9), speed_of_sound=c,
                            mixed=True)
    for xm, xc in zip(mixed.solutions, cold.solutions):
        assert np.linalg.norm(xm - xc) / np.linalg.norm(xc) < 1e-5
    # each frequency's solution is that frequency's own system's (single solve, same beta)
    ph = gpu.PhysicsParams.new(freqs[3], c)
    beta = ph.burton_miller_beta(4.0)
    op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
    b = gpu.rhs_plane_wave(mesh, ph, beta, [0, 0, 1])[:, 0]
    x = gpu.gmres(op, b, gpu.GmresConfig(max_iterations=200, restart=30, tolerance=1e-10)).x
    assert np.linalg.norm(warm.solutions[3] - x) / np.linalg.norm(x) < 1e-7
    op.close()


def test_batch_half_inner_matches_single_instance(gpu, oracle):
    """SB_INNER_FP16 on a batch: every instance's solution equals the single-instance FP16-inner
    solve of the same complex64 matrix (same algorithm per instance) and the batch's own FP32-inner
    solution to the solver tolerance; the copies are rebuilt after a re-assembly; restarts inside
    the inner solves (inner_restart 8, inner tolerance 1e-5) take the residual on the half copies; an odd size covers
    the column tail."""
    from sonium_b200.sweep import SweepBatch

    meshes, phys, betas = _instances(gpu, oracle, SPEC)
    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    meshes.append(gpu.Mesh(nodes, tris[:-1]))
    ph = gpu.PhysicsParams.for_wavenumber(1.7)
    phys.append(ph)
    betas.append(ph.burton_miller_beta())
    batch = SweepBatch(meshes, phys, betas)
    batch.assemble()
    batch.set_rhs_plane_wave([0.0, 0.0, 1.0])
    cfg32 = gpu.IrConfig(tolerance=1e-8)
    s32 = batch.solve(cfg32)
    x32 = [batch.solution(i) for i in range(len(batch))]
    batch.set_inner_precision(gpu.SB_INNER_FP16)
    for cfg16 in (gpu.IrConfig(tolerance=1e-8, inner_tolerance=1e-3),
                  gpu.IrConfig(tolerance=1e-8, inner_tolerance=1e-5, inner_restart=8)):
        s16 = batch.solve(cfg16)
        for i, (m, ph_i, be) in enumerate(zip(meshes, phys, betas)):
            x = batch.solution(i)
            assert s16[i].converged and s16[i].residual < 1e-8, (i, s16[i])
            assert np.linalg.norm(x - x32[i]) / np.linalg.norm(x32[i]) < 1e-6, i
        if cfg16.inner_restart == 8:  # inner solves to 1e-5 need more than 8 steps
            assert sum(st.restarts for st in s16) > 0
        # single-instance FP16-inner solve of instance 4: the same iterations within rounding noise
        m, ph_i, be = meshes[4], phys[4], betas[4]
        b = gpu.rhs_plane_wave(m, ph_i, be, [0, 0, 1])[:, 0]
        op = gpu.build_tbem_system_with_beta(m, ph_i, be, precision=gpu.SB_PRECISION_FP32)
        op.set_inner_precision(gpu.SB_INNER_FP16)
        single = gpu.gmres_mixed(op, b, cfg16)
        assert abs(s16[4].iterations - single.iterations) <= max(2, single.iterations // 10)
        assert np.linalg.norm(batch.solution(4) - single.x) / np.linalg.norm(single.x) < 1e-6
        op.close()
    # re-assembly at other wavenumbers: the half copies follow the new matrices
    phys2 = [gpu.PhysicsParams.for_wavenumber(0.9 * p.wave_number) for p in phys]
    betas2 = [p.burton_miller_beta() for p in phys2]
    batch.close()
    batch = SweepBatch(meshes, phys2, betas2)
    batch.set_inner_precision(gpu.SB_INNER_FP16)
    batch.assemble()
    batch.set_rhs_plane_wave([1.0, 0.0, 0.0])
    a = batch.solve(gpu.IrConfig(tolerance=1e-8, inner_tolerance=1e-3))
    xa = [batch.solution(i) for i in range(len(batch))]
    batch.assemble()  # same matrices again: the copies are rebuilt and the answers repeat
    b2 = batch.solve(gpu.IrConfig(tolerance=1e-8, inner_tolerance=1e-3))
    assert [s.iterations for s in a] == [s.iterations for s in b2]
    assert all(np.array_equal(batch.solution(i), xa[i]) for i in range(len(batch)))
    batch.set_inner_precision(gpu.SB_INNER_FP32)
    c = batch.solve(gpu.IrConfig(tolerance=1e-8))
    assert all(s.converged for s in c)
    assert all(np.linalg.norm(batch.solution(i) - xa[i]) / np.linalg.norm(xa[i]) < 1e-6 for i in range(len(batch)))
    with pytest.raises(gpu.SoniumError):
        batch.set_inner_precision(5)
    batch.close()


def test_batch_block_jacobi_matches_single_instance(gpu, oracle):
    """SB_INNER_PRECOND_BLOCK_JACOBI on a batch (FP32 and complex-half inner products): every
    instance converges to the batch's unpreconditioned solution with no more inner iterations;
    instance 4 matches the single-instance preconditioned solve; inner restarts (inner_restart 8)
    take the preconditioned residual; an odd size covers the partial last block."""
    from sonium_b200.sweep import SweepBatch

    meshes, phys, betas = _instances(gpu, oracle, SPEC)
    nodes, tris = oracle.icosphere(1.0, 2, (1.0, 0.6, 0.4))
    meshes.append(gpu.Mesh(nodes, tris[:-1]))
    ph = gpu.PhysicsParams.for_wavenumber(1.7)
    phys.append(ph)
    betas.append(ph.burton_miller_beta())
    batch = SweepBatch(meshes, phys, betas)
    batch.assemble()
    batch.set_rhs_plane_wave([0.0, 0.0, 1.0])
    for inner, tol in ((gpu.SB_INNER_FP32, 1e-5), (gpu.SB_INNER_FP16, 1e-3)):
        batch.set_inner_precision(inner)
        batch.set_inner_preconditioner(gpu.SB_INNER_PRECOND_NONE, 64)
        cfg = gpu.IrConfig(tolerance=1e-8, inner_tolerance=tol)
        s0 = batch.solve(cfg)
        x0 = [batch.solution(i) for i in range(len(batch))]
        for bs, restart in ((64, 50), (32, 8)):
            batch.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, bs)
            cfg_b = gpu.IrConfig(tolerance=1e-8, inner_tolerance=tol, inner_restart=restart)
            s1 = batch.solve(cfg_b)
            for i in range(len(batch)):
                assert s1[i].converged and s1[i].residual < 1e-8, (i, s1[i])
                assert np.linalg.norm(batch.solution(i) - x0[i]) / np.linalg.norm(x0[i]) < 1e-6, i
            if restart == 50:
                assert sum(s.iterations for s in s1) < sum(s.iterations for s in s0)
                m, ph_i, be = meshes[4], phys[4], betas[4]
                b = gpu.rhs_plane_wave(m, ph_i, be, [0, 0, 1])[:, 0]
                op = gpu.build_tbem_system_with_beta(m, ph_i, be, precision=gpu.SB_PRECISION_FP32)
                op.set_inner_precision(inner)
                op.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, bs)
                single = gpu.gmres_mixed(op, b, cfg_b)
                assert abs(s1[4].iterations - single.iterations) <= max(2, single.iterations // 10)
                assert np.linalg.norm(batch.solution(4) - single.x) / np.linalg.norm(single.x) < 1e-6
                op.close()
    with pytest.raises(gpu.SoniumError):
        batch.set_inner_preconditioner(gpu.SB_INNER_PRECOND_BLOCK_JACOBI, 100)
    batch.close()
