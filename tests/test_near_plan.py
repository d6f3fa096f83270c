"""The recorded near-pair subdivision plan against the subdividing near kernel.

A mesh's first near-pair assembly subdivides each near pair as it integrates (k_near, the
generate_subelements recursion of crates/sonium-bem/src/core/integration/singular.rs:1372-1540); the
second records the kept leaves once (they depend on the geometry alone) and every later assembly
evaluates the recorded leaves (k_near_cached) in the same level and point order. These tests check
that the recorded path reproduces the subdividing one bit for bit: in FP64 and FP32, at the wave
number of the recording and at another, and with a right-hand side from a prescribed boundary value.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _fresh(gpu, nodes, tris, k, prec, bc=None):
    """Matrix and RHS from a new mesh's first assembly (the subdividing kernel)."""
    mesh = gpu.Mesh(nodes, tris)
    if bc is not None:
        mesh.set_boundary_conditions(*bc)
    ph = gpu.PhysicsParams.for_wavenumber(k)
    op = gpu.build_tbem_system_with_beta(mesh, ph, ph.burton_miller_beta(), prec)
    out = (op.matrix, op.rhs)
    op.close()
    mesh.close()
    return out


@pytest.mark.parametrize("prec_name", ["SB_PRECISION_FP64", "SB_PRECISION_FP32"])
def test_recorded_plan_bit_identical(gpu, oracle, prec_name):
    prec = getattr(gpu, prec_name)
    nodes, tris = oracle.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    ref5 = _fresh(gpu, nodes, tris, 5.0, prec)
    ref9 = _fresh(gpu, nodes, tris, 9.0, prec)
    mesh = gpu.Mesh(nodes, tris)
    ph5 = gpu.PhysicsParams.for_wavenumber(5.0)
    ph9 = gpu.PhysicsParams.for_wavenumber(9.0)
    op = gpu.build_tbem_system_with_beta(mesh, ph5, ph5.burton_miller_beta(), prec)  # subdividing
    assert np.array_equal(op.matrix, ref5[0])
    op.reassemble(ph5, ph5.burton_miller_beta())  # records the plan, then evaluates it
    assert np.array_equal(op.matrix, ref5[0])
    op.reassemble(ph9, ph9.burton_miller_beta())  # the recorded plan at another wave number
    assert np.array_equal(op.matrix, ref9[0])
    op2 = gpu.build_tbem_system_with_beta(mesh, ph9, ph9.burton_miller_beta(), prec)  # a second operator
    assert np.array_equal(op2.matrix, ref9[0])
    op.close()
    op2.close()
    mesh.close()


def test_recorded_plan_with_boundary_rhs(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 2)
    m = len(tris)
    rng = np.random.default_rng(3)
    kind = np.where(rng.random(m) < 0.3, 1, 0).astype(np.int32)
    value = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    bc = (kind, value)
    ref = _fresh(gpu, nodes, tris, 4.0, gpu.SB_PRECISION_FP64, bc)
    mesh = gpu.Mesh(nodes, tris)
    mesh.set_boundary_conditions(*bc)
    ph = gpu.PhysicsParams.for_wavenumber(4.0)
    op = gpu.build_tbem_system_with_beta(mesh, ph, ph.burton_miller_beta(), gpu.SB_PRECISION_FP64)
    op.reassemble(ph, ph.burton_miller_beta())
    op.reassemble(ph, ph.burton_miller_beta())
    assert np.array_equal(op.matrix, ref[0])
    assert np.array_equal(op.rhs, ref[1])
    op.close()
    mesh.close()
