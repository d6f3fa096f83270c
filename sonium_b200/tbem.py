"""Python mirror of the reference's dense TBEM interface over the sonium-b200 C ABI.

Names follow the reference (sonium-bem / sonium-solvers): ``PhysicsParams``,
``build_tbem_system_with_beta`` (crates/sonium-bem/src/core/assembly/tbem.rs:1196),
``LinearOperator.apply_into`` / ``apply_block`` (crates/sonium-solvers/crates/sonium-solvers-core/
src/traits.rs:2949-3120), ``GmresConfig`` / ``gmres`` / ``GmresSolution``
(crates/sonium-solvers/crates/sonium-solvers-iterative/src/gmres.rs:26-47, 93-118, 286) and
``IncidentField.compute_rhs_with_beta`` for plane waves (crates/sonium-bem/src/core/incident.rs:
807-833). Every call goes to the CUDA library; failures raise ``SoniumError``.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import SoniumError, check


def _p(a: np.ndarray):
    return a.ctypes.data_as(ct.c_void_p)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def device_count() -> int:
    n = ct.c_int(0)
    check(L.load().sb_device_count(ct.byref(n)))
    return n.value


@dataclass
class PhysicsParams:
    """PhysicsParams (crates/sonium-bem/src/core/types.rs:34-53)."""

    frequency: float
    speed_of_sound: float
    density: float
    wave_number: float
    omega: float
    wave_length: float
    harmonic_factor: float
    pressure_factor: float
    tau: float

    @classmethod
    def new(cls, frequency: float, speed_of_sound: float = 343.0, density: float = 1.21,
            is_internal: bool = False) -> "PhysicsParams":
        s = L.SbPhysics()
        check(L.load().sb_physics_new(frequency, speed_of_sound, density, int(is_internal), ct.byref(s)))
        return cls(*(getattr(s, f) for f, _ in L.SbPhysics._fields_))

    @classmethod
    def for_wavenumber(cls, k: float, speed_of_sound: float = 343.0, density: float = 1.21,
                       is_internal: bool = False) -> "PhysicsParams":
        return cls.new(k * speed_of_sound / (2.0 * np.pi), speed_of_sound, density, is_internal)

    def _struct(self) -> L.SbPhysics:
        return L.SbPhysics(*(getattr(self, f) for f, _ in L.SbPhysics._fields_))

    def burton_miller_beta(self, scale: float = 1.0) -> complex:
        out = L.SbComplex()
        check(L.load().sb_burton_miller_beta(ct.byref(self._struct()), scale, ct.byref(out)))
        return complex(out.re, out.im)


def icosphere(radius: float, level: int, scale=None):
    """generate_icosphere_mesh (crates/sonium-bem/src/core/mesh/generators.rs:309-397) nodes/tris."""
    lib = L.load()
    nn, nt = ct.c_int64(), ct.c_int64()
    check(lib.sb_icosphere_counts(level, ct.byref(nn), ct.byref(nt)))
    nodes = np.zeros((nn.value, 3))
    tris = np.zeros((nt.value, 3), np.uint32)
    sc = None if scale is None else np.ascontiguousarray(scale, np.float64)
    check(lib.sb_icosphere(radius, level, None if sc is None else _p(sc), _p(nodes), _p(tris)))
    return nodes, tris


class Mesh:
    """A device-resident Tri3 constant-panel mesh (element e owns DOF e)."""

    def __init__(self, nodes, tris, device: int = 0):
        self.nodes = np.ascontiguousarray(nodes, np.float64)
        self.tris = np.ascontiguousarray(tris, np.uint32)
        if self.nodes.ndim != 2 or self.nodes.shape[1] != 3 or self.tris.ndim != 2 or self.tris.shape[1] != 3:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "nodes must be (n, 3) and tris (m, 3)")
        h = ct.c_void_p()
        check(L.load().sb_mesh_create(_p(self.nodes), self.nodes.shape[0], _p(self.tris),
                                      self.tris.shape[0], device, ct.byref(h)))
        self._h = h
        self.device = device

    @classmethod
    def quad4(cls, nodes, quads, device: int = 0) -> "Mesh":
        """A Quad4 mesh of constant panels (quads: (m, 4) vertex indices)."""
        self = cls.__new__(cls)
        self.nodes = np.ascontiguousarray(nodes, np.float64)
        self.tris = np.ascontiguousarray(quads, np.uint32)
        if self.nodes.ndim != 2 or self.nodes.shape[1] != 3 or self.tris.ndim != 2 or self.tris.shape[1] != 4:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "nodes must be (n, 3) and quads (m, 4)")
        h = ct.c_void_p()
        check(L.load().sb_mesh_create_quad4(_p(self.nodes), self.nodes.shape[0], _p(self.tris), self.tris.shape[0],
                                            device, ct.byref(h)))
        self._h = h
        self.device = device
        return self

    @classmethod
    def icosphere(cls, radius: float, level: int, scale=None, device: int = 0) -> "Mesh":
        nodes, tris = icosphere(radius, level, scale)
        return cls(nodes, tris, device)

    @property
    def handle(self):
        if self._h is None:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "mesh has been closed")
        return self._h

    @property
    def num_elements(self) -> int:
        return self.tris.shape[0]

    def info(self) -> L.SbMeshInfo:
        i = L.SbMeshInfo()
        check(L.load().sb_mesh_info_get(self.handle, ct.byref(i)))
        return i

    def element_geometry(self):
        m = self.num_elements
        c, n, a = np.zeros((m, 3)), np.zeros((m, 3)), np.zeros(m)
        check(L.load().sb_mesh_element_geometry(self.handle, _p(c), _p(n), _p(a)))
        return c, n, a

    def collocation(self, basis: int = L.SB_BASIS_CONSTANT):
        """Collocation points and normals of a basis: (m, 3) each for the constant basis (centroids),
        (3m, 3) for the linear basis (DOF 3e + c)."""
        rows = self.num_elements * {L.SB_BASIS_LINEAR: 3, L.SB_BASIS_QUADRATIC: 6}.get(basis, 1)
        pts = np.zeros((rows, 3))
        nrm = np.zeros((rows, 3))
        check(L.load().sb_mesh_collocation(self.handle, basis, _p(pts), _p(nrm)))
        return pts, nrm

    def set_boundary_conditions(self, kind=None, value=None, admittance=None):
        """Per-element BoundaryCondition; ``admittance`` uses NaN for 'no admittance'."""
        m = self.num_elements
        k = None if kind is None else np.ascontiguousarray(np.broadcast_to(kind, (m,)), np.int32)
        v = None if value is None else _c128(np.broadcast_to(value, (m,)))
        has = adm = None
        if admittance is not None:
            a = np.asarray(np.broadcast_to(admittance, (m,)), np.complex128)
            has = np.ascontiguousarray(~np.isnan(a.real), np.uint8)
            adm = _c128(np.nan_to_num(a))
        check(L.load().sb_mesh_set_bc(self.handle, None if k is None else _p(k), None if v is None else _p(v),
                                      None if has is None else _p(has), None if adm is None else _p(adm)))

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.load().sb_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LinearOperator:
    """LinearOperator<Complex64> (traits.rs:2949-3120)."""

    def num_rows(self) -> int:
        raise NotImplementedError

    def num_cols(self) -> int:
        raise NotImplementedError

    def apply_into(self, x, y) -> None:
        raise NotImplementedError

    def apply(self, x):
        y = np.zeros(self.num_rows(), np.complex128)
        self.apply_into(x, y)
        return y


class TbemOperator(LinearOperator):
    """The assembled TbemSystem kept on the device, as a dense LinearOperator."""

    def __init__(self, mesh: Mesh, handle, physics: PhysicsParams, beta: complex, precision: int):
        self.mesh = mesh
        self._h = handle
        self.physics = physics
        self.beta = beta
        self.precision = precision
        self.n = mesh.num_elements
        self.basis = L.SB_BASIS_CONSTANT

    @property
    def handle(self):
        if self._h is None:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "operator has been closed")
        return self._h

    def num_rows(self) -> int:
        return self.n

    def num_cols(self) -> int:
        return self.n

    def info(self) -> L.SbOperatorInfo:
        i = L.SbOperatorInfo()
        check(L.load().sb_operator_info_get(self.handle, ct.byref(i)))
        return i

    def set_inner_precision(self, inner: int) -> None:
        """Matrix of gmres_mixed's inner GMRES: SB_INNER_FP32 (the complex64 copy, default) or
        SB_INNER_FP16 (a power-of-two-scaled complex-half copy, half the bytes per product; pair it
        with IrConfig(inner_tolerance=1e-3)). Needs a complex64 matrix."""
        check(L.load().sb_operator_set_inner_precision(self.handle, int(inner)))

    def set_inner_preconditioner(self, kind: int, block_size: int = 128) -> None:
        """Right preconditioner of gmres_mixed's inner GMRES: SB_INNER_PRECOND_NONE (default) or
        SB_INNER_PRECOND_BLOCK_JACOBI (inverted diagonal blocks of block_size spatially close
        elements; 32, 64, 96 or 128). The converged solution is unchanged; the inner solves need fewer
        iterations. Needs a complex64 matrix."""
        check(L.load().sb_operator_set_inner_preconditioner(self.handle, int(kind), int(block_size)))

    def reassemble(self, physics: PhysicsParams, beta: complex) -> None:
        check(L.load().sb_assemble_into(self.handle, ct.byref(physics._struct()), L.SbComplex(beta.real, beta.imag)))
        self.physics, self.beta = physics, beta

    @property
    def matrix(self) -> np.ndarray:
        A = np.zeros((self.n, self.n), np.complex128)
        check(L.load().sb_operator_copy_to_host(self.handle, _p(A), None))
        return A

    @property
    def rhs(self) -> np.ndarray:
        r = np.zeros(self.n, np.complex128)
        check(L.load().sb_operator_copy_to_host(self.handle, None, _p(r)))
        return r

    def rows(self, r0: int, r1: int) -> np.ndarray:
        A = np.zeros((r1 - r0, self.n), np.complex128)
        check(L.load().sb_operator_copy_rows_to_host(self.handle, r0, r1, _p(A)))
        return A

    def matrix_c64(self) -> np.ndarray:
        A = np.zeros((self.n, self.n), np.complex64)
        check(L.load().sb_operator_copy_to_host_c64(self.handle, _p(A)))
        return A

    def _apply(self, trans: int, x, y) -> None:
        x = _c128(x)
        if x.shape != (self.n,) or y.shape != (self.n,) or y.dtype != np.complex128 or not y.flags.c_contiguous:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "apply: vectors must be length-n complex128")
        check(L.load().sb_operator_apply(self.handle, trans, _p(x), _p(y)))

    def apply_into(self, x, y) -> None:
        self._apply(L.SB_OP_N, x, y)

    def apply_transpose_into(self, x, y) -> None:
        self._apply(L.SB_OP_T, x, y)

    def apply_hermitian_into(self, x, y) -> None:
        self._apply(L.SB_OP_C, x, y)

    def apply_block(self, X) -> np.ndarray:
        X = _c128(X)
        if X.ndim != 2 or X.shape[0] != self.n:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "apply_block: X must be n x r")
        Y = np.zeros_like(X)
        check(L.load().sb_operator_apply_block(self.handle, _p(X), _p(Y), X.shape[1]))
        return Y

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.load().sb_operator_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DenseMatrixOperator(TbemOperator):
    """DenseMatrixOperator (crates/sonium-bem/src/core/bem_solver.rs:6548-6590) over a caller's
    n x n matrix, copied to the device: the LinearOperator of any dense system, with the same
    products and solvers as an assembled operator (no mesh: no re-assembly, zero BC right-hand side)."""

    def __init__(self, matrix, precision: int = L.SB_PRECISION_FP64, device: int = 0):
        A = np.ascontiguousarray(matrix, np.complex128)
        if A.ndim != 2 or A.shape[0] != A.shape[1] or A.shape[0] == 0:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "dense operator: matrix must be square and non-empty")
        h = ct.c_void_p()
        check(L.load().sb_operator_from_dense(device, A.shape[0], _p(A), precision, ct.byref(h)))
        self.mesh = None
        self._h = h
        self.physics = None
        self.beta = None
        self.precision = precision
        self.n = A.shape[0]

    def reassemble(self, physics: PhysicsParams, beta: complex) -> None:
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "a dense operator has no mesh to re-assemble")


class JacobiPreconditioner:
    """Preconditioner<Complex64> (traits.rs:3645-3720): y = diag(A)^-1 x."""

    kind = L.SB_PRECOND_JACOBI

    def __init__(self, op: TbemOperator):
        self.op = op

    def apply_into(self, x, y) -> None:
        x = _c128(x)
        check(L.load().sb_preconditioner_apply(self.op.handle, self.kind, _p(x), _p(y)))


class BlockJacobiPreconditioner:
    """Block-Jacobi right preconditioner of the FP64 gmres (no reference counterpart; the
    Preconditioner<Complex64>::apply_into interface, traits.rs:3645-3720): y = M^-1 x, M the
    diagonal blocks of block_size spatially close elements (32, 64, 96 or 128) of the complex128
    matrix, inverted on the device after each assembly."""

    kind = L.SB_PRECOND_BLOCK_JACOBI

    def __init__(self, op: TbemOperator, block_size: int = 128):
        self.op = op
        check(L.load().sb_operator_set_block_jacobi_size(op.handle, int(block_size)))

    def apply_into(self, x, y) -> None:
        x = _c128(x)
        check(L.load().sb_preconditioner_apply(self.op.handle, self.kind, _p(x), _p(y)))


def build_tbem_system_with_beta(mesh: Mesh, physics: PhysicsParams, beta: complex,
                                precision: int = L.SB_PRECISION_FP64) -> TbemOperator:
    """build_tbem_system_with_beta (tbem.rs:1196-1203): assemble on the device.
    SB_PRECISION_FP32_HALF: SB_PRECISION_FP32 whose first assembly also writes the complex-half
    copy for gmres_mixed's inner products (SB_INNER_FP16 set from the start)."""
    h = ct.c_void_p()
    check(L.load().sb_assemble(mesh.handle, ct.byref(physics._struct()), L.SbComplex(beta.real, beta.imag),
                               precision, ct.byref(h)))
    return TbemOperator(mesh, h, physics, beta,
                        L.SB_PRECISION_FP32 if precision == L.SB_PRECISION_FP32_HALF else precision)


def build_tbem_system_linear(mesh: Mesh, physics: PhysicsParams, beta: complex) -> TbemOperator:
    """build_tbem_system_linear (tbem.rs:1490-1620): the discontinuous linear Tri3 basis, three DOFs
    per element (DOF 3e + c), a 3m x 3m complex128 operator on the device."""
    h = ct.c_void_p()
    check(L.load().sb_assemble_linear(mesh.handle, ct.byref(physics._struct()), L.SbComplex(beta.real, beta.imag),
                                      ct.byref(h)))
    op = TbemOperator(mesh, h, physics, beta, L.SB_PRECISION_FP64)
    op.n = 3 * mesh.num_elements
    op.basis = L.SB_BASIS_LINEAR
    return op


def build_tbem_system_discontinuous_stabilized(mesh: Mesh, physics: PhysicsParams, sign: float = 1.0,
                                               beta_scale: float = 1.0,
                                               basis: int = L.SB_BASIS_QUADRATIC) -> TbemOperator:
    """build_tbem_system_{linear,quadratic}_stabilized (tbem.rs:2993-3030): the discontinuous
    linear (3 DOFs per element) or quadratic (6) basis, every entry times sign, beta =
    burton_miller_beta_scaled(beta_scale)."""
    beta = physics.burton_miller_beta(beta_scale)
    h = ct.c_void_p()
    check(L.load().sb_assemble_discontinuous(mesh.handle, ct.byref(physics._struct()),
                                             L.SbComplex(beta.real, beta.imag), basis, float(sign), ct.byref(h)))
    op = TbemOperator(mesh, h, physics, beta, L.SB_PRECISION_FP64)
    op.n = (6 if basis == L.SB_BASIS_QUADRATIC else 3) * mesh.num_elements
    op.basis = basis
    return op


def build_tbem_system_quadratic_stabilized(mesh: Mesh, physics: PhysicsParams, sign: float = 1.0,
                                           beta_scale: float = 1.0) -> TbemOperator:
    """build_tbem_system_quadratic_stabilized (tbem.rs:3010-3030)."""
    return build_tbem_system_discontinuous_stabilized(mesh, physics, sign, beta_scale, L.SB_BASIS_QUADRATIC)


def rhs_plane_wave_at(points, normals, physics: PhysicsParams, beta: complex, directions, amplitudes=None,
                      device: int = 0) -> np.ndarray:
    """IncidentField::compute_rhs_with_beta (incident.rs:807-833) at arbitrary collocation points
    and normals (np x 3 each), computed on the device: (np, r) complex128."""
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    nrm = np.ascontiguousarray(normals, np.float64).reshape(-1, 3)
    if pts.shape != nrm.shape:
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "points and normals must have the same shape")
    d = np.ascontiguousarray(np.atleast_2d(directions), np.float64)
    r = d.shape[0]
    a = None if amplitudes is None else _c128(np.broadcast_to(amplitudes, (r,)))
    out = np.zeros((pts.shape[0], r), np.complex128)
    check(L.load().sb_rhs_plane_wave_points(device, pts.shape[0], _p(pts), _p(nrm), ct.byref(physics._struct()),
                                            L.SbComplex(beta.real, beta.imag), _p(d), None if a is None else _p(a),
                                            r, _p(out)))
    return out


def build_tbem_system(mesh: Mesh, physics: PhysicsParams, precision: int = L.SB_PRECISION_FP64) -> TbemOperator:
    """build_tbem_system (tbem.rs:877-883): beta = i/k."""
    return build_tbem_system_with_beta(mesh, physics, physics.burton_miller_beta(), precision)


def rhs_plane_wave(mesh: Mesh, physics: PhysicsParams, beta: complex, directions, amplitudes=None) -> np.ndarray:
    """IncidentField::compute_rhs_with_beta for plane waves: (n, r) complex128."""
    d = np.ascontiguousarray(np.atleast_2d(directions), np.float64)
    r = d.shape[0]
    a = None if amplitudes is None else _c128(np.broadcast_to(amplitudes, (r,)))
    out = np.zeros((mesh.num_elements, r), np.complex128)
    check(L.load().sb_rhs_plane_wave(mesh.handle, ct.byref(physics._struct()), L.SbComplex(beta.real, beta.imag),
                                     _p(d), None if a is None else _p(a), r, _p(out)))
    return out


@dataclass
class GmresConfig:
    """GmresConfig (gmres.rs:26-47): max_iterations = restart cycles."""

    max_iterations: int = 100
    restart: int = 30
    tolerance: float = 1e-6
    convergence_check_interval: int = 1

    def _struct(self):
        return L.SbGmresConfig(self.max_iterations, self.restart, self.tolerance, self.convergence_check_interval)


@dataclass
class IrConfig:
    """Mixed-precision refinement: FP64 outer residual, FP32 inner GMRES."""

    max_refinements: int = 20
    tolerance: float = 1e-8
    inner_restart: int = 50
    inner_max_iterations: int = 20
    inner_tolerance: float = 1e-5

    def _struct(self):
        return L.SbIrConfig(self.max_refinements, self.tolerance, self.inner_restart, self.inner_max_iterations,
                            self.inner_tolerance)


STATUS_NAMES = {0: "Converged", 1: "MaxIterationsReached", 2: "Breakdown", 3: "NumericalError"}


@dataclass
class GmresSolution:
    """GmresSolution (gmres.rs:93-118)."""

    x: np.ndarray
    iterations: int
    restarts: int
    residual: float
    estimated_residual: float
    backward_error: float
    converged: bool
    status: str
    matvecs: int = 0
    matvecs_fp32: int = 0
    refinements: int = 0
    device_ms: float = 0.0
    extra: dict = field(default_factory=dict)

    @classmethod
    def _from(cls, x, st: L.SbGmresStats) -> "GmresSolution":
        return cls(x=x, iterations=st.iterations, restarts=st.restarts, residual=st.residual,
                   estimated_residual=st.estimated_residual, backward_error=st.backward_error,
                   converged=bool(st.converged), status=STATUS_NAMES.get(st.status, str(st.status)),
                   matvecs=st.matvecs, matvecs_fp32=st.matvecs_fp32, refinements=st.refinements,
                   device_ms=st.device_ms)


def gmres(operator: TbemOperator, b, config: GmresConfig = GmresConfig(), x0=None,
          preconditioner: JacobiPreconditioner | BlockJacobiPreconditioner | None = None) -> GmresSolution:
    """gmres / gmres_preconditioned (gmres.rs:286-305) on the device-resident operator (Jacobi
    preconditioning on the left as the reference; block-Jacobi on the right)."""
    b = _c128(b)
    if b.shape != (operator.n,):
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "gmres: b must have length n")
    x = np.zeros(operator.n, np.complex128)
    x0a = None if x0 is None else _c128(x0)
    st = L.SbGmresStats()
    pk = L.SB_PRECOND_IDENTITY if preconditioner is None else preconditioner.kind
    check(L.load().sb_gmres(operator.handle, _p(b), None if x0a is None else _p(x0a), ct.byref(config._struct()),
                            pk, _p(x), ct.byref(st)))
    return GmresSolution._from(x, st)


def gmres_mixed(operator: TbemOperator, b, config: IrConfig = IrConfig(), x0=None) -> GmresSolution:
    """FP32-inner / FP64-refined GMRES (needs a SB_PRECISION_FP64_FP32 operator)."""
    b = _c128(b)
    x = np.zeros(operator.n, np.complex128)
    x0a = None if x0 is None else _c128(x0)
    st = L.SbGmresStats()
    check(L.load().sb_gmres_mixed(operator.handle, _p(b), None if x0a is None else _p(x0a),
                                  ct.byref(config._struct()), _p(x), ct.byref(st)))
    return GmresSolution._from(x, st)


def block_residual(operator: TbemOperator, B, X):
    """R = B - A X for n x r blocks on the operator's complex128 matrix (the block residual of block
    GMRES, crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:829): integer
    slices on the INT8 tensor cores, FP64-grade (not bit-identical to an FP64 GEMM)."""
    B = _c128(B)
    X = _c128(X)
    if B.ndim != 2 or B.shape[0] != operator.n or X.shape != B.shape:
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "block_residual: B and X must be n x r")
    R = np.zeros_like(B)
    check(L.load().sb_operator_block_residual(operator.handle, _p(B), _p(X), B.shape[1], _p(R)))
    return R


def gmres_multi(operator: TbemOperator, B, config: IrConfig = IrConfig()):
    """Many right-hand sides of one operator (the block_gmres_preconditioned role,
    crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:163): B is n x r, returns
    (X n x r, [GmresSolution without x per right-hand side]). Inner products on the tensor cores,
    FP64 refinement; the operator must hold the complex128 matrix."""
    B = _c128(B)
    if B.ndim != 2 or B.shape[0] != operator.n:
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "gmres_multi: B must be n x r")
    r = B.shape[1]
    X = np.zeros_like(B)
    stats = (L.SbGmresStats * r)()
    check(L.load().sb_gmres_multi(operator.handle, _p(B), r, ct.byref(config._struct()), _p(X),
                                  ct.cast(stats, ct.c_void_p)))
    return X, [GmresSolution._from(None, stats[i]) for i in range(r)]


class GcroDrSubspace:
    """GcroDrSubspace (crates/sonium-solvers/crates/sonium-solvers-iterative/src/gcro_dr.rs:65-110):
    up to k orthonormal recycled vectors kept on one device across GCRO-DR solves."""

    def __init__(self, k: int, device: int = 0):
        h = ct.c_void_p()
        check(L.load().sb_gcro_subspace_create(device, int(k), ct.byref(h)))
        self._h = h

    @property
    def handle(self):
        if self._h is None:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "subspace has been closed")
        return self._h

    def _info(self):
        c, t, n = ct.c_int64(), ct.c_int64(), ct.c_int64()
        check(L.load().sb_gcro_subspace_info(self.handle, ct.byref(c), ct.byref(t), ct.byref(n)))
        return c.value, t.value, n.value

    def num_vectors(self) -> int:
        return self._info()[0]

    def target_size(self) -> int:
        return self._info()[1]

    def is_populated(self) -> bool:
        return self.num_vectors() > 0

    def reset(self) -> None:
        check(L.load().sb_gcro_subspace_reset(self.handle))

    def vectors(self) -> np.ndarray:
        """The held vectors, (num_vectors, n) complex128."""
        c, _, n = self._info()
        u = np.zeros((c, n), np.complex128)
        if c:
            check(L.load().sb_gcro_subspace_get_vectors(self.handle, _p(u)))
        return u

    def replace_vectors(self, u) -> None:
        u = np.ascontiguousarray(np.atleast_2d(u), np.complex128)
        check(L.load().sb_gcro_subspace_set_vectors(self.handle, u.shape[0], u.shape[1] if u.shape[0] else 0,
                                                    _p(u) if u.size else None))

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.load().sb_gcro_subspace_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class GcroDrConfig:
    """GcroDrConfig (gcro_dr.rs:114-160): restart cycles, Krylov dimension per cycle, relative
    tolerance."""

    max_iterations: int = 100
    restart: int = 50
    tolerance: float = 1e-6

    @classmethod
    def from_gmres(cls, g: GmresConfig) -> "GcroDrConfig":
        return cls(g.max_iterations, g.restart, g.tolerance)

    def _struct(self):
        return L.SbGmresConfig(self.max_iterations, self.restart, self.tolerance, 1)


def gcro_dr(operator: TbemOperator, b, subspace: GcroDrSubspace, config: GcroDrConfig = GcroDrConfig(),
            x0=None, preconditioner: JacobiPreconditioner | None = None) -> GmresSolution:
    """gcro_dr / gcro_dr_preconditioned (gcro_dr.rs:164-260) on the device: consumes the recycled
    subspace and leaves the updated one in it."""
    b = _c128(b)
    if b.shape != (operator.n,):
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "gcro_dr: b must have length n")
    x = np.zeros(operator.n, np.complex128)
    x0a = None if x0 is None else _c128(x0)
    st = L.SbGmresStats()
    pk = L.SB_PRECOND_IDENTITY if preconditioner is None else preconditioner.kind
    check(L.load().sb_gcro_dr(operator.handle, _p(b), None if x0a is None else _p(x0a), subspace.handle,
                              ct.byref(config._struct()), pk, _p(x), ct.byref(st)))
    return GmresSolution._from(x, st)


def compute_scattered_field(mesh: Mesh, physics: PhysicsParams, surface_pressure, points,
                            surface_velocity=None) -> np.ndarray:
    """compute_scattered_field_checked (crates/sonium-bem/src/core/postprocess/pressure.rs:250):
    scattered pressure at points (m x 3) from constant surface pressure / velocity."""
    p = _c128(surface_pressure)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    if p.shape != (mesh.num_elements,):
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "surface_pressure must have one value per element")
    v = None if surface_velocity is None else _c128(np.broadcast_to(surface_velocity, p.shape))
    out = np.zeros(pts.shape[0], np.complex128)
    check(L.load().sb_field_eval(mesh.handle, ct.byref(physics._struct()), _p(p), None if v is None else _p(v),
                                 _p(pts), pts.shape[0], _p(out)))
    return out


def compute_total_field(mesh: Mesh, physics: PhysicsParams, surface_pressure, points, direction=(0.0, 0.0, 1.0),
                        amplitude: complex = 1.0, surface_velocity=None) -> np.ndarray:
    """compute_total_field_checked (pressure.rs:501): scattered field plus the incident plane wave
    A exp(i k d.x) (IncidentField::evaluate_pressure, incident.rs:216-245)."""
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    d = np.asarray(direction, np.float64)
    d = d / np.linalg.norm(d)
    inc = amplitude * np.exp(1j * physics.harmonic_factor * physics.wave_number * (pts @ d))
    return compute_scattered_field(mesh, physics, surface_pressure, pts, surface_velocity) + inc


def fibonacci_sphere_directions(n: int) -> np.ndarray:
    """Unit vectors on a Fibonacci sphere (the reference's fibonacci_sphere_directions,
    crates/sonium-bem/src/core/assembly/mlfmm.rs:8012-8024)."""
    golden = (1.0 + np.sqrt(5.0)) / 2.0
    i = np.arange(n, dtype=np.float64)
    theta = np.arccos(1.0 - 2.0 * (i + 0.5) / n)
    phi = 2.0 * np.pi * i / golden
    return np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], axis=1)


def inject_failure(point: int) -> None:
    check(L.load().sb_inject_failure(point))
