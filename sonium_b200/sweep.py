"""Batched frequency sweep over the sonium-b200 C ABI.

Mirrors the reference's sweep lifecycle (crates/sonium-bem/src/core/solver/frequency_sweep.rs:
``FrequencySweepConfig`` at :43-170, ``FrequencySweepResult`` at :175-230, the per-frequency loop of
``frequency_sweep_with_physics_and_admittances`` at :592-700), but instead of assembling and solving
one frequency after another, every instance (mesh, physics, Burton-Miller beta) is assembled in one
persistent launch and all are solved together by the batched mixed-precision GMRES
(``sb_batch_*`` in ``include/sonium_b200.h``). Instances may use different meshes, so a sweep can
refine the mesh with frequency.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import SoniumError, check
from .tbem import (GmresConfig, GmresSolution, IrConfig, Mesh, PhysicsParams, _c128, _p,
                   build_tbem_system_with_beta, gmres, gmres_mixed, rhs_plane_wave)


class SweepBatch:
    """Device-resident batch of TBEM instances (complex64 matrices, FP64-refined solves)."""

    def __init__(self, meshes, physics, betas):
        meshes = list(meshes)
        physics = list(physics)
        betas = [complex(b) for b in betas]
        if not (len(meshes) == len(physics) == len(betas)) or not meshes:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "batch: meshes, physics and betas must have one "
                                                         "entry per instance")
        self.meshes = meshes  # the batch refers to the meshes' device data: keep them alive
        self.physics = physics
        self.betas = betas
        n = len(meshes)
        handles = (ct.c_void_p * n)(*[m.handle.value for m in meshes])
        phys = (L.SbPhysics * n)(*[p._struct() for p in physics])
        bet = (L.SbComplex * n)(*[L.SbComplex(b.real, b.imag) for b in betas])
        h = ct.c_void_p()
        check(L.load().sb_batch_create(n, ct.cast(handles, ct.c_void_p), ct.cast(phys, ct.c_void_p),
                                       ct.cast(bet, ct.c_void_p), ct.byref(h)))
        self._h = h

    @property
    def handle(self):
        if self._h is None:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "batch has been closed")
        return self._h

    def __len__(self) -> int:
        return len(self.meshes)

    def sizes(self):
        return [m.num_elements for m in self.meshes]

    def assemble(self) -> float:
        """Assemble every instance; returns the device time in ms."""
        check(L.load().sb_batch_assemble(self.handle))
        return self.timings()[0]

    def set_assembly_mode(self, mode: int) -> None:
        """SB_BATCH_ASM_AUTO (autotuned), SB_BATCH_ASM_PERSISTENT or SB_BATCH_ASM_STREAMS."""
        check(L.load().sb_batch_set_assembly_mode(self.handle, int(mode)))

    def assembly_tuning(self):
        """(form used by the last assembly, autotuner's persistent ms, autotuner's streams ms)."""
        c, a, b = ct.c_int(), ct.c_double(), ct.c_double()
        check(L.load().sb_batch_assembly_tuning(self.handle, ct.byref(c), ct.byref(a), ct.byref(b)))
        return c.value, a.value, b.value

    def assembly_split(self):
        """(far CTA slots per SM of the persistent form's two-launch layout, 0 = one launch;
        {layout: autotuner ms}, layouts "one_launch", "far_2", "far_3", "far_4", 0 when it did not run)."""
        c = ct.c_int()
        t = np.zeros(5, np.float64)
        check(L.load().sb_batch_assembly_split(self.handle, ct.byref(c), _p(t)))
        return c.value, {"one_launch": t[0], "far_2": t[2], "far_3": t[3], "far_4": t[4]}

    def set_inner_precision(self, inner: int) -> None:
        """SB_INNER_FP32 (the complex64 matrices) or SB_INNER_FP16 (complex-half copies, built by
        the first solve after each assembly; pair with IrConfig(inner_tolerance=1e-3))."""
        check(L.load().sb_batch_set_inner_precision(self.handle, int(inner)))

    def set_inner_preconditioner(self, kind: int, block_size: int = 64) -> None:
        """SB_INNER_PRECOND_NONE or SB_INNER_PRECOND_BLOCK_JACOBI (blocks of block_size spatially
        close elements per instance, inverted by the first solve after each assembly)."""
        check(L.load().sb_batch_set_inner_preconditioner(self.handle, int(kind), int(block_size)))

    def set_rhs_plane_wave(self, direction=(0.0, 0.0, 1.0)) -> None:
        d = np.ascontiguousarray(direction, np.float64)
        check(L.load().sb_batch_set_rhs_plane_wave(self.handle, _p(d)))

    def set_rhs(self, index: int, b) -> None:
        b = _c128(b)
        if b.shape != (self.meshes[index].num_elements,):
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "batch: right-hand side length must be n")
        check(L.load().sb_batch_set_rhs(self.handle, index, _p(b)))

    def solve(self, config: IrConfig = IrConfig()) -> list:
        """Batched FP32-inner / FP64-refined GMRES; one GmresSolution (without x) per instance."""
        n = len(self)
        stats = (L.SbGmresStats * n)()
        check(L.load().sb_batch_solve(self.handle, ct.byref(config._struct()), ct.cast(stats, ct.c_void_p)))
        return [GmresSolution._from(None, stats[i]) for i in range(n)]

    def solution(self, index: int) -> np.ndarray:
        x = np.zeros(self.meshes[index].num_elements, np.complex128)
        check(L.load().sb_batch_solution(self.handle, index, _p(x)))
        return x

    def matrix_c64(self, index: int) -> np.ndarray:
        m = self.meshes[index].num_elements
        a = np.zeros((m, m), np.complex64)
        check(L.load().sb_batch_matrix_c64(self.handle, index, _p(a)))
        return a

    def timings(self):
        """(assembly_ms, solve_ms) of the last assemble / solve."""
        a, s = ct.c_double(), ct.c_double()
        check(L.load().sb_batch_timings(self.handle, ct.byref(a), ct.byref(s)))
        return a.value, s.value

    def close(self):
        if getattr(self, "_h", None) is not None:
            L.load().sb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class FrequencySweepResult:
    """FrequencySweepResult (frequency_sweep.rs:175-230) of a batched sweep."""

    solutions: list
    frequencies: list
    iteration_counts: list
    converged: list
    exact_relative_residuals: list
    assembly_ms: float
    solve_ms: float
    stats: list = field(default_factory=list)
    assembly_times: list = field(default_factory=list)  # seconds per frequency (sequential sweep)
    solve_times: list = field(default_factory=list)
    recycled_subspace_eligible: list = field(default_factory=list)  # sequential sweep (:196)

    def total_iterations(self) -> int:
        return int(sum(self.iteration_counts))

    def average_iterations(self) -> float:
        return self.total_iterations() / len(self.iteration_counts) if self.iteration_counts else 0.0

    def num_converged(self) -> int:
        return int(sum(bool(c) for c in self.converged))


def frequency_sweep_batched(meshes, physics, betas, direction=(0.0, 0.0, 1.0),
                            config: IrConfig = IrConfig()) -> FrequencySweepResult:
    """Assemble and solve every instance of a plane-wave scattering sweep in one batch."""
    batch = SweepBatch(meshes, physics, betas)
    try:
        batch.assemble()
        batch.set_rhs_plane_wave(direction)
        stats = batch.solve(config)
        sols = [batch.solution(i) for i in range(len(batch))]
        a_ms, s_ms = batch.timings()
    finally:
        batch.close()
    return FrequencySweepResult(
        solutions=sols, frequencies=[p.frequency for p in physics],
        iteration_counts=[s.iterations for s in stats], converged=[s.converged for s in stats],
        exact_relative_residuals=[s.residual for s in stats], assembly_ms=a_ms, solve_ms=s_ms, stats=stats)


@dataclass
class FrequencySweepConfig:
    """FrequencySweepConfig (frequency_sweep.rs:43-170): frequencies (Hz, strictly increasing),
    GMRES tolerance / restarts / restart length, warm start from the previous frequency's solution
    (recycle_solution), Burton-Miller beta scale."""

    frequencies: list = field(default_factory=list)
    tolerance: float = 1e-6
    max_iterations: int = 200
    recycle_solution: bool = True
    gmres_restart: int = 30
    beta_scale: float = 4.0
    # GCRO-DR vectors recycled between adjacent frequencies (0 = warm start only), and the largest
    # relative frequency step |f_new - f_old| / max(f_new, f_old) that keeps the subspace (:60-68).
    recycle_subspace_size: int = 0
    max_recycle_relative_frequency_delta: float = 0.1

    def validate(self) -> None:
        """FrequencySweepConfig::validate (frequency_sweep.rs:88-114) and validate_frequency_grid
        (:306-320)."""
        if not (np.isfinite(self.tolerance) and self.tolerance > 0):
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "frequency-sweep tolerance must be finite and positive")
        if self.max_iterations <= 0 or self.gmres_restart <= 0:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT,
                              "frequency-sweep iteration and restart limits must be non-zero")
        if not (np.isfinite(self.beta_scale) and self.beta_scale > 0):
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "Burton-Miller beta scale must be finite and positive")
        d = self.max_recycle_relative_frequency_delta
        if not (np.isfinite(d) and d >= 0):
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT,
                              "frequency-sweep recycle frequency bound must be finite and non-negative")
        if self.recycle_subspace_size < 0:
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "recycle_subspace_size must be non-negative")
        f = np.asarray(self.frequencies, np.float64)
        if f.size == 0 or not np.all(np.isfinite(f)) or np.any(f <= 0) or np.any(np.diff(f) <= 0):
            raise SoniumError(L.SB_ERR_INVALID_ARGUMENT,
                              "frequency sweep frequencies must be finite, positive, and strictly increasing")

    @classmethod
    def linear(cls, start_hz: float, end_hz: float, num_points: int) -> "FrequencySweepConfig":
        step = (end_hz - start_hz) / (num_points - 1) if num_points > 1 else 0.0
        return cls(frequencies=[start_hz + i * step for i in range(num_points)])

    @classmethod
    def logarithmic(cls, start_hz: float, end_hz: float, num_points: int) -> "FrequencySweepConfig":
        a, b = np.log(start_hz), np.log(end_hz)
        step = (b - a) / (num_points - 1) if num_points > 1 else 0.0
        return cls(frequencies=[float(np.exp(a + i * step)) for i in range(num_points)])


def frequency_sweep(mesh: Mesh, config: FrequencySweepConfig, direction=(0.0, 0.0, 1.0),
                    speed_of_sound: float = 343.0, density: float = 1.21, mixed: bool = False,
                    ir: IrConfig | None = None) -> FrequencySweepResult:
    """The reference's sequential sweep (frequency_sweep_with_physics_and_admittances,
    frequency_sweep.rs:592-850, dense branch): per frequency, re-assemble the dense system into one
    device operator (the CudaTbemAssemblyWorkspace pattern), add the incident plane wave to the
    boundary-condition right-hand side, solve with the previous frequency's solution as the
    initial guess when recycle_solution is set, and accept the point only if the exact relative
    residual is within max(20 tol, 1e-10) (:790-799). With recycle_subspace_size > 0 every solve is
    GCRO-DR (solve_sweep_operator, :495-508) on one recycled subspace, started afresh whenever the
    relative step from the previous frequency exceeds max_recycle_relative_frequency_delta
    (:636-647, relative_frequency_delta of crates/sonium-bem/src/core/mesh/lineage.rs:548).
    `mixed` solves with the FP32-inner / FP64-refined GMRES instead of FP64 GMRES (no recycling)."""
    import time

    from .tbem import GcroDrConfig, GcroDrSubspace, gcro_dr

    config.validate()
    if mixed and config.recycle_subspace_size > 0:
        raise SoniumError(L.SB_ERR_INVALID_ARGUMENT, "subspace recycling runs the FP64 solver: mixed must be False")
    op = None
    prev = None
    prev_f = None
    sub = None
    res = FrequencySweepResult([], [], [], [], [], 0.0, 0.0)
    try:
        for f in config.frequencies:
            eligible = prev_f is not None and abs(f - prev_f) / max(abs(prev_f), abs(f)) <= \
                config.max_recycle_relative_frequency_delta
            if config.recycle_subspace_size > 0 and (sub is None or not eligible):
                if sub is not None:
                    sub.close()
                sub = GcroDrSubspace(config.recycle_subspace_size, mesh.device)
            ph = PhysicsParams.new(f, speed_of_sound, density)
            beta = ph.burton_miller_beta(config.beta_scale)
            t0 = time.perf_counter()
            if op is None:
                op = build_tbem_system_with_beta(mesh, ph, beta,
                                                 L.SB_PRECISION_FP64_FP32 if mixed else L.SB_PRECISION_FP64)
            else:
                op.reassemble(ph, beta)
            b = op.rhs + rhs_plane_wave(mesh, ph, beta, [direction])[:, 0]
            t1 = time.perf_counter()
            x0 = prev if (config.recycle_solution and prev is not None) else None
            if mixed:
                cfg = ir or IrConfig(tolerance=config.tolerance, inner_restart=config.gmres_restart)
                sol = gmres_mixed(op, b, cfg, x0=x0)
            elif sub is not None:
                sol = gcro_dr(op, b, sub, GcroDrConfig(config.max_iterations, config.gmres_restart, config.tolerance),
                              x0=x0)
            else:
                sol = gmres(op, b, GmresConfig(max_iterations=config.max_iterations, restart=config.gmres_restart,
                                               tolerance=config.tolerance), x0=x0)
            t2 = time.perf_counter()
            tol = max(20.0 * config.tolerance, 1e-10)
            if not np.isfinite(sol.residual) or sol.residual > tol:
                raise SoniumError(L.SB_ERR_NOT_FINITE,
                                  f"frequency sweep at {f:.3f} Hz: residual {sol.residual:.3e} above {tol:.3e}")
            prev = sol.x
            res.solutions.append(sol.x)
            res.frequencies.append(f)
            res.iteration_counts.append(sol.iterations)
            res.converged.append(sol.converged)
            res.exact_relative_residuals.append(sol.residual)
            res.assembly_times.append(t1 - t0)
            res.solve_times.append(t2 - t1)
            res.stats.append(sol)
            res.recycled_subspace_eligible.append(bool(eligible))
            prev_f = f
    finally:
        if op is not None:
            op.close()
        if sub is not None:
            sub.close()
    res.assembly_ms = 1e3 * sum(res.assembly_times)
    res.solve_ms = 1e3 * sum(res.solve_times)
    return res


# Sweep workload: ka log-spaced on a triaxial ellipsoid, mesh refined with frequency.
ELLIPSOID_AXES = (1.0, 0.6, 0.4)


def max_edge_length(nodes: np.ndarray, tris: np.ndarray) -> float:
    e = [np.linalg.norm(nodes[tris[:, i]] - nodes[tris[:, (i + 1) % 3]], axis=1).max() for i in range(3)]
    return float(max(e))


def level_for_wavenumber(k: float, edge_by_level: dict, elements_per_wavelength: float = 8.0) -> int:
    """Smallest icosphere level whose longest edge gives `elements_per_wavelength` per wavelength
    (the finest level offered when none does)."""
    lam = 2.0 * np.pi / k
    for level in sorted(edge_by_level):
        if lam / edge_by_level[level] >= elements_per_wavelength:
            return level
    return max(edge_by_level)


def ellipsoid_sweep_plan(count: int = 64, ka_min: float = 1.0, ka_max: float = 32.0,
                         axes=ELLIPSOID_AXES, levels=(2, 3, 4, 5), elements_per_wavelength: float = 8.0):
    """[(ka, k, level)] for `count` instances with ka = k * axes[0] log-spaced in [ka_min, ka_max]."""
    from .tbem import icosphere
    edges = {}
    for lv in levels:
        nodes, tris = icosphere(1.0, lv, axes)
        edges[lv] = max_edge_length(nodes, tris)
    plan = []
    for ka in np.geomspace(ka_min, ka_max, count):
        k = float(ka) / axes[0]
        plan.append((float(ka), k, level_for_wavenumber(k, edges, elements_per_wavelength)))
    return plan


def build_ellipsoid_sweep(plan, axes=ELLIPSOID_AXES, device: int = 0, speed_of_sound: float = 343.0,
                          density: float = 1.21):
    """Meshes (one per level, shared by the instances of that level), physics and betas of a plan."""
    meshes_by_level = {}
    meshes, physics, betas = [], [], []
    for _, k, level in plan:
        if level not in meshes_by_level:
            meshes_by_level[level] = Mesh.icosphere(1.0, level, axes, device=device)
        ph = PhysicsParams.for_wavenumber(k, speed_of_sound, density)
        meshes.append(meshes_by_level[level])
        physics.append(ph)
        betas.append(ph.burton_miller_beta())
    return meshes, physics, betas
