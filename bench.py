"""Benchmark: BEM solves/s (dense Burton-Miller TBEM: assembly + GMRES) on B200.

Workload (default): rigid sphere, icosphere level 5 (N = 20480 flat triangles, constant panels
collocated at centroids), k = 10, incident plane wave exp(i k z), beta = i/k. One step = one
solve: re-assembly of the dense system on the device, the incident right-hand side, and GMRES.

  * `value`  -- the fastest mixed-precision form whose solution is within 1e-5 of the plain FP64
                one (`headline_mode`): FP32 assembly (FP64 phase, near and self terms) and FP64
                refinement to 1e-8 around an inner GMRES(50) with FP32 vectors, on the complex64
                matrix (`mixed`, inner tolerance 1e-5) or on its power-of-two-scaled complex-half
                copy (`mixed_half`, inner tolerance 1e-3), the latter also with a block-Jacobi
                right preconditioner of the inner solve (`mixed_half_bj`, blocks of 128 spatially
                close elements); `mixed_fp64_matrix` refines on the complex128 matrix. Inputs resident in HBM, device time by CUDA events on the
                operator's stream; every mode's error against the plain FP64 solution is reported.
  * `plain_fp64` -- the same solve with complex128 only and FP64 GMRES(50) to 1e-8; `plain_fp64_bj`
                the same with the headline's block-Jacobi right preconditioner (blocks of 128), the
                like-for-like FP64 form: the line reports the speed-up against both.
  * `e2e`    -- the headline form through the C ABI with host buffers: mesh upload, assembly,
                host RHS, solve with host b / x (all copies inside the timed region).
  * `cpu_baseline` / `--impl reference` -- the CPU restatement of the reference path (oracle) on
                the host cores: whole solves (all N rows of the assembly, the RHS, GMRES(50) from
                x0 = 0 to 1e-8 with its real iteration count), one per step, same metric string.

  * `sweep`  -- the batched frequency sweep: 64 instances (ka 1 -> 32 on the (1, 0.6, 0.4) ellipsoid,
                levels 2-5) assembled together (the autotuned form: one persistent launch or
                per-instance kernels on two streams) and solved by the batched mixed GMRES,
                against the same instances solved one after another in plain FP64 (and in FP64 with
                the sweep's block-Jacobi preconditioner).
  * `multi_rhs` -- 256 plane-wave right-hand sides of one operator (ellipsoid level 5, k = 16)
                solved together with tensor-core block products, against plain FP64 GMRES per
                right-hand side; carries the tensor kernel's roofline.
  * `precision_form` -- N = 81920, k = 40 (complex128 + complex64, ~165 GB): FP64 and mixed solves
                to 1e-10, their difference and both surface errors against the Mie series
                (skipped with the free memory it found when the device has less).
  * `reference_gpu_assembly` -- the reference's own CUDA pair kernel (compiled from its source) on
                its quadrature charts, beside this library's FP64 assembly of the same system.
  Legs alone: `--precision-form`, `--sweep-only`, `--multi-rhs`.

With torchrun (N > 1 ranks): the single-solve headline runs one replica per rank (a solve has no
exchange step to split); value = all ranks' solves / max-over-ranks time. The sweep shares its 64
instances out over the ranks (balanced by N^2) and the multi-RHS leg its groups of 128
right-hand sides (sonium_b200/shard.py): all instances / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import csv
import ctypes as ct
import io
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RADIUS = 1.0
LEVEL = 5
K = 10.0
RESTART = 50
TOL = 1e-8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=LEVEL)
    ap.add_argument("--k", type=float, default=K)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 timing")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the batched frequency-sweep leg")
    ap.add_argument("--sweep-count", type=int, default=64, help="instances of the frequency sweep")
    ap.add_argument("--sweep-only", action="store_true", help="run only the sweep leg and print its JSON")
    ap.add_argument("--multi-rhs", action="store_true",
                    help="run only the 256-right-hand-side tensor-core leg and print its JSON")
    ap.add_argument("--rhs", type=int, default=256, help="right-hand sides of the multi-RHS leg")
    ap.add_argument("--no-multi", action="store_true", help="skip the multi-RHS leg in the default run")
    ap.add_argument("--no-precision-form", action="store_true",
                    help="skip the N = 81920, k = 40 precision-form leg (~165 GB) in the default run")
    ap.add_argument("--no-gemv-bar", action="store_true",
                    help="skip the cuBLAS Cgemv / Zgemv comparison of the matrix-vector products")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the leg that times the reference's own CUDA assembly kernel beside ours")
    ap.add_argument("--precision-form", action="store_true",
                    help="run only the N = 81920, k = 40 precision-form leg (~165 GB) and print its JSON")
    ap.add_argument("--single", action="store_true",
                    help="one untimed solve per precision mode at --level (profiling driver), no JSON line")
    ap.add_argument("--single-mode", choices=sorted(MODES), default=None,
                    help="with --single: run only this mode")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# distributed plumbing (only used when launched by torchrun)
# ---------------------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons around a timed region.

    The sampler runs at 25 ms; start() waits for its first sample so that the timed region is
    covered from its beginning, and stop() keeps the samples taken between mark() and stop()
    (plus the one just before mark(), so that a region shorter than the period still has one).
    """
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 25

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.rows = []
        self.t_mark = None
        self.thread = None

    def _reader(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), line))

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", str(self.PERIOD_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._reader, daemon=True)
        self.thread.start()
        t0 = time.perf_counter()
        while not self.rows and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.005)
        self.t_mark = time.perf_counter()

    def mark(self):
        self.t_mark = time.perf_counter()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(self.PERIOD_MS / 1000.0 * 1.5)  # one more sample after the region
        t_stop = time.perf_counter()
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=10)
        rows = list(self.rows)
        before = [r for r in rows if r[0] < self.t_mark]
        inside = [r for r in rows if self.t_mark <= r[0] <= t_stop]
        keep = (before[-1:] if before else []) + inside
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in csv.reader(io.StringIO("".join(line for _, line in keep))):
            if len(row) < 9:
                continue
            try:
                sm.append(float(row[1]))
                smax.append(float(row[2]))
            except ValueError:
                continue
            for nm, v in zip(names, row[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "sm_mhz_min": min(sm), "period_ms": self.PERIOD_MS}


def mie_rigid_surface(k: float, radius: float, theta: np.ndarray, terms: int) -> np.ndarray:
    """Total surface pressure of a plane wave exp(i k z) on a rigid sphere (Mie series,
    crates/sonium-wave/src/analytical/solutions_3d.rs:315-366, 769-806): sum over n of
    (2n + 1) i^n (j_n(ka) - a_n h_n(ka)) P_n(cos theta), a_n = j_n'(ka) / h_n'(ka), h_n = j_n + i y_n."""
    from scipy.special import eval_legendre, spherical_jn, spherical_yn

    ka = k * radius
    nn = np.arange(terms)
    jp, yp = spherical_jn(nn, ka, derivative=True), spherical_yn(nn, ka, derivative=True)
    j, y = spherical_jn(nn, ka), spherical_yn(nn, ka)
    coef = (2 * nn + 1) * (1j ** nn) * (j - jp / (jp + 1j * yp) * (j + 1j * y))
    ct_ = np.cos(theta)
    out = np.zeros(theta.shape, complex)
    for m in range(terms):
        out += coef[m] * eval_legendre(m, ct_)
    return out


def mie_surface_error(x: np.ndarray, centers: np.ndarray, areas: np.ndarray, k: float, radius: float) -> float:
    """Area-weighted relative L2 error of surface pressure x (element centroids) against the Mie
    series (rigid_sphere_surface_relative_l2_error, crates/sonium-qa/src/lib.rs:319-358; terms
    max(4 ceil(ka) + 16, 17) as suggested_sphere_terms, solutions_3d.rs:241-249)."""
    ka = k * radius
    terms = max(int(np.ceil(ka)) * 4 + 16, 17)
    theta = np.arccos(np.clip(centers[:, 2] / np.linalg.norm(centers, axis=1), -1.0, 1.0))
    ref = mie_rigid_surface(k, radius, theta, terms)
    return float(np.sqrt(np.sum(areas * np.abs(x - ref) ** 2) / np.sum(areas * np.abs(ref) ** 2)))


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ---------------------------------------------------------------------------------------------
# CPU path (oracle restatement of the reference CPU code): whole solves, nothing extrapolated
# ---------------------------------------------------------------------------------------------
METRIC = "BEM solves/s at <=1e-5 rel err vs FP64 (mixed-precision solve, dense Burton-Miller TBEM)"


def cpu_solve(level: int, k: float):
    """One whole solve of the workload on the host cores by the oracle (C++ restatement of the
    reference CPU path, OpenMP over rows): assembly of all N rows (build_tbem_system_with_beta_parallel,
    tbem.rs:1284-1466), the incident right-hand side, and restarted GMRES(50) from x0 = 0 to rtol 1e-8
    with its real iteration count (gmres.rs:631-1000). Returns the timings and counts."""
    from oracle import oracle as O

    O.build()
    nodes, tris = O.icosphere(RADIUS, level)
    n = tris.shape[0]
    ph = O.physics_for_k(k)
    beta = O.bm_beta(ph)
    t0 = time.perf_counter()
    A, _ = O.assemble(nodes, tris, ph, beta)
    t1 = time.perf_counter()
    c, nrm, _ = O.element_geometry(nodes, tris)
    b = O.rhs_plane_wave(c, nrm, ph, beta, np.array([[0.0, 0.0, 1.0]]))[:, 0]
    x, res = O.gmres(A, b, restart=RESTART, max_iterations=100, tol=TOL)
    t2 = time.perf_counter()
    del A
    return {"n": n, "s": t2 - t0, "assembly_s": t1 - t0, "solve_s": t2 - t1, "iterations": int(res.iterations),
            "matvecs": int(res.matvecs), "converged": bool(res.converged), "residual": float(res.residual)}


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample_text(r) -> str:
    return (f"oracle (C++ restatement of the reference CPU path, OpenMP {cpu_threads()} threads): one whole "
            f"solve of N={r['n']}: assembly of all {r['n']} rows ({r['assembly_s']:.2f} s) + incident RHS + "
            f"GMRES({RESTART}) from x0 = 0 to rtol {TOL}: {r['iterations']} iterations, {r['matvecs']} "
            f"complex128 matvecs ({r['solve_s']:.2f} s), converged={r['converged']}")


def cpu_baseline(level: int, k: float):
    r = cpu_solve(level, k)
    return {"value": 1.0 / r["s"], "unit": "solves/s", "cores": cpu_threads(), "kind": "port",
            "sample": cpu_sample_text(r), "assembly_s": r["assembly_s"], "solve_s": r["solve_s"]}


def reference_arm(a, dist: Dist):
    """--impl reference: the reference's CPU path (its C++ restatement, oracle/) on this host's
    cores, one whole solve of the same workload per step (W untimed, K timed, wall clock)."""
    if dist.rank != 0:
        return
    for _ in range(a.warmup):
        cpu_solve(a.level, a.k)
    t0 = time.perf_counter()
    runs = [cpu_solve(a.level, a.k) for _ in range(a.steps)]
    t = time.perf_counter() - t0
    v = a.steps / t
    n = runs[-1]["n"]
    line = {
        "impl": "reference", "metric": METRIC,
        "value": v, "unit": "solves/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * t / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic (icosphere geometry, analytic incident plane wave)",
        "config": {"workload": f"rigid sphere icosphere L{a.level} (N={n}), k={a.k}, beta=i/k, plane wave +z; "
                               f"one step = assembly of all rows + RHS + GMRES({RESTART}) from x0 = 0 to rtol {TOL} "
                               "(FP64 throughout: error vs FP64 is zero)",
                   "N": n, "parallelism": "host cores (rank 0 only)"},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cpu_threads(), "kind": "port",
                         "sample": cpu_sample_text(runs[-1]) + f"; {a.steps} timed solves, wall clock"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": [r["iterations"] for r in runs],
        "assembly_s_median": float(np.median([r["assembly_s"] for r in runs])),
        "solve_s_median": float(np.median([r["solve_s"] for r in runs])),
        "note": "the Rust reference cannot be built here (no rustc/cargo); this arm times its C++ restatement "
                "(oracle/), whole solves, on the host cores",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------
MODES = {
    # name: (assembly precision, solver)
    "mixed_half_bj": ("SB_PRECISION_FP32", "ir16bj"),
    "mixed_half": ("SB_PRECISION_FP32", "ir16"),
    "mixed": ("SB_PRECISION_FP32", "ir"),
    "mixed_fp64_matrix": ("SB_PRECISION_FP64_FP32", "ir"),
    "plain_fp64": ("SB_PRECISION_FP64", "fp64"),
    # FP64 GMRES(50) with the same block-Jacobi right preconditioner as `mixed_half_bj` (blocks of
    # BJ_BLOCK): the like-for-like FP64 form of the preconditioned headline
    "plain_fp64_bj": ("SB_PRECISION_FP64", "fp64bj"),
}
# Inner tolerance of the refinement with the complex-half inner matrix: the half copy limits each
# refinement to about three digits, so a tighter inner solve buys nothing.
HALF_INNER_TOL = 1e-3
# DRAM bytes per matrix entry of one k_gemv_n_c16 launch: dram__bytes_read.sum +
# dram__bytes_write.sum = 108.19 MB at N = 5120 (ncu, cold caches).
GEMV16_TRAFFIC_PER_ENTRY = 4.13
# Modes that may carry the headline (fastest first when both meet the accuracy bar), with the
# kernel class of their dominant matrix-vector product.
HEADLINE_MODES = {"mixed_half_bj": "SB_PROF_GEMV16", "mixed_half": "SB_PROF_GEMV16", "mixed": "SB_PROF_GEMV32"}
# Block sizes of the block-Jacobi inner preconditioner: the single-solve `mixed_half_bj` form
# (N = 20480, k = 10: blocks of 128 take 33 inner iterations, 64 take 36; measured 26.9 vs 27.5 ms
# per step in one call) and the batched sweep (64, measured).
BJ_BLOCK = 128
BJ_BLOCK_SWEEP = 64


def main():
    a = parse()
    dist = Dist()
    if a.impl == "reference":
        reference_arm(a, dist)
        dist.close()
        return
    import sonium_b200 as sb
    from sonium_b200 import _lib as L
    from sonium_b200 import build as sb_build

    sb_build.build()
    lib = L.load()
    dev = dist.local
    if a.single:
        single_solves(sb, a.level, a.k, dev, a.single_mode and [a.single_mode])
        return
    assert sb.device_count() > dev, "no CUDA device for this rank"
    if a.sweep_only or a.precision_form or a.multi_rhs:
        name, leg = (("sweep", sweep_leg) if a.sweep_only else ("precision_form", precision_leg)
                     if a.precision_form else ("multi_rhs", multi_rhs_leg))
        out = leg(sb, a, dist, dev, _cudart())
        if dist.rank == 0:
            print(json.dumps({name: out}), flush=True)
        dist.close()
        return

    nodes, tris = sb.icosphere(RADIUS, a.level)
    n = tris.shape[0]
    ph = sb.PhysicsParams.for_wavenumber(a.k)
    beta = ph.burton_miller_beta()
    mesh = sb.Mesh(nodes, tris, device=dev)
    near_pairs = float(mesh.info().n_near_pairs)  # pairs the near kernel owns (the far kernel skips them)
    dirs = np.array([[0.0, 0.0, 1.0]])
    rt = _cudart()
    b_d = _dev_alloc(rt, 16 * n)  # device-resident b and x (caller-owned device memory)
    x_d = _dev_alloc(rt, 16 * n)
    phys = ph._struct()
    bta = L.SbComplex(beta.real, beta.imag)
    ir = L.SbIrConfig(20, TOL, RESTART, 20, 1e-5)
    ir16 = L.SbIrConfig(20, TOL, RESTART, 20, HALF_INNER_TOL)
    gc = L.SbGmresConfig(100, RESTART, TOL, 1)
    st = L.SbGmresStats()
    ev0, ev1 = ct.c_void_p(), ct.c_void_p()
    L.check(lib.sb_event_create(ct.byref(ev0)))
    L.check(lib.sb_event_create(ct.byref(ev1)))

    def make_step(op, solver):
        def step():
            L.check(lib.sb_assemble_into(op.handle, ct.byref(phys), bta))
            L.check(lib.sb_rhs_plane_wave_device(op.handle, dirs.ctypes.data, None, 1, b_d))
            if solver in ("ir", "ir16", "ir16bj"):
                cfg = ir if solver == "ir" else ir16
                L.check(lib.sb_gmres_mixed_device(op.handle, b_d, x_d, 0, ct.byref(cfg), ct.byref(st)))
            else:
                pk = L.SB_PRECOND_BLOCK_JACOBI if solver == "fp64bj" else L.SB_PRECOND_IDENTITY
                L.check(lib.sb_gmres_device(op.handle, b_d, x_d, 0, ct.byref(gc), pk, ct.byref(st)))
            return L.SbGmresStats.from_buffer_copy(st)
        return step

    def timed(step, handle, steps):
        dist.barrier()
        rt.cudaDeviceSynchronize()
        L.check(lib.sb_event_record(ev0, handle))
        stats = [step() for _ in range(steps)]
        L.check(lib.sb_event_record(ev1, handle))
        ms = ct.c_float()
        L.check(lib.sb_event_elapsed_ms(ev0, ev1, ct.byref(ms)))
        rt.cudaDeviceSynchronize()
        dist.barrier()
        return dist.max(ms.value / 1e3), stats

    results, x_ref = {}, None
    live = {}  # per headline-capable mode: (live profile, class breakdown, clocks, launches)
    for name in ("plain_fp64", "plain_fp64_bj", "mixed_fp64_matrix", "mixed", "mixed_half", "mixed_half_bj"):
        prec, solver = MODES[name]
        op = sb.build_tbem_system_with_beta(mesh, ph, beta, getattr(sb, prec))
        if solver == "fp64bj":
            L.check(lib.sb_operator_set_block_jacobi_size(op.handle, BJ_BLOCK))
        if solver in ("ir16", "ir16bj"):
            op.set_inner_precision(sb.SB_INNER_FP16)
        if solver == "ir16bj":
            op.set_inner_preconditioner(sb.SB_INNER_PRECOND_BLOCK_JACOBI, BJ_BLOCK)
        step = make_step(op, solver)
        s0 = step()  # untimed: solution for the accuracy check
        x = _to_host(rt, x_d, n)
        if x_ref is None:
            x_ref = x
        for _ in range(a.warmup):
            step()
        cls = HEADLINE_MODES.get(name)
        if cls:
            count = L.SbProfile()
            L.check(lib.sb_profile_read(ct.byref(count), 1))  # resets the counters
            clocks = Clocks(dev)
            clocks.start()
        t, stats = timed(step, op.handle, a.steps)
        if cls:
            clk = clocks.stop()
            L.check(lib.sb_profile_read(ct.byref(count), 1))  # kernels launched in the timed steps
            # The timed steps carry no profiling events (an event pair around each launch inside
            # the captured cycles costs ~3 ms a step). The matrix-vector product's launch times
            # come from a repetition of the same K steps with CUDA events around each launch of
            # that class on its stream; the kernel-class breakdown from a third repetition with
            # every class timed.
            live_prof = L.SbProfile()
            L.check(lib.sb_profile_enable_classes((1 << getattr(L, cls)) | (1 << L.SB_PROF_FAR)))
            for _ in range(a.steps):
                step()
            rt.cudaDeviceSynchronize()
            L.check(lib.sb_profile_enable_classes(0))
            L.check(lib.sb_profile_read(ct.byref(live_prof), 1))
            prof = L.SbProfile()
            L.check(lib.sb_profile_enable(1))
            for _ in range(a.steps):
                step()
            rt.cudaDeviceSynchronize()
            L.check(lib.sb_profile_enable(0))
            L.check(lib.sb_profile_read(ct.byref(prof), 1))
            live[name] = (live_prof, prof, clk, int(count.kernels))
        results[name] = {
            "value": dist.world * a.steps / t, "unit": "solves/s", "ms_per_step": 1e3 * t / a.steps,
            "assembly": prec, "error_vs_fp64": float(np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)),
            "iterations": int(s0.iterations), "matvecs": int(s0.matvecs), "matvecs_fp32": int(s0.matvecs_fp32),
            "refinements": int(s0.refinements), "residual": s0.residual,
        }
        if solver in ("ir16", "ir16bj"):
            results[name]["inner"] = "complex-half matrix, inner tolerance %g" % HALF_INNER_TOL
        if solver == "ir16bj":
            results[name]["inner"] += ", block-Jacobi right preconditioner (blocks of %d)" % BJ_BLOCK
        if solver == "fp64bj":
            results[name]["preconditioner"] = "block-Jacobi, right, blocks of %d (as mixed_half_bj)" % BJ_BLOCK
        op.close()
    # Headline: the fastest mixed form whose solution is within 1e-5 of the FP64 one.
    ok = [m for m in HEADLINE_MODES if results[m]["error_vs_fp64"] <= 1e-5]
    head_mode = max(ok, key=lambda m: results[m]["value"]) if ok else "mixed"
    prof_live, prof_main, clk, launches_timed = live[head_mode]

    # ---- e2e through the C ABI with host buffers ----
    e2e = None
    if not a.no_e2e:
        mesh.close()
        ts = []
        for i in range(1 + a.steps):
            rt.cudaDeviceSynchronize()
            dist.barrier()
            t0 = time.perf_counter()
            m2 = sb.Mesh(nodes, tris, device=dev)
            # the complex-half forms assemble with the half copy written by the first assembly
            o2 = sb.build_tbem_system_with_beta(m2, ph, beta, sb.SB_PRECISION_FP32 if head_mode == "mixed"
                                                else sb.SB_PRECISION_FP32_HALF)
            if head_mode == "mixed_half_bj":
                o2.set_inner_preconditioner(sb.SB_INNER_PRECOND_BLOCK_JACOBI, BJ_BLOCK)
            bh = sb.rhs_plane_wave(m2, ph, beta, dirs)[:, 0]
            sb.gmres_mixed(o2, bh, sb.IrConfig(20, TOL, RESTART, 20,
                                               1e-5 if head_mode == "mixed" else HALF_INNER_TOL))
            o2.close()
            m2.close()
            rt.cudaDeviceSynchronize()
            dt = time.perf_counter() - t0
            dist.barrier()
            if i > 0:
                ts.append(dist.max(dt))
        h2d = nodes.nbytes + tris.nbytes + 16 * n + 24  # nodes, tris, b, direction
        d2h = 16 * n + 16 * n                           # RHS and solution
        e2e = {"value": dist.world * len(ts) / sum(ts), "unit": "solves/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "sb_mesh_create + sb_assemble("
                       + ("SB_PRECISION_FP32) + " if head_mode == "mixed" else "SB_PRECISION_FP32_HALF) + ")
                       + ("sb_operator_set_inner_preconditioner(SB_INNER_PRECOND_BLOCK_JACOBI, %d) + " % BJ_BLOCK
                          if head_mode == "mixed_half_bj" else "")
                       + "sb_rhs_plane_wave + sb_gmres_mixed (host buffers), wall clock"}

    # ---- batched frequency sweep ----
    sweep = None if a.no_sweep else sweep_leg(sb, a, dist, dev, rt)
    multi = None
    if not a.no_multi:
        lvl = a.level
        a.level = LEVEL
        multi = multi_rhs_leg(sb, a, dist, dev, rt)
        a.level = lvl

    extra_legs = {}
    if not a.no_precision_form:
        extra_legs["precision_form"] = precision_leg(sb, a, dist, dev, rt, reps=1)
    if not a.no_ref_gpu:
        extra_legs["reference_gpu_assembly"] = reference_gpu_leg(sb, L, lib, dev)
    if not a.no_gemv_bar:
        extra_legs["gemv_bar"] = gemv_bar_leg(sb, L, lib, dev, rt)

    # ---- roofline of the dominant kernel of the headline step ----
    pk, pk_kind = peaks()
    names = L.PROF_NAMES
    prof = prof_main
    ms = {names[i]: prof.ms[i] for i in range(L.SB_PROF_KINDS)}
    launches = {names[i]: prof.launches[i] for i in range(L.SB_PROF_KINDS)}
    total_ms = sum(ms.values())
    dominant = max(ms, key=lambda kk: ms[kk])
    # complex-half matvec: 4 N^2 bytes of matrix per launch (+ 8 N x, 8 N y); complex64: 8 N^2;
    # complex128: 16 N^2
    bytes_mv = {"gemv16": 4.0 * n * n + 16.0 * n, "gemv32": 8.0 * n * n + 16.0 * n,
                "gemv64": 16.0 * n * n + 32.0 * n}
    hbm_kind = "gemv32" if head_mode == "mixed" else "gemv16"
    hbm_cls = getattr(L, HEADLINE_MODES[head_mode])
    # average working launch of the matvec, from the events recorded inside the timed region
    live_ms = prof_live.ms[hbm_cls]
    live_n = prof_live.launches[hbm_cls]
    avg = live_ms / max(live_n, 1) / 1e3
    achieved = bytes_mv[hbm_kind] / avg / 1e9
    # DRAM traffic per launch from one ncu capture of the same kernel at N = 5120, scaled by the
    # entries of this launch: dram__bytes_read.sum + dram__bytes_write.sum per matrix entry.
    traffic_per_entry = {"gemv16": GEMV16_TRAFFIC_PER_ENTRY, "gemv32": 8.47}
    tpe = traffic_per_entry.get(hbm_kind)
    traffic = None if tpe is None else tpe * n * n
    kernel_names = {"gemv16": "k_gemv_n_c16 (complex-half matrix, FP32 vectors)",
                    "gemv32": "k_gemv_n_c64 (complex64 matrix; FP32 or FP64 vectors)"}
    roof_gemv = {"kernel": kernel_names[hbm_kind],
                 "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                 "frac": achieved / pk["hbm_gbs"], "traffic": traffic, "peak_source": pk_kind,
                 "bytes_per_launch": bytes_mv[hbm_kind], "avg_launch_ms": avg * 1e3,
                 "launches": int(live_n), "share_of_kernel_time": ms[hbm_kind] / max(total_ms, 1e-9),
                 "measured": "CUDA events on the operator's stream around each matvec launch, in a repetition of "
                             "the K timed steps (the timed steps themselves carry no events)"}
    # Far field (FP32 kernel): point evaluations of the 13-point far leaf over the far pairs, in
    # the assembly convention of 90 FP64-equivalent flops per evaluation (sincos, sqrt and
    # reciprocals not counted), against the FP32 FMA rate measured on this device.
    far_pairs = float(n) * (n - 1) - near_pairs
    evals = 13.0 * far_pairs
    far_n = prof_live.launches[L.SB_PROF_FAR]
    far_avg = prof_live.ms[L.SB_PROF_FAR] / max(far_n, 1) / 1e3
    fp32_s, fp32_p = ct.c_double(), ct.c_double()
    L.check(lib.sb_measure_fp32_rate(dev, ct.byref(fp32_s), ct.byref(fp32_p)))
    fp32_peak = max(fp32_s.value, fp32_p.value)
    far_tflops = 90.0 * evals / far_avg / 1e12
    # bytes the far kernel must write: the complex64 entries of the far pairs and, with the
    # complex-half copy, their FP16 pairs
    far_bytes = far_pairs * (8.0 + (0.0 if head_mode == "mixed" else 4.0))
    roof_far = {"kernel": "k_far32 (FP32 far field, FP64 phase, packed f32x2)",
                "bound": "fp32 (FMA pipe with the special-function unit)",
                "achieved": far_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": far_tflops / fp32_peak, "traffic": None, "peak_source":
                    "measured on this device (sb_measure_fp32_rate: FMA chains on every SM, best of scalar %.1f "
                    "and packed f32x2 %.1f TFLOP/s)" % (fp32_s.value, fp32_p.value),
                "flop_convention": "90 FP64-equivalent flop per point evaluation, 13 evaluations per far pair "
                                   "(%.4g far pairs)" % far_pairs,
                "evals_per_s": evals / far_avg, "avg_launch_ms": far_avg * 1e3, "launches": int(far_n),
                "bytes_written_per_launch": far_bytes,
                "write_gbs": far_bytes / far_avg / 1e9,
                "share_of_kernel_time": ms["far"] / max(total_ms, 1e-9),
                "measured": "CUDA events on the operator's stream around each far-kernel launch, in the same "
                            "repetition of the K timed steps"}
    if ms["far"] >= ms[hbm_kind]:
        roof, roof2 = roof_far, roof_gemv
    else:
        roof, roof2 = roof_gemv, roof_far
    roof["dominant_kernel_class"] = dominant
    assembly = {"far_kernel_ms": far_avg * 1e3, "far_evals_per_s": evals / far_avg,
                "near_kernel_ms": ms["near"] / max(launches["near"], 1),
                "self_kernel_ms": ms["self"] / max(launches["self"], 1),
                "near_pairs": int(near_pairs),
                "share_of_kernel_time": (ms["far"] + ms["near"] + ms["self"]) / max(total_ms, 1e-9),
                "fp32_fma_rate_tflops": {"scalar": fp32_s.value, "packed": fp32_p.value}}

    cpu = None
    if not a.no_cpu and dist.rank == 0:
        cpu = cpu_baseline(a.level, a.k)
    head = results[head_mode]
    # The FP64 form with the same preconditioner as the headline's (like for like), else plain.
    like = "plain_fp64_bj" if head_mode == "mixed_half_bj" else "plain_fp64"
    line = {
        "metric": METRIC,
        "value": head["value"], "unit": "solves/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("c64 matrix (FP64 phase, near/self, refinement)" if head_mode == "mixed" else
                  "c64 matrix + complex-half (FP16 pair, per-row power-of-two scale) inner copy; FP64 phase, "
                  "near/self, refinement"),
        "data": "synthetic (icosphere geometry, analytic incident plane wave)",
        "config": {"workload": f"rigid sphere icosphere L{a.level} (N={n}), k={a.k}, beta=i/k, plane wave +z; "
                               f"one step = assembly + RHS + GMRES({RESTART}) inner solve on the "
                               f"{'complex64' if head_mode == 'mixed' else 'complex-half'} matrix with FP32 "
                               f"vectors{' and block-Jacobi right preconditioning' if head_mode == 'mixed_half_bj' else ''}"
                               f" / FP64-refined on the complex64 matrix to rtol {TOL}",
                   "N": n, "l2": "inputs larger than L2 (complex64 matrix %.1f GB)" % (8 * n * n / 1e9),
                   "parallelism": f"replicas x{dist.world}"},
        "headline_mode": head_mode,
        "error_vs_fp64": head["error_vs_fp64"],
        "speedup_vs_plain_fp64": head["value"] / results["plain_fp64"]["value"],
        "speedup_vs_plain_fp64_bj": head["value"] / results["plain_fp64_bj"]["value"],
        "roofline": roof,
        "roofline_second": roof2,
        "gpu_launches": launches_timed,
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": None if cpu is None else {kk: cpu[kk] for kk in ("value", "unit", "cores", "kind", "sample")},
        "modes": results,
        "assembly": assembly,
        "kernel_ms_per_step": {kk: v / a.steps for kk, v in ms.items() if v > 0},
        "sweep": sweep,
        "multi_rhs": multi,
    }
    line.update(extra_legs)
    # Compact summary last (the part of the line that a truncated log tail keeps).
    summ = {"headline": head_mode, "like_for_like": like,
            "ms_per_step": {m: round(r["ms_per_step"], 3) for m, r in results.items()},
            "speedup_vs_plain_fp64": round(line["speedup_vs_plain_fp64"], 3),
            "speedup_vs_plain_fp64_bj": round(line["speedup_vs_plain_fp64_bj"], 3),
            "iterations": {m: r["iterations"] for m, r in results.items()},
            "error_vs_fp64": {m: float("%.3g" % r["error_vs_fp64"]) for m, r in results.items()}}
    if sweep:
        summ["sweep"] = {"value": round(sweep["value"], 2), "form": sweep["inner_form"],
                         "speedup_vs_plain_fp64": round(sweep["speedup_vs_plain_fp64"], 3),
                         "speedup_vs_plain_fp64_bj": round(sweep["speedup_vs_plain_fp64_bj"], 3),
                         "max_error_vs_fp64": float("%.3g" % sweep["max_error_vs_fp64"])}
    if multi:
        summ["multi_rhs"] = {"rhs_solves_per_s": round(multi["rhs_solves_per_s"], 1),
                             "speedup_vs_plain_fp64": round(multi["speedup_vs_plain_fp64"], 2),
                             "tensor_frac": round(multi["tensor_kernel"]["frac"], 3)}
    summ["roofline_frac"] = {"gemv_hbm": round(roof_gemv["frac"], 3), "far32_fp32": round(roof_far["frac"], 3)}
    summ["far32_ms"] = round(far_avg * 1e3, 3)
    if cpu is not None:
        summ["cpu_solves_per_s"] = float("%.4g" % cpu["value"])
    pf = extra_legs.get("precision_form") or {}
    if "mixed_error_vs_fp64" in pf:
        summ["precision_form"] = {"mixed_error_vs_fp64": float("%.3g" % pf["mixed_error_vs_fp64"]),
                                  "mie_fp64": float("%.4g" % pf["mie_surface_error"]["fp64"]),
                                  "mie_mixed": float("%.4g" % pf["mie_surface_error"]["mixed"]),
                                  "solve_speedup": round(pf["solve_speedup"], 2)}
    rg = extra_legs.get("reference_gpu_assembly") or {}
    if "N1280_k2_all_pairs" in rg:
        summ["reference_gpu_assembly_speedup_per_pair"] = {
            kk: round(rg[kk]["speedup_per_pair"], 1) for kk in ("N1280_k2_all_pairs", "N20480_k10_rows0_128") if kk in rg}
    gb = extra_legs.get("gemv_bar") or {}
    if "c64" in gb:
        summ["gemv_vs_cublas"] = {kk: round(gb[kk]["ours_over_cublas"], 3) for kk in ("c64", "c128")}
    line["summary"] = summ
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    rt.cudaFree(b_d)
    rt.cudaFree(x_d)
    dist.close()


def gemv_bar_leg(sb, L, lib, dev, rt, reps=20):
    """The matrix-vector products against cuBLAS on the same device (the reference's backend calls
    cublasCgemv / cublasZgemv, crates/sonium-compute/src/cuda/cublas_blas23.rs:126,165): at the
    config-2 size (N = 20480), torch.mv on random complex64 / complex128 device matrices (cuBLAS)
    and this library's product on the assembled complex64 / complex128 operators of the headline
    mesh (sb_operator_apply_device, complex128 vectors), each timed over back-to-back calls between
    CUDA events after warm-up; matrix bytes per product over the time, against the measured HBM
    copy bandwidth."""
    import torch

    n = 20 * 4 ** LEVEL
    pk, pk_kind = peaks()
    out = {"n": n, "peak_gbs": pk["hbm_gbs"], "peak_source": pk_kind}
    torch.cuda.set_device(dev)
    for key, dt in (("c64", torch.complex64), ("c128", torch.complex128)):
        A = torch.randn(n, n, dtype=dt, device=f"cuda:{dev}")
        x = torch.randn(n, dtype=dt, device=f"cuda:{dev}")
        for _ in range(3):
            y = torch.mv(A, x)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            y = torch.mv(A, x)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        nbytes = A.element_size() * n * n
        out[key] = {"cublas_ms": ms, "cublas_gbs": nbytes / ms / 1e6}
        del A, x, y
        torch.cuda.empty_cache()
    nodes, tris = sb.icosphere(RADIUS, LEVEL)
    mesh = sb.Mesh(nodes, tris, device=dev)
    ph = sb.PhysicsParams.for_wavenumber(K)
    beta = ph.burton_miller_beta()
    xv = np.ascontiguousarray(np.exp(1j * np.arange(n) * 0.37))
    x_d, y_d = _dev_alloc(rt, xv.nbytes), _dev_alloc(rt, xv.nbytes)
    rt.cudaMemcpy(x_d, xv.ctypes.data, xv.nbytes, 1)
    e0, e1 = ct.c_void_p(), ct.c_void_p()
    L.check(lib.sb_event_create(ct.byref(e0)))
    L.check(lib.sb_event_create(ct.byref(e1)))
    for key, prec, esize in (("c64", sb.SB_PRECISION_FP32, 8), ("c128", sb.SB_PRECISION_FP64, 16)):
        op = sb.build_tbem_system_with_beta(mesh, ph, beta, prec)
        for _ in range(3):
            L.check(lib.sb_operator_apply_device(op.handle, 0, x_d, y_d))
        L.check(lib.sb_event_record(e0, op.handle))
        for _ in range(reps):
            L.check(lib.sb_operator_apply_device(op.handle, 0, x_d, y_d))
        L.check(lib.sb_event_record(e1, op.handle))
        ems = ct.c_float()
        L.check(lib.sb_event_elapsed_ms(e0, e1, ct.byref(ems)))
        ms = ems.value / reps
        gbs = esize * n * n / ms / 1e6
        out[key].update({"ours_ms": ms, "ours_gbs": gbs, "ours_over_cublas": out[key]["cublas_ms"] / ms,
                         "ours_frac": gbs / pk["hbm_gbs"], "cublas_frac": out[key]["cublas_gbs"] / pk["hbm_gbs"]})
        op.close()
    lib.sb_event_destroy(e0)
    lib.sb_event_destroy(e1)
    rt.cudaFree(x_d)
    rt.cudaFree(y_d)
    mesh.close()
    return out


def reference_gpu_leg(sb, L, lib, dev):
    """Baseline leg: the reference's CUDA assembly kernel on the same B200.

    The reference's GPU path (tbem.rs:5165-5405) builds a quadrature chart per pair on the host
    and integrates every pair with its kernel sonium_bem_quadrature_pair_c64 (bem_kernels.cu:
    839-967), one thread per pair, 128 threads per block. That kernel, compiled from the reference's
    source (oracle/_ref/), is timed here on the oracle's restatement of those charts (inputs
    resident on the device, kernel time by CUDA events, best of a few launches) against this
    library's FP64 assembly of the same system (far tiles + near-pair replay + self terms, device
    time of sb_assemble_into). The small configuration (N = 1280, k = 2) runs in full; at N = 20480
    the charts of all pairs would take 0.5 TB, so the reference kernel runs on the first 128 rows
    (2.6 M pairs) and the per-pair rates are compared."""
    from oracle import oracle as O
    from oracle import ref_kernels as RK

    try:
        if RK.build() is None:
            return {"unavailable": "oracle/_ref/bem_kernels.cubin is missing (built where the reference tree is)"}
        kern = RK.RefPairKernel(dev)
        out = {"kernel": "sonium_bem_quadrature_pair_c64 (reference source, compiled unchanged for compute_100)",
               "timing": "kernel only, charts resident on the device, CUDA events, best of the launches"}
        for name, level, k, rows in (("N1280_k2_all_pairs", 3, 2.0, None), ("N20480_k10_rows0_128", 5, 10.0, (0, 128))):
            nodes, tris = O.icosphere(RADIUS, level)
            n = tris.shape[0]
            t0 = time.perf_counter()
            pairs, samples = O.chart(nodes, tris, k, rows=rows)
            t_chart = time.perf_counter() - t0
            kern.run(pairs, samples, k, 1.0, reps=1)  # warm-up
            ms_ref = min(kern.run(pairs, samples, k, 1.0, reps=1)[1] for _ in range(3))
            npairs = pairs.shape[0]
            nsamp = samples.shape[0]
            del pairs, samples
            mesh = sb.Mesh(nodes, tris, device=dev)
            ph = sb.PhysicsParams.for_wavenumber(k)
            beta = ph.burton_miller_beta()
            op = sb.build_tbem_system_with_beta(mesh, ph, beta)
            ours = []
            for _ in range(3):
                op.reassemble(ph, beta)
                ours.append(op.info().assembly_ms)
            ms_ours = min(ours)
            op.close()
            mesh.close()
            ref_per_pair = ms_ref / npairs
            ours_per_pair = ms_ours / (n * n)
            out[name] = {"N": n, "k": k, "pairs": int(npairs), "samples": int(nsamp),
                         "reference_kernel_ms": ms_ref, "reference_host_chart_s": t_chart,
                         "ours_fp64_assembly_ms": ms_ours,
                         "ns_per_pair": {"reference": 1e6 * ref_per_pair, "ours": 1e6 * ours_per_pair},
                         "speedup_per_pair": ref_per_pair / ours_per_pair,
                         "scope": ("all pairs" if rows is None else f"reference on rows {rows[0]}-{rows[1]} of {n} "
                                   "(per-pair rate), ours on the whole matrix")}
        return out
    except Exception as e:  # a baseline leg never fails the bench line
        return {"unavailable": f"{type(e).__name__}: {e}"}


def sweep_leg(sb, a, dist, dev, rt):
    """Batched frequency sweep: 64 instances, ka log-spaced 1 -> 32 on the (1, 0.6, 0.4) ellipsoid,
    icosphere level per instance for >= 8 elements per wavelength (levels 2-5), plane wave +z.

    One step = batched assembly of all 64 complex64 matrices (the form the autotuner chose on the
    first, untimed step), the incident right-hand sides, and the batched mixed GMRES to rtol 1e-8
    (FP64 refinement on the complex64 matrices around FP32-vector inner solves). Three forms of
    the inner solves are timed: products on the complex64 matrices (inner tolerance 1e-5), on
    complex-half copies built inside each solve (inner tolerance 1e-3), and the latter with the
    block-Jacobi right preconditioner (blocks of 64, inverted inside each solve); `value` is the
    fastest form whose solutions are all within 1e-5 of the FP64 ones. Baseline: the same 64 instances solved one
    after another in plain FP64 (complex128 assembly re-done into one operator per mesh level,
    FP64 GMRES(50) to 1e-8), timed once. Wall clock around device-synchronised work on both sides;
    the per-instance error of the batched solution against the FP64 one is reported as its
    maximum."""
    from sonium_b200.sweep import SweepBatch, build_ellipsoid_sweep, ellipsoid_sweep_plan

    from sonium_b200 import shard

    plan = ellipsoid_sweep_plan(count=a.sweep_count)
    # With several ranks each solves its share of the instances (balanced by N^2, no exchange
    # until the end); the whole job's rate is all instances over the slowest rank's time.
    levels_all = [p[2] for p in plan]
    mine = shard.partition_by_cost(shard.dense_solve_costs([20 * 4 ** lv for lv in levels_all]),
                                   dist.world)[dist.rank]
    plan_all, plan = plan, [plan[i] for i in mine]
    meshes, physics, betas = build_ellipsoid_sweep(plan, device=dev)
    sizes = [m.num_elements for m in meshes]
    cfg = sb.IrConfig(20, TOL, RESTART, 20, 1e-5)
    cfg16 = sb.IrConfig(20, TOL, RESTART, 20, HALF_INNER_TOL)
    batch = SweepBatch(meshes, physics, betas)

    def wall(fn):
        rt.cudaDeviceSynchronize()
        dist.barrier()
        t0 = time.perf_counter()
        out = fn()
        rt.cudaDeviceSynchronize()
        dt = time.perf_counter() - t0
        dist.barrier()
        return dist.max(dt), out

    # Two forms of the batched inner products: the complex64 matrices, and their complex-half
    # copies (built inside each solve, after each assembly).
    forms = {}
    for form_name, inner, bj, cfg_f in (("fp32_inner", sb.SB_INNER_FP32, False, cfg),
                                        ("half_inner", sb.SB_INNER_FP16, False, cfg16),
                                        ("half_inner_bj", sb.SB_INNER_FP16, True, cfg16)):
        batch.set_inner_precision(inner)
        batch.set_inner_preconditioner(sb.SB_INNER_PRECOND_BLOCK_JACOBI if bj else sb.SB_INNER_PRECOND_NONE,
                                       BJ_BLOCK_SWEEP)

        def step():
            batch.assemble()
            batch.set_rhs_plane_wave([0.0, 0.0, 1.0])
            return batch.solve(cfg_f)

        st0 = step()
        xb = [batch.solution(i) for i in range(len(batch))]
        for _ in range(a.warmup):
            step()
        t_batch, _ = wall(lambda: [step() for _ in range(a.steps)])
        asm_ms, solve_ms = batch.timings()  # the last timed step
        forms[form_name] = {"t": t_batch, "st0": st0, "xb": xb, "assembly_ms": asm_ms, "solve_ms": solve_ms}
    form, tune_p, tune_s = batch.assembly_tuning()
    split, layout_ms = batch.assembly_split()
    batch.close()
    # plain FP64 baseline, one instance after another; and the same with the sweep's block-Jacobi
    # right preconditioner (blocks of BJ_BLOCK_SWEEP, as the half_inner_bj form)
    ops = {}

    def fp64_sweep(bj=False):
        out = []
        for m, ph, be in zip(meshes, physics, betas):
            key = id(m)
            if key not in ops:
                ops[key] = sb.build_tbem_system_with_beta(m, ph, be)
            else:
                ops[key].reassemble(ph, be)
            b = sb.rhs_plane_wave(m, ph, be, [[0.0, 0.0, 1.0]])[:, 0]
            pre = sb.BlockJacobiPreconditioner(ops[key], BJ_BLOCK_SWEEP) if bj else None
            out.append(sb.gmres(ops[key], b, sb.GmresConfig(100, RESTART, TOL), preconditioner=pre))
        return out

    fp64_sweep()  # warm-up: allocations, graphs
    t_fp64, sols = wall(fp64_sweep)
    fp64_sweep(True)
    t_fp64_bj, sols_bj = wall(lambda: fp64_sweep(True))
    fp64_iters = [int(s.iterations) for s in sols]
    fp64_bj_iters = [int(s.iterations) for s in sols_bj]
    bj_err = dist.max(max(float(np.linalg.norm(sb_.x - s.x) / np.linalg.norm(s.x)) for sb_, s in zip(sols_bj, sols)))
    for f in forms.values():
        f["errs"] = [float(np.linalg.norm(f["xb"][i] - s.x) / np.linalg.norm(s.x)) for i, s in enumerate(sols)]
        f["max_err"] = dist.max(max(f["errs"]))  # over every rank's instances
        f["value"] = len(plan_all) * a.steps / f["t"]
    for o in ops.values():
        o.close()
    plain = len(plan_all) / t_fp64
    plain_bj = len(plan_all) / t_fp64_bj
    # the fastest form within the metric's 1e-5 of the FP64 solutions
    ok = [k for k, f in forms.items() if f["max_err"] <= 1e-5]
    best = max(ok, key=lambda k: forms[k]["value"]) if ok else "fp32_inner"
    fb = forms[best]
    batched, t_batch, st0, errs = fb["value"], fb["t"], fb["st0"], fb["errs"]
    asm_ms, solve_ms = fb["assembly_ms"], fb["solve_ms"]
    levels = levels_all
    return {
        "workload": (f"{len(plan_all)} instances, ka log-spaced {plan_all[0][0]:g} -> {plan_all[-1][0]:g} on the ellipsoid "
                     "(1, 0.6, 0.4), icosphere level per instance for >= 8 elements per wavelength "
                     f"(levels {min(levels)}-{max(levels)}: " +
                     ", ".join(f"L{lv} x{levels.count(lv)}" for lv in sorted(set(levels))) +
                     f"), plane wave +z, rtol {TOL}"),
        "value": batched, "unit": "solves/s", "ms_per_step": 1e3 * t_batch / a.steps,
        "plain_fp64": plain, "plain_fp64_ms_per_sweep": 1e3 * t_fp64,
        "speedup_vs_plain_fp64": batched / plain,
        "plain_fp64_bj": plain_bj, "plain_fp64_bj_ms_per_sweep": 1e3 * t_fp64_bj,
        "speedup_vs_plain_fp64_bj": batched / plain_bj,
        "plain_fp64_bj_max_error_vs_fp64": bj_err,
        "max_error_vs_fp64": fb["max_err"], "median_error_vs_fp64_this_rank": float(np.median(errs)),
        "all_converged": bool(all(s.converged for s in st0)),
        "max_residual": float(max(s.residual for s in st0)),
        "matrix_gb_c64": float(sum(8.0 * n * n for n in sizes) / 1e9),
        "assembly_ms": asm_ms, "solve_ms": solve_ms,
        "assembly_form": {1: "persistent", 2: "streams"}.get(form, str(form)),
        "assembly_autotune_ms": {"persistent": tune_p, "streams": tune_s},
        "assembly_persistent_layout": {"far_slots_per_sm": split, "autotune_ms": layout_ms},
        "iterations_total": {"batched": int(sum(s.iterations for s in st0)), "fp64": int(sum(fp64_iters)),
                             "fp64_bj": int(sum(fp64_bj_iters))},
        "inner_form": best,
        "forms": {k: {"value": f["value"], "ms_per_step": 1e3 * f["t"] / a.steps, "assembly_ms": f["assembly_ms"],
                      "solve_ms": f["solve_ms"], "max_error_vs_fp64": f["max_err"],
                      "speedup_vs_plain_fp64": f["value"] / plain,
                      "speedup_vs_plain_fp64_bj": f["value"] / plain_bj,
                      "inner_tolerance": cfg.inner_tolerance if k == "fp32_inner" else cfg16.inner_tolerance,
                      "block_jacobi": BJ_BLOCK_SWEEP if k == "half_inner_bj" else None,
                      "iterations_total": int(sum(s.iterations for s in f["st0"]))}
                  for k, f in forms.items()},
        "timing": "wall clock around device-synchronised steps, max over ranks",
        "ranks": dist.world,
        "scaling": "strong: the instances are shared out over the ranks (balanced by N^2), solutions gathered "
                   "at the end" if dist.world > 1 else "one rank",
        "instances_this_rank": len(plan),
    }


def multi_rhs_leg(sb, a, dist, dev, rt):
    """Multi-RHS tensor-core form: ellipsoid (1, 0.6, 0.4) icosphere level 5 (N = 20480; --level
    changes it), k = 16, 256 plane waves along Fibonacci-sphere directions, complex128 assembly.

    A step = one sb_gmres_multi_device solve of all 256 right-hand sides (device-resident b and x):
    FP32-inner GMRES(50) with every step's 256 products as one tensor-core block product (BF16
    hi/lo split, FP32 accumulation) and FP64 refinement to rtol 1e-8 by one integer-slice block
    residual (INT8 tensor cores, FP64-grade) per refinement. Device time from the solver (CUDA
    events on its stream). Baseline: plain FP64 GMRES(50) to 1e-8, one right-hand side after another, timed on a sample of 16 directions and
    reported per right-hand side; the error of the multi-RHS solutions against those FP64 solutions."""
    from sonium_b200 import _lib as L

    level, k, r = a.level, 16.0, a.rhs
    nodes, tris = sb.icosphere(RADIUS, level, (1.0, 0.6, 0.4))
    n = tris.shape[0]
    mesh = sb.Mesh(nodes, tris, device=dev)
    ph = sb.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    op = sb.build_tbem_system_with_beta(mesh, ph, beta, sb.SB_PRECISION_FP64)
    B = sb.rhs_plane_wave(mesh, ph, beta, sb.fibonacci_sphere_directions(r))  # n x r
    # With several ranks each solves its groups of 128 right-hand sides (no exchange); the whole
    # job's rate is all right-hand sides over the slowest rank's time.
    from sonium_b200 import shard

    r_total = r
    cols = [c for start, stop in shard.rhs_groups(r, dist.world)[dist.rank] for c in range(start, stop)]
    B = np.ascontiguousarray(B[:, cols])
    r = len(cols)
    lib = L.load()
    bt = np.ascontiguousarray(B.T)  # right-hand-side-major
    b_d = _dev_alloc(rt, bt.nbytes)
    x_d = _dev_alloc(rt, bt.nbytes)
    if rt.cudaMemcpy(b_d, bt.ctypes.data, bt.nbytes, 1) != 0:
        raise RuntimeError("cudaMemcpy failed")
    ir = L.SbIrConfig(20, TOL, RESTART, 20, 1e-5)
    stats = (L.SbGmresStats * r)()

    def solve():
        L.check(lib.sb_gmres_multi_device(op.handle, b_d, r, ct.byref(ir), x_d, ct.cast(stats, ct.c_void_p)))
        return stats[0].device_ms

    solve()
    X = np.zeros((r, n), np.complex128)
    rt.cudaDeviceSynchronize()
    rt.cudaMemcpy(X.ctypes.data, x_d, X.nbytes, 2)
    first = [L.SbGmresStats.from_buffer_copy(stats[i]) for i in range(r)]
    for _ in range(a.warmup):
        solve()
    times = [solve() for _ in range(a.steps)]
    t_block = dist.max(float(np.median(times)) / 1e3)
    # The block product alone, for its roofline: K launches on the operator's stream between two
    # CUDA events (all 256 right-hand sides, inputs resident, split planes 3.4 GB > L2).
    x32 = np.ascontiguousarray(bt.astype(np.complex64))
    x32_d = _dev_alloc(rt, x32.nbytes)
    y32_d = _dev_alloc(rt, x32.nbytes)
    rt.cudaMemcpy(x32_d, x32.ctypes.data, x32.nbytes, 1)
    for _ in range(2):
        L.check(lib.sb_operator_apply_block_tensor_device(op.handle, x32_d, y32_d, r))
    e0, e1 = ct.c_void_p(), ct.c_void_p()
    L.check(lib.sb_event_create(ct.byref(e0)))
    L.check(lib.sb_event_create(ct.byref(e1)))
    reps = max(a.steps, 3) * 4
    L.check(lib.sb_event_record(e0, op.handle))
    for _ in range(reps):
        L.check(lib.sb_operator_apply_block_tensor_device(op.handle, x32_d, y32_d, r))
    L.check(lib.sb_event_record(e1, op.handle))
    ems = ct.c_float()
    L.check(lib.sb_event_elapsed_ms(e0, e1, ct.byref(ems)))
    rt.cudaFree(x32_d)
    rt.cudaFree(y32_d)
    live = (ems.value / reps, reps)
    # The FP64-grade block residual alone (integer slices on the INT8 tensor cores), for its
    # roofline: the same event bracket around back-to-back residuals of all right-hand sides.
    res_d = _dev_alloc(rt, bt.nbytes)
    for _ in range(2):
        L.check(lib.sb_operator_block_residual_device(op.handle, b_d, x_d, r, res_d))
    rreps = max(a.steps, 3) * 2
    L.check(lib.sb_event_record(e0, op.handle))
    for _ in range(rreps):
        L.check(lib.sb_operator_block_residual_device(op.handle, b_d, x_d, r, res_d))
    L.check(lib.sb_event_record(e1, op.handle))
    L.check(lib.sb_event_elapsed_ms(e0, e1, ct.byref(ems)))
    R = np.zeros((r, n), np.complex128)
    Xr = np.zeros((r, n), np.complex128)
    rt.cudaMemcpy(R.ctypes.data, res_d, R.nbytes, 2)
    rt.cudaMemcpy(Xr.ctypes.data, x_d, Xr.nbytes, 2)
    rt.cudaFree(res_d)
    live_res = (ems.value / rreps, rreps, R, Xr)
    lib.sb_event_destroy(e0)
    lib.sb_event_destroy(e1)
    # all kernel classes from a separate profiled pass (their event pairs stay out of the timed solves)
    prof = L.SbProfile()
    L.check(lib.sb_profile_enable(1))
    for _ in range(a.steps):
        solve()
    L.check(lib.sb_profile_enable(0))
    L.check(lib.sb_profile_read(ct.byref(prof), 1))
    out = multi_rhs_report(sb, L, a, op, mesh, B, X, first, prof, live, t_block, rt, b_d, x_d, n, r, level, k,
                           live_res)
    out["rhs_solves_per_s"] = r_total / t_block
    out["speedup_vs_plain_fp64"] = out["rhs_solves_per_s"] / out["plain_fp64_rhs_solves_per_s"]
    out["ranks"] = dist.world
    out["rhs_this_rank"] = r
    if dist.world > 1:
        out["scaling"] = "strong: groups of 128 right-hand sides shared out over the ranks"
    return out


def multi_rhs_report(sb, L, a, op, mesh, B, X, first, prof, live, t_block, rt, b_d, x_d, n, r, level, k,
                     live_res):
    """FP64 baseline on a sample of right-hand sides and the tensor-kernel rooflines of the leg."""
    sample = list(range(0, r, max(1, r // 16)))[:16]
    # the block residual of the solutions against numpy's FP64 residual on the same sample
    A = op.matrix
    absA = np.abs(A)
    res_err = 0.0
    for c in sample:
        xr = live_res[3][c]
        ref = B[:, c] - A @ xr
        scale = absA @ np.abs(xr) + np.abs(B[:, c])
        res_err = max(res_err, float(np.max(np.abs(live_res[2][c] - ref) / scale)))
    del A, absA
    gc = sb.GmresConfig(100, RESTART, TOL)
    rt.cudaDeviceSynchronize()
    t0 = time.perf_counter()
    errs, it64 = [], []
    for c in sample:
        s = sb.gmres(op, B[:, c], gc)
        errs.append(float(np.linalg.norm(X[c] - s.x) / np.linalg.norm(s.x)))
        it64.append(int(s.iterations))
    rt.cudaDeviceSynchronize()
    t64 = (time.perf_counter() - t0) / len(sample)
    rt.cudaFree(b_d)
    rt.cudaFree(x_d)
    op.close()
    mesh.close()
    pk, pk_kind = peaks()
    names = L.PROF_NAMES
    ms = {names[i]: prof.ms[i] for i in range(L.SB_PROF_KINDS)}
    launches = {names[i]: prof.launches[i] for i in range(L.SB_PROF_KINDS)}
    tl = launches["tensor"]
    avg = live[0] / 1e3
    executed = 24.0 * n * n * 128 * ((r + 127) // 128)  # 3 BF16 terms x real GEMM (2N x 2R x N)
    algorithmic = 8.0 * n * n * r                         # complex flops of A X
    achieved = executed / max(avg, 1e-12) / 1e12
    return {
        "workload": f"ellipsoid (1, 0.6, 0.4) icosphere L{level} (N={n}), k={k}, {r} plane waves on "
                    f"Fibonacci-sphere directions, complex128 assembly, rtol {TOL}",
        "rhs_solves_per_s": r / t_block, "block_solve_ms": 1e3 * t_block,
        "plain_fp64_rhs_solves_per_s": 1.0 / t64, "plain_fp64_ms_per_rhs": 1e3 * t64,
        "speedup_vs_plain_fp64": (r / t_block) * t64,
        "max_error_vs_fp64": max(errs), "error_sample": len(sample),
        "all_converged": bool(all(s.converged for s in first)),
        "max_residual": float(max(s.residual for s in first)),
        "iterations_median": float(np.median([s.iterations for s in first])),
        "refinements_median": float(np.median([s.refinements for s in first])),
        "fp64_iterations_median": float(np.median(it64)),
        "tensor_kernel": {"kernel": "k_block_bf16x3 (tcgen05 BF16 hi/lo split, TMA, TMEM)",
                          "launches_per_solve": tl / max(a.steps, 1), "avg_launch_ms": avg * 1e3,
                          "measured": f"{live[1]} back-to-back block products of all {r} right-hand sides "
                                      "between CUDA events on the operator's stream",
                          "bound": "tensor", "achieved": achieved, "unit": "TFLOP/s",
                          "peak": pk["bf16_tflops"], "frac": achieved / pk["bf16_tflops"],
                          "peak_source": pk_kind, "executed_flop_per_launch": executed,
                          "algorithmic_complex_flop_per_launch": algorithmic,
                          "share_of_kernel_time": ms["tensor"] / max(sum(ms.values()), 1e-9)},
        "residual_kernel": residual_roofline(n, r, live_res, pk, pk_kind, ms, launches, a.steps, res_err),
        "gram_schmidt_kernels": gram_schmidt_roofline(n, first, ms["arnoldi"] / max(a.steps, 1), pk, pk_kind),
        "kernel_ms_per_solve": {kk: v / max(a.steps, 1) for kk, v in ms.items() if v > 0},
    }


def gram_schmidt_roofline(n, stats, ms_per_solve, pk, pk_kind):
    """Roofline of the many-right-hand-side Gram-Schmidt (k_bdots, k_bproject and their small
    reductions, the `arnoldi` kernel class). Algorithmic bytes per right-hand side and Arnoldi step
    with k basis vectors: two classical Gram-Schmidt passes (the DGKS second pass, which these
    solves take at every step), each reading the k complex64 basis vectors twice (dots, projection)
    plus w three times (8 bytes per entry): 2 (2 k + 3) 8 n. A right-hand side's inner iterations
    are split evenly over its refinements (k counts from 1 in every inner solve)."""
    total = 0.0
    for st in stats:
        solves = max(int(st.refinements), 1)
        its = int(st.iterations)
        for q in range(solves):
            steps = its // solves + (1 if q < its % solves else 0)
            total += sum(2.0 * (2 * k + 3) * 8.0 * n for k in range(1, steps + 1))
    achieved = total / max(ms_per_solve / 1e3, 1e-12) / 1e9
    return {"kernels": "k_bdots + k_bproject (+ k_breduce, k_bsum_partials, k_bnext, Givens / control)",
            "bound": "hbm", "algorithmic_bytes_per_solve": total, "ms_per_solve": ms_per_solve,
            "achieved": achieved, "unit": "GB/s", "peak": pk["hbm_gbs"], "frac": achieved / pk["hbm_gbs"],
            "peak_source": pk_kind}


OZAKI_PRODUCTS = 36  # slice products of the block residual: diagonals 2..9 of 8 x 8 INT8 slices


def residual_roofline(n, r, live_res, pk, pk_kind, ms, launches, steps, res_err):
    """Roofline of the integer-slice block residual (k_ozaki_residual with its slicing and combine
    kernels): INT8 tensor work = 36 slice products of the real 2N x 2R x N GEMM per launch; peak =
    2 x the measured BF16 GEMM rate (the INT8 tensor rate per SM and clock is twice the BF16 one)."""
    avg_s = live_res[0] / 1e3
    ops = OZAKI_PRODUCTS * 2.0 * (2 * n) * (2 * r) * n
    achieved = ops / max(avg_s, 1e-12) / 1e12
    peak = 2.0 * pk["bf16_tflops"]
    return {"kernel": "k_ozaki_residual (tcgen05 kind::i8, 8 INT8 slices, 36 products, TMA, TMEM) + slicing + combine",
            "avg_launch_ms": live_res[0], "measured": f"{live_res[1]} back-to-back residuals of all {r} right-hand "
                                                      "sides between CUDA events on the operator's stream",
            "bound": "tensor", "achieved": achieved, "unit": "TOP/s (INT8)", "peak": peak,
            "frac": achieved / peak, "peak_source": f"2 x {pk_kind} bf16 GEMM", "int8_ops_per_launch": ops,
            "fp64_equivalent_tflops": 8.0 * n * n * r / max(avg_s, 1e-12) / 1e12,
            "launches_per_solve": launches["residual"] / max(steps, 1),
            "share_of_kernel_time": ms["residual"] / max(sum(ms.values()), 1e-9),
            "max_error_vs_numpy_fp64": res_err}


def precision_leg(sb, a, dist, dev, rt, reps=None):
    """Precision form: rigid sphere, icosphere level 6 (N = 81920), k = 40, plane wave +z.

    The complex128 matrix (107 GB) and its complex64 copy (54 GB) come from one assembly; a step
    solves to rtol 1e-10 once in plain FP64 GMRES(50) and once with FP32-inner GMRES(50) to 1e-5 and
    FP64 refinement on the complex128 matrix. Device times from the solver statistics (CUDA events
    on the operator's stream); error of the mixed solution against the FP64 one, and both
    solutions' surface error against the Mie series (mie_surface_error)."""
    reps = a.steps if reps is None else reps
    from sonium_b200 import _lib as L

    level, k = 6, 40.0
    import gc

    gc.collect()
    L.check(L.load().sb_memory_trim(-1))  # cached blocks of the other legs back to the driver
    free, total = ct.c_size_t(), ct.c_size_t()
    rt.cudaMemGetInfo.argtypes = [ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_size_t)]
    rt.cudaMemGetInfo(ct.byref(free), ct.byref(total))
    if free.value < 170e9:
        return {"unavailable": f"needs ~170 GB of free device memory, {free.value / 1e9:.1f} GB free"}
    nodes, tris = sb.icosphere(RADIUS, level)
    n = tris.shape[0]
    mesh = sb.Mesh(nodes, tris, device=dev)
    ph = sb.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    op = sb.build_tbem_system_with_beta(mesh, ph, beta, sb.SB_PRECISION_FP64_FP32)
    asm_ms = op.info().assembly_ms
    b = sb.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    gc = sb.GmresConfig(max_iterations=400, restart=RESTART, tolerance=1e-10)
    ir = sb.IrConfig(max_refinements=20, tolerance=1e-10, inner_restart=RESTART, inner_max_iterations=40,
                     inner_tolerance=1e-5)
    t64, tmix = [], []
    s64 = mix = None
    for i in range(max(1, reps)):
        s64 = sb.gmres(op, b, gc)
        mix = sb.gmres_mixed(op, b, ir)
        t64.append(s64.device_ms)
        tmix.append(mix.device_ms)
    c, _, areas = mesh.element_geometry()
    op.close()
    mesh.close()
    L.check(L.load().sb_memory_trim(-1))
    err = float(np.linalg.norm(mix.x - s64.x) / np.linalg.norm(s64.x))
    e64 = mie_surface_error(s64.x, c, areas, k, RADIUS)
    emix = mie_surface_error(mix.x, c, areas, k, RADIUS)
    return {
        "workload": f"rigid sphere icosphere L{level} (N={n}), k={k}, complex128 + complex64 matrices "
                    f"({16 * n * n / 1e9:.0f} + {8 * n * n / 1e9:.0f} GB), rtol 1e-10",
        "mie_surface_error": {"fp64": e64, "mixed": emix, "difference": abs(emix - e64)},
        "assembly_ms": asm_ms,
        "fp64_solve_ms": float(np.median(t64)), "mixed_solve_ms": float(np.median(tmix)),
        "solve_speedup": float(np.median(t64) / np.median(tmix)),
        "fp64": {"iterations": s64.iterations, "matvecs": s64.matvecs, "residual": s64.residual},
        "mixed": {"iterations": mix.iterations, "matvecs": mix.matvecs, "matvecs_fp32": mix.matvecs_fp32,
                  "refinements": mix.refinements, "residual": mix.residual},
        "mixed_error_vs_fp64": err,
    }


def single_solves(sb, level, k, dev, modes=None):
    """One solve per precision mode, untimed: the small case the ncu captures profile."""
    nodes, tris = sb.icosphere(RADIUS, level)
    ph = sb.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    mesh = sb.Mesh(nodes, tris, device=dev)
    b = sb.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    for name in (modes or ("mixed", "mixed_half", "mixed_half_bj", "plain_fp64")):
        prec, solver = MODES[name]
        op = sb.build_tbem_system_with_beta(mesh, ph, beta, getattr(sb, prec))
        if solver in ("ir16", "ir16bj"):
            op.set_inner_precision(sb.SB_INNER_FP16)
            if solver == "ir16bj":
                op.set_inner_preconditioner(sb.SB_INNER_PRECOND_BLOCK_JACOBI, BJ_BLOCK)
            s = sb.gmres_mixed(op, b, sb.IrConfig(20, TOL, RESTART, 20, HALF_INNER_TOL))
        elif solver == "ir":
            s = sb.gmres_mixed(op, b, sb.IrConfig(20, TOL, RESTART, 20, 1e-5))
        else:
            pre = sb.BlockJacobiPreconditioner(op, BJ_BLOCK) if solver == "fp64bj" else None
            s = sb.gmres(op, b, sb.GmresConfig(100, RESTART, TOL), preconditioner=pre)
        print(f"{name}: N={tris.shape[0]} iterations {s.iterations} matvecs {s.matvecs} residual {s.residual:.2e}")
        op.close()


def _cudart():
    for name in ("libcudart.so.12", "libcudart.so", "/usr/local/cuda/lib64/libcudart.so.12"):
        try:
            rt = ct.CDLL(name)
            break
        except OSError:
            continue
    else:
        raise RuntimeError("libcudart not found")
    rt.cudaMalloc.argtypes = [ct.POINTER(ct.c_void_p), ct.c_size_t]
    rt.cudaFree.argtypes = [ct.c_void_p]
    rt.cudaMemcpy.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_size_t, ct.c_int]
    return rt


def _dev_alloc(rt, nbytes):
    p = ct.c_void_p()
    if rt.cudaMalloc(ct.byref(p), nbytes) != 0:
        raise RuntimeError("cudaMalloc failed")
    return p


def _to_host(rt, p, n):
    out = np.zeros(n, np.complex128)
    rt.cudaDeviceSynchronize()
    if rt.cudaMemcpy(out.ctypes.data, p, 16 * n, 2) != 0:
        raise RuntimeError("cudaMemcpy failed")
    return out


if __name__ == "__main__":
    main()
