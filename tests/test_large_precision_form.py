"""Precision form at full size: rigid sphere, icosphere level 6 (N = 81920), k = 40.

The complex128 matrix (107 GB) and its complex64 copy (54 GB) are assembled by one epilogue;
the plain FP64 GMRES(50) and the FP32-inner GMRES(50) with FP64 refinement both solve to a
1e-10 relative residual. Bars: the mixed solution within 1e-5 (the metric's tolerance) of the
FP64 one, and the same surface error against the Mie series (area-weighted relative L2,
crates/sonium-qa/src/lib.rs:319-358) to 1e-5.

Needs about 165 GB of device memory: it runs whenever the device has that much free (after the
library's cached blocks are returned), which a whole B200 has, and is skipped with that reason
otherwise (SB_LARGE_TESTS=0 skips it always). With SB_LARGE_REPORT=<path> it also writes its
numbers as JSON there.
"""
import ctypes as ct
import gc
import json
import os
import time

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("SB_LARGE_TESTS") == "0", reason="SB_LARGE_TESTS=0")]

NEED_BYTES = 170e9  # complex128 + complex64 matrices at N = 81920 (161 GB) and the solver's vectors


def _free_device_bytes():
    for name in ("libcudart.so.12", "libcudart.so", "/usr/local/cuda/lib64/libcudart.so.12"):
        try:
            rt = ct.CDLL(name)
            break
        except OSError:
            continue
    else:
        return 0
    free, total = ct.c_size_t(), ct.c_size_t()
    if rt.cudaMemGetInfo(ct.byref(free), ct.byref(total)) != 0:
        return 0
    return free.value


def test_precision_form_level6_k40(sb, oracle):
    from sonium_b200 import _lib as L

    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible")
    gc.collect()
    L.check(L.load().sb_memory_trim(-1))  # cached blocks of earlier tests back to the driver
    free = _free_device_bytes()
    if free < NEED_BYTES:
        pytest.skip(f"needs ~{NEED_BYTES / 1e9:.0f} GB of free device memory, {free / 1e9:.1f} GB free")
    k = 40.0
    nodes, tris = oracle.icosphere(1.0, 6)
    mesh = sb.Mesh(nodes, tris)
    ph = sb.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    t0 = time.perf_counter()
    op = sb.build_tbem_system_with_beta(mesh, ph, beta, sb.SB_PRECISION_FP64_FP32)
    t_asm = time.perf_counter() - t0
    b = sb.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
    s64 = sb.gmres(op, b, sb.GmresConfig(max_iterations=400, restart=50, tolerance=1e-10))
    mix = sb.gmres_mixed(op, b, sb.IrConfig(max_refinements=20, tolerance=1e-10, inner_restart=50,
                                            inner_max_iterations=40, inner_tolerance=1e-5))
    assert s64.converged and mix.converged
    err = float(np.linalg.norm(mix.x - s64.x) / np.linalg.norm(s64.x))
    c, _, a = mesh.element_geometry()
    e64 = oracle.rigid_sphere_surface_error(s64.x, c, a, k, 1.0)
    emix = oracle.rigid_sphere_surface_error(mix.x, c, a, k, 1.0)
    report = {
        "N": int(tris.shape[0]), "k": k, "assembly_s_wall": t_asm,
        "fp64": {"iterations": s64.iterations, "matvecs": s64.matvecs, "residual": s64.residual,
                 "device_ms": s64.device_ms, "mie_surface_error": e64},
        "mixed": {"iterations": mix.iterations, "matvecs": mix.matvecs, "matvecs_fp32": mix.matvecs_fp32,
                  "refinements": mix.refinements, "residual": mix.residual, "device_ms": mix.device_ms,
                  "mie_surface_error": emix},
        "mixed_error_vs_fp64": err,
    }
    path = os.environ.get("SB_LARGE_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report))
    op.close()
    mesh.close()
    L.check(L.load().sb_memory_trim(-1))
    assert err < 1e-5
    assert abs(emix - e64) < 1e-5
    assert mix.residual < 1e-10 and s64.residual < 1e-10
