"""CPU tests of the C ABI: symbols, host-side logic and input validation (no GPU needed).

The library must load without a GPU, export every function the header declares, validate its
inputs before touching a device (validate_cuda_tbem_inputs, crates/sonium-bem/src/core/assembly/
tbem.rs:4659-4798) and fail loudly -- never fall back to the CPU -- when no device exists.
"""
import ctypes as ct
import os
import sys

import numpy as np
import pytest

import sonium_b200 as sb
from sonium_b200 import _lib as L


def test_library_exports_every_header_symbol(sb):
    lib = L.load()
    syms = L.header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert missing == []
    # and the binding declares all of them
    assert sorted(L._SIGNATURES) == syms


def test_physics_params_follow_reference(sb, oracle):
    for f, c, rho in [(343.0 / (2 * np.pi), 343.0, 1.21), (1000.0, 340.0, 1.2), (5e3, 1500.0, 1000.0)]:
        p = sb.PhysicsParams.new(f, c, rho)
        o = oracle.physics(f, c, rho)
        for name, _ in L.SbPhysics._fields_:
            assert getattr(p, name) == getattr(o, name), name
        assert p.burton_miller_beta() == oracle.bm_beta(o)
        assert p.burton_miller_beta(0.2) == oracle.bm_beta(o, 0.2)
    pi = sb.PhysicsParams.new(100.0, is_internal=True)
    assert pi.tau == -1.0 and pi.burton_miller_beta() == 0j


@pytest.mark.parametrize("f,c,rho", [(0.0, 343.0, 1.2), (-1.0, 343.0, 1.2), (100.0, float("nan"), 1.2),
                                     (100.0, 343.0, 0.0)])
def test_physics_rejects_invalid_input(sb, f, c, rho):
    with pytest.raises(sb.SoniumError) as e:
        sb.PhysicsParams.new(f, c, rho)
    assert e.value.status == L.SB_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("level", [0, 1, 2, 3, 4])
def test_icosphere_matches_oracle(sb, oracle, level):
    n1, t1 = sb.icosphere(1.0, level)
    n2, t2 = oracle.icosphere(1.0, level)
    assert np.array_equal(n1, n2) and np.array_equal(t1, t2)
    n1, t1 = sb.icosphere(0.5, level, scale=(1.0, 0.6, 0.4))
    n2, t2 = oracle.icosphere(0.5, level, (1.0, 0.6, 0.4))
    assert np.array_equal(n1, n2) and np.array_equal(t1, t2)


def test_icosphere_counts(sb):
    for level, (nn, nt) in {0: (12, 20), 3: (642, 1280), 5: (10242, 20480), 6: (40962, 81920)}.items():
        a, b = ct.c_int64(), ct.c_int64()
        L.check(L.load().sb_icosphere_counts(level, ct.byref(a), ct.byref(b)))
        assert (a.value, b.value) == (nn, nt)


def test_mesh_validation_happens_before_device_work(sb):
    nodes, tris = sb.icosphere(1.0, 1)
    bad = tris.copy()
    bad[3, 1] = 10_000
    with pytest.raises(sb.SoniumError) as e:
        sb.Mesh(nodes, bad)
    assert e.value.status == L.SB_ERR_INVALID_ARGUMENT
    nan_nodes = nodes.copy()
    nan_nodes[2, 0] = np.nan
    with pytest.raises(sb.SoniumError) as e:
        sb.Mesh(nan_nodes, tris)
    assert e.value.status == L.SB_ERR_INVALID_ARGUMENT
    degen = tris.copy()
    degen[5] = [degen[5, 0], degen[5, 0], degen[5, 1]]
    with pytest.raises(sb.SoniumError) as e:
        sb.Mesh(nodes, degen)
    assert e.value.status == L.SB_ERR_UNSUPPORTED_ELEMENT
    with pytest.raises(sb.SoniumError):
        sb.Mesh(nodes[:, :2], tris)


def test_no_cpu_fallback_without_device(sb):
    if sb.device_count() > 0:
        pytest.skip("a CUDA device is present")
    nodes, tris = sb.icosphere(1.0, 1)
    with pytest.raises(sb.SoniumError) as e:
        sb.Mesh(nodes, tris)
    assert e.value.status == L.SB_ERR_CUDA
    x = np.zeros(4)
    s = np.zeros(4)
    c = np.zeros(4)
    st = L.load().sb_math_sincos(0, x.ctypes.data, 4, s.ctypes.data, c.ctypes.data)
    assert st == L.SB_ERR_CUDA


def test_null_and_bad_arguments(sb):
    lib = L.load()
    assert lib.sb_mesh_create(None, 0, None, 0, 0, None) == L.SB_ERR_INVALID_ARGUMENT
    assert "null" in L.last_error()
    assert lib.sb_assemble(None, None, L.SbComplex(0, 0), 0, None) == L.SB_ERR_INVALID_ARGUMENT
    assert lib.sb_inject_failure(99) == L.SB_ERR_INVALID_ARGUMENT
    assert lib.sb_inject_failure(0) == L.SB_OK
    assert lib.sb_mesh_destroy(None) == L.SB_OK
    assert lib.sb_operator_destroy(None) == L.SB_OK
    assert lib.sb_icosphere_counts(12, None, None) == L.SB_ERR_INVALID_ARGUMENT


def test_ellipsoid_sweep_plan_levels(sb):
    """The sweep plan: 64 instances, ka 1 -> 32, level refined with frequency, N 320 -> 20480."""
    from sonium_b200.sweep import ellipsoid_sweep_plan

    plan = ellipsoid_sweep_plan()
    assert len(plan) == 64
    ka = np.array([p[0] for p in plan])
    assert ka[0] == pytest.approx(1.0) and ka[-1] == pytest.approx(32.0)
    levels = [p[2] for p in plan]
    assert levels == sorted(levels) and levels[0] == 2 and levels[-1] == 5


def test_umma_descriptors_match_cutlass(tmp_path):
    """The tcgen05 instruction / shared-memory descriptor encoders agree bit for bit with CUTLASS's
    cute::UMMA descriptor types (compiled host-side; skipped when nvcc or the headers are absent)."""
    import glob
    import shutil
    import subprocess

    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    cands = [p for p in glob.glob(os.path.join(sys.prefix, "lib", "python3*", "site-packages", "*", "data",
                                               "cutlass", "include"))
             + glob.glob(os.path.join(sys.prefix, "lib", "python3*", "site-packages", "*", "3rdparty",
                                      "cutlass", "include"))
             if os.path.exists(os.path.join(p, "cute", "arch", "mma_sm100_desc.hpp"))]
    if not cands:
        pytest.skip("no CUTLASS headers with sm100 descriptors in this environment")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "umma_desc_check")
    cmd = [nvcc, "-std=c++17", "-Wno-deprecated-gpu-targets", "-I" + cands[0],
           "-I" + os.path.join(root, "sonium_b200", "csrc"), os.path.join(root, "tests", "native", "umma_desc_check.cu"),
           "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout


def test_frequency_sweep_config_validation(sb):
    """FrequencySweepConfig::validate / validate_frequency_grid (frequency_sweep.rs:88-114, 306-320)."""
    ok = sb.FrequencySweepConfig.linear(100.0, 200.0, 3)
    ok.validate()
    assert ok.frequencies == [100.0, 150.0, 200.0]
    lg = sb.FrequencySweepConfig.logarithmic(10.0, 1000.0, 3)
    assert np.allclose(lg.frequencies, [10.0, 100.0, 1000.0])
    for bad in (sb.FrequencySweepConfig(frequencies=[]), sb.FrequencySweepConfig(frequencies=[200.0, 100.0]),
                sb.FrequencySweepConfig(frequencies=[100.0, 100.0]), sb.FrequencySweepConfig(frequencies=[-1.0]),
                sb.FrequencySweepConfig(frequencies=[100.0], tolerance=0.0),
                sb.FrequencySweepConfig(frequencies=[100.0], gmres_restart=0),
                sb.FrequencySweepConfig(frequencies=[100.0], beta_scale=float("nan"))):
        with pytest.raises(sb.SoniumError):
            bad.validate()
