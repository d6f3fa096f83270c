"""The allocation-free transposed / Hermitian product (sb_operator_apply_device_noalloc).

It exists for callers that must not allocate device memory through the driver: a host whose GPU
memory is already owned by its own pool, or one that cannot take the device-wide wait of
cudaFree. The test calls it through the C ABI on device buffers that the test itself owns and
checks it against the regular entry point, sb_operator_apply_device, on two calls in a row (the
second call reuses the shared scratch the first one left behind), within the 1e-12 relative bar
of the other matvec tests. This file is collected last on purpose.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cudart():
    for name in ("libcudart.so.12", "libcudart.so", "/usr/local/cuda/lib64/libcudart.so.12"):
        try:
            rt = ct.CDLL(name)
            break
        except OSError:
            continue
    else:
        pytest.fail("libcudart not found")
    rt.cudaMalloc.argtypes = [ct.POINTER(ct.c_void_p), ct.c_size_t]
    rt.cudaFree.argtypes = [ct.c_void_p]
    rt.cudaMemcpy.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_size_t, ct.c_int]
    return rt


def test_noalloc_transposed_apply_matches_regular_entry(sb):
    from sonium_b200 import _lib as L

    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    lib = L.load()
    rt = _cudart()
    nodes, tris = sb.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    mesh = sb.Mesh(nodes, tris)
    ph = sb.PhysicsParams.for_wavenumber(5.0)
    op = sb.build_tbem_system(mesh, ph)
    n = tris.shape[0]
    rng = np.random.default_rng(0x5EED)
    bufs = []
    for _ in range(3):
        p = ct.c_void_p()
        assert rt.cudaMalloc(ct.byref(p), 16 * n) == 0
        bufs.append(p)
    x_d, y_ref_d, y_na_d = bufs
    try:
        for call, trans in enumerate((L.SB_OP_T, L.SB_OP_C, L.SB_OP_T)):
            x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
            assert rt.cudaMemcpy(x_d, x.ctypes.data, 16 * n, 1) == 0
            L.check(lib.sb_operator_apply_device(op.handle, trans, x_d, y_ref_d))
            L.check(lib.sb_operator_apply_device_noalloc(op.handle, trans, x_d, y_na_d))
            y_ref = np.zeros(n, np.complex128)
            y_na = np.zeros(n, np.complex128)
            assert rt.cudaMemcpy(y_ref.ctypes.data, y_ref_d, 16 * n, 2) == 0
            assert rt.cudaMemcpy(y_na.ctypes.data, y_na_d, 16 * n, 2) == 0
            err = np.linalg.norm(y_na - y_ref) / np.linalg.norm(y_ref)
            assert err < 1e-12, (call, err)
        # the forward product through the same entry point
        L.check(lib.sb_operator_apply_device(op.handle, L.SB_OP_N, x_d, y_ref_d))
        L.check(lib.sb_operator_apply_device_noalloc(op.handle, L.SB_OP_N, x_d, y_na_d))
        y_ref = np.zeros(n, np.complex128)
        y_na = np.zeros(n, np.complex128)
        rt.cudaMemcpy(y_ref.ctypes.data, y_ref_d, 16 * n, 2)
        rt.cudaMemcpy(y_na.ctypes.data, y_na_d, 16 * n, 2)
        assert np.array_equal(y_ref, y_na)
        # bad arguments are rejected before any device work
        assert lib.sb_operator_apply_device_noalloc(op.handle, 7, x_d, y_na_d) == L.SB_ERR_INVALID_ARGUMENT
    finally:
        for p in bufs:
            rt.cudaFree(p)
        op.close()
        mesh.close()
