"""The allocation-free transposed / Hermitian product (sb_operator_apply_device_noalloc).

It exists for callers that must not allocate device memory through the driver: a host whose GPU
memory is already owned by its own pool, or one that cannot take the device-wide wait of
cudaFree. The tests call it through the C ABI on device buffers that the tests themselves own:

* on a fresh operator that has never run a transposed product, its first call leaves the
  library's allocator (sb_memory_stats) and the device's free memory (cudaMemGetInfo) unchanged;
  the device set-up (the lookup of the scratch array's address, which also loads the library's
  device code for it) is done beforehand by a call on another operator;
* its A^T x and A^H x match numpy on the oracle-assembled matrix (the assembly parity bar, 1e-10)
  and the regular entry point, sb_operator_apply_device, within 1e-12 on two calls in a row (the
  second call reuses the shared scratch the first one left behind);
* at N = 20480 the row chunks are capped by the scratch size (25 chunks of 820 rows) and the
  result still matches the regular entry point.

This file is collected last on purpose.
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
    rt.cudaMemGetInfo.argtypes = [ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_size_t)]
    return rt


class _Bufs:
    """Device vectors owned by the test (cudaMalloc'd here, never by the entry point)."""

    def __init__(self, rt, n, count):
        self.rt, self.n, self.p = rt, n, []
        for _ in range(count):
            p = ct.c_void_p()
            assert rt.cudaMalloc(ct.byref(p), 16 * n) == 0
            self.p.append(p)

    def put(self, i, v):
        v = np.ascontiguousarray(v, np.complex128)
        assert self.rt.cudaMemcpy(self.p[i], v.ctypes.data, 16 * self.n, 1) == 0

    def get(self, i):
        out = np.zeros(self.n, np.complex128)
        assert self.rt.cudaMemcpy(out.ctypes.data, self.p[i], 16 * self.n, 2) == 0
        return out

    def free(self):
        for p in self.p:
            self.rt.cudaFree(p)


def _memory(L, lib, rt):
    used, cached = ct.c_int64(), ct.c_int64()
    L.check(lib.sb_memory_stats(0, ct.byref(used), ct.byref(cached)))
    free, total = ct.c_size_t(), ct.c_size_t()
    assert rt.cudaMemGetInfo(ct.byref(free), ct.byref(total)) == 0
    return int(used.value), int(cached.value), int(free.value)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def env(sb):
    from sonium_b200 import _lib as L

    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb, L, L.load(), _cudart()


def test_noalloc_first_call_allocates_nothing_and_matches_numpy(env, oracle):
    sb, L, lib, rt = env
    # device set-up on another operator: the scratch address lookup (and the loading of the
    # entry point's device code) happen on a device's first call
    A_small = np.eye(16, dtype=complex) * 2.0
    small = sb.DenseMatrixOperator(A_small, sb.SB_PRECISION_FP64)
    sbuf = _Bufs(rt, 16, 2)
    try:
        sbuf.put(0, np.arange(16) + 1j)
        for trans in (L.SB_OP_T, L.SB_OP_C, L.SB_OP_N):
            L.check(lib.sb_operator_apply_device_noalloc(small.handle, trans, sbuf.p[0], sbuf.p[1]))
        assert np.allclose(sbuf.get(1), 2.0 * (np.arange(16) + 1j))  # the last call: N, x = k + i
    finally:
        sbuf.free()
        small.close()

    nodes, tris = sb.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    n = tris.shape[0]
    k = 5.0
    mesh = sb.Mesh(nodes, tris)
    ph = sb.PhysicsParams.for_wavenumber(k)
    beta = ph.burton_miller_beta()
    op = sb.build_tbem_system_with_beta(mesh, ph, beta)
    A_ref, _ = oracle.assemble(nodes, tris, oracle.physics_for_k(k), beta)
    rng = np.random.default_rng(0x5EED)
    bufs = _Bufs(rt, n, 3)
    try:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        bufs.put(0, x)
        rt.cudaDeviceSynchronize()
        before = _memory(L, lib, rt)
        # the first transposed product this operator ever runs
        L.check(lib.sb_operator_apply_device_noalloc(op.handle, L.SB_OP_T, bufs.p[0], bufs.p[2]))
        rt.cudaDeviceSynchronize()
        after = _memory(L, lib, rt)
        assert after == before, (before, after)
        assert _rel(bufs.get(2), A_ref.T @ x) < 1e-10
        L.check(lib.sb_operator_apply_device_noalloc(op.handle, L.SB_OP_C, bufs.p[0], bufs.p[2]))
        rt.cudaDeviceSynchronize()
        assert _memory(L, lib, rt) == before
        assert _rel(bufs.get(2), A_ref.conj().T @ x) < 1e-10
        # two calls in a row against the regular entry point
        for call, trans in enumerate((L.SB_OP_T, L.SB_OP_C, L.SB_OP_T)):
            x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
            bufs.put(0, x)
            L.check(lib.sb_operator_apply_device(op.handle, trans, bufs.p[0], bufs.p[1]))
            L.check(lib.sb_operator_apply_device_noalloc(op.handle, trans, bufs.p[0], bufs.p[2]))
            y_ref, y_na = bufs.get(1), bufs.get(2)
            assert _rel(y_na, y_ref) < 1e-12, (call, _rel(y_na, y_ref))
            ref_np = (A_ref.T if trans == L.SB_OP_T else A_ref.conj().T) @ x
            assert _rel(y_na, ref_np) < 1e-10
        # the forward product through the same entry point
        L.check(lib.sb_operator_apply_device(op.handle, L.SB_OP_N, bufs.p[0], bufs.p[1]))
        L.check(lib.sb_operator_apply_device_noalloc(op.handle, L.SB_OP_N, bufs.p[0], bufs.p[2]))
        assert np.array_equal(bufs.get(1), bufs.get(2))
        # bad arguments are rejected before any device work
        assert lib.sb_operator_apply_device_noalloc(op.handle, 7, bufs.p[0], bufs.p[2]) == L.SB_ERR_INVALID_ARGUMENT
        assert lib.sb_operator_apply_device_noalloc(op.handle, L.SB_OP_T, None, bufs.p[2]) == L.SB_ERR_INVALID_ARGUMENT
    finally:
        bufs.free()
        op.close()
        mesh.close()


def test_noalloc_capped_row_chunks_at_n20480(env):
    """N = 20480: 8 MiB of scratch holds 25 chunks of 16-byte partial sums per column, fewer than
    the 80 chunks of 256 rows the product would take, so the rows are split in 25 chunks of 820."""
    sb, L, lib, rt = env
    nodes, tris = sb.icosphere(1.0, 5)
    n = tris.shape[0]
    assert n == 20480 and (8 << 20) // (16 * n) == 25
    mesh = sb.Mesh(nodes, tris)
    ph = sb.PhysicsParams.for_wavenumber(10.0)
    op = sb.build_tbem_system(mesh, ph)
    rng = np.random.default_rng(20480)
    bufs = _Bufs(rt, n, 3)
    try:
        for call, trans in enumerate((L.SB_OP_T, L.SB_OP_C)):
            x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
            bufs.put(0, x)
            L.check(lib.sb_operator_apply_device(op.handle, trans, bufs.p[0], bufs.p[1]))
            L.check(lib.sb_operator_apply_device_noalloc(op.handle, trans, bufs.p[0], bufs.p[2]))
            assert _rel(bufs.get(2), bufs.get(1)) < 1e-12, call
            # rows of the host matrix: a sample of columns checked against numpy
            cols = np.arange(0, n, 997)
            A_cols = np.zeros((n, cols.size), complex)
            for r0 in range(0, n, 2048):
                rows = op.rows(r0, min(n, r0 + 2048))
                A_cols[r0:r0 + rows.shape[0]] = rows[:, cols]
            M = A_cols.T if trans == L.SB_OP_T else A_cols.conj().T
            assert _rel(bufs.get(2)[cols], M @ x) < 1e-12
    finally:
        bufs.free()
        op.close()
        mesh.close()
