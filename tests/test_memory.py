"""The caching device allocator behind every device buffer (sb_memory_stats / sb_memory_trim):
released blocks are reused by the next allocation of the same rounded size, results do not
change when buffers come from the cache, and trim hands the cache back to the driver."""
import ctypes as ct
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("SB_DEVICE_CACHE", "1").startswith("0"),
                                 reason="the device cache is switched off (SB_DEVICE_CACHE=0)")]


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _stats(L):
    a, c = ct.c_int64(), ct.c_int64()
    L.check(L.load().sb_memory_stats(0, ct.byref(a), ct.byref(c)))
    return a.value, c.value


def test_blocks_are_reused_and_trimmed(gpu):
    from sonium_b200 import _lib as L

    nodes, tris = gpu.icosphere(1.0, 3)
    ph = gpu.PhysicsParams.for_wavenumber(3.0)
    beta = ph.burton_miller_beta()
    b = None
    results = []
    for rep in range(3):
        mesh = gpu.Mesh(nodes, tris)
        op = gpu.build_tbem_system_with_beta(mesh, ph, beta)
        if b is None:
            b = gpu.rhs_plane_wave(mesh, ph, beta, [0.0, 0.0, 1.0])[:, 0]
        results.append((op.matrix, gpu.gmres(op, b, gpu.GmresConfig(50, 30, 1e-10)).x))
        in_use, cached_before = _stats(L)
        assert in_use > 0
        op.close()
        mesh.close()
        in_use_after, cached = _stats(L)
        assert in_use_after < in_use and cached > cached_before
    for A, x in results[1:]:
        assert np.array_equal(A, results[0][0]) and np.array_equal(x, results[0][1])
    L.check(L.load().sb_memory_trim(-1))
    assert _stats(L)[1] == 0
