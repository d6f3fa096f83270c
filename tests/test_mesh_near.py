"""The near-pair classifier of mesh creation against a brute-force count, and mesh validation.

The near list is the superset of the reference's level-0 "must subdivide" test (ratdis < 3,
crates/sonium-bem/src/core/integration/singular.rs:1431): a pair (i, j), i != j, is near when the
squared distance from row i's centroid to column j's level-0 subdivision centre is below
9.000000009 * area_j, with correctly rounded operations in a fixed order. The device classifier
skips chunks of 256 columns whose bounding box lies beyond the chunk's largest threshold from the
box of 32 rows; these tests check that the pair count and the assembled matrix do not depend on
it: an ellipsoid, the same mesh with its elements shuffled (chunks then span the whole surface and
are rarely skipped), and two far-apart spheres (whole chunks skipped).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return sb


def _near_count(nodes, tris):
    """Brute-force near pairs with the classifier's operation order (numpy float64 operations are
    correctly rounded and not contracted)."""
    v0, v1, v2 = (nodes[tris[:, a]] for a in range(3))
    c = ((0.0 + v0) + v1 + v2) / 3.0
    cr = np.cross(v1 - v0, v2 - v0)
    area = np.sqrt((cr[:, 0] * cr[:, 0] + cr[:, 1] * cr[:, 1]) + cr[:, 2] * cr[:, 2]) / 2.0
    third = 1.0 / 3.0
    sf0 = (1.0 - third) - third
    g = ((0.0 + sf0 * v0) + third * v1) + third * v2
    thr = 9.000000009 * area
    count = 0
    for i in range(len(tris)):
        d = g - c[i]
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        near = d2 < thr
        near[i] = False
        count += int(near.sum())
    return count


def test_near_count_ellipsoid_and_shuffled(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 3, (1.0, 0.6, 0.4))
    rng = np.random.default_rng(11)
    perm = rng.permutation(len(tris))
    ref = _near_count(nodes, tris)
    assert ref > 0
    m1 = gpu.Mesh(nodes, tris)
    m2 = gpu.Mesh(nodes, tris[perm])
    assert m1.info().n_near_pairs == ref
    assert m2.info().n_near_pairs == ref
    ph = gpu.PhysicsParams.for_wavenumber(5.0)
    A1 = gpu.build_tbem_system(m1, ph).matrix
    A2 = gpu.build_tbem_system(m2, ph).matrix
    P = A1[np.ix_(perm, perm)]
    assert np.max(np.abs(A2 - P)) <= 1e-12 * np.max(np.abs(A1))
    m1.close()
    m2.close()


def test_near_count_two_spheres(gpu, oracle):
    n1, t1 = oracle.icosphere(1.0, 3)
    n2, t2 = oracle.icosphere(0.5, 2)
    nodes = np.vstack([n1, n2 + np.array([6.0, 0.0, 0.0])])
    tris = np.vstack([t1, t2 + len(n1)]).astype(np.uint32)
    ref = _near_count(nodes, tris)
    m = gpu.Mesh(nodes, tris)
    assert m.info().n_near_pairs == ref == _near_count(n1, t1) + _near_count(n2, t2)
    m.close()


def test_degenerate_triangle_rejected(gpu, oracle):
    nodes, tris = oracle.icosphere(1.0, 1)
    tris = tris.copy()
    tris[5] = [tris[5][0], tris[5][0], tris[5][1]]  # two equal vertices: zero area
    with pytest.raises(gpu.SoniumError, match="degenerate triangle 5"):
        gpu.Mesh(nodes, tris)
