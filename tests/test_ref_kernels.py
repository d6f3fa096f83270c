"""The reference's own CUDA pair kernel as a checker of the oracle and of the product.

The reference's CUDA assembly path (tbem.rs:5165-5405) integrates every pair over a host-built
quadrature chart with its kernel ``sonium_bem_quadrature_pair_c64``
(crates/sonium-compute/src/cuda/kernels/bem_kernels.cu:839-967). ``oracle/Makefile`` compiles that
kernel unchanged from the reference's source into ``oracle/_ref/``; the oracle restates the chart
construction (tbem.rs:4998-5161) and ``oracle/ref_kernels.py`` launches the kernel as the
reference's backend does. This pins the oracle's per-sample channel arithmetic (regular points,
the Duffy bulk of the self term and its regularised hypersingular edge integral) to the
reference's own code:

* CPU: the charts have the reference's structure (sample counts per pair, weights summing to the
  element area, the self rule of QuadratureParams::for_ka);
* GPU: per pair (G, H, H^T, E) of the reference kernel equals the oracle's CPU integration
  (or_regular_pair / or_singular_pair) on far, near (subdivided) and self pairs of all four self
  brackets, to 1e-12 relative (1e-11 for the self E channel, whose edge terms cancel);
* GPU: the whole N = 1280, k = 2 matrix assembled from the reference kernel's channels equals the
  oracle's matrix (1e-12) and the product's FP64 matrix (1e-10 per entry, the assembly parity bar).
"""
import numpy as np
import pytest

from oracle import ref_kernels as RK


def _pair_channels_oracle(oracle, nodes, tris, ph, pairs_ij):
    c, nrm, area = oracle.element_geometry(nodes, tris)
    out = np.zeros((len(pairs_ij), 4), complex)
    for q, (i, j) in enumerate(pairs_ij):
        coords = nodes[tris[j]]
        if i == j:
            out[q] = oracle.singular_pair(c[i], nrm[i], coords, ph)
        else:
            out[q] = oracle.regular_pair(c[i], nrm[i], coords, area[j], ph)
    return out


def test_chart_structure(oracle):
    nodes, tris = oracle.icosphere(1.0, 2)
    n = tris.shape[0]
    c, nrm, area = oracle.element_geometry(nodes, tris)
    for k, edge_pts, bulk_pts in ((0.5, 3 * 4 * 3, 3 * 2 * 16), (2.0, 3 * 6 * 4, 3 * 2 * 25),
                                  (8.0, 3 * 8 * 5, 3 * 3 * 36), (20.0, 3 * 10 * 6, 3 * 4 * 49)):
        pairs, samples = oracle.chart(nodes, tris, k, rows=(0, 4))
        assert pairs.shape[0] == 4 * n
        for i in range(4):
            p = pairs[i * n + i]  # the self pair
            s = samples[p["sample_offset"]:p["sample_offset"] + p["sample_count"]]
            assert np.count_nonzero(s["kind"] == 2) == edge_pts
            assert np.count_nonzero(s["kind"] == 1) == bulk_pts
            # the Duffy bulk integrates the element's area; the edge weights its perimeter
            assert abs(s["weight"][s["kind"] == 1].sum() - area[i]) < 1e-12 * area[i] * 100
            edges = nodes[tris[i][[1, 2, 0]]] - nodes[tris[i]]
            assert abs(s["weight"][s["kind"] == 2].sum() - np.linalg.norm(edges, axis=1).sum()) < 1e-12
            assert np.allclose(p["source_point"], c[i]) and np.allclose(p["source_normal"], nrm[i])
        jf = int(np.argmax(np.linalg.norm(c - c[0], axis=1)))  # the element farthest from element 0
        far = pairs[jf]
        assert far["sample_count"] == 13  # a far pair: one leaf of the 13-point rule
        s = samples[far["sample_offset"]:far["sample_offset"] + far["sample_count"]]
        assert np.all(s["kind"] == 0) and abs(s["weight"].sum() - area[jf]) < 1e-14
    # contiguous, ordered sample ranges
    assert np.all(pairs["sample_offset"][1:] == pairs["sample_offset"][:-1] + pairs["sample_count"][:-1])


@pytest.fixture(scope="module")
def refk(sb):
    if sb.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return RK.RefPairKernel(0)


@pytest.mark.gpu
@pytest.mark.parametrize("level,k,scale", [(3, 2.0, (1.0, 1.0, 1.0)), (2, 10.0, (1.0, 0.6, 0.4)),
                                           (1, 4.0, (1.0, 1.0, 1.0)), (2, 3.0, (1.0, 1.0, 1.0)),
                                           (1, 40.0, (1.0, 1.0, 1.0)), (1, 90.0, (1.0, 0.6, 0.4))])
def test_reference_kernel_matches_oracle_pairs(oracle, refk, level, k, scale):
    nodes, tris = oracle.icosphere(1.0, level, scale)
    n = tris.shape[0]
    ph = oracle.physics_for_k(k)
    rows = (0, min(n, 24))
    pairs, samples = oracle.chart(nodes, tris, k, rows=rows)
    ch, _ = refk.run(pairs, samples, k, ph.harmonic_factor)
    ij = [(i, j) for i in range(rows[0], rows[1]) for j in range(n)]
    ref = _pair_channels_oracle(oracle, nodes, tris, ph, ij)
    counts = pairs["sample_count"]
    selfm = np.array([i == j for i, j in ij])
    nearm = (counts > 13) & ~selfm
    assert nearm.any() and (~nearm & ~selfm).any()  # far and subdivided near pairs both present
    # relative per entry, with a floor of a fraction of the pair's largest channel for channels
    # that vanish up to rounding (H and H^T of a flat self element: r.n_y = 0 in the element's
    # plane, so both sums are rounding noise of the G-sized terms)
    pair_scale = np.abs(ref).max(axis=1)
    for m, tol_e, floor in ((~selfm, 1e-12, 1e-6), (selfm, 1e-11, 1e-4)):
        for c in range(4):
            d = np.abs(ch[m, c] - ref[m, c]) / np.maximum(np.abs(ref[m, c]), floor * pair_scale[m])
            tol = tol_e if c == 3 else 1e-12
            assert d.max() < tol, (c, float(d.max()))


@pytest.mark.gpu
def test_reference_kernel_matrix_config1(oracle, sb, refk):
    """N = 1280, k = 2 (the small plain configuration): all 1.64 M pairs through the reference
    kernel, combined with the CPU path's coefficients, against the oracle and the product."""
    k = 2.0
    nodes, tris = oracle.icosphere(1.0, 3)
    ph = oracle.physics_for_k(k)
    beta = oracle.bm_beta(ph)
    pairs, samples = oracle.chart(nodes, tris, k)
    ch, _ = refk.run(pairs, samples, k, ph.harmonic_factor)
    A_refk, _ = oracle.assemble_from_channels(nodes, tris, ph, beta, ch)
    A_or, _ = oracle.assemble(nodes, tris, ph, beta)
    floor = 1e-8 * np.abs(A_or).max()
    err_or = float(np.max(np.abs(A_refk - A_or) / np.maximum(np.abs(A_or), floor)))
    assert err_or < 1e-12, err_or
    mesh = sb.Mesh(nodes, tris)
    op = sb.build_tbem_system_with_beta(mesh, sb.PhysicsParams.for_wavenumber(k), beta)
    A = op.matrix
    err_gpu = float(np.max(np.abs(A - A_refk) / np.maximum(np.abs(A_refk), floor)))
    assert err_gpu < 1e-10, err_gpu
    op.close()
    mesh.close()
