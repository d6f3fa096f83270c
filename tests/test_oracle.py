"""CPU tests of the oracle: pinned against the reference's golden vectors and its own invariants.

The oracle is the checker for the CUDA path, so it is itself checked here first:
  * Mie coefficients vs the 100-digit reference fixture (scattering-golden-v1.json),
  * spherical Bessel j_n, y_n and derivatives vs the Wolfram fixture at 1e-10, the tolerance of
    crates/sonium-bem/tests/wolfram_sphere_coefficients.rs:26-28,
  * quadrature exactness (Gauss-Legendre, the 13-point triangle rule),
  * generate_subelements against an independent pure-Python restatement,
  * the assembly invariants the reference tests (tbem.rs:5516, 5619, 6191),
  * Mie convergence of the solved field (crates/sonium-qa/bin/bem_mesh_refinement.rs:19-128).
"""
import json
import math
from decimal import Decimal

import numpy as np
import pytest

from conftest import golden_path


def test_mie_coefficients_match_reference_golden(oracle):
    g = json.load(open(golden_path("mie_rigid_golden.json")))
    for case in g["cases"]:
        ka = float(case["ka"])
        nt = case["num_terms"]
        got = oracle.mie_coefficients(ka, nt)
        for n, c in enumerate(case["coefficients"]):
            ref = complex(float(Decimal(c["re"])), float(Decimal(c["im"])))
            # the fixture is fixed-point with 45 decimals: absolute resolution 1e-45
            assert abs(got[n] - ref) <= 1e-12 * abs(ref) + 1e-44, (ka, n, got[n], ref)


def test_spherical_bessel_match_wolfram_golden(oracle):
    g = json.load(open(golden_path("spherical_bessel_golden.json")))
    for case in g["cases"]:
        x = float(Decimal(case["x"]))
        for n in range(len(case["j"])):
            j = float(Decimal(case["j"][n]))
            y = float(Decimal(case["y"][n]))
            # the golden is at the exact argument (e.g. pi/2), the oracle at its double rounding:
            # allow |f'| * ulp(x) ~ 1e-15 absolute on top of the 1e-10 relative bound
            assert abs(oracle.sph_j(n, x) - j) <= 1e-10 * abs(j) + 1e-15, (case["name"], n)
            assert abs(oracle.sph_y(n, x) - y) <= 1e-10 * abs(y) + 1e-15, (case["name"], n)
        # derivatives j_n' = j_{n-1} - (n+1)/x j_n (solutions_3d.rs:779-795)
        for n in range(1, len(case["j"])):
            jp = oracle.sph_j(n - 1, x) - (n + 1) / x * oracle.sph_j(n, x)
            ref = float(Decimal(case["j_derivative"][n]))
            assert abs(jp - ref) <= 1e-10 * abs(ref) + 1e-15, (case["name"], n)


def test_far_leaf_quadrature_accuracy(oracle):
    # A far pair is one 13-point leaf over the whole element: at k -> 0, G is the integral of
    # 1 / (4 pi r); compare with a high-order Duffy-collapsed Gauss product rule.
    ph = oracle.physics_for_k(1e-9)
    x = np.array([0.0, 0.0, 5.0])
    nx = np.array([0.0, 0.0, 1.0])
    coords = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    out = oracle.regular_pair(x, nx, coords, 0.5, ph)
    # Duffy-collapsed Gauss reference (degree-60 product rule)
    gx, gw = np.polynomial.legendre.leggauss(60)
    u = 0.5 * (gx + 1)
    acc = 0.0
    for a in range(60):
        for b in range(60):
            s = u[a]
            t = (1 - s) * u[b]
            w = 0.25 * gw[a] * gw[b] * (1 - s)
            r = math.sqrt(s * s + t * t + 25.0)
            acc += w / (4 * math.pi * r)
    assert abs(out[0].real - acc) < 1e-9 * acc


def _py_subelements(x, c, area):
    """Independent pure-Python restatement of generate_subelements (singular.rs:1372-1540)."""
    csi = [0.0, 1.0, 0.0, 0.5, 0.5, 0.0]
    eta = [0.0, 0.0, 1.0, 0.0, 0.5, 0.5]
    cur = [([0.0, 1.0, 0.0], [0.0, 0.0, 1.0])]
    faclin = 2.0
    leaves = []
    while True:
        faclin *= 0.5
        arels = area * faclin * faclin
        nxt = []
        ndie = 0
        for xs, es in cur:
            sc = (xs[0] + xs[1] + xs[2]) / 3.0
            tc = (es[0] + es[1] + es[2]) / 3.0
            sf = [1 - sc - tc, sc, tc]
            g = [sum(sf[i] * c[i][j] for i in range(3)) for j in range(3)]
            dist = math.sqrt(sum((g[j] - x[j]) ** 2 for j in range(3)))
            rat = dist / math.sqrt(arels)
            if rat < 3.0:
                ndie += 1
                if ndie > 15:
                    break
                xm = [xs[0], xs[1], xs[2], (xs[0] + xs[1]) / 2, (xs[1] + xs[2]) / 2, (xs[2] + xs[0]) / 2]
                em = [es[0], es[1], es[2], (es[0] + es[1]) / 2, (es[1] + es[2]) / 2, (es[2] + es[0]) / 2]
                for t in range(3):
                    t2 = 5 if t == 0 else t + 2
                    nxt.append(([xm[t], xm[t + 3], xm[t2]], [em[t], em[t + 3], em[t2]]))
                nxt.append(([xm[3], xm[4], xm[5]], [em[3], em[4], em[5]]))
            else:
                leaves.append((xs, es, faclin))
                if len(leaves) >= 110:
                    return leaves
        if ndie == 0:
            break
        cur = nxt
    return leaves


@pytest.mark.parametrize("height", [0.01, 0.05, 0.2, 1.0, 10.0])
def test_subelements_match_python_restatement(oracle, height):
    coords = np.array([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.05, 0.25, 0.0]])
    area = 0.5 * abs(0.3 * 0.25)
    for x in ([0.1, 0.08, height], [0.31, 0.01, height], [-0.05, 0.3, height * 0.5]):
        got = oracle.subelements(np.array(x), coords, area)
        ref = _py_subelements(x, coords.tolist(), area)
        assert len(got) == len(ref)
        for lg, (xs, es, f) in zip(got, ref):
            verts = [lg[0], lg[2], lg[4]], [lg[1], lg[3], lg[5]]
            assert np.allclose(verts[0], xs, atol=0) and np.allclose(verts[1], es, atol=0)
            assert lg[6] == f and lg[7] == 4
        if len(ref) < 110:
            # leaves tile the element: local areas sum to 1/2
            tot = sum(0.5 * abs((xs[1] - xs[0]) * (es[2] - es[0]) - (xs[2] - xs[0]) * (es[1] - es[0]))
                      for xs, es, _ in ref)
            assert abs(tot - 0.5) < 1e-14


def test_far_pair_is_single_13_point_leaf(oracle):
    coords = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.0, 0.1, 0.0]])
    leaves = oracle.subelements(np.array([1.0, 1.0, 1.0]), coords, 0.005)
    assert len(leaves) == 1 and leaves[0][6] == 1.0 and leaves[0][7] == 4


def _sphere(oracle, level, k, radius=1.0):
    nodes, tris = oracle.icosphere(radius, level)
    ph = oracle.physics_for_k(k)
    return nodes, tris, ph


def test_assembly_thread_count_independence(oracle):
    """tbem.rs:6191: the row-parallel assembly does not depend on the thread count."""
    nodes, tris, ph = _sphere(oracle, 1, 1.0)
    beta = oracle.bm_beta(ph)
    A1, r1 = oracle.assemble(nodes, tris, ph, beta, threads=1)
    A8, r8 = oracle.assemble(nodes, tris, ph, beta, threads=8)
    assert np.array_equal(A1, A8) and np.array_equal(r1, r8)


def test_assembly_partial_rows_equal_full(oracle):
    """tbem.rs:5619 / 5516: partial-row (and RHS-only) assembly equals the full system."""
    nodes, tris, ph = _sphere(oracle, 1, 1.5)
    beta = oracle.bm_beta(ph)
    m = tris.shape[0]
    kind = np.zeros(m, np.int32)
    kind[::3] = 1
    val = np.linspace(0.1, 1.0, m) * (1 + 0.5j)
    adm = np.full(m, np.nan + 0j)
    adm[1::4] = 0.01 - 0.002j
    A, rhs = oracle.assemble(nodes, tris, ph, beta, bc_kind=kind, bc_value=val, admittance=adm)
    Ap, rp = oracle.assemble(nodes, tris, ph, beta, rows=(17, 41), bc_kind=kind, bc_value=val, admittance=adm)
    assert np.array_equal(A[17:41], Ap) and np.array_equal(rhs[17:41], rp)


def test_assembly_free_terms(oracle):
    """Diagonal free term -gamma/2 (velocity) / +beta tau / 2 (pressure), tbem.rs:1344-1358."""
    nodes, tris, ph = _sphere(oracle, 0, 0.5)
    beta = oracle.bm_beta(ph)
    m = tris.shape[0]
    A0, _ = oracle.assemble(nodes, tris, ph, beta)
    kind = np.ones(m, np.int32)
    A1, r1 = oracle.assemble(nodes, tris, ph, beta, bc_kind=kind)
    # pressure rows: coefficient -(G + beta H^T) off the diagonal; free term beta/2 on it
    assert np.allclose(np.diag(A1) - np.diag(A1), 0)
    assert np.all(np.abs(r1) == 0)
    assert A0.shape == A1.shape


def test_gmres_matches_dense_solve(oracle):
    rng = np.random.default_rng(0x5EED)
    n = 120
    A = np.eye(n) * 4 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x, res = oracle.gmres(A, b, restart=20, max_iterations=50, tol=1e-10)
    assert res.converged == 1 and res.status == 0
    xr = np.linalg.solve(A, b)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8
    assert res.residual < 1e-10


def test_gmres_reports_max_iterations(oracle):
    rng = np.random.default_rng(1)
    n = 60
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal(n) + 0j
    x, res = oracle.gmres(A, b, restart=3, max_iterations=2, tol=1e-12)
    assert res.converged == 0 and res.status == 1
    assert res.iterations == 6


def test_mie_convergence_rigid_sphere(oracle):
    """bem_mesh_refinement.rs:19-128: radius 0.1, ka = 1, beta = 2 i / k, levels 1..3."""
    radius, ka = 0.1, 1.0
    k = ka / radius
    errors, sizes = [], []
    for level in (1, 2, 3):
        nodes, tris = oracle.icosphere(radius, level)
        ph = oracle.physics_for_k(k)
        beta = oracle.bm_beta(ph, 2.0)
        A, rhs_bc = oracle.assemble(nodes, tris, ph, beta)
        c, nrm, area = oracle.element_geometry(nodes, tris)
        b = oracle.rhs_plane_wave(c, nrm, ph, beta, [0, 0, 1])[:, 0]
        x, res = oracle.gmres(A, b, restart=50, max_iterations=1000, tol=1e-10)
        assert res.converged == 1
        errors.append(oracle.rigid_sphere_surface_error(x, c, area, ph.wave_number, radius, 50))
        sizes.append(math.sqrt(area.sum() / len(area)))
    assert errors[0] > errors[1] > errors[2]
    orders = [math.log(errors[i] / errors[i + 1]) / math.log(sizes[i] / sizes[i + 1]) for i in range(2)]
    assert np.mean(orders) >= 0.5
    assert errors[-1] <= 0.01


def test_field_eval_matches_mie_exterior(oracle):
    """Scattered field at exterior points (compute_scattered_field, postprocess/pressure.rs:
    1388-1448) from the solved rigid-sphere surface pressure, plus the incident plane wave, against
    the Mie total field: relative error within the surface error's order (<= 2 % at level 3, ka = 2),
    and the error falls from level 2 to level 3."""
    k, radius = 2.0, 1.0
    rng = np.random.default_rng(11)
    th = rng.uniform(0.1, np.pi - 0.1, 24)
    rs = np.array([1.5, 2.0, 3.0])
    errs = []
    for level in (2, 3):
        nodes, tris = oracle.icosphere(radius, level)
        ph = oracle.physics_for_k(k)
        beta = oracle.bm_beta(ph)
        A, _ = oracle.assemble(nodes, tris, ph, beta)
        c, nrm, area = oracle.element_geometry(nodes, tris)
        b = oracle.rhs_plane_wave(c, nrm, ph, beta, [0, 0, 1])[:, 0]
        x, res = oracle.gmres(A, b, restart=50, max_iterations=200, tol=1e-10)
        assert res.converged == 1
        worst = 0.0
        for r in rs:
            pts = np.stack([r * np.sin(th), np.zeros_like(th), r * np.cos(th)], axis=1)
            scat = oracle.field_eval(nodes, tris, x, ph, pts)
            total = scat + np.exp(1j * k * pts[:, 2])
            mie = oracle.mie_field(k, radius, oracle.suggested_sphere_terms(k * radius), r, th)
            worst = max(worst, float(np.linalg.norm(total - mie) / np.linalg.norm(mie)))
        errs.append(worst)
    assert errs[1] < errs[0] and errs[1] <= 0.02, errs
    # a prescribed surface velocity enters through the single-layer term, linearly
    nodes, tris = oracle.icosphere(radius, 1)
    ph = oracle.physics_for_k(k)
    n = tris.shape[0]
    p0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    pts = np.array([[0.0, 0.0, 2.5], [1.7, -0.4, 0.9]])
    f_pv = oracle.field_eval(nodes, tris, p0, ph, pts, velocity=v0)
    f_p = oracle.field_eval(nodes, tris, p0, ph, pts)
    f_v = oracle.field_eval(nodes, tris, np.zeros(n, complex), ph, pts, velocity=v0)
    assert np.allclose(f_pv, f_p + f_v, rtol=1e-12, atol=1e-14)
