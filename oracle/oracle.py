"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is a plain C++ restatement of the reference (sonium-bem) CPU path, built from
``oracle/tbem_oracle.cpp`` by ``oracle/Makefile``. Only the tests, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` import this module; the product library never does.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtbem_oracle.so")
_lib = None


class OrC128(ct.Structure):
    _fields_ = [("re", ct.c_double), ("im", ct.c_double)]


class OrPhysics(ct.Structure):
    _fields_ = [(n, ct.c_double) for n in (
        "frequency", "speed_of_sound", "density", "wave_number", "omega", "wave_length",
        "harmonic_factor", "pressure_factor", "tau")]


class OrBc(ct.Structure):
    _fields_ = [("kind", ct.c_void_p), ("value", ct.c_void_p), ("has_adm", ct.c_void_p),
                ("adm", ct.c_void_p)]


class OrGmresResult(ct.Structure):
    _fields_ = [("iterations", ct.c_int64), ("restarts", ct.c_int64), ("matvecs", ct.c_int64),
                ("residual", ct.c_double), ("estimated_residual", ct.c_double),
                ("backward_error", ct.c_double), ("converged", ct.c_int32),
                ("status", ct.c_int32)]


def build() -> str:
    """Compile the oracle library with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ct.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    P = ct.c_void_p
    L.or_physics_new.argtypes = [ct.c_double, ct.c_double, ct.c_double, ct.c_int,
                                 ct.POINTER(OrPhysics)]
    L.or_icosphere_counts.argtypes = [ct.c_int, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)]
    L.or_icosphere.argtypes = [ct.c_double, ct.c_int, ct.c_double, ct.c_double, ct.c_double, P, P]
    L.or_element_geometry.argtypes = [ct.c_int64, P, P, P, P, P]
    L.or_assemble_rows.argtypes = [ct.c_int64, P, ct.c_int64, P, ct.POINTER(OrBc),
                                   ct.POINTER(OrPhysics), OrC128, ct.c_int64, ct.c_int64,
                                   ct.c_int, P, P]
    L.or_regular_pair.argtypes = [P, P, P, ct.c_double, ct.POINTER(OrPhysics), P]
    L.or_singular_pair.argtypes = [P, P, P, ct.POINTER(OrPhysics), P]
    L.or_subelements.argtypes = [P, P, ct.c_double, P, ct.c_int]
    L.or_rhs_plane_wave.argtypes = [ct.c_int64, P, P, ct.POINTER(OrPhysics), OrC128,
                                    ct.c_int64, P, P, P]
    L.or_gmres.argtypes = [ct.c_int64, P, P, P, ct.c_int64, ct.c_int64, ct.c_double, ct.c_int,
                           P, ct.POINTER(OrGmresResult)]
    L.or_matvec.argtypes = [ct.c_int64, P, P, P, ct.c_int]
    L.or_sph_j.argtypes = [ct.c_int, ct.c_double]
    L.or_sph_j.restype = ct.c_double
    L.or_sph_y.argtypes = [ct.c_int, ct.c_double]
    L.or_sph_y.restype = ct.c_double
    L.or_mie_rigid_coefficients.argtypes = [ct.c_double, ct.c_int, P]
    L.or_mie_rigid_field.argtypes = [ct.c_double, ct.c_double, ct.c_int, ct.c_double,
                                     ct.c_int64, P, P]
    L.or_field_eval.argtypes = [P, P, ct.c_int64, P, P, ct.c_double, ct.c_double, ct.c_double, P,
                                ct.c_int64, ct.c_int, P]
    L.or_linear_collocation.argtypes = [ct.c_int64, P, P, P, P]
    L.or_quad_geometry.argtypes = [ct.c_int64, P, P, P, P, P]
    L.or_assemble_quad.argtypes = [ct.c_int64, P, ct.c_int64, P, ct.POINTER(OrBc), ct.POINTER(OrPhysics), OrC128,
                                   ct.c_int, P, P]
    L.or_regular_pair_disc.argtypes = [P, P, P, ct.c_double, ct.POINTER(OrPhysics), ct.c_int, P]
    L.or_singular_pair_disc.argtypes = [P, P, P, ct.POINTER(OrPhysics), ct.c_int, P]
    L.or_disc_collocation.argtypes = [ct.c_int64, P, P, ct.c_int, P, P]
    L.or_assemble_discontinuous.argtypes = [ct.c_int64, P, ct.c_int64, P, ct.POINTER(OrBc), ct.POINTER(OrPhysics),
                                            OrC128, ct.c_int, ct.c_double, ct.c_int, P, P]
    L.or_assemble_linear.argtypes = [ct.c_int64, P, ct.c_int64, P, ct.POINTER(OrBc), ct.POINTER(OrPhysics),
                                     OrC128, ct.c_int, P, P]
    L.or_assemble_rows_from_channels.argtypes = [ct.c_int64, P, ct.c_int64, P, ct.POINTER(OrBc),
                                                 ct.POINTER(OrPhysics), OrC128, ct.c_int64, ct.c_int64, P,
                                                 ct.c_int, P, P]
    L.or_chart_rows.argtypes = [ct.c_int64, P, ct.c_int64, P, ct.c_double, ct.c_int64, ct.c_int64, ct.c_int, P, P,
                                ct.c_int64]
    L.or_chart_rows.restype = ct.c_int64


# Record layouts of the reference CUDA path's chart-driven pair kernel (bem_kernels.cu:818-833).
CHART_SAMPLE = np.dtype([("position", "<f8", 3), ("field_normal", "<f8", 3), ("edge_direction", "<f8", 3),
                         ("weight", "<f8"), ("basis_weight", "<f8"), ("kind", "<u4"), ("pad", "<u4")])
CHART_PAIR = np.dtype([("source_point", "<f8", 3), ("source_normal", "<f8", 3), ("sample_offset", "<u8"),
                       ("sample_count", "<u8")])
assert CHART_SAMPLE.itemsize == 96 and CHART_PAIR.itemsize == 64


def _p(a: np.ndarray):
    return a.ctypes.data_as(ct.c_void_p)


def physics(frequency: float, speed_of_sound: float = 343.0, density: float = 1.21,
            internal: bool = False) -> OrPhysics:
    out = OrPhysics()
    lib().or_physics_new(frequency, speed_of_sound, density, int(internal), ct.byref(out))
    return out


def physics_for_k(k: float, speed_of_sound: float = 343.0, density: float = 1.21) -> OrPhysics:
    return physics(k * speed_of_sound / (2.0 * np.pi), speed_of_sound, density)


def bm_beta(ph: OrPhysics, scale: float = 1.0) -> complex:
    """burton_miller_beta (crates/sonium-bem/src/core/types.rs:314-320), times ``scale``."""
    if ph.tau > 0.0:
        return complex(0.0, scale * ph.harmonic_factor / ph.wave_number)
    return 0j


def icosphere(radius: float, level: int, scale=(1.0, 1.0, 1.0)):
    nn, nt = ct.c_int64(), ct.c_int64()
    if lib().or_icosphere_counts(level, ct.byref(nn), ct.byref(nt)):
        raise ValueError("bad icosphere level")
    nodes = np.zeros((nn.value, 3), np.float64)
    tris = np.zeros((nt.value, 3), np.uint32)
    rc = lib().or_icosphere(radius, level, scale[0], scale[1], scale[2], _p(nodes), _p(tris))
    if rc:
        raise RuntimeError("icosphere failed")
    return nodes, tris


def element_geometry(nodes: np.ndarray, tris: np.ndarray):
    m = tris.shape[0]
    c = np.zeros((m, 3)); n = np.zeros((m, 3)); a = np.zeros(m)
    lib().or_element_geometry(m, _p(np.ascontiguousarray(nodes, np.float64)),
                              _p(np.ascontiguousarray(tris, np.uint32)), _p(c), _p(n), _p(a))
    return c, n, a


def _bc_struct(m, bc_kind=None, bc_value=None, admittance=None, keep=None):
    b = OrBc()
    if bc_kind is not None:
        k = np.ascontiguousarray(bc_kind, np.int32); keep.append(k); b.kind = k.ctypes.data
    if bc_value is not None:
        v = np.ascontiguousarray(bc_value, np.complex128); keep.append(v); b.value = v.ctypes.data
    if admittance is not None:
        adm = np.asarray(admittance, np.complex128)
        has = np.ascontiguousarray(~np.isnan(adm.real), np.uint8)
        adm = np.ascontiguousarray(np.nan_to_num(adm), np.complex128)
        keep += [has, adm]
        b.has_adm = has.ctypes.data
        b.adm = adm.ctypes.data
    return b


def assemble(nodes, tris, ph: OrPhysics, beta: complex, rows=None, bc_kind=None, bc_value=None,
             admittance=None, threads: int = 0):
    """Rows [r0, r1) of the dense TBEM matrix and RHS (build_tbem_system_with_beta_parallel).

    ``admittance`` holds NaN for elements without admittance."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    tris = np.ascontiguousarray(tris, np.uint32)
    m = tris.shape[0]
    r0, r1 = (0, m) if rows is None else rows
    A = np.zeros((r1 - r0, m), np.complex128)
    rhs = np.zeros(r1 - r0, np.complex128)
    keep = []
    b = _bc_struct(m, bc_kind, bc_value, admittance, keep)
    rc = lib().or_assemble_rows(nodes.shape[0], _p(nodes), m, _p(tris), ct.byref(b),
                                ct.byref(ph), OrC128(beta.real, beta.imag), r0, r1, threads,
                                _p(A), _p(rhs))
    if rc:
        raise ValueError("oracle assembly rejected its input")
    return A, rhs


def assemble_from_channels(nodes, tris, ph: OrPhysics, beta: complex, channels, rows=None, threads: int = 0):
    """Rows of the TBEM matrix with the CPU path's free terms and coefficients over the given
    (G, H, H^T, E) channels of every pair of the rows (rigid surface): channels is
    (rows x n x 4) complex128."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    tris = np.ascontiguousarray(tris, np.uint32)
    m = tris.shape[0]
    r0, r1 = (0, m) if rows is None else rows
    ch = np.ascontiguousarray(channels, np.complex128)
    if ch.size != (r1 - r0) * m * 4:
        raise ValueError("channels must hold 4 values per pair of the rows")
    A = np.zeros((r1 - r0, m), np.complex128)
    rhs = np.zeros(r1 - r0, np.complex128)
    b = OrBc()
    rc = lib().or_assemble_rows_from_channels(nodes.shape[0], _p(nodes), m, _p(tris), ct.byref(b), ct.byref(ph),
                                              OrC128(beta.real, beta.imag), r0, r1, _p(ch), threads, _p(A),
                                              _p(rhs))
    if rc:
        raise ValueError("oracle assembly rejected its input")
    return A, rhs


def chart(nodes, tris, k: float, rows=None, threads: int = 0):
    """Quadrature charts of the reference CUDA assembly path for the pairs of rows [r0, r1) x all
    elements (pair index (i - r0) * n + j): (pairs, samples) as CHART_PAIR / CHART_SAMPLE arrays."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    tris = np.ascontiguousarray(tris, np.uint32)
    m = tris.shape[0]
    r0, r1 = (0, m) if rows is None else rows
    L = lib()
    total = L.or_chart_rows(nodes.shape[0], _p(nodes), m, _p(tris), k, r0, r1, threads, None, None, 0)
    if total < 0:
        raise ValueError("oracle chart rejected its input")
    pairs = np.zeros((r1 - r0) * m, CHART_PAIR)
    samples = np.zeros(total, CHART_SAMPLE)
    got = L.or_chart_rows(nodes.shape[0], _p(nodes), m, _p(tris), k, r0, r1, threads, _p(pairs), _p(samples), total)
    if got != total:
        raise ValueError("oracle chart changed size between its two passes")
    return pairs, samples


def quad_geometry(nodes, quads):
    """Quad4 element geometry: centres, normals, areas (generators.rs:771-850)."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    quads = np.ascontiguousarray(quads, np.uint32)
    m = quads.shape[0]
    c, n, a = np.zeros((m, 3)), np.zeros((m, 3)), np.zeros(m)
    lib().or_quad_geometry(m, _p(nodes), _p(quads), _p(c), _p(n), _p(a))
    return c, n, a


def assemble_quad(nodes, quads, ph: OrPhysics, beta: complex, bc_kind=None, bc_value=None, admittance=None,
                  threads: int = 0):
    """The constant-panel system of a Quad4 mesh: (m x m matrix, rhs)."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    quads = np.ascontiguousarray(quads, np.uint32)
    m = quads.shape[0]
    A = np.zeros((m, m), np.complex128)
    rhs = np.zeros(m, np.complex128)
    keep = []
    b = _bc_struct(m, bc_kind, bc_value, admittance, keep)
    rc = lib().or_assemble_quad(nodes.shape[0], _p(nodes), m, _p(quads), ct.byref(b), ct.byref(ph),
                                OrC128(beta.real, beta.imag), threads, _p(A), _p(rhs))
    if rc:
        raise ValueError("oracle assembly rejected its input")
    return A, rhs


def cubed_sphere(radius: float, n: int, scale=(1.0, 1.0, 1.0)):
    """Quad4 test mesh: the six faces of a cube split into n x n quads, projected onto the sphere
    (then scaled per axis), shared nodes merged, vertex order such that (p2 - p0) x (p3 - p1)
    points outward."""
    faces = []
    t = np.linspace(-1.0, 1.0, n + 1)
    for axis in range(3):
        for sgn in (1.0, -1.0):
            u, v = np.meshgrid(t, t, indexing="ij")
            p = np.zeros((n + 1, n + 1, 3))
            p[..., axis] = sgn
            p[..., (axis + 1) % 3] = u
            p[..., (axis + 2) % 3] = v
            faces.append((p, axis, sgn))
    pts, quads, index = [], [], {}

    def node(x):
        key = tuple(np.round(x, 12))
        if key not in index:
            index[key] = len(pts)
            pts.append(x)
        return index[key]

    for p, axis, sgn in faces:
        for i in range(n):
            for j in range(n):
                q = [p[i, j], p[i + 1, j], p[i + 1, j + 1], p[i, j + 1]]
                ids = [node(x / np.linalg.norm(x)) for x in q]
                if sgn < 0:
                    ids = ids[::-1]
                quads.append(ids)
    nodes = np.array(pts) * radius * np.asarray(scale)
    return nodes, np.array(quads, np.uint32)


def disc_collocation(nodes, tris, nbas: int = 3):
    """Collocation points and normals of a discontinuous basis (nbas 3 or 6): (nbas m, 3) each."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    tris = np.ascontiguousarray(tris, np.uint32)
    m = tris.shape[0]
    pts = np.zeros((nbas * m, 3))
    nrm = np.zeros((nbas * m, 3))
    lib().or_disc_collocation(m, _p(nodes), _p(tris), nbas, _p(pts), _p(nrm))
    return pts, nrm


def linear_collocation(nodes, tris):
    """Collocation points and normals of the discontinuous linear basis: (3m, 3) each, DOF 3e + c."""
    return disc_collocation(nodes, tris, 3)


def assemble_discontinuous(nodes, tris, ph: OrPhysics, beta: complex, nbas: int = 3, sign: float = 1.0,
                           bc_kind=None, bc_value=None, admittance=None, threads: int = 0):
    """build_tbem_system_discontinuous_stabilized (tbem.rs:2810-2990): ((nbas m)^2 matrix, rhs)."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    tris = np.ascontiguousarray(tris, np.uint32)
    m = tris.shape[0]
    n = nbas * m
    A = np.zeros((n, n), np.complex128)
    rhs = np.zeros(n, np.complex128)
    keep = []
    b = _bc_struct(m, bc_kind, bc_value, admittance, keep)
    rc = lib().or_assemble_discontinuous(nodes.shape[0], _p(nodes), m, _p(tris), ct.byref(b), ct.byref(ph),
                                         OrC128(beta.real, beta.imag), nbas, float(sign), threads, _p(A), _p(rhs))
    if rc:
        raise ValueError("oracle assembly rejected its input")
    return A, rhs


def assemble_linear(nodes, tris, ph: OrPhysics, beta: complex, bc_kind=None, bc_value=None, admittance=None,
                    threads: int = 0):
    """build_tbem_system_linear (tbem.rs:1490-1620): (3m x 3m matrix, 3m rhs)."""
    return assemble_discontinuous(nodes, tris, ph, beta, 3, 1.0, bc_kind, bc_value, admittance, threads)


def regular_pair_disc(x, nx, coords, area, ph, nbas: int = 3):
    """(nbas, 4) channels (g, h, ht, e) per basis function, regular integration."""
    out = np.zeros(4 * nbas, np.complex128)
    x, nx, c = (np.ascontiguousarray(v, np.float64) for v in (x, nx, coords))
    lib().or_regular_pair_disc(_p(x), _p(nx), _p(c), float(area), ct.byref(ph), nbas, _p(out))
    return out.reshape(nbas, 4)


def singular_pair_disc(x, nx, coords, ph, nbas: int = 3):
    """(nbas, 4) channels (g, h, ht, e) per basis function, self element."""
    out = np.zeros(4 * nbas, np.complex128)
    x, nx, c = (np.ascontiguousarray(v, np.float64) for v in (x, nx, coords))
    lib().or_singular_pair_disc(_p(x), _p(nx), _p(c), ct.byref(ph), nbas, _p(out))
    return out.reshape(nbas, 4)


def regular_pair_linear(x, nx, coords, area, ph):
    return regular_pair_disc(x, nx, coords, area, ph, 3)


def singular_pair_linear(x, nx, coords, ph):
    return singular_pair_disc(x, nx, coords, ph, 3)


def regular_pair(x, nx, coords, area, ph):
    out = np.zeros(4, np.complex128)
    lib().or_regular_pair(_p(np.ascontiguousarray(x, np.float64)),
                          _p(np.ascontiguousarray(nx, np.float64)),
                          _p(np.ascontiguousarray(coords, np.float64)), area, ct.byref(ph),
                          _p(out))
    return out


def singular_pair(x, nx, coords, ph):
    out = np.zeros(4, np.complex128)
    lib().or_singular_pair(_p(np.ascontiguousarray(x, np.float64)),
                           _p(np.ascontiguousarray(nx, np.float64)),
                           _p(np.ascontiguousarray(coords, np.float64)), ct.byref(ph), _p(out))
    return out


def subelements(x, coords, area, cap=256):
    leaves = np.zeros((cap, 8))
    n = lib().or_subelements(_p(np.ascontiguousarray(x, np.float64)),
                             _p(np.ascontiguousarray(coords, np.float64)), area, _p(leaves), cap)
    return leaves[:min(n, cap)]


def rhs_plane_wave(centers, normals, ph, beta, dirs, amps=None):
    centers = np.ascontiguousarray(centers, np.float64)
    normals = np.ascontiguousarray(normals, np.float64)
    dirs = np.ascontiguousarray(np.atleast_2d(dirs), np.float64)
    n, r = centers.shape[0], dirs.shape[0]
    out = np.zeros((n, r), np.complex128)
    a = None if amps is None else np.ascontiguousarray(amps, np.complex128)
    lib().or_rhs_plane_wave(n, _p(centers), _p(normals), ct.byref(ph),
                            OrC128(beta.real, beta.imag), r, _p(dirs),
                            None if a is None else _p(a), _p(out))
    return out


def gmres(A, b, restart=30, max_iterations=100, tol=1e-8, x0=None, threads=0):
    A = np.ascontiguousarray(A, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    n = b.shape[0]
    x = np.zeros(n, np.complex128)
    res = OrGmresResult()
    x0a = None if x0 is None else np.ascontiguousarray(x0, np.complex128)
    lib().or_gmres(n, _p(A), _p(b), None if x0a is None else _p(x0a), max_iterations, restart,
                   tol, threads, _p(x), ct.byref(res))
    return x, res


def matvec(A, x, threads=0):
    A = np.ascontiguousarray(A, np.complex128)
    x = np.ascontiguousarray(x, np.complex128)
    y = np.zeros(A.shape[0], np.complex128)
    lib().or_matvec(A.shape[0], _p(A), _p(x), _p(y), threads)
    return y


def sph_j(n, x):
    return lib().or_sph_j(n, x)


def sph_y(n, x):
    return lib().or_sph_y(n, x)


def mie_coefficients(ka, num_terms):
    out = np.zeros(num_terms, np.complex128)
    lib().or_mie_rigid_coefficients(ka, num_terms, _p(out))
    return out


def mie_field(k, radius, num_terms, r, theta):
    theta = np.ascontiguousarray(theta, np.float64)
    out = np.zeros(theta.shape[0], np.complex128)
    lib().or_mie_rigid_field(k, radius, num_terms, r, theta.shape[0], _p(theta), _p(out))
    return out


def field_eval(nodes, tris, pressure, ph: OrPhysics, points, velocity=None, threads: int = 0):
    """Scattered field at exterior points (compute_scattered_field with explicit surface velocity,
    crates/sonium-bem/src/core/postprocess/pressure.rs:1388-1448; 7-point rule per element)."""
    nodes = np.ascontiguousarray(nodes, np.float64)
    tris = np.ascontiguousarray(tris, np.uint32)
    p = np.ascontiguousarray(pressure, np.complex128)
    v = None if velocity is None else np.ascontiguousarray(velocity, np.complex128)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    out = np.zeros(pts.shape[0], np.complex128)
    lib().or_field_eval(_p(nodes), _p(tris), tris.shape[0], _p(p), None if v is None else _p(v),
                        ph.wave_number, ph.harmonic_factor, ph.pressure_factor, _p(pts), pts.shape[0],
                        threads, _p(out))
    return out


def suggested_sphere_terms(ka: float) -> int:
    """suggested_sphere_terms (crates/sonium-wave/src/analytical/solutions_3d.rs:241-249)."""
    if np.isfinite(ka) and ka > 0:
        return max(int(np.ceil(ka)) * 4 + 16, 17)
    return 16


def weighted_relative_l2(computed, reference, weights):
    """weighted_relative_l2_error (crates/sonium-qa/src/lib.rs:264-311)."""
    d = np.sum(weights * np.abs(computed - reference) ** 2)
    r = np.sum(weights * np.abs(reference) ** 2)
    return float(np.sqrt(d / r))


def rigid_sphere_surface_error(x, centers, areas, k, radius, num_terms=None):
    """rigid_sphere_surface_relative_l2_error (crates/sonium-qa/src/lib.rs:319-358)."""
    if num_terms is None:
        num_terms = suggested_sphere_terms(k * radius)
    rad = np.linalg.norm(centers, axis=1)
    theta = np.arccos(np.clip(centers[:, 2] / rad, -1.0, 1.0))
    ref = mie_field(k, radius, num_terms, radius, theta)
    return weighted_relative_l2(x, ref, areas)
