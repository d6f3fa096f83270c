/*
 * CPU oracle for the dense Burton-Miller TBEM path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker the CUDA product is compared against. It is a
 * plain C++ restatement of the reference (sonium-bem, Rust) CPU algorithms;
 * only tests, the smoke check and the CPU-baseline leg of the benchmark may
 * load it. Nothing in the product library links or calls it.
 *
 * Parity pins: the Mie/spherical-Bessel parts are pinned by the reference's
 * golden fixtures (crates/sonium-wave/fixtures/scattering-golden-v1.json and
 * special-golden-wolfram-v1.json, extracted into tests/golden/). The TBEM
 * matrix itself has no golden vector in the reference; it is pinned through
 * the reference's own invariants (thread-count independence, RHS-only ==
 * full, partial rows == full) and the Mie convergence of the solved field.
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef SONIUM_TBEM_ORACLE_H
#define SONIUM_TBEM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_c128 {
    double re, im;
} or_c128;

/* Mirrors PhysicsParams (crates/sonium-bem/src/core/types.rs:34-53,165-190). */
typedef struct or_physics {
    double frequency, speed_of_sound, density, wave_number, omega, wave_length;
    double harmonic_factor, pressure_factor, tau;
} or_physics;

void or_physics_new(double frequency, double speed_of_sound, double density, int is_internal,
                    or_physics* out);

/* generate_icosphere_mesh (crates/sonium-bem/src/core/mesh/generators.rs:309-397) with an
 * optional per-axis vertex scale applied after the radius (ellipsoid configs). */
int or_icosphere_counts(int level, int64_t* n_nodes, int64_t* n_tris);
int or_icosphere(double radius, int level, double sx, double sy, double sz, double* nodes,
                 uint32_t* tris);

/* compute_element_geometry (generators.rs:771-830): centroid, unit normal, area. */
void or_element_geometry(int64_t n_tris, const double* nodes, const uint32_t* tris,
                         double* centers, double* normals, double* areas);

/* Boundary condition per element: kind 0 = velocity (Neumann), 1 = pressure (Dirichlet);
 * value = the element's (averaged) prescribed value; has_adm/adm = surface admittance.
 * Null pointers mean rigid (velocity 0, no admittance). */
typedef struct or_bc {
    const int32_t* kind;
    const or_c128* value;
    const uint8_t* has_adm;
    const or_c128* adm;
} or_bc;

/* build_tbem_system_with_beta_parallel (crates/sonium-bem/src/core/assembly/tbem.rs:1284-1466)
 * for source rows [row0, row1). A is (row1-row0) x n_tris row-major, rhs has row1-row0 entries.
 * threads <= 0 uses all OpenMP threads. */
int or_assemble_rows(int64_t n_nodes, const double* nodes, int64_t n_tris, const uint32_t* tris,
                     const or_bc* bc, const or_physics* phys, or_c128 beta, int64_t row0,
                     int64_t row1, int threads, or_c128* A, or_c128* rhs);

/* The same rows assembled from given channels instead of the CPU integration rules: channels holds
 * (G, H, H^T, E) of every pair of the rows, ((i - row0) * n_tris + j) * 4, e.g. the reference CUDA
 * kernel's output for the same pairs; the free terms and BC coefficients are the CPU path's. */
int or_assemble_rows_from_channels(int64_t n_nodes, const double* nodes, int64_t n_tris, const uint32_t* tris,
                                   const or_bc* bc, const or_physics* phys, or_c128 beta, int64_t row0,
                                   int64_t row1, const or_c128* channels, int threads, or_c128* A,
                                   or_c128* rhs);

/* Quadrature charts of the reference CUDA assembly path (crates/sonium-bem/src/core/assembly/
 * tbem.rs:4998-5161, pairs as at :5189-5275) in the record layouts of its chart-driven kernel
 * (SoniumBemQuadratureSampleC64 / SoniumBemQuadraturePairC64, crates/sonium-compute/src/cuda/
 * kernels/bem_kernels.cu:818-833): kind 0 = regular sample, 1 = singular bulk, 2 = hypersingular
 * edge. */
typedef struct or_chart_sample {
    double position[3];
    double field_normal[3];
    double edge_direction[3];
    double weight;
    double basis_weight;
    uint32_t kind;
    uint32_t pad;
} or_chart_sample;
typedef struct or_chart_pair {
    double source_point[3];
    double source_normal[3];
    uint64_t sample_offset;
    uint64_t sample_count;
} or_chart_pair;
/* Charts of the pairs (i, j), i in [row0, row1), all j (pair index (i - row0) * n_tris + j).
 * Returns the sample count; with null pairs / samples only counts; -1 on bad input or when
 * capacity (samples) is too small. */
int64_t or_chart_rows(int64_t n_nodes, const double* nodes, int64_t n_tris, const uint32_t* tris, double k,
                      int64_t row0, int64_t row1, int threads, or_chart_pair* pairs, or_chart_sample* samples,
                      int64_t capacity);

/* Single-pair channel integrals (G, H, H^T, E) as 4 complex numbers, for unit tests.
 * regular_integration (crates/sonium-bem/src/core/integration/regular.rs:124-321) and
 * singular_integration (crates/sonium-bem/src/core/integration/singular.rs:297-614). */
void or_regular_pair(const double* x, const double* nx, const double* coords9, double area,
                     const or_physics* phys, or_c128* out4);
void or_singular_pair(const double* x, const double* nx, const double* coords9,
                      const or_physics* phys, or_c128* out4);

/* generate_subelements (singular.rs:1372-1540): returns the leaf count, writes up to cap
 * leaves as [v0x v0y v1x v1y v2x v2y factor order]. */
int or_subelements(const double* x, const double* coords9, double area, double* leaves, int cap);

/* IncidentField::compute_rhs_with_beta for a plane wave (crates/sonium-bem/src/core/incident.rs:
 * 216-245, 315-331, 807-833). dirs: r x 3, amps: r; rhs: n x r row-major. */
void or_rhs_plane_wave(int64_t n, const double* centers, const double* normals,
                       const or_physics* phys, or_c128 beta, int64_t r, const double* dirs,
                       const or_c128* amps, or_c128* rhs);

/* Restarted GMRES (crates/sonium-solvers/crates/sonium-solvers-iterative/src/gmres.rs:631-1047,
 * finalize 159-247), dense row-major operator, identity preconditioner. */
typedef struct or_gmres_result {
    int64_t iterations, restarts, matvecs;
    double residual, estimated_residual, backward_error;
    int32_t converged, status; /* status: 0 converged, 1 max iterations, 2 breakdown, 3 numerical */
} or_gmres_result;

int or_gmres(int64_t n, const or_c128* A, const or_c128* b, const or_c128* x0,
             int64_t max_iterations, int64_t restart, double tolerance, int threads,
             or_c128* x, or_gmres_result* res);

/* Dense complex matvec y = A x (row-major), the reference CPU GEMV
 * (crates/sonium-solvers/crates/sonium-solvers-core/src/dense.rs:416-427). */
void or_matvec(int64_t n, const or_c128* A, const or_c128* x, or_c128* y, int threads);

/* Spherical Bessel j_n, y_n (crates/sonium-wave/src/analytical/solutions_3d.rs:808-900),
 * rigid-sphere Mie coefficients (solutions_3d.rs:769-806) and the surface field
 * (solutions_3d.rs:315-366). */
double or_sph_j(int n, double x);
double or_sph_y(int n, double x);
void or_mie_rigid_coefficients(double ka, int num_terms, or_c128* out);
void or_mie_rigid_field(double k, double radius, int num_terms, double r, int64_t n_theta,
                        const double* theta, or_c128* out);
/* Scattered field at m exterior points from constant Tri3 surface pressure / velocity
 * (velocity may be NULL = rigid); compute_scattered_field, postprocess/pressure.rs:1388-1448. */
/* Discontinuous linear Tri3 basis: collocation points / normals (3 per element, DOF 3e + c) and
 * build_tbem_system_linear (A: 3m x 3m row-major, rhs: 3m). */
void or_linear_collocation(int64_t n_tris, const double* nodes, const uint32_t* tris, double* points,
                           double* normals);
int or_assemble_linear(int64_t n_nodes, const double* nodes, int64_t n_tris, const uint32_t* tris,
                       const or_bc* bc, const or_physics* phys, or_c128 beta, int threads, or_c128* A,
                       or_c128* rhs);

/* Discontinuous-basis channels of one pair: out = (g, h, ht, e) for each of nbas (3 or 6) basis
 * functions. */
void or_regular_pair_disc(const double* x, const double* nx, const double* coords9, double area,
                          const or_physics* phys, int nbas, or_c128* out);
void or_singular_pair_disc(const double* x, const double* nx, const double* coords9,
                           const or_physics* phys, int nbas, or_c128* out);
/* Any discontinuous basis (nbas 3 or 6) and sign +-1: collocation and assembly. */
void or_disc_collocation(int64_t n_tris, const double* nodes, const uint32_t* tris, int nbas, double* points,
                         double* normals);
int or_assemble_discontinuous(int64_t n_nodes, const double* nodes, int64_t n_tris, const uint32_t* tris,
                              const or_bc* bc, const or_physics* phys, or_c128 beta, int nbas, double sign,
                              int threads, or_c128* A, or_c128* rhs);

/* Quad4 constant panels: element geometry (centre, diagonal-cross normal, mean-split area) and
 * the m x m constant-panel system. */
void or_quad_geometry(int64_t n_quads, const double* nodes, const uint32_t* quads, double* centers,
                      double* normals, double* areas);
int or_assemble_quad(int64_t n_nodes, const double* nodes, int64_t n_quads, const uint32_t* quads,
                     const or_bc* bc, const or_physics* phys, or_c128 beta, int threads, or_c128* A,
                     or_c128* rhs);

void or_field_eval(const double* nodes, const uint32_t* tris, int64_t n_tris, const or_c128* pressure,
                   const or_c128* velocity, double k, double harmonic_factor, double pressure_factor,
                   const double* points, int64_t m, int threads, or_c128* out);

#ifdef __cplusplus
}
#endif
#endif
