/*
 * sonium-b200 C ABI: dense constant-panel Burton-Miller TBEM on one NVIDIA B200 (sm_100a).
 *
 * The entry points below are what the reference's Rust side would bind over FFI to replace
 * its dense collocation path: the assembly entry points of crates/sonium-bem/src/core/
 * assembly/tbem.rs, the incident-field right-hand side of crates/sonium-bem/src/core/
 * incident.rs, the LinearOperator / Preconditioner surface of crates/sonium-solvers/crates/
 * sonium-solvers-core/src/traits.rs and the restarted GMRES of crates/sonium-solvers/crates/
 * sonium-solvers-iterative/src/gmres.rs. Citations are relative to the sonium workspace root.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, POD structs. Complex numbers are interleaved
 *    (re, im) doubles (sb_complex) or floats (sb_complex32), layout-compatible with
 *    num_complex::Complex64 / Complex32.
 *  - Matrices are row-major (row = source/collocation DOF, column = field DOF), as
 *    DenseMatrix<Complex64> in tbem.rs:135.
 *  - Constant panels: element e owns DOF e (the dof_addresses = [e] numbering that
 *    generate_icosphere_mesh produces, generators.rs:700-712).
 *  - Every function returns an int status (SB_OK = 0). On failure sb_last_error() returns a
 *    message. Errors are never silently replaced by a CPU computation: there is no CPU
 *    fallback in this library, and a missing or unusable GPU is SB_ERR_CUDA.
 *  - Host pointers are caller-owned and only read/written during the call. Handles are
 *    thread-safe per handle, not across handles that share a mesh.
 */
#ifndef SONIUM_B200_H
#define SONIUM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SB_API __attribute__((visibility("default")))
#else
#define SB_API
#endif

/* ---- status codes: CudaTbemAssemblyError (tbem.rs:3693-3718) + MissingSourceDof (:108-129) ---- */
#define SB_OK 0
#define SB_ERR_INVALID_ARGUMENT 1   /* InvalidInput { reason } */
#define SB_ERR_UNSUPPORTED_ELEMENT 2 /* UnsupportedElement (degenerate Tri3) */
#define SB_ERR_OUT_OF_MEMORY 3
#define SB_ERR_CUDA 4               /* Backend(..): launch / runtime failure, no device */
#define SB_ERR_DEVICE_CHECK 5       /* a kernel reported a bounded failure in its status word */
#define SB_ERR_INJECTED 6           /* host-side fault injection (sb_inject_failure) */
#define SB_ERR_NOT_FINITE 7         /* non-finite input or output (try_apply contract) */

/* ---- basic types ---- */
typedef struct sb_complex {
    double re, im;
} sb_complex;

typedef struct sb_complex32 {
    float re, im;
} sb_complex32;

/* PhysicsParams (crates/sonium-bem/src/core/types.rs:34-53). */
typedef struct sb_physics {
    double frequency, speed_of_sound, density, wave_number, omega, wave_length;
    double harmonic_factor, pressure_factor, tau;
} sb_physics;

/* Message of the last failure on this thread (empty when none). Returns the message length. */
SB_API int sb_last_error(char* buf, size_t len);
SB_API int sb_version(int* major, int* minor, int* patch);
/* Number of visible CUDA devices (0 when none); never falls back. */
SB_API int sb_device_count(int* count);

/* PhysicsParams::new / try_new (types.rs:120-160,165-190): k = 2 pi f / c, harmonic factor +1
 * (conventions.rs:308-313), pressure_factor = rho * omega, tau = +1 exterior / -1 interior. */
SB_API int sb_physics_new(double frequency, double speed_of_sound, double density,
                          int is_internal, sb_physics* out);
/* PhysicsParams::validate (types.rs:238-300). */
SB_API int sb_physics_validate(const sb_physics* p);
/* burton_miller_beta_scaled (types.rs:314-320, 418): i * harmonic_factor * scale / k for
 * exterior problems, 0 for interior ones. */
SB_API int sb_burton_miller_beta(const sb_physics* p, double scale, sb_complex* beta);

/* ---- mesh ---- */
/* generate_icosphere_mesh (crates/sonium-bem/src/core/mesh/generators.rs:309-397) on the host,
 * vertices scaled per axis by scale[3] (NULL = sphere) after the radius. */
SB_API int sb_icosphere_counts(int level, int64_t* n_nodes, int64_t* n_tris);
SB_API int sb_icosphere(double radius, int level, const double* scale, double* nodes,
                        uint32_t* tris);

typedef struct sb_mesh sb_mesh;

typedef struct sb_mesh_info {
    int64_t n_nodes, n_elements, n_near_pairs;
    int32_t device;
    int32_t reserved;
} sb_mesh_info;

/* Upload a Tri3 constant-panel mesh to `device` (validate_cuda_tbem_inputs, tbem.rs:4659-4798:
 * finite coordinates, in-range connectivity, non-degenerate triangles) and precompute the
 * element geometry (compute_element_geometry, generators.rs:771-830), the far-field quadrature
 * points and the near-pair list. The default boundary condition is rigid (velocity 0). */
SB_API int sb_mesh_create(const double* nodes, int64_t n_nodes, const uint32_t* tris,
                          int64_t n_tris, int device, sb_mesh** out);
/* A Quad4 mesh (constant panels, element e owns DOF e): quads[e * 4 + v], vertices ordered
 * around the element so that the bilinear map of (1, 1), (-1, 1), (-1, -1), (1, -1) runs through
 * them; the element normal is that of the diagonals, (p2 - p0) x (p3 - p1) (compute_element_geometry,
 * crates/sonium-bem/src/core/mesh/generators.rs:771-850). sb_assemble builds its constant-panel
 * system with the Quad4 branches of the regular and singular integration (bilinear geometry,
 * tensor Gauss-Legendre rules, four-quad subdivision; SB_PRECISION_FP64 only, no prescribed
 * boundary values); the batched, tensor-core, field and discontinuous-basis entry points take
 * Tri3 meshes only (SB_ERR_UNSUPPORTED_ELEMENT). */
SB_API int sb_mesh_create_quad4(const double* nodes, int64_t n_nodes, const uint32_t* quads, int64_t n_quads,
                                int device, sb_mesh** out);
SB_API int sb_mesh_destroy(sb_mesh* mesh);
SB_API int sb_mesh_info_get(const sb_mesh* mesh, sb_mesh_info* info);
/* Element centroid (collocation point), unit normal and area, each n_elements long. */
SB_API int sb_mesh_element_geometry(const sb_mesh* mesh, double* centers, double* normals,
                                    double* areas);

/* Boundary conditions per element (BoundaryCondition, types.rs:582-640; get_bc_type_and_value,
 * crates/sonium-bem/src/core/assembly/common.rs:283-293): kind 0 = velocity (Neumann),
 * 1 = pressure (Dirichlet); value = the element's averaged prescribed value; has_admittance /
 * admittance = VelocityWithAdmittance. Any pointer may be NULL (0 / none). */
#define SB_BC_VELOCITY 0
#define SB_BC_PRESSURE 1
SB_API int sb_mesh_set_bc(sb_mesh* mesh, const int32_t* kind, const sb_complex* value,
                          const uint8_t* has_admittance, const sb_complex* admittance);

/* ---- assembly ---- */
#define SB_PRECISION_FP64 0      /* complex128 matrix only */
#define SB_PRECISION_FP64_FP32 1 /* complex128 matrix plus a complex64 copy from one epilogue */
#define SB_PRECISION_FP32 2      /* complex64 matrix only: far pairs in FP32 with the phase
                                  * argument k r in FP64, near and self pairs in FP64; products
                                  * with FP64 vectors accumulate in FP64 */
#define SB_PRECISION_FP32_HALF 3 /* SB_PRECISION_FP32 with SB_INNER_FP16 set from the start (accepted
                                  * by sb_assemble only): the first assembly already writes the
                                  * complex-half copy the mixed solver's inner products read;
                                  * sb_operator_info_get reports SB_PRECISION_FP32 */

typedef struct sb_operator sb_operator;

typedef struct sb_operator_info {
    int64_t n;
    int32_t precision;
    int32_t device;
    double assembly_ms;          /* device time of the last assembly */
    uint64_t bytes_fp64, bytes_fp32;
} sb_operator_info;

/* build_tbem_system_with_beta (tbem.rs:1196-1203 -> build_tbem_system_with_beta_parallel
 * :1284-1466): dense Burton-Miller collocation matrix (G, H, H^T, E channels; adaptive
 * regular quadrature regular.rs:124-321 with generate_subelements singular.rs:1372-1540;
 * self term singular.rs:297-614) plus the boundary-condition RHS, resident on the device. */
SB_API int sb_assemble(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta,
                       int precision, sb_operator** out);
/* Re-assemble an existing operator for a new frequency / beta in place
 * (CudaTbemAssemblyWorkspace::assemble, tbem.rs:4230-4389). */
SB_API int sb_assemble_into(sb_operator* op, const sb_physics* physics, sb_complex beta);
/* Discontinuous linear Tri3 basis: build_tbem_system_linear (crates/sonium-bem/src/core/assembly/
 * tbem.rs:1490-1620) with regular_integration_linear (integration/regular.rs:337-470) and
 * singular_integration_linear (integration/singular.rs:719-1170). Every element carries three
 * DOFs, DOF 3e + c collocated at local point c of (1/6, 1/6), (2/3, 1/6), (1/6, 2/3)
 * (mesh/element.rs:91-99) with the element normal, basis 2 lambda_c - 1/3 (element.rs:229-236);
 * the operator is 3m x 3m complex128 (SB_PRECISION_FP64). Boundary conditions as sb_mesh_set_bc,
 * without prescribed values (rigid, zero-pressure and admittance surfaces): a mesh with nonzero
 * prescribed values gives SB_ERR_INVALID_ARGUMENT. sb_assemble_into re-assembles it at another
 * frequency; sb_rhs_plane_wave_device evaluates the incident field at its collocation points. */
#define SB_BASIS_CONSTANT 0
#define SB_BASIS_LINEAR 1
#define SB_BASIS_QUADRATIC 2
SB_API int sb_assemble_linear(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta,
                              sb_operator** out);
/* build_tbem_system_linear_stabilized / build_tbem_system_quadratic_stabilized (tbem.rs:2993-3030
 * -> build_tbem_system_discontinuous_stabilized :2810-2990): the same assembly for
 * SB_BASIS_LINEAR or SB_BASIS_QUADRATIC (six DOFs per element, DOF 6e + c collocated at the
 * six interior points of element.rs:108-115, quadratic Lagrange basis), every matrix entry
 * multiplied by sign (+1 or -1); pass beta = burton_miller_beta_scaled(beta_scale). */
SB_API int sb_assemble_discontinuous(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta,
                                     int basis, double sign, sb_operator** out);
/* Collocation points and normals of a basis (host arrays, DOF-major x 3): m of them for
 * SB_BASIS_CONSTANT (the centroids), 3m for SB_BASIS_LINEAR, 6m for SB_BASIS_QUADRATIC. */
SB_API int sb_mesh_collocation(const sb_mesh* mesh, int basis, double* points, double* normals);
/* IncidentField::compute_rhs_with_beta (incident.rs:807-833) for plane waves at np arbitrary
 * collocation points with normals (host arrays np x 3), on the device: rhs[i * r + q]. */
SB_API int sb_rhs_plane_wave_points(int device, int64_t np, const double* points, const double* normals,
                                    const sb_physics* physics, sb_complex beta, const double* dirs,
                                    const sb_complex* amps, int64_t r, sb_complex* rhs);

/* DenseMatrixOperator over a caller's matrix (crates/sonium-bem/src/core/bem_solver.rs:6548-6590:
 * the LinearOperator<Complex64> of any dense row-major matrix): matrix is n x n complex128,
 * row-major, copied to the device. SB_PRECISION_FP64 keeps it in complex128, SB_PRECISION_FP64_FP32
 * adds the complex64 copy of the mixed solver, SB_PRECISION_FP32 keeps only the complex64 copy.
 * The operator has no mesh: sb_assemble_into and sb_rhs_plane_wave_device return
 * SB_ERR_INVALID_ARGUMENT for it, its boundary-condition right-hand side is zero; the products,
 * the preconditioner and every solver accept it. Non-finite entries: SB_ERR_NOT_FINITE. */
SB_API int sb_operator_from_dense(int device, int64_t n, const sb_complex* matrix, int precision,
                                  sb_operator** out);
SB_API int sb_operator_destroy(sb_operator* op);
SB_API int sb_operator_info_get(const sb_operator* op, sb_operator_info* info);
/* TbemSystem { matrix, rhs } (tbem.rs:134-150) copied to host; either pointer may be NULL. */
SB_API int sb_operator_copy_to_host(const sb_operator* op, sb_complex* matrix, sb_complex* rhs);
SB_API int sb_operator_copy_rows_to_host(const sb_operator* op, int64_t row0, int64_t row1,
                                         sb_complex* rows);
SB_API int sb_operator_copy_to_host_c64(const sb_operator* op, sb_complex32* matrix);

/* LinearOperator<Complex64> (traits.rs:2949-3120) over DenseMatrixOperator
 * (crates/sonium-bem/src/core/bem_solver.rs:6548-6590): apply_into (y = A x),
 * apply_transpose_into (y = A^T x), Hermitian (y = A^H x) and apply_block (Y = A X, X/Y row-major
 * n x r). Host buffers; non-finite input or output returns SB_ERR_NOT_FINITE (try_apply). */
#define SB_OP_N 0
#define SB_OP_T 1
#define SB_OP_C 2
SB_API int sb_operator_apply(const sb_operator* op, int trans, const sb_complex* x,
                             sb_complex* y);
SB_API int sb_operator_apply_block(const sb_operator* op, const sb_complex* X, sb_complex* Y,
                                   int64_t r);
/* Same on device pointers (n complex128 each), on the operator's stream, synchronised. */
SB_API int sb_operator_apply_device(const sb_operator* op, int trans, const sb_complex* x_dev,
                                    sb_complex* y_dev);

/* Same product without any device allocation. This entry point has no counterpart in the
 * reference: it serves callers that must not call cudaMalloc / cudaFree, such as a host that has
 * already given the GPU's memory to its own pool (a driver allocation would fail or fragment it)
 * or one that keeps other streams busy and cannot take the device-wide wait of cudaFree. The
 * partial sums of op(A) x live in one fixed 8 MiB device array per GPU, held until the process
 * exits, so n is limited to 524288 (larger operators: SB_ERR_INVALID_ARGUMENT). The first call on
 * a device looks that array's address up once; make it before any stream capture. All calls on a
 * device share the array: calls whose kernels overlap on the GPU race. */
SB_API int sb_operator_apply_device_noalloc(const sb_operator* op, int trans,
                                            const sb_complex* x_dev, sb_complex* y_dev);

/* Preconditioner<Complex64>::apply_into (traits.rs:3645-3720): identity or Jacobi (A_ii^-1).
 * SB_PRECOND_BLOCK_JACOBI (no reference counterpart; the interface is the same apply_into):
 * y = M^-1 x with M the block diagonal of the complex128 matrix in blocks of the size set by
 * sb_operator_set_block_jacobi_size (default 128) spatially close elements (consecutive in the
 * Morton order of the element centroids; index order without a mesh), each block rounded to
 * complex64 and inverted on the device (Gauss-Jordan with partial pivoting, FP32; a singular
 * block keeps the identity) after each assembly, applied with FP64 vectors and accumulation.
 * Needs the complex128 matrix. */
#define SB_PRECOND_IDENTITY 0
#define SB_PRECOND_JACOBI 1
#define SB_PRECOND_BLOCK_JACOBI 2
SB_API int sb_preconditioner_apply(const sb_operator* op, int precond, const sb_complex* x,
                                   sb_complex* y);
/* Block size (32, 64, 96 or 128) of SB_PRECOND_BLOCK_JACOBI and of the block-Jacobi inner
 * preconditioner of sb_gmres_mixed (no reference counterpart). */
SB_API int sb_operator_set_block_jacobi_size(sb_operator* op, int block_size);

/* IncidentField::compute_rhs_with_beta for plane waves (incident.rs:216-245,315-331,807-833):
 * rhs[i*r+q] = -(gamma p_inc + beta tau dp_inc/dn) at the element centroids, for r directions
 * dirs[q] (unit vectors) with amplitudes amps[q] (NULL = 1). */
SB_API int sb_rhs_plane_wave(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta,
                             const double* dirs, const sb_complex* amps, int64_t r,
                             sb_complex* rhs);

/* ---- GMRES ---- */
/* GmresConfig (gmres.rs:26-47): max_iterations counts restart cycles, restart is the Krylov
 * dimension, tolerance is relative to ||b||. */
typedef struct sb_gmres_config {
    int64_t max_iterations;
    int64_t restart;
    double tolerance;
    int64_t convergence_check_interval;
} sb_gmres_config;

/* GmresSolution (gmres.rs:93-118). status: SB_SOLVER_* below. */
#define SB_SOLVER_CONVERGED 0
#define SB_SOLVER_MAX_ITERATIONS 1
#define SB_SOLVER_BREAKDOWN 2
#define SB_SOLVER_NUMERICAL_ERROR 3
typedef struct sb_gmres_stats {
    int64_t iterations;         /* Krylov steps (outer + inner for the mixed solver) */
    int64_t restarts;
    int64_t matvecs;            /* all operator applications incl. residual checks */
    int64_t matvecs_fp32;       /* of which on the complex64 copy (mixed solver) */
    int64_t refinements;        /* FP64 refinement steps (mixed solver) */
    double residual;            /* ||b - A x|| / ||b|| with the complex128 operator */
    double estimated_residual;
    double backward_error;
    double device_ms;           /* device time of the solve */
    int32_t converged;
    int32_t status;
} sb_gmres_stats;

/* gmres / gmres_preconditioned (gmres.rs:286-305, 631-1047, finalize 159-247) with CGS + one
 * DGKS pass (0.707), Givens on the host in FP64. b, x0 (NULL = 0) and x are host buffers.
 * precond: SB_PRECOND_IDENTITY, SB_PRECOND_JACOBI (left, as gmres_preconditioned) or
 * SB_PRECOND_BLOCK_JACOBI (right: GMRES on (A M^-1) z = b - A x0, x = x0 + M^-1 z; convergence is
 * tested on b - A x relative to ||b|| as without a preconditioner). */
SB_API int sb_gmres(const sb_operator* op, const sb_complex* b, const sb_complex* x0,
                    const sb_gmres_config* cfg, int precond, sb_complex* x, sb_gmres_stats* stats);
/* Same with device-resident b / x (x holds x0 on entry when x0_given != 0). */
SB_API int sb_gmres_device(const sb_operator* op, const sb_complex* b_dev, sb_complex* x_dev,
                           int x0_given, const sb_gmres_config* cfg, int precond,
                           sb_gmres_stats* stats);

/* Mixed-precision iterative refinement (the FGMRES-IR precedent of crates/sonium-compute/src/
 * gmres_ir.rs:1-80, 665): an FP64 outer loop r = b - A x on the complex128 matrix, an inner
 * GMRES on the complex64 copy with FP32 vectors and FP32-accumulated products (Hessenberg /
 * Givens in FP64), x += d in FP64. Needs an SB_PRECISION_FP64_FP32 operator. */
typedef struct sb_ir_config {
    int64_t max_refinements;
    double tolerance;            /* outer relative residual target */
    int64_t inner_restart;
    int64_t inner_max_iterations;
    double inner_tolerance;
} sb_ir_config;
SB_API int sb_gmres_mixed(const sb_operator* op, const sb_complex* b, const sb_complex* x0,
                          const sb_ir_config* cfg, sb_complex* x, sb_gmres_stats* stats);
/* Matrix of the inner GMRES of sb_gmres_mixed (no reference counterpart: a storage choice of this
 * library). SB_INNER_FP32 (default): the complex64 copy. SB_INNER_FP16: a complex-half copy of the
 * complex64 matrix (real and imaginary parts times one power-of-two scale s, chosen so that the
 * largest part maps to [2^13, 2^14), rounded to FP16; products divide by s exactly), built on the
 * device on the first mixed solve after each assembly. The inner products read 4 bytes per entry
 * instead of 8; the outer residual stays on the complex64 (or complex128) matrix with FP64
 * vectors, so the converged solution is that of the complex64 system, as with SB_INNER_FP32. The
 * copy perturbs the inner operator by about 2^-11 of each entry, so each refinement gains about
 * three digits: inner_tolerance near 1e-3 avoids inner iterations that cannot pay. Needs an
 * operator with a complex64 matrix (SB_PRECISION_FP64_FP32 or SB_PRECISION_FP32). */
#define SB_INNER_FP32 0
#define SB_INNER_FP16 1
SB_API int sb_operator_set_inner_precision(sb_operator* op, int inner);
/* Right preconditioner of sb_gmres_mixed's inner GMRES (no reference counterpart: an inner-solver
 * choice of this library; the reference's preconditioner interface is Preconditioner::apply_into,
 * crates/sonium-solvers/crates/sonium-solvers-core/src/traits.rs:3645). SB_INNER_PRECOND_NONE
 * (default) or SB_INNER_PRECOND_BLOCK_JACOBI: the unknowns in blocks of block_size (32, 64, 96 or 128)
 * spatially close elements (consecutive in the Morton order of the element centroids; index
 * order for an operator without a mesh or with a discontinuous basis), each diagonal block of the
 * complex64 matrix inverted on the device (Gauss-Jordan with partial pivoting, FP32; a singular
 * block keeps the identity) on the first mixed solve after each assembly. The inner solve works
 * on A M^-1 and the correction is M^-1 y, so the outer refinement and the converged solution are
 * unchanged; fewer inner iterations are needed. Needs a complex64 matrix. */
#define SB_INNER_PRECOND_NONE 0
#define SB_INNER_PRECOND_BLOCK_JACOBI 1
SB_API int sb_operator_set_inner_preconditioner(sb_operator* op, int kind, int block_size);
SB_API int sb_gmres_mixed_device(const sb_operator* op, const sb_complex* b_dev,
                                 sb_complex* x_dev, int x0_given, const sb_ir_config* cfg,
                                 sb_gmres_stats* stats);

/* GCRO-DR: Krylov subspace recycling across a sequence of related systems (consecutive
 * frequencies of a sweep). gcro_dr / gcro_dr_preconditioned (crates/sonium-solvers/crates/
 * sonium-solvers-iterative/src/gcro_dr.rs:164-260, core :339-760) with the recycled subspace of
 * GcroDrSubspace (:65-110): a subspace keeps up to k orthonormal vectors U (k = its target size,
 * 0..100) on one device. Each solve rebuilds C = orth(M^-1 A U) for the operator it is given
 * (k extra products; columns whose projected norm falls below 1e-12 are dropped, as build_c_r
 * :769-850), runs restarted Arnoldi cycles of the restart length whose vectors are projected
 * against C twice before CGS + DGKS against the cycle basis, tests convergence every step and
 * the exact residual when a cycle claims convergence, and on an accepted solution (or after the
 * last cycle without one) replaces U by the harmonic Ritz vectors of smallest magnitude of the
 * augmented (k + m) problem (update_recycled_subspace :922-1050). An empty subspace gives plain
 * GMRES with a convergence check every step. cfg as sb_gmres (max_iterations = restart cycles;
 * convergence_check_interval is not used). stats: iterations, restarts, matvecs (incl. the
 * rebuild of C and residual checks), residual = backward_error = exact relative residual.
 * A subspace holding vectors of another length than the operator's n gives
 * status SB_SOLVER_NUMERICAL_ERROR (x = x0) without touching it. Host entry: b, x0 (NULL = 0), x
 * host buffers; non-finite b or x0 return SB_ERR_NOT_FINITE before any device work. */
typedef struct sb_gcro_subspace sb_gcro_subspace;
SB_API int sb_gcro_subspace_create(int device, int64_t k, sb_gcro_subspace** out);
SB_API int sb_gcro_subspace_destroy(sb_gcro_subspace* s);
/* GcroDrSubspace::reset: drop every vector (the next solve seeds a fresh subspace). */
SB_API int sb_gcro_subspace_reset(sb_gcro_subspace* s);
/* num_vectors held now, target size, vector length (0 while empty); any pointer may be NULL. */
SB_API int sb_gcro_subspace_info(const sb_gcro_subspace* s, int64_t* num_vectors, int64_t* target,
                                 int64_t* n);
/* The held vectors to host memory (num_vectors x n, vector i at u + i * n) and back (the
 * validated checkpoint round trip of GcroDrSubspace::vectors / replace_vectors, :98-110; count <=
 * target, finite entries; the vectors are taken as given, orthonormal ones expected). */
SB_API int sb_gcro_subspace_get_vectors(const sb_gcro_subspace* s, sb_complex* u);
SB_API int sb_gcro_subspace_set_vectors(sb_gcro_subspace* s, int64_t count, int64_t n,
                                        const sb_complex* u);
SB_API int sb_gcro_dr(const sb_operator* op, const sb_complex* b, const sb_complex* x0,
                      sb_gcro_subspace* s, const sb_gmres_config* cfg, int precond, sb_complex* x,
                      sb_gmres_stats* stats);
/* Same with device-resident b / x (x holds x0 on entry when x0_given != 0). */
SB_API int sb_gcro_dr_device(const sb_operator* op, const sb_complex* b_dev, sb_complex* x_dev,
                             int x0_given, sb_gcro_subspace* s, const sb_gmres_config* cfg,
                             int precond, sb_gmres_stats* stats);

/* Plane-wave RHS written to device memory (n x r complex128) on the operator's stream. */
SB_API int sb_rhs_plane_wave_device(const sb_operator* op, const double* dirs,
                                    const sb_complex* amps, int64_t r, sb_complex* rhs_dev);

/* ---- exterior field ----
 * compute_scattered_field_checked (crates/sonium-bem/src/core/postprocess/pressure.rs:250-289 ->
 * compute_scattered_field_with_incident :1388-1448, integrate_element_field :1566-1606 with the
 * 7-point triangle rule, integrate_quad_point :1987-2042): the scattered pressure at m points
 * (points: m x 3) from the constant surface pressure (n values, e.g. the solution of a rigid or
 * admittance problem) and the surface normal velocity (n values, NULL = rigid). FP64. Add the
 * incident field for the total field (compute_total_field_checked, :501). Points on the surface
 * give a non-finite result (SB_ERR_NOT_FINITE), as the reference's checked form. */
SB_API int sb_field_eval(const sb_mesh* mesh, const sb_physics* physics, const sb_complex* surface_pressure,
                         const sb_complex* surface_velocity, const double* points, int64_t m, sb_complex* field);

/* ---- tensor-core block product ----
 * The block product of LinearOperator::apply_block (crates/sonium-solvers/crates/
 * sonium-solvers-core/src/traits.rs:2949-3120 -> DenseMatrix::matmul_into, dense.rs:450-490) as
 * used by block GMRES (crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:
 * 163), on the tensor cores: every real operand is split into two BF16 terms (hi + lo, 16
 * significant bits) and the three leading cross products are accumulated in FP32, so each entry
 * of Y = A X carries a relative error of order 1e-5 of the row's magnitude (not an FP64
 * product: sb_operator_apply_block is the exact one). prepare builds the split planes of the
 * operator's matrix (4 N^2 * 2 bytes); re-assembly drops them. apply: x and y hold r complex64
 * vectors of length n, vector c at x + c * n (host memory). */
SB_API int sb_operator_prepare_block_tensor(sb_operator* op);
SB_API int sb_operator_apply_block_tensor(const sb_operator* op, const sb_complex32* x, sb_complex32* y, int64_t r);
/* Device-resident variant: x_dev and y_dev hold vector c at + c * n (complex64), on the operator's
 * device; the product runs on the operator's stream and is complete on return. */
SB_API int sb_operator_apply_block_tensor_device(const sb_operator* op, const sb_complex32* x_dev,
                                                 sb_complex32* y_dev, int64_t r);

/* ---- FP64-grade block residual ----
 * R = B - A X for r right-hand sides on the operator's complex128 matrix: the block residual of
 * block GMRES (crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:829 and
 * block_true_metrics :571-620, one FP64 complex GEMM there) on the INT8 tensor cores. Every row
 * of A and every vector is split into 8 signed 8-bit slices of a power-of-two scale (exact to
 * 2^-56 of the scale); the slice products are exact in INT32 and summed by diagonal in FP64, 36
 * of the 64 kept: per term an error below 9.05 * 2^-56 of (row scale x vector scale), the size of
 * an FP64 rounding of a term near the largest entries (not bit-identical to an FP64 GEMM). The
 * operator must hold the complex128 matrix; its slices (8 x 2 N^2 bytes) are built on first use
 * and dropped by re-assembly. Host variant: b, x, res n x r row-major (b[i * r + c]). */
SB_API int sb_operator_block_residual(const sb_operator* op, const sb_complex* b, const sb_complex* x, int64_t r,
                                      sb_complex* res);
/* Device-resident variant: vector c at + c * n (complex128), on the operator's device; complete on
 * return. */
SB_API int sb_operator_block_residual_device(const sb_operator* op, const sb_complex* b_dev, const sb_complex* x_dev,
                                             int64_t r, sb_complex* res_dev);

/* Many right-hand sides of one operator (the role of block_gmres_preconditioned,
 * crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:163, called via
 * solve_compressed_many, bem_solver.rs:4072-4110): r systems A x_c = b_c solved in lockstep by
 * FP32-inner GMRES with FP64 refinement, every right-hand side with its own Krylov basis and
 * convergence state (the reference's block method shares one basis across right-hand sides; this
 * one shares the products instead). Each step's products for all right-hand sides are one
 * tensor-core block product (the BF16 split of sb_operator_apply_block_tensor); the refinement
 * residual of all of them is one sb_operator_block_residual on the complex128 matrix, so the
 * operator must hold it (SB_PRECISION_FP64 or SB_PRECISION_FP64_FP32). The split planes are built on first use. b and
 * x: n x r row-major (b[i * r + c], the reference's DenseMatrix block layout); stats: r entries,
 * the sb_gmres_mixed statistics per right-hand side (device_ms = the whole block's time). */
SB_API int sb_gmres_multi(const sb_operator* op, const sb_complex* b, int64_t r, const sb_ir_config* cfg,
                          sb_complex* x, sb_gmres_stats* stats);
/* Device-resident variant: b_dev and x_dev hold right-hand side c at + c * n (complex128). */
SB_API int sb_gmres_multi_device(const sb_operator* op, const sb_complex* b_dev, int64_t r,
                                 const sb_ir_config* cfg, sb_complex* x_dev, sb_gmres_stats* stats);

/* ---- batched frequency sweep ----
 * Replaces the reference's per-frequency loop (crates/sonium-bem/src/core/solver/
 * frequency_sweep.rs:541-600: build_tbem_system_stabilized at :20, then one GMRES solve per
 * frequency) for many independent instances (mesh, physics, beta) on one device: one persistent
 * assembly launch writes every instance's complex64 matrix (the SB_PRECISION_FP32 arithmetic of
 * sb_assemble), and one batched mixed-precision solve (the sb_gmres_mixed algorithm and
 * statistics per instance, zero initial guess) advances all instances in lockstep, each with its
 * own convergence state. Meshes must carry no prescribed boundary values (rigid or admittance
 * surfaces; the right-hand side is an incident field): SB_ERR_INVALID_ARGUMENT otherwise. The
 * meshes must outlive the batch. */
typedef struct sb_batch sb_batch;
SB_API int sb_batch_create(int64_t count, sb_mesh* const* meshes, const sb_physics* physics,
                           const sb_complex* betas, sb_batch** out);
SB_API int sb_batch_destroy(sb_batch* batch);
SB_API int sb_batch_assemble(sb_batch* batch);
/* Incident plane wave of unit amplitude along `direction` (3 doubles) for every instance. */
SB_API int sb_batch_set_rhs_plane_wave(sb_batch* batch, const double* direction);
/* Right-hand side of one instance from host memory (n complex128). */
SB_API int sb_batch_set_rhs(sb_batch* batch, int64_t index, const sb_complex* b);
/* stats: count entries, one per instance (device_ms is the whole batch's time). */
SB_API int sb_batch_solve(sb_batch* batch, const sb_ir_config* cfg, sb_gmres_stats* stats);
/* Matrix of the batched inner products, as sb_operator_set_inner_precision: SB_INNER_FP32 (the
 * complex64 matrices, default) or SB_INNER_FP16 (complex-half copies of every instance's matrix,
 * each with its own power-of-two scale, built on the device by the first solve after each
 * sb_batch_assemble and counted in its time; 4 bytes per entry of extra device memory). */
SB_API int sb_batch_set_inner_precision(sb_batch* batch, int inner);
/* Block-Jacobi right preconditioner of the batched inner solves, as
 * sb_operator_set_inner_preconditioner: every instance's blocks of its own Morton order, inverted
 * on the device by the first solve after each sb_batch_assemble (counted in its time). */
SB_API int sb_batch_set_inner_preconditioner(sb_batch* batch, int kind, int block_size);
SB_API int sb_batch_solution(const sb_batch* batch, int64_t index, sb_complex* x);
/* The assembled complex64 matrix of one instance, row-major n x n. */
SB_API int sb_batch_matrix_c64(const sb_batch* batch, int64_t index, sb_complex32* matrix);
/* Assembly form of sb_batch_assemble (no reference counterpart: the execution choice of this
 * implementation). SB_BATCH_ASM_PERSISTENT: persistent CTAs walk flattened work lists of every
 * instance's far tiles, near pairs and self terms, either as one launch (each CTA alternating far
 * tiles with near / self items) or as two persistent launches side by side (the far tiles on some
 * of each SM's CTA slots, the near / self items on the others; sb_batch_assembly_split).
 * SB_BATCH_ASM_STREAMS: per-instance far kernels on the batch's stream with the near and self
 * kernels on a second, higher-priority stream beside them. All run the same device functions and
 * write the same entries. SB_BATCH_ASM_AUTO (default): the first assembly of a batch shape
 * (device, unknowns and near pairs per instance) runs one untimed assembly, then times the
 * persistent layouts and the streams form once each, keeps the fastest for every later batch of
 * that shape in the process, and reports the times through sb_batch_assembly_tuning and
 * sb_batch_assembly_split. */
#define SB_BATCH_ASM_AUTO 0
#define SB_BATCH_ASM_PERSISTENT 1
#define SB_BATCH_ASM_STREAMS 2
SB_API int sb_batch_set_assembly_mode(sb_batch* batch, int mode);
/* The form the last sb_batch_assemble used, and the autotuner's measurements of the two forms in
 * milliseconds (0 when this batch did not run the autotuner). Any pointer may be NULL. */
SB_API int sb_batch_assembly_tuning(const sb_batch* batch, int* chosen, double* persistent_ms,
                                    double* streams_ms);
/* The persistent form's layout: far CTA slots per SM when it runs as two persistent launches (the
 * far tiles of every instance on those slots, the near pairs and self terms on the SM's other slots,
 * or, with all slots, on the slots the far launch frees at its end; 0 = one launch alternating
 * both), and in layout_ms[0..4] (may be NULL) the autotuner's times of the one-launch layout (index
 * 0) and of far tiles on 2, 3 and 4 slots (indices 2..4; 0 when it did not run). No counterpart in
 * the reference (its sweep assembles one frequency after another). */
SB_API int sb_batch_assembly_split(const sb_batch* batch, int* far_slots_per_sm, double* layout_ms);
/* Device time of the last sb_batch_assemble and sb_batch_solve, milliseconds. */
SB_API int sb_batch_timings(const sb_batch* batch, double* assembly_ms, double* solve_ms);

/* ---- device memory (no reference counterpart: the allocator of this implementation) ----
 * Device buffers of meshes, operators, solvers and batches come from a per-device cache of
 * released blocks of the same size (rounded to 2 MiB, or 512 B below 1 MiB) before cudaMalloc is
 * asked; a released block enters the cache after a device synchronisation (as cudaFree waits)
 * while the cache holds at most 96 GiB per device, and an allocation that fails empties the
 * cache and retries. The solver workspaces of destroyed operators (vectors, pinned host memory,
 * captured cycle graphs) are likewise kept, four per process, for the next operator of the same
 * size. trim frees the kept workspaces and returns every cached block of a device (device < 0:
 * all devices) to the driver; stats reports the bytes held by live buffers (kept workspaces
 * included) and by the cache. */
SB_API int sb_memory_trim(int device);
SB_API int sb_memory_stats(int device, int64_t* in_use_bytes, int64_t* cached_bytes);

/* ---- timing (no reference counterpart: instrumentation, the PerfModel / runtime-stats role of
 * crates/sonium-compute/src/perf.rs:1-30) ---- */
/* Kernel classes timed by CUDA events recorded on their launching stream when profiling is on. */
#define SB_PROF_FAR 0        /* far-field assembly tiles */
#define SB_PROF_NEAR 1       /* near-pair subdivision kernel */
#define SB_PROF_SELF 2       /* self (singular) kernel */
#define SB_PROF_GEMV64 3     /* complex128 matvec (incl. fused residual) */
#define SB_PROF_GEMV32 4     /* complex64 matvec (FP32 or FP64 vectors) */
#define SB_PROF_ARNOLDI 5    /* Gram-Schmidt dots / projections / basis updates */
#define SB_PROF_OTHER 6      /* geometry, coefficients, RHS reductions, plane waves */
#define SB_PROF_TENSOR 7     /* tensor-core block product (BF16 split, tcgen05) */
#define SB_PROF_GEMV16 8     /* complex-half matvec of the FP16 inner solve (incl. its copy) */
#define SB_PROF_RESIDUAL 9   /* integer-slice FP64 block residual (INT8 slices, tcgen05 kind::i8) */
#define SB_PROF_KINDS 10
typedef struct sb_profile {
    double ms[SB_PROF_KINDS];
    int64_t launches[SB_PROF_KINDS];
    int64_t kernels; /* all kernels launched by the library (counted whether profiling is on or not) */
} sb_profile;
SB_API int sb_profile_enable(int on);
/* Profile only the kernel classes whose bit (1 << SB_PROF_*) is set in mask (0 = off): timing one
 * class adds fewer event records to the work it measures. */
SB_API int sb_profile_enable_classes(unsigned mask);
/* Totals since the last reset (synchronises the recorded events); reset != 0 clears them. */
SB_API int sb_profile_read(sb_profile* out, int reset);
/* FP32 fused multiply-add rate of `device` in TFLOP/s (2 flop per lane and FMA), measured by a
 * kernel of 8 independent FMA chains per thread on every SM, scalar (fmaf) and packed (sm_100's
 * f32x2 FMA): the denominator of the FP32 far-field kernel's roofline. No reference counterpart. */
SB_API int sb_measure_fp32_rate(int device, double* scalar_tflops, double* packed_tflops);
/* CUDA event helpers on an operator's stream, for timing whole solves on the device. */
SB_API int sb_event_create(void** event);
SB_API int sb_event_destroy(void* event);
SB_API int sb_event_record(void* event, const sb_operator* op);
SB_API int sb_event_elapsed_ms(void* start, void* stop, float* ms);

/* ---- diagnostics ---- */
/* The device sine/cosine used by every kernel phase exp(i k r) (the reference's exp_i,
 * crates/sonium-fastmath/src/api.rs:450-456): s[i] = sin(x[i]), c[i] = cos(x[i]) computed on
 * `device`, for testing it against golden values. */
SB_API int sb_math_sincos(int device, const double* x, int64_t n, double* s, double* c);

/* ---- fault injection (tbem.rs:6740-6794, injection point crates/sonium-compute/src/cuda/
 * cublas.rs:3128): the next library call that reaches `point` fails with SB_ERR_INJECTED
 * before any device work, releasing its transient buffers. ---- */
#define SB_INJECT_NONE 0
#define SB_INJECT_ALLOC 1
#define SB_INJECT_LAUNCH 2
SB_API int sb_inject_failure(int point);

#ifdef __cplusplus
}
#endif
#endif
