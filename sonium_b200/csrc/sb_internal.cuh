// Internal declarations shared by the sonium-b200 CUDA sources (not part of the C ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/sonium_b200.h"

namespace sb {

// ---------------------------------------------------------------------------------------------
// Error handling: every entry point converts failures into an sb status plus a message that
// sb_last_error() returns. Nothing throws across the C ABI.
// ---------------------------------------------------------------------------------------------
struct Error {
    int status;
    std::string msg;
};

void set_error(int status, const std::string& msg);
void clear_error();

// Runs the body of a C-ABI entry point and turns whatever it throws into a status code with its
// message: Error as raised, a failed host allocation as SB_ERR_OUT_OF_MEMORY, any other standard
// exception as SB_ERR_CUDA with its what().
template <class F>
int abi_guard(F&& f) {
    try {
        clear_error();
        f();
        return SB_OK;
    } catch (const Error& e) {
        set_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_error(SB_ERR_OUT_OF_MEMORY, "host allocation failed");
        return SB_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_error(SB_ERR_CUDA, e.what());
        return SB_ERR_CUDA;
    } catch (...) {
        set_error(SB_ERR_CUDA, "unknown failure");
        return SB_ERR_CUDA;
    }
}

#define SB_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            throw ::sb::Error{SB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
        }                                                                                    \
    } while (0)

#define SB_REQUIRE(cond, status, msg)                        \
    do {                                                     \
        if (!(cond)) throw ::sb::Error{(status), (msg)};     \
    } while (0)

// Number of kernels this library has launched (reported by sb_profile_read).
void count_launch();

// Host fault injection (points from the header's SB_INJECT_* values).
extern int g_inject_point;
void maybe_inject(int point);

// Device memory with ownership; allocation failures surface as SB_ERR_OUT_OF_MEMORY. Blocks come
// from a per-device cache of released blocks of the same rounded size when one is free (a
// released block enters the cache after a device synchronisation, as cudaFree would wait), and
// from cudaMalloc otherwise; an allocation that fails empties the cache and retries once.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;  // requested size
    size_t cap = 0;    // rounded size of the block
    int dev = -1;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void alloc(size_t n);
    void release();
    void swap(DevBuf& o) {
        std::swap(p, o.p);
        std::swap(bytes, o.bytes);
        std::swap(cap, o.cap);
        std::swap(dev, o.dev);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};
// Host-to-device copy / device memset on the legacy default stream that are complete on return.
// The legacy stream does not order work on the library's non-blocking streams, and a copy from
// pageable host memory may return before its DMA has landed, so every upload or fill that a
// kernel on another stream reads goes through these.
void h2d_sync(void* dst, const void* src, size_t bytes);
void memset_sync(void* dst, int value, size_t bytes);
// Frees every cached block of `device` (all devices when device < 0).
void memory_trim(int device);
// Bytes held by live DevBufs and by the cache on `device`.
void memory_stats(int device, int64_t* in_use, int64_t* cached);

// ---------------------------------------------------------------------------------------------
// Quadrature tables in constant memory (uploaded once per device by ensure_tables()).
// ---------------------------------------------------------------------------------------------
constexpr int kMaxGL = 8;              // Gauss-Legendre orders 1..8
constexpr int kGLTotal = kMaxGL * (kMaxGL + 1) / 2;
constexpr int kTriOrders = 4;          // regular leaf orders 4..7
constexpr int kTriTotal = 13 + 25 + 36 + 49;
constexpr int kFarPoints = 13;         // order-4 rule: the far-field single leaf

void ensure_tables(int device);
void host_gauss_legendre(int n, double* x, double* w);
// Triangle rule of leaf order `order` (4..7) as (xi, eta, w) with weights summing to 0.5.
int host_triangle_rule(int order, double* xi, double* eta, double* w);

// ---------------------------------------------------------------------------------------------
// Device-resident mesh
// ---------------------------------------------------------------------------------------------
// Element record fields in the SoA `elem` array: elem[f * ld + e].
enum ElemField {
    EV0X = 0, EV0Y, EV0Z, EV1X, EV1Y, EV1Z, EV2X, EV2Y, EV2Z,  // vertices
    ECX, ECY, ECZ,                                          // centroid (collocation point)
    ENX, ENY, ENZ,                                          // unit normal
    EAREA, EJAC,                                            // area, |dx/ds x dx/dt|
    EGX, EGY, EGZ,                                          // level-0 subdivision centre
    ESQA,                                                   // sqrt(area)
    EV3X, EV3Y, EV3Z,                                       // fourth vertex (Quad4 meshes)
    EFIELDS
};

constexpr int kFarTile = 128;  // field elements per far-kernel column tile

struct Mesh {
    int device = 0;
    int64_t n = 0, n_nodes = 0, ld = 0, n_tiles = 0;
    double coord_bound = 0.0;  // largest |coordinate| of the nodes (bounds FP32 rounding of positions)
    std::vector<double> h_nodes;
    std::vector<uint32_t> h_tris;
    // host copy of the element SoA (ld stride), read back on first use (mesh_host_elem)
    mutable std::vector<double> h_elem;
    mutable std::mutex h_elem_mu;
    DevBuf nodes, tris, elem, qp, qp32;
    // near-pair CSR (superset of the reference's subdivision criterion; excludes the diagonal)
    int64_t nnz = 0;
    DevBuf near_ptr, near_col, near_row;  // near_row: the row of each near pair
    // The near pairs' recorded subdivision leaves (geometry only), built on the mesh's second
    // near-pair assembly when memory allows; near_plan_off has nnz + 1 entries.
    DevBuf near_plan, near_plan_off;
    int near_assemblies = 0;
    bool near_plan_ready = false, near_plan_declined = false;
    std::mutex near_plan_mu;
    // Quad4 meshes: four vertices per element (EV0..EV3), far points of the 4 x 4 rule with their
    // normals, qq[(q * 7 + f) * ld + e] for f = x, y, z, w J, nx, ny, nz.
    bool quad = false;
    DevBuf qq;
    // boundary conditions
    std::vector<int32_t> h_bc_kind;
    std::vector<double> h_bc_value, h_adm;  // interleaved complex
    std::vector<uint8_t> h_has_adm;
    bool any_bc_value = false, any_adm = false;
    DevBuf bc_kind, bc_value, has_adm, adm;
};

// A second stream, of the device's highest priority, for work independent of the main stream's
// (the batched near-pair and self kernels beside the far-field tiles: they write disjoint matrix
// entries).
// begin() makes it wait for the main stream's work so far; end() makes the main stream wait for it.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    void ensure();
    void release();
    void begin(cudaStream_t main);
    void end(cudaStream_t main);
};

// ---------------------------------------------------------------------------------------------
// Device-resident operator (assembled TBEM system)
// ---------------------------------------------------------------------------------------------
struct Operator {
    Mesh* mesh = nullptr;
    int device = 0;
    int precision = SB_PRECISION_FP64;
    int64_t n = 0;
    sb_physics phys{};
    double beta_re = 0, beta_im = 0;
    int64_t lda32 = 0;           // even leading dimension of the complex64 copy
    DevBuf A64, A32, rhs, diag;  // rhs: BC-induced RHS (N complex); diag: A_ii for Jacobi
    DevBuf coef, far_part, near_rhs, self_rhs, scratch, status;
    void* work = nullptr;        // solver workspace (gmres.cu), released by destroy_solve_work
    void* tensor = nullptr;      // BF16 split planes for the tensor-core block product (tensor.cu)
    void* ozaki = nullptr;       // INT8 slices of the complex128 matrix for the block residual (ozaki.cu)
    void* multi = nullptr;       // many-right-hand-side solver workspace (batch.cu)
    // Discontinuous bases (n = 3 or 6 x elements): collocation points / normals (SoA) and the
    // near-pair CSR of the collocation rows.
    int basis = SB_BASIS_CONSTANT;
    double sign = 1.0;  // the stabilised discontinuous systems' sign (every entry times sign)
    DevBuf lin_cp, lin_cn, lin_ptr, lin_col;
    int64_t lin_nnz = 0;
    // Complex-half copy of the complex64 matrix for the inner solve of the mixed solver
    // (SB_INNER_FP16): FP16 (re, im) pairs of row i's entries times a power-of-two scale s_i,
    // rows lda16 entries apart; half_scale = [s (n floats), 1 / s (n floats)]; half_flag = 1 when
    // an entry the assembly converted left the FP16 range (checked by the first solve).
    int inner = SB_INNER_FP32;
    DevBuf A16, half_scale, half_flag;
    bool half_check = false;
    // Block-Jacobi preconditioner of the inner solve (SB_INNER_PRECOND_BLOCK_JACOBI): unknowns in
    // blocks of bj_size consecutive entries of bj_perm (Morton order of the element centroids),
    // the transposed inverses of the complex64 diagonal blocks in bj_inv (rebuilt after assembly).
    int inner_precond = SB_INNER_PRECOND_NONE;
    int bj_size = 128;
    DevBuf bj_perm, bj_inv, bj_status;
    bool bj_valid = false;
    // The FP64 solver's block-Jacobi right preconditioner (SB_PRECOND_BLOCK_JACOBI): the same
    // blocks of the complex128 matrix, inverted in FP32 (rebuilt after assembly).
    DevBuf bj64_inv;
    bool bj64_valid = false;
    // Near-pair and self kernels of the constant-basis Tri3 assembly run here, concurrently with
    // the far kernel (they write disjoint entries; the far kernel is FMA / special-function bound,
    // the near kernel FP64 and latency bound).
    SideStream side;
    int64_t lda16 = 0;
    bool half_valid = false;
    cudaStream_t stream = nullptr;
    double last_assembly_ms = 0.0;
};

// Batched assembly (assembly.cu): one persistent launch over all instances of a batch.
struct BatchAsmInst {
    const double* elem;
    const float* qp32;
    double coord_bound;  // the mesh's largest |coordinate| (FP32 near-pair margin test)
    const double* coef;
    double2* diag;
    float2* A32;
    int64_t n, ld, n_tiles, lda32;
    double k;
    const int64_t* near_ptr;
    const int32_t* near_col;
    const int32_t* near_row;
    int64_t nnz;
    unsigned* amax;  // when set: the largest |re|, |im| written (FP32 bits), for the complex-half copy
    Mesh* mesh;      // host side only: the instance's mesh (its recorded near-pair plan)
};
// The persistent form: one launch over every instance's far tiles, near pairs and self elements
// (far_per_sm = 0), or two persistent launches side by side, the far tiles on far_per_sm CTA slots
// per SM and the near / self items on the rest (side stream).
void assemble_batch(const std::vector<BatchAsmInst>& h_inst, const BatchAsmInst* d_inst, DevBuf& pre_buf,
                    cudaStream_t s, int device, SideStream* side = nullptr, int far_per_sm = 0);
// The same batch as per-instance launches: far tiles on s, near pairs and self terms on the side
// stream (same device functions, so the same entries).
// With amax, instance b's largest matrix part lands in amax[4 b] (float bits; the complex-half
// copies' scales then need no scan).
void assemble_batch_streams(const std::vector<BatchAsmInst>& h_inst, cudaStream_t s, SideStream& side,
                            unsigned* amax = nullptr);
void coefficients_for(const Mesh& m, const sb_physics& ph, double beta_re, double beta_im, double* coef,
                      cudaStream_t s);
int coefficient_fields();

// Assembly (assembly.cu)
void assemble(Operator& op, const sb_physics& ph, double beta_re, double beta_im);
// The discontinuous linear / quadratic bases (op.basis, op.sign).
void assemble_discontinuous(Operator& op, const sb_physics& ph, double beta_re, double beta_im);
// Collocation points / normals of a discontinuous basis (SoA, 3 x (NB n) device arrays).
void lin_collocation(const Mesh& m, int basis, double* cp_dev, double* cn_dev);
// Plane-wave right-hand side at np points with normals (SoA, component c of point i at c * stride
// + i), on the device.
void incident_plane_wave_at(int device, const double* pts_dev, const double* nrm_dev, int64_t np, int64_t stride,
                            const sb_physics& ph, double beta_re, double beta_im, const double* dirs_host,
                            const double* amps_host, int64_t r, double2* rhs_dev, cudaStream_t s);
void incident_plane_wave(const Mesh& m, const sb_physics& ph, double beta_re, double beta_im,
                         const double* dirs_host, const double* amps_host, int64_t r,
                         double2* rhs_dev, cudaStream_t s, bool accumulate);

void device_sincos(int device, const double* x, int64_t n, double* s, double* c);

// Mesh (assembly.cu)
Mesh* mesh_create(const double* nodes, int64_t n_nodes, const uint32_t* tris, int64_t n_tris,
                  int device);
Mesh* mesh_create_quad(const double* nodes, int64_t n_nodes, const uint32_t* quads, int64_t n_quads, int device);
void assemble_quad(Operator& op, const sb_physics& ph, double beta_re, double beta_im);
void mesh_set_bc(Mesh& m, const int32_t* kind, const sb_complex* value, const uint8_t* has_adm,
                 const sb_complex* adm);
// The element SoA on the host (EFIELDS x ld doubles), copied from the device on first use.
const std::vector<double>& mesh_host_elem(const Mesh& m);

enum class Trans { N = 0, T = 1, C = 2 };

// GMRES (gmres.cu)
void gmres_fp64(const Operator& op, const double2* b_dev, double2* x_dev, bool x0_given,
                const sb_gmres_config& cfg, int precond, sb_gmres_stats& st);
void gmres_mixed_ir(const Operator& op, const double2* b_dev, double2* x_dev, bool x0_given,
                    const sb_ir_config& cfg, sb_gmres_stats& st);

void destroy_solve_work(Operator& op);
// Frees the kept solver workspaces of `device` (all devices when device < 0).
void solve_work_pool_trim(int device);
struct Gate;
// Builds the complex-half copy of the complex64 matrix on the operator's stream, unless the FP32
// assembly wrote it (blas.cu); half_alloc sizes its buffers.
void half_prepare(Operator& op);
void half_alloc(Operator& op);
// Block-Jacobi inner preconditioner (precond.cu): build the block inverses; y = M^-1 x (FP32).
void bj_prepare(Operator& op);
void bj_apply(const Operator& op, const float2* x, float2* y, Gate g);
// The FP64 solver's block-Jacobi right preconditioner: inverses of the complex128 matrix's blocks;
// y = M^-1 x with FP64 vectors.
void bj64_prepare(Operator& op);
void bj64_apply(const Operator& op, const double2* x, double2* y, Gate g);
// Morton (Z-order) permutation of a mesh's element centroids (precond.cu).
std::vector<int32_t> element_morton_order(const Mesh& m);
// Products with FP64 vectors on whichever matrix the operator holds (gmres.cu).
void op_gemv64(const Operator& op, const double2* x, double2* y, Gate g);
void op_residual64(const Operator& op, const double2* x, const double2* b, double2* r, double* part);
int64_t op_residual64_partials(const Operator& op);  // entries op_residual64 writes to part

int device_sm_count(int device);

// Scattered field at m points from constant surface pressure / velocity (field.cu); device
// pointers, velocity may be null (rigid surface).
void field_eval(const Mesh& mesh, const sb_physics& ph, const double2* pressure, const double2* velocity,
                const double* points, int64_t m, double2* out, cudaStream_t s);

// Tensor-core block product (tensor.cu): BF16 hi/lo split planes of the operator's matrix, then
// Y = A X for r complex64 vectors (vector c at x + c * ldx, result at y + c * ldy).
void tensor_prepare(Operator& op);
void tensor_release(Operator& op);
// 2-D tiled TMA descriptor over rows x ldk elements of elem_bytes (row pitch ldk elements), box of
// box_rows x box_inner elements, with the given swizzle.
CUtensorMap make_tmap_2d(void* base, CUtensorMapDataType type, int elem_bytes, int64_t rows, int64_t ldk,
                         int box_inner, int box_rows, CUtensorMapSwizzle swizzle);
// R = B - A X for r complex128 vectors on the operator's complex128 matrix (ozaki.cu): integer
// slices on the INT8 tensor cores, FP64-grade; b_c at b + c * ldb, x_c at x + c * ldx, r_c at
// res + c * ldr. Builds the matrix slices on first use; tensor_release drops them.
void ozaki_residual(const Operator& op, const double2* b, int64_t ldb, const double2* x, int64_t ldx, int r,
                    double2* res, int64_t ldr, cudaStream_t s);
void ozaki_release(Operator& op);
int ozaki_status(const Operator& op, bool reset);
bool tensor_ready(const Operator& op);
// block_gate (optional, one int per group of kTensorRhsTile vectors): a group whose entry is 0
// is skipped; its results are unspecified (zero or left as they were).
constexpr int kTensorRhsTile = 128;
void tensor_block_product(const Operator& op, const float2* x, int64_t ldx, int r, float2* y, int64_t ldy,
                          cudaStream_t s, const int* block_gate = nullptr);
int tensor_status(const Operator& op, bool reset);
// Split planes for up to r vectors, allocated ahead of any stream capture.
void tensor_reserve(const Operator& op, int r);
// Changes whenever the planes (and so the tensor maps baked into captured graphs) change.
uint64_t tensor_generation(const Operator& op);

// Many right-hand sides of one operator (batch.cu): r systems solved in lockstep, products for all
// of them on the tensor cores, FP64 refinement residual by one complex128 GEMM.
void multi_solve_device(Operator& op, const double2* b, int64_t ldb, int r, double2* x, int64_t ldx,
                        const sb_ir_config& cfg, sb_gmres_stats* stats);
void multi_release(Operator& op);

// GCRO-DR with a recycled subspace kept across solves (gcro.cu).
struct RecycleSpace;
RecycleSpace* recycle_create(int device, int64_t k);
void recycle_destroy(RecycleSpace* s);
void recycle_reset(RecycleSpace& s);
void recycle_info(const RecycleSpace& s, int64_t* count, int64_t* target, int64_t* n);
void recycle_get(const RecycleSpace& s, double2* host);  // count x n, vector i at host + i * n
void recycle_set(RecycleSpace& s, int64_t count, int64_t n, const double2* host);
void gcro_dr(const Operator& op, const double2* b_dev, double2* x_dev, bool x0_given, RecycleSpace& sp,
             const sb_gmres_config& cfg, int precond, sb_gmres_stats& st);

}  // namespace sb
