// Block-Jacobi preconditioner of the inner solve of the mixed solver (no reference counterpart:
// an inner-solver choice of this library; the reference's preconditioned GMRES interface is
// Preconditioner::apply_into, crates/sonium-solvers/crates/sonium-solvers-core/src/traits.rs:3645).
//
// The unknowns are grouped into blocks of spatially close elements (consecutive in the Morton
// order of the element centroids; index order for an operator without a mesh). Each diagonal
// block of the complex64 matrix is gathered into shared memory by one CTA and inverted in place
// by Gauss-Jordan elimination with partial pivoting (FP32); the inverse is stored transposed so
// that the apply kernel's loads are coalesced. The inner GMRES is preconditioned on the right:
// it solves (A M^-1) y = r and the correction is d = M^-1 y, so the outer refinement (and the
// converged answer) is unchanged; only the inner iteration count drops. The preconditioner is
// rebuilt after each assembly on the first mixed solve that uses it.
//
// The FP64 solver takes the same preconditioner on the right (SB_PRECOND_BLOCK_JACOBI): the
// diagonal blocks of the complex128 matrix, rounded to complex64 and inverted by the same kernel,
// applied to FP64 vectors with FP64 accumulation. Right preconditioning leaves the residual that
// decides convergence, b - A x, untouched, so the FP64 solution meets the same tolerance.

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "sb_blas.cuh"
#include "sb_device.cuh"
#include "sb_internal.cuh"
#include "sb_precond.cuh"
#include "sb_profile.cuh"

namespace sb {

namespace {

template <int BS>
__global__ void __launch_bounds__(bj_threads(BS)) k_bj_invert(const float2* __restrict__ A, int64_t lda, int64_t n,
                                                              const int32_t* __restrict__ perm,
                                                              float2* __restrict__ out, int* __restrict__ status) {
    extern __shared__ float2 M[];  // BS x BS, row-major
    const int64_t base = blockIdx.x * (int64_t)BS;
    const int rows = static_cast<int>(n - base < BS ? n - base : BS);
    bj_invert_block<BS, bj_threads(BS)>(A, lda, rows, perm + base, out + blockIdx.x * (int64_t)BS * BS, status, M);
}

// The same blocks of the complex128 matrix (row-major, leading dimension n), rounded to complex64
// before the inversion: the FP64 solver's right preconditioner is then the same linear map as the
// mixed solver's.
template <int BS>
__global__ void __launch_bounds__(bj_threads(BS)) k_bj_invert64(const double2* __restrict__ A, int64_t n,
                                                                const int32_t* __restrict__ perm,
                                                                float2* __restrict__ out, int* __restrict__ status) {
    extern __shared__ float2 M[];
    const int64_t base = blockIdx.x * (int64_t)BS;
    const int rows = static_cast<int>(n - base < BS ? n - base : BS);
    bj_invert_block<BS, bj_threads(BS), double2>(A, n, rows, perm + base, out + blockIdx.x * (int64_t)BS * BS, status,
                                                 M);
}

// y = M^-1 x: one CTA of BS * kBjSplit threads per block; V = float2 (FP32 vectors) or double2.
template <int BS, class V>
__global__ void __launch_bounds__(BS * kBjSplit) k_bj_apply(const float2* __restrict__ invT, int64_t n,
                                                 const int32_t* __restrict__ perm, const V* __restrict__ x,
                                                 V* __restrict__ y, Gate gate) {
    if ((gate.a && *gate.a == 0) || (gate.b && *gate.b == 0)) return;
    const int64_t base = blockIdx.x * (int64_t)BS;
    const int rows = static_cast<int>(n - base < BS ? n - base : BS);
    bj_apply_block<BS, V>(invT + blockIdx.x * (int64_t)BS * BS, rows, perm + base, x, y);
}

}  // namespace

namespace {

// Bounds of the element centroids: one CTA, bounds[0..2] the smallest and [3..5] the largest
// coordinate along each axis.
constexpr int kMortonThreads = 1024;
__global__ void __launch_bounds__(kMortonThreads) k_centroid_bounds(const double* __restrict__ elem, int64_t n,
                                                                     int64_t ld, double* __restrict__ bounds) {
    __shared__ double red[kMortonThreads / 32][6];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int64_t e = tid; e < n; e += kMortonThreads)
        for (int d = 0; d < 3; ++d) {
            const double x = elem[(ECX + d) * ld + e];
            v[d] = fmin(v[d], x);
            v[3 + d] = fmax(v[3 + d], x);
        }
#pragma unroll
    for (int o = 16; o; o >>= 1)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = fmin(v[d], __shfl_xor_sync(0xffffffffu, v[d], o));
            v[3 + d] = fmax(v[3 + d], __shfl_xor_sync(0xffffffffu, v[3 + d], o));
        }
    if (lane == 0)
        for (int c = 0; c < 6; ++c) red[warp][c] = v[c];
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kMortonThreads / 32; ++w)
            for (int d = 0; d < 3; ++d) {
                v[d] = fmin(v[d], red[w][d]);
                v[3 + d] = fmax(v[3 + d], red[w][3 + d]);
            }
        for (int c = 0; c < 6; ++c) bounds[c] = v[c];
    }
}

// Two zero bits after each of the low 21 bits of x (bit b moves to bit 3 b).
__device__ __forceinline__ uint64_t spread3(uint64_t x) {
    x &= 0x1fffffull;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

// Morton (Z-order) code of every element centroid: each coordinate normalised by the largest
// extent of the box, clamped to [0, 1], scaled to 21 bits (truncated), bits interleaved x, y, z
// from the lowest. Correctly rounded operations, so the code does not depend on contraction.
__global__ void k_morton_codes(const double* __restrict__ elem, int64_t n, int64_t ld,
                               const double* __restrict__ bounds, uint64_t* __restrict__ code) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double span = fmax(fmax(fmax(__dsub_rn(bounds[3], bounds[0]), __dsub_rn(bounds[4], bounds[1])),
                                  __dsub_rn(bounds[5], bounds[2])), 1e-300);
    uint64_t c = 0;
    for (int d = 0; d < 3; ++d) {
        const double t = __ddiv_rn(__dsub_rn(elem[(ECX + d) * ld + e], bounds[d]), span);
        const uint64_t q = static_cast<uint64_t>(__dmul_rn(fmin(fmax(t, 0.0), 1.0), 2097151.0));
        c |= spread3(q) << d;
    }
    code[e] = c;
}

// Indices sorted by code, equal codes in index order (least-significant-digit radix sort, 8 bits
// a pass over the 63 code bits).
std::vector<int32_t> order_by_code(const std::vector<uint64_t>& code) {
    const size_t n = code.size();
    std::vector<int32_t> a(n), b(n);
    std::iota(a.begin(), a.end(), 0);
    if (n == 0) return a;
    for (int shift = 0; shift < 64; shift += 8) {
        size_t cnt[257] = {0};
        for (size_t i = 0; i < n; ++i) ++cnt[((code[a[i]] >> shift) & 0xff) + 1];
        if (cnt[1 + ((code[a[0]] >> shift) & 0xff)] == n) continue;  // one digit value: order kept
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (size_t i = 0; i < n; ++i) b[cnt[(code[a[i]] >> shift) & 0xff]++] = a[i];
        a.swap(b);
    }
    return a;
}

}  // namespace

// Morton order of a mesh's element centroids: codes on the device, the stable sort on the host.
std::vector<int32_t> element_morton_order(const Mesh& m) {
    SB_CUDA(cudaSetDevice(m.device));
    DevBuf bounds, dcode;
    bounds.alloc(sizeof(double) * 6);
    dcode.alloc(sizeof(uint64_t) * std::max<int64_t>(m.n, 1));
    k_centroid_bounds<<<1, kMortonThreads>>>(m.elem.as<double>(), m.n, m.ld, bounds.as<double>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    k_morton_codes<<<static_cast<unsigned>((m.n + 255) / 256), 256>>>(m.elem.as<double>(), m.n, m.ld,
                                                                      bounds.as<double>(), dcode.as<uint64_t>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    std::vector<uint64_t> code(m.n);
    SB_CUDA(cudaMemcpy(code.data(), dcode.p, sizeof(uint64_t) * m.n, cudaMemcpyDeviceToHost));
    return order_by_code(code);
}

namespace {

template <int BS>
void bj_build(Operator& op, int* status) {
    const int64_t nb = (op.n + BS - 1) / BS;
    const size_t smem = sizeof(float2) * BS * BS;
    SB_CUDA(cudaFuncSetAttribute(k_bj_invert<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    k_bj_invert<BS><<<static_cast<unsigned>(nb), bj_threads(BS), smem, op.stream>>>(
        op.A32.as<float2>(), op.lda32, op.n, op.bj_perm.as<int32_t>(), op.bj_inv.as<float2>(), status);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

template <int BS>
void bj_build64(Operator& op, int* status) {
    const int64_t nb = (op.n + BS - 1) / BS;
    const size_t smem = sizeof(float2) * BS * BS;
    SB_CUDA(cudaFuncSetAttribute(k_bj_invert64<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    k_bj_invert64<BS><<<static_cast<unsigned>(nb), bj_threads(BS), smem, op.stream>>>(
        op.A64.as<double2>(), op.n, op.bj_perm.as<int32_t>(), op.bj64_inv.as<float2>(), status);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

template <int BS, class V>
void bj_launch(const Operator& op, const float2* inv, const V* x, V* y, cudaStream_t s, Gate g) {
    const int64_t nb = (op.n + BS - 1) / BS;
    k_bj_apply<BS, V><<<static_cast<unsigned>(nb), BS * kBjSplit, 0, s>>>(inv, op.n, op.bj_perm.as<int32_t>(), x, y,
                                                                          g);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

template <class V>
void bj_dispatch(const Operator& op, const float2* inv, const V* x, V* y, Gate g) {
    ProfScope prof(SB_PROF_ARNOLDI, op.stream);
    switch (op.bj_size) {
        case 32: bj_launch<32, V>(op, inv, x, y, op.stream, g); break;
        case 64: bj_launch<64, V>(op, inv, x, y, op.stream, g); break;
        case 96: bj_launch<96, V>(op, inv, x, y, op.stream, g); break;
        default: bj_launch<128, V>(op, inv, x, y, op.stream, g); break;
    }
}

// The blocks' permutation (Morton order of the element centroids, else index order), built once
// per operator.
void bj_ensure_perm(Operator& op) {
    if (op.bj_perm.p) return;
    const int64_t n = op.n;
    std::vector<int32_t> perm(n);
    if (op.mesh && op.basis == SB_BASIS_CONSTANT) {
        perm = element_morton_order(*op.mesh);
    } else {
        std::iota(perm.begin(), perm.end(), 0);
    }
    op.bj_perm.alloc(sizeof(int32_t) * n);
    h2d_sync(op.bj_perm.p, perm.data(), sizeof(int32_t) * n);
}

}  // namespace

void bj64_prepare(Operator& op) {
    if (op.bj64_valid) return;
    SB_REQUIRE(op.A64.p, SB_ERR_INVALID_ARGUMENT,
               "block-Jacobi preconditioner of the FP64 solver: the operator has no complex128 matrix");
    const int bs = op.bj_size;
    const int64_t nb = (op.n + bs - 1) / bs;
    bj_ensure_perm(op);
    const size_t bytes = sizeof(float2) * static_cast<size_t>(nb) * bs * bs;
    if (op.bj64_inv.bytes != bytes) {
        op.bj64_inv.release();
        op.bj64_inv.alloc(bytes);
    }
    if (!op.bj_status.p) op.bj_status.alloc(sizeof(int));
    ProfScope prof(SB_PROF_OTHER, op.stream);
    SB_CUDA(cudaMemsetAsync(op.bj_status.p, 0, sizeof(int), op.stream));
    switch (bs) {
        case 32: bj_build64<32>(op, op.bj_status.as<int>()); break;
        case 64: bj_build64<64>(op, op.bj_status.as<int>()); break;
        case 96: bj_build64<96>(op, op.bj_status.as<int>()); break;
        default: bj_build64<128>(op, op.bj_status.as<int>()); break;
    }
    op.bj64_valid = true;
}

void bj64_apply(const Operator& op, const double2* x, double2* y, Gate g) {
    bj_dispatch<double2>(op, op.bj64_inv.as<float2>(), x, y, g);
}

void bj_prepare(Operator& op) {
    if (op.bj_valid) return;
    SB_REQUIRE(op.A32.p, SB_ERR_INVALID_ARGUMENT, "block-Jacobi inner preconditioner: no complex64 matrix");
    const int bs = op.bj_size;
    const int64_t nb = (op.n + bs - 1) / bs;
    bj_ensure_perm(op);
    const size_t bytes = sizeof(float2) * static_cast<size_t>(nb) * bs * bs;
    if (op.bj_inv.bytes != bytes) {
        op.bj_inv.release();
        op.bj_inv.alloc(bytes);
    }
    if (!op.bj_status.p) op.bj_status.alloc(sizeof(int));
    ProfScope prof(SB_PROF_OTHER, op.stream);
    SB_CUDA(cudaMemsetAsync(op.bj_status.p, 0, sizeof(int), op.stream));
    switch (bs) {
        case 32: bj_build<32>(op, op.bj_status.as<int>()); break;
        case 64: bj_build<64>(op, op.bj_status.as<int>()); break;
        case 96: bj_build<96>(op, op.bj_status.as<int>()); break;
        default: bj_build<128>(op, op.bj_status.as<int>()); break;
    }
    op.bj_valid = true;
}

void bj_apply(const Operator& op, const float2* x, float2* y, Gate g) {
    bj_dispatch<float2>(op, op.bj_inv.as<float2>(), x, y, g);
}

}  // namespace sb
