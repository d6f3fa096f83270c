// Allocation-free variant of the transposed / Hermitian matvec (sb_operator_apply_device_noalloc).
//
// Why it exists: the regular entry points allocate their scratch with cudaMalloc on first use
// (and free it with cudaFree, which waits for the whole device). Some callers cannot allow that:
// a host that has already handed the GPU's memory to its own pool or arena, where a driver
// allocation fails or fragments that pool, and a host that keeps several streams busy and cannot
// accept the device-wide wait that cudaFree implies. This variant takes its scratch from a
// fixed, file-scope device array instead and allocates nothing.
//
// Limits and sharing:
//  - the array holds kNoAllocScratchBytes (8 MiB) on every GPU that loads the library, until the
//    process exits;
//  - y = A^T x needs 16 bytes of partial sums per column and row chunk, so n may be at most
//    kNoAllocScratchBytes / 16 = 524288; larger operators are rejected with SB_ERR_INVALID_ARGUMENT;
//  - every call on a device shares the one array and leaves its partial sums in it. Each call
//    writes every partial sum it later reads, so nothing needs to start at zero, but two calls
//    whose kernels overlap on the GPU (different streams, different operators on one device, or
//    different host threads) overwrite each other's partial sums and race.
//  - the first call on a device looks up the array's device address (cudaGetSymbolAddress, with
//    that device current) and keeps it; make that first call before any stream capture. The kept
//    address belongs to the device's current context: a host that calls cudaDeviceReset (which
//    unloads the library's device code) must not call this entry point on that device again in
//    the same process, since the kept address would then point at released memory.

#include <mutex>

#include "sb_blas.cuh"
#include "sb_internal.cuh"

struct sb_operator {
    sb::Operator* op;
};

namespace sb {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_na_mu;
void* g_na_addr[64] = {};

// Device address of the scratch array on the current device (looked up once per device).
double2* noalloc_scratch(int device) {
    std::lock_guard<std::mutex> lock(g_na_mu);
    SB_REQUIRE(device >= 0 && device < 64, SB_ERR_INVALID_ARGUMENT, "device index out of range");
    if (!g_na_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error{SB_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                         cudaGetErrorString(e)};
        }
        g_na_addr[device] = p;
    }
    return static_cast<double2*>(g_na_addr[device]);
}

// Column sums of A (optionally conjugated) times x over row chunks of `rows` rows:
// part[chunk * n + j] = sum_{i in chunk} op(A)_{ij} x_i.
template <bool CONJ>
__global__ void __launch_bounds__(256) k_gemv_t_rows(const double2* __restrict__ A, int64_t n, int64_t rows,
                                                     const double2* __restrict__ x, double2* __restrict__ part) {
    const int64_t j = blockIdx.x * 256LL + threadIdx.x;
    const int64_t r0 = blockIdx.y * rows;
    const int64_t r1 = (r0 + rows < n) ? r0 + rows : n;
    if (j >= n) return;
    double ar = 0.0, ai = 0.0;
    for (int64_t i = r0; i < r1; ++i) {
        const double2 a = __ldcs(A + i * n + j);
        const double2 xv = __ldg(x + i);
        const double ay = CONJ ? -a.y : a.y;
        ar = fma(a.x, xv.x, fma(-ay, xv.y, ar));
        ai = fma(a.x, xv.y, fma(ay, xv.x, ai));
    }
    part[blockIdx.y * n + j] = make_double2(ar, ai);
}

__global__ void k_sum_rows_chunks(const double2* __restrict__ part, int64_t n, int64_t chunks,
                                  double2* __restrict__ y) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double sr = 0.0, si = 0.0;
    for (int64_t c = 0; c < chunks; ++c) {
        const double2 v = part[c * n + j];
        sr += v.x;
        si += v.y;
    }
    y[j] = make_double2(sr, si);
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" SB_API int sb_operator_apply_device_noalloc(const sb_operator* op, int trans, const sb_complex* x_dev,
                                                       sb_complex* y_dev) {
    return abi_guard([&] {
        SB_REQUIRE(op && op->op && x_dev && y_dev, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_REQUIRE(trans == SB_OP_N || trans == SB_OP_T || trans == SB_OP_C, SB_ERR_INVALID_ARGUMENT,
                   "trans must be N, T or C");
        Operator& o = *op->op;
        const int64_t n = o.n;
        SB_REQUIRE(n > 0, SB_ERR_INVALID_ARGUMENT, "empty operator");
        SB_CUDA(cudaSetDevice(o.device));
        const double2* x = reinterpret_cast<const double2*>(x_dev);
        double2* y = reinterpret_cast<double2*>(y_dev);
        if (trans == SB_OP_N) {
            // The forward product keeps no partial sums: the regular kernels allocate nothing.
            op_gemv64(o, x, y, Gate{});
        } else {
            SB_REQUIRE(o.A64.p, SB_ERR_INVALID_ARGUMENT,
                       "transposed products need the complex128 matrix (SB_PRECISION_FP64 or SB_PRECISION_FP64_FP32)");
            const int64_t max_chunks = static_cast<int64_t>(kNoAllocScratchBytes / (sizeof(double2) * n));
            SB_REQUIRE(max_chunks >= 1, SB_ERR_INVALID_ARGUMENT,
                       "operator too large for the allocation-free transposed product: n = " + std::to_string(n) +
                           " exceeds " + std::to_string(kNoAllocScratchBytes / sizeof(double2)));
            double2* part = noalloc_scratch(o.device);
            const int64_t want = (n + 255) / 256;  // about 256 rows per chunk when the scratch allows
            const int64_t chunks = want < max_chunks ? want : max_chunks;
            const int64_t rows = (n + chunks - 1) / chunks;
            const dim3 grid(static_cast<unsigned>((n + 255) / 256), static_cast<unsigned>((n + rows - 1) / rows));
            if (trans == SB_OP_T)
                k_gemv_t_rows<false><<<grid, 256, 0, o.stream>>>(o.A64.as<double2>(), n, rows, x, part);
            else
                k_gemv_t_rows<true><<<grid, 256, 0, o.stream>>>(o.A64.as<double2>(), n, rows, x, part);
            count_launch();
            SB_CUDA(cudaGetLastError());
            k_sum_rows_chunks<<<(n + 255) / 256, 256, 0, o.stream>>>(part, n, grid.y, y);
            count_launch();
            SB_CUDA(cudaGetLastError());
        }
        SB_CUDA(cudaStreamSynchronize(o.stream));
    });
}
