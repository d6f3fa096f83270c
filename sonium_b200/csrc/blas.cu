// Dense complex matvec and Arnoldi building blocks on sm_100a.
//
// Reference: DenseMatrix::matvec_into -> gemv_c64 (crates/sonium-solvers/crates/sonium-solvers-core/
// src/dense.rs:416-427, traits.rs:1430-1452) on the CPU and cublasZgemv / cublasCgemv
// (crates/sonium-compute/src/cuda/cublas_blas23.rs:126,165) on the GPU; the Arnoldi helpers follow
// batched_dots_flat_into / batched_project_flat / fused_basis_update_flat (crates/sonium-solvers/
// crates/sonium-solvers-iterative/src/cgs_orth.rs:180-300) and the fused CUDA multi-dot / axpy
// kernels (crates/sonium-compute/src/cuda/kernels/multi_dot_kernels.cu:173-306).
//
// The matvec is HBM-bound (16 N^2 bytes per complex128 product): each CTA owns a few rows and
// streams them with 128-bit evict-first loads, several loads in flight per thread, reusing each
// x element across its rows.

#include <algorithm>

#include "sb_blas.cuh"
#include "sb_device.cuh"
#include "sb_gemv.cuh"
#include "sb_internal.cuh"
#include "sb_profile.cuh"

namespace sb {

static inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Gates: a kernel launched inside a captured Krylov cycle returns at once when its gate is
// closed (the instance converged or the step needs no second Gram-Schmidt pass).
__device__ __forceinline__ bool closed(Gate g) {
    return (g.a && *g.a == 0) || (g.b && *g.b == 0);
}

// ---------------------------------------------------------------------------------------------
// y = A x (complex128), or y = b - A x with per-CTA partial ||y||^2 when b != null.
// ---------------------------------------------------------------------------------------------
template <int ROWS, int THREADS, int UNROLL>
__global__ void __launch_bounds__(THREADS) k_gemv_n_c128(const double2* __restrict__ A, int64_t n,
                                                         const double2* __restrict__ x,
                                                         double2* __restrict__ y,
                                                         const double2* __restrict__ b,
                                                         double* __restrict__ part, Gate gate) {
    if (closed(gate)) return;
    __shared__ double red[(THREADS / 32) * 2 * ROWS];
    const int64_t row0 = blockIdx.x * (int64_t)ROWS;
    const int nr = static_cast<int>((n - row0) < ROWS ? (n - row0) : ROWS);
    double acc[2 * ROWS];
#pragma unroll
    for (int r = 0; r < 2 * ROWS; ++r) acc[r] = 0.0;
    const double2* Ar = A + row0 * n;
    int64_t c = threadIdx.x;
    for (; c + (UNROLL - 1) * THREADS < n; c += UNROLL * THREADS) {
        double2 xv[UNROLL];
        double2 av[UNROLL][ROWS];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            xv[u] = __ldg(x + c + u * THREADS);
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
                av[u][r] = (r < nr) ? ld_stream(Ar + r * n + c + u * THREADS) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                acc[2 * r] = fma(av[u][r].x, xv[u].x, fma(-av[u][r].y, xv[u].y, acc[2 * r]));
                acc[2 * r + 1] = fma(av[u][r].x, xv[u].y, fma(av[u][r].y, xv[u].x, acc[2 * r + 1]));
            }
    }
    for (; c < n; c += THREADS) {
        const double2 xv = __ldg(x + c);
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            if (r < nr) {
                const double2 a = ld_stream(Ar + r * n + c);
                acc[2 * r] = fma(a.x, xv.x, fma(-a.y, xv.y, acc[2 * r]));
                acc[2 * r + 1] = fma(a.x, xv.y, fma(a.y, xv.x, acc[2 * r + 1]));
            }
        }
    }
    block_sum<2 * ROWS, THREADS>(acc, red);
    if (threadIdx.x == 0) {
        double nrm = 0.0;
        for (int r = 0; r < nr; ++r) {
            double2 v = make_double2(acc[2 * r], acc[2 * r + 1]);
            if (b) {
                const double2 bb = b[row0 + r];
                v = make_double2(bb.x - v.x, bb.y - v.y);
                nrm += v.x * v.x + v.y * v.y;
            }
            y[row0 + r] = v;
        }
        if (part) part[blockIdx.x] = nrm;
    }
}

// y = A^T x or A^H x (complex128): column-per-thread over row chunks, then a chunk reduction.
constexpr int kTRows = 256;
template <bool CONJ>
__global__ void __launch_bounds__(256) k_gemv_t_c128(const double2* __restrict__ A, int64_t n,
                                                     const double2* __restrict__ x,
                                                     double2* __restrict__ part) {
    const int64_t j = blockIdx.x * 256LL + threadIdx.x;
    const int64_t r0 = blockIdx.y * (int64_t)kTRows;
    const int64_t r1 = (r0 + kTRows < n) ? r0 + kTRows : n;
    if (j >= n) return;
    double ar = 0.0, ai = 0.0;
    for (int64_t i = r0; i < r1; ++i) {
        const double2 a = ld_stream(A + i * n + j);
        const double2 xv = __ldg(x + i);
        const double ay = CONJ ? -a.y : a.y;
        ar = fma(a.x, xv.x, fma(-ay, xv.y, ar));
        ai = fma(a.x, xv.y, fma(ay, xv.x, ai));
    }
    part[blockIdx.y * n + j] = make_double2(ar, ai);
}

__global__ void k_sum_chunks(const double2* __restrict__ part, int64_t n, int64_t chunks,
                             double2* __restrict__ y) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double2 s = make_double2(0.0, 0.0);
    for (int64_t c = 0; c < chunks; ++c) s = cadd(s, part[c * n + j]);
    y[j] = s;
}

// ---------------------------------------------------------------------------------------------
// Complex64 matrix: FP32 vectors with FP32 accumulation, or FP64 vectors with FP64 accumulation.
// ---------------------------------------------------------------------------------------------
template <int ROWS, int THREADS, int UNROLL, bool X64>
__global__ void __launch_bounds__(THREADS) k_gemv_n_c64(const float2* __restrict__ A, int64_t n,
                                                        int64_t lda,
                                                        const void* __restrict__ xv_,
                                                        void* __restrict__ yv_,
                                                        const void* __restrict__ bv_,
                                                        double* __restrict__ part, Gate gate) {
    if (closed(gate)) return;
    gemv_c64_block<ROWS, THREADS, UNROLL, X64>(A, n, lda, xv_, yv_, bv_, part, blockIdx.x);
}

// ---------------------------------------------------------------------------------------------
// Arnoldi helpers, templated on the vector element (double2 / float2); reductions in FP64.
// ---------------------------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ double2 to_d(T v) {
    return make_double2(static_cast<double>(v.x), static_cast<double>(v.y));
}

constexpr int kDotRows = 256;
constexpr int kDotVecs = 8;

// part[(chunk * (k + 1)) + i] = sum over the chunk of conj(V_i) w  (i < k), and |w|^2 at i = k.
// With cnt (one counter per blockIdx.y, zero between launches) the last CTA of each column of the
// grid also reduces the partials into out, in chunk order as k_reduce_part does, and resets the
// counter: one launch instead of two.
template <class T>
__global__ void __launch_bounds__(kDotRows) k_dots(const T* __restrict__ V, int64_t ldv, int k,
                                                   const T* __restrict__ w, int64_t n,
                                                   double2* __restrict__ part, Gate gate,
                                                   double2* __restrict__ out = nullptr,
                                                   unsigned* __restrict__ cnt = nullptr) {
    if (closed(gate)) return;
    __shared__ double red[(kDotRows / 32) * 2 * kDotVecs];
    const int64_t r = blockIdx.x * (int64_t)kDotRows + threadIdx.x;
    const int i0 = blockIdx.y * kDotVecs;
    double acc[2 * kDotVecs];
#pragma unroll
    for (int t = 0; t < 2 * kDotVecs; ++t) acc[t] = 0.0;
    if (r < n) {
        const double2 wv = to_d(w[r]);
#pragma unroll
        for (int t = 0; t < kDotVecs; ++t) {
            const int i = i0 + t;
            if (i < k) {
                const double2 v = to_d(V[i * ldv + r]);
                acc[2 * t] = v.x * wv.x + v.y * wv.y;
                acc[2 * t + 1] = v.x * wv.y - v.y * wv.x;
            } else if (i == k) {
                acc[2 * t] = wv.x * wv.x + wv.y * wv.y;
            }
        }
    }
    block_sum<2 * kDotVecs, kDotRows>(acc, red);
    if (threadIdx.x == 0) {
        for (int t = 0; t < kDotVecs; ++t) {
            const int i = i0 + t;
            if (i <= k) part[blockIdx.x * (int64_t)(k + 1) + i] = make_double2(acc[2 * t], acc[2 * t + 1]);
        }
    }
    if (!cnt) return;
    __shared__ int last;
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's partials are visible before its count
        last = atomicAdd(&cnt[blockIdx.y], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // warp t reduces vector i0 + t (kDotRows / 32 == kDotVecs warps)
    const int t = threadIdx.x >> 5, lane = threadIdx.x & 31, i = i0 + t;
    if (i <= k) {
        double sr = 0.0, si = 0.0;
        for (int64_t c = lane; c < gridDim.x; c += 32) {
            const double2 v = __ldcg(part + c * (k + 1) + i);
            sr += v.x;
            si += v.y;
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) out[i] = make_double2(sr, si);
    }
    if (threadIdx.x == 0) cnt[blockIdx.y] = 0;
}
static_assert(kDotRows / 32 == kDotVecs, "one reducing warp per vector of a dots CTA");
static_assert((kMaxKrylov + kDotVecs) / kDotVecs <= kArnoldiCounters, "a counter per column of the dots grid");

// out[i] = sum over chunks of part[c][i], i <= k (one warp per output).
__global__ void k_reduce_part(const double2* __restrict__ part, int64_t chunks, int kp1,
                              double2* __restrict__ out, Gate gate) {
    if (closed(gate)) return;
    const int i = blockIdx.x;
    double sr = 0.0, si = 0.0;
    for (int64_t c = threadIdx.x; c < chunks; c += 32) {
        const double2 v = part[c * kp1 + i];
        sr += v.x;
        si += v.y;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (threadIdx.x == 0) out[i] = make_double2(sr, si);
}

// w -= sum_i coeff[i] V_i, and a per-CTA partial of |w|^2.
// With cnt the last CTA also sums the partials into *out (as k_sum_real does) and resets *cnt.
template <class T>
__global__ void __launch_bounds__(256) k_project(const T* __restrict__ V, int64_t ldv, int k,
                                                 const double2* __restrict__ coeff,
                                                 T* __restrict__ w, int64_t n,
                                                 double* __restrict__ part, Gate gate,
                                                 double* __restrict__ out = nullptr,
                                                 unsigned* __restrict__ cnt = nullptr) {
    if (closed(gate)) return;
    __shared__ double2 sc[kMaxKrylov + 1];
    __shared__ double red[8];
    for (int t = threadIdx.x; t < k; t += blockDim.x) sc[t] = coeff[t];
    __syncthreads();
    const int64_t r = blockIdx.x * 256LL + threadIdx.x;
    double nr2[1] = {0.0};
    if (r < n) {
        double2 acc = to_d(w[r]);
        int i = 0;
        for (; i + 4 <= k; i += 4) {
            double2 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = to_d(V[(i + u) * ldv + r]);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                acc.x -= sc[i + u].x * v[u].x - sc[i + u].y * v[u].y;
                acc.y -= sc[i + u].x * v[u].y + sc[i + u].y * v[u].x;
            }
        }
        for (; i < k; ++i) {
            const double2 v = to_d(V[i * ldv + r]);
            acc.x -= sc[i].x * v.x - sc[i].y * v.y;
            acc.y -= sc[i].x * v.y + sc[i].y * v.x;
        }
        T o;
        o.x = acc.x;
        o.y = acc.y;
        w[r] = o;
        const double2 ad = to_d(o);
        nr2[0] = ad.x * ad.x + ad.y * ad.y;
    }
    block_sum<1, 256>(nr2, red);
    if (threadIdx.x == 0) part[blockIdx.x] = nr2[0];
    if (!cnt) return;
    __shared__ int last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(cnt, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    __threadfence();
    double sum = 0.0;
    for (int64_t c = threadIdx.x; c < gridDim.x; c += 32) sum += __ldcg(part + c);
    sum = warp_sum(sum);
    if (threadIdx.x == 0) {
        *out = sum;
        *cnt = 0;
    }
}

// One CTA sums m partial norms (m up to one per row of the residual products).
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_sum_real(const double* __restrict__ part, int64_t m,
                                                          double* __restrict__ out, Gate gate) {
    if (closed(gate)) return;
    __shared__ double red[kSumThreads / 32];
    double s = 0.0;
    for (int64_t c = threadIdx.x; c < m; c += kSumThreads) s += part[c];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < kSumThreads / 32 ? red[threadIdx.x] : 0.0;
        s = warp_sum(s);
        if (threadIdx.x == 0) *out = s;
    }
}

// y = alpha * x with type conversion; alpha from the host, or *alpha_dev when given.
template <class TI, class TO>
__global__ void k_scale(const TI* __restrict__ x, double alpha, const double* __restrict__ alpha_dev,
                        TO* __restrict__ y, int64_t n, Gate gate) {
    if (closed(gate)) return;
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    const double a = alpha_dev ? *alpha_dev : alpha;
    TO o;
    o.x = static_cast<double>(x[r].x) * a;
    o.y = static_cast<double>(x[r].y) * a;
    y[r] = o;
}

// x += alpha * sum_i y_i V_i (y on device), x of type TX, V of type T.
template <class T, class TX>
__global__ void k_update(const T* __restrict__ V, int64_t ldv, int k, const int* __restrict__ k_dev,
                         const double2* __restrict__ yc, double alpha, TX* __restrict__ x, int64_t n) {
    __shared__ double2 sc[kMaxKrylov + 1];
    const int kk = k_dev ? *k_dev : k;
    for (int t = threadIdx.x; t < kk; t += blockDim.x) sc[t] = yc[t];
    __syncthreads();
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < kk; ++i) {
        const double2 v = to_d(V[i * ldv + r]);
        sr += sc[i].x * v.x - sc[i].y * v.y;
        si += sc[i].x * v.y + sc[i].y * v.x;
    }
    TX o = x[r];
    o.x = static_cast<double>(o.x) + alpha * sr;
    o.y = static_cast<double>(o.y) + alpha * si;
    x[r] = o;
}

// y = diag^-1 x (Jacobi), complex division with the FP64 diagonal.
template <class T>
__global__ void k_jacobi(const double2* __restrict__ d, const T* __restrict__ x, T* __restrict__ y,
                         int64_t n, Gate gate) {
    if (closed(gate)) return;
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    const double2 a = d[r];
    const double2 v = to_d(x[r]);
    const double den = a.x * a.x + a.y * a.y;
    T o;
    o.x = (v.x * a.x + v.y * a.y) / den;
    o.y = (v.y * a.x - v.x * a.y) / den;
    y[r] = o;
}

// ---------------------------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------------------------

// Launch shape of the complex128 product (rows per CTA, 16-byte loads in flight per row and
// thread): 1 x 4, measured at N = 20480 on B200 0.93-0.99 ms against 0.98-1.02 ms for 4 x 2.
constexpr int kGemv128Rows = 1, kGemv128Unroll = 4;

// gemv_partials counts the partial norms of both the complex128 and the FP32-vector complex64
// residuals, and callers size partial-norm buffers by it for every residual product.
static_assert(kGemv64Rows == kGemv128Rows, "one partial count for the c128 and c64 residuals");
static_assert(kGemvX64Rows >= kGemv128Rows && kGemv16PRows >= kGemv128Rows,
              "gemv_partials bounds every residual's partial count");

void gemv_c128(const double2* A, int64_t n, const double2* x, double2* y, Trans t,
               cudaStream_t s, DevBuf& scratch, Gate gate) {
    ProfScope prof(SB_PROF_GEMV64, s);
    if (t == Trans::N) {
        k_gemv_n_c128<kGemv128Rows, kGemvThreads, kGemv128Unroll>
            <<<cdiv(n, kGemv128Rows), kGemvThreads, 0, s>>>(A, n, x, y, nullptr, nullptr, gate);
        count_launch();
        SB_CUDA(cudaGetLastError());
        return;
    }
    const int64_t chunks = cdiv(n, kTRows);
    const size_t need = sizeof(double2) * chunks * n;
    if (scratch.bytes < need) {
        scratch.release();
        scratch.alloc(need);
    }
    dim3 grid(static_cast<unsigned>(cdiv(n, 256)), static_cast<unsigned>(chunks));
    if (t == Trans::T)
        k_gemv_t_c128<false><<<grid, 256, 0, s>>>(A, n, x, scratch.as<double2>());
    else
        k_gemv_t_c128<true><<<grid, 256, 0, s>>>(A, n, x, scratch.as<double2>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    k_sum_chunks<<<cdiv(n, 256), 256, 0, s>>>(scratch.as<double2>(), n, chunks, y);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

void gemv_residual_c128(const double2* A, int64_t n, const double2* x, const double2* b,
                        double2* r, double* part, cudaStream_t s, Gate gate) {
    ProfScope prof(SB_PROF_GEMV64, s);
    k_gemv_n_c128<kGemv128Rows, kGemvThreads, kGemv128Unroll>
        <<<cdiv(n, kGemv128Rows), kGemvThreads, 0, s>>>(A, n, x, r, b, part, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}
int64_t gemv_partials(int64_t n) { return cdiv(n, kGemv128Rows); }

void gemv_c64(const float2* A, int64_t n, int64_t lda, const float2* x, float2* y,
              const float2* b, double* part, cudaStream_t s, Gate gate) {
    ProfScope prof(SB_PROF_GEMV32, s);
    k_gemv_n_c64<kGemv64Rows, kGemvThreads, kGemv64Unroll, false>
        <<<cdiv(n, kGemv64Rows), kGemvThreads, 0, s>>>(A, n, lda, x, y, b, part, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

int64_t gemv_x64_partials(int64_t n) { return cdiv(n, kGemvX64Rows); }

void gemv_c64_x64(const float2* A, int64_t n, int64_t lda, const double2* x, double2* y,
                  const double2* b, double* part, cudaStream_t s, Gate gate) {
    ProfScope prof(SB_PROF_GEMV32, s);
    k_gemv_n_c64<kGemvX64Rows, kGemvThreads, kGemvX64Unroll, true>
        <<<cdiv(n, kGemvX64Rows), kGemvThreads, 0, s>>>(A, n, lda, x, y, b, part, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------------------
// Complex-half matrix (the row-block body, the largest-part scan and the conversion are shared
// with the batched solver: sb_gemv.cuh).
// ---------------------------------------------------------------------------------------------
template <int ROWS, int THREADS, int UNROLL>
__global__ void __launch_bounds__(THREADS) k_gemv_n_c16(const uint32_t* __restrict__ A, int64_t n, int64_t lda,
                                                        const float* __restrict__ inv_scale,
                                                        const float2* __restrict__ x, float2* __restrict__ y,
                                                        const float2* __restrict__ b, double* __restrict__ part,
                                                        Gate gate) {
    if (closed(gate)) return;
    gemv_c16_block<ROWS, THREADS, UNROLL, true>(A, n, lda, inv_scale, x, y, b, part, blockIdx.x);
}

int64_t gemv16_partials(int64_t n) { return cdiv(n, kGemv16PRows); }

void gemv_c16(const uint32_t* A, int64_t n, int64_t lda, const float* inv_scale, const float2* x, float2* y,
              const float2* b, double* part, cudaStream_t s, Gate gate) {
    ProfScope prof(SB_PROF_GEMV16, s);
    k_gemv_n_c16<kGemv16PRows, kGemvThreads, kGemv16PUnroll>
        <<<cdiv(n, kGemv16PRows), kGemvThreads, 0, s>>>(A, n, lda, inv_scale, x, y, b, part, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

// Per-row scales of a complex64 matrix: one CTA per row (grid-stride) takes the row's largest
// |re|, |im| and writes its power-of-two scale s[row] and inverse inv[row].
__global__ void __launch_bounds__(kHalfThreads) k_row_scale_full(const float2* __restrict__ A, int64_t n,
                                                                 int64_t lda, float* __restrict__ s,
                                                                 float* __restrict__ inv) {
    __shared__ float red[kHalfThreads / 32];
    for (int64_t row = blockIdx.x; row < n; row += gridDim.x) {
        float m = 0.f;
        const float4* r4 = reinterpret_cast<const float4*>(A + row * lda);  // lda even
        for (int64_t c = threadIdx.x; c < (n >> 1); c += kHalfThreads) {
            const float4 v = __ldcs(r4 + c);
            const float a = fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w)));
            m = (a <= 3.4e38f) ? fmaxf(m, a) : INFINITY;
        }
        if ((n & 1) && threadIdx.x == 0) {
            const float2 v = A[row * lda + n - 1];
            const float a = fmaxf(fabsf(v.x), fabsf(v.y));
            m = (a <= 3.4e38f) ? fmaxf(m, a) : INFINITY;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < kHalfThreads / 32; ++w) m = fmaxf(m, red[w]);
            const float sc = half_scale_for(m);
            s[row] = sc;
            inv[row] = 1.f / sc;
        }
        __syncthreads();
    }
}

// H[row][c] = FP16(s[row] A[row][c]) for c < n, four entries a thread, one CTA per row.
__global__ void __launch_bounds__(kHalfThreads) k_c64_to_c16_rows(const float2* __restrict__ A, int64_t n,
                                                                  int64_t lda32, const float* __restrict__ s,
                                                                  uint32_t* __restrict__ H, int64_t lda16) {
    const int64_t q = lda16 >> 2;
    for (int64_t row = blockIdx.x; row < n; row += gridDim.x) {
        const float sc = s[row];
        int bad = 0;
        for (int64_t c4 = threadIdx.x; c4 < q; c4 += kHalfThreads) {
            const int64_t c = 4 * c4;
            float2 v[4];
            if (c + 3 < n) {
                const float4* p = reinterpret_cast<const float4*>(A + row * lda32 + c);  // lda32 and c even
                const float4 a = __ldcs(p), bq = __ldcs(p + 1);
                v[0] = make_float2(a.x, a.y);
                v[1] = make_float2(a.z, a.w);
                v[2] = make_float2(bq.x, bq.y);
                v[3] = make_float2(bq.z, bq.w);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = (c + j < n) ? A[row * lda32 + c + j] : make_float2(0.f, 0.f);
            }
            uint32_t w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) w[j] = half_pack(v[j], sc, &bad);
            __stcs(reinterpret_cast<uint4*>(H + row * lda16 + c), make_uint4(w[0], w[1], w[2], w[3]));
        }
    }
}

void half_prepare(Operator& op) {
    const cudaStream_t s = op.stream;
    if (op.half_valid && op.half_check) {
        // The FP32 assembly wrote the copy with scales from each row's near and diagonal entries;
        // a far entry beyond the FP16 range (never seen on resolved meshes) sends it to the full
        // rebuild below.
        int bad = 0;
        SB_CUDA(cudaMemcpyAsync(&bad, op.half_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        op.half_check = false;
        if (bad) op.half_valid = false;
    }
    if (op.half_valid) return;
    SB_REQUIRE(op.A32.p, SB_ERR_INVALID_ARGUMENT, "FP16 inner solve: the operator has no complex64 matrix");
    const int64_t n = op.n;
    half_alloc(op);
    ProfScope prof(SB_PROF_OTHER, s);
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>(n, 8 * device_sm_count(op.device)));
    float* sc = op.half_scale.as<float>();
    k_row_scale_full<<<grid, kHalfThreads, 0, s>>>(op.A32.as<float2>(), n, op.lda32, sc, sc + n);
    k_c64_to_c16_rows<<<grid, kHalfThreads, 0, s>>>(op.A32.as<float2>(), n, op.lda32, sc, op.A16.as<uint32_t>(),
                                                    op.lda16);
    count_launch();
    count_launch();
    SB_CUDA(cudaGetLastError());
    op.half_valid = true;
}

void half_alloc(Operator& op) {
    const int64_t n = op.n;
    const int64_t lda16 = (n + 3) / 4 * 4;
    const size_t bytes = sizeof(uint32_t) * static_cast<size_t>(n) * lda16;
    if (op.A16.bytes != bytes) {
        op.A16.release();
        op.A16.alloc(bytes);
    }
    if (op.half_scale.bytes != sizeof(float) * 2 * n) {
        op.half_scale.release();
        op.half_scale.alloc(sizeof(float) * 2 * n);
    }
    if (!op.half_flag.p) op.half_flag.alloc(sizeof(int));
    op.lda16 = lda16;
}

template <class T>
void arnoldi_dots(const T* V, int64_t ldv, int k, const T* w, int64_t n, double2* part,
                  double2* out, cudaStream_t s, Gate gate, unsigned* cnt) {
    ProfScope prof(SB_PROF_ARNOLDI, s);
    const int64_t chunks = cdiv(n, kDotRows);
    dim3 grid(static_cast<unsigned>(chunks), static_cast<unsigned>(cdiv(k + 1, kDotVecs)));
    k_dots<T><<<grid, kDotRows, 0, s>>>(V, ldv, k, w, n, part, gate, out, cnt);
    count_launch();
    SB_CUDA(cudaGetLastError());
    if (cnt) return;
    k_reduce_part<<<k + 1, 32, 0, s>>>(part, chunks, k + 1, out, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}
int64_t arnoldi_dot_chunks(int64_t n) { return cdiv(n, kDotRows); }

template <class T>
void arnoldi_project(const T* V, int64_t ldv, int k, const double2* coeff, T* w, int64_t n,
                     double* part, double* out_norm2, cudaStream_t s, Gate gate, unsigned* cnt) {
    ProfScope prof(SB_PROF_ARNOLDI, s);
    const int64_t nb = cdiv(n, 256);
    k_project<T><<<nb, 256, 0, s>>>(V, ldv, k, coeff, w, n, part, gate, out_norm2, cnt);
    count_launch();
    SB_CUDA(cudaGetLastError());
    if (cnt) return;
    k_sum_real<<<1, kSumThreads, 0, s>>>(part, nb, out_norm2, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

void sum_real(const double* part, int64_t m, double* out, cudaStream_t s, Gate gate) {
    k_sum_real<<<1, kSumThreads, 0, s>>>(part, m, out, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

template <class TI, class TO>
void scale_vec(const TI* x, double alpha, const double* alpha_dev, TO* y, int64_t n, cudaStream_t s,
               Gate gate) {
    k_scale<TI, TO><<<cdiv(n, 256), 256, 0, s>>>(x, alpha, alpha_dev, y, n, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

template <class T, class TX>
void basis_update(const T* V, int64_t ldv, int k, const int* k_dev, const double2* y, double alpha,
                  TX* x, int64_t n, cudaStream_t s) {
    ProfScope prof(SB_PROF_ARNOLDI, s);
    k_update<T, TX><<<cdiv(n, 256), 256, 0, s>>>(V, ldv, k, k_dev, y, alpha, x, n);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

template <class T>
void jacobi_apply(const double2* d, const T* x, T* y, int64_t n, cudaStream_t s, Gate gate) {
    k_jacobi<T><<<cdiv(n, 256), 256, 0, s>>>(d, x, y, n, gate);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

// Explicit instantiations.
template void arnoldi_dots<double2>(const double2*, int64_t, int, const double2*, int64_t, double2*, double2*, cudaStream_t, Gate, unsigned*);
template void arnoldi_dots<float2>(const float2*, int64_t, int, const float2*, int64_t, double2*, double2*, cudaStream_t, Gate, unsigned*);
template void arnoldi_project<double2>(const double2*, int64_t, int, const double2*, double2*, int64_t, double*, double*, cudaStream_t, Gate, unsigned*);
template void arnoldi_project<float2>(const float2*, int64_t, int, const double2*, float2*, int64_t, double*, double*, cudaStream_t, Gate, unsigned*);
template void scale_vec<double2, double2>(const double2*, double, const double*, double2*, int64_t, cudaStream_t, Gate);
template void scale_vec<float2, float2>(const float2*, double, const double*, float2*, int64_t, cudaStream_t, Gate);
template void scale_vec<double2, float2>(const double2*, double, const double*, float2*, int64_t, cudaStream_t, Gate);
template void scale_vec<float2, double2>(const float2*, double, const double*, double2*, int64_t, cudaStream_t, Gate);
template void basis_update<double2, double2>(const double2*, int64_t, int, const int*, const double2*, double, double2*, int64_t, cudaStream_t);
template void basis_update<float2, float2>(const float2*, int64_t, int, const int*, const double2*, double, float2*, int64_t, cudaStream_t);
template void basis_update<float2, double2>(const float2*, int64_t, int, const int*, const double2*, double, double2*, int64_t, cudaStream_t);
template void jacobi_apply<double2>(const double2*, const double2*, double2*, int64_t, cudaStream_t, Gate);
template void jacobi_apply<float2>(const double2*, const float2*, float2*, int64_t, cudaStream_t, Gate);

}  // namespace sb
