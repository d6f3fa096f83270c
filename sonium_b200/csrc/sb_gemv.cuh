// Row-block body of the complex64 matrix-vector product, shared by the single-instance kernel
// (blas.cu) and the batched sweep kernel (batch.cu) (internal).
//
// Reference: DenseMatrix::matvec_into -> gemv_c64 (crates/sonium-solvers/crates/sonium-solvers-core/
// src/dense.rs:416-427) and cublasCgemv (crates/sonium-compute/src/cuda/cublas_blas23.rs:165).
// HBM-bound: each CTA owns ROWS rows, streams them with 128-bit evict-first loads (UNROLL loads in
// flight per row and thread) and reuses each x element across its rows.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "sb_device.cuh"

namespace sb {

// Launch shape of the matrix-vector products: rows per CTA, threads per CTA, loads in flight.
constexpr int kGemvRows = 4;
constexpr int kGemvThreads = 256;
constexpr int kGemvUnroll = 2;

__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }

// Block-wide sum of NV doubles held per thread; result valid in thread 0.
template <int NV, int THREADS>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < NV; ++t) v[t] = warp_sum(v[t]);
    if (lane == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) red[warp * NV + t] = v[t];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            double s = 0.0;
            for (int w = 0; w < THREADS / 32; ++w) s += red[w * NV + t];
            v[t] = s;
        }
    }
}

// Rows [blk * ROWS, blk * ROWS + ROWS) of y = A x, FP32 vectors / FP32 accumulation, or FP64
// vectors / FP64 accumulation (X64). With b != null the rows get b - A x and part[blk] gets their
// squared norm. Called by every thread of a THREADS-wide CTA.
template <int ROWS, int THREADS, int UNROLL, bool X64>
__device__ __forceinline__ void gemv_c64_block(const float2* __restrict__ A, int64_t n, int64_t lda,
                                               const void* __restrict__ xv_, void* __restrict__ yv_,
                                               const void* __restrict__ bv_, double* __restrict__ part,
                                               int64_t blk) {
    using Acc = typename std::conditional<X64, double, float>::type;
    __shared__ double red[(THREADS / 32) * 2 * ROWS];
    const int64_t row0 = blk * (int64_t)ROWS;
    const int nr = static_cast<int>((n - row0) < ROWS ? (n - row0) : ROWS);
    Acc acc[2 * ROWS];
#pragma unroll
    for (int r = 0; r < 2 * ROWS; ++r) acc[r] = 0;
    const int64_t n2 = n >> 1;     // float4 = two complex64 entries
    const int64_t ld2 = lda >> 1;  // lda is even, so every row starts 16-byte aligned
    const float4* A4 = reinterpret_cast<const float4*>(A + row0 * lda);
    int64_t c = threadIdx.x;
    for (; c + (UNROLL - 1) * THREADS < n2; c += UNROLL * THREADS) {
        Acc xr[UNROLL][4];
        float4 av[UNROLL][ROWS];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const int64_t cc = c + u * THREADS;
            if (X64) {
                const double2* x = static_cast<const double2*>(xv_);
                const double2 p = __ldg(x + 2 * cc), q = __ldg(x + 2 * cc + 1);
                xr[u][0] = p.x; xr[u][1] = p.y; xr[u][2] = q.x; xr[u][3] = q.y;
            } else {
                const float4 p = __ldg(static_cast<const float4*>(xv_) + cc);
                xr[u][0] = p.x; xr[u][1] = p.y; xr[u][2] = p.z; xr[u][3] = p.w;
            }
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
                av[u][r] = (r < nr) ? ld_stream(A4 + r * ld2 + cc) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                const Acc a0 = av[u][r].x, a1 = av[u][r].y, a2 = av[u][r].z, a3 = av[u][r].w;
                acc[2 * r] = fma(a0, xr[u][0], fma(-a1, xr[u][1], acc[2 * r]));
                acc[2 * r + 1] = fma(a0, xr[u][1], fma(a1, xr[u][0], acc[2 * r + 1]));
                acc[2 * r] = fma(a2, xr[u][2], fma(-a3, xr[u][3], acc[2 * r]));
                acc[2 * r + 1] = fma(a2, xr[u][3], fma(a3, xr[u][2], acc[2 * r + 1]));
            }
    }
    for (; c < n2; c += THREADS) {
        Acc x0r, x0i, x1r, x1i;
        if (X64) {
            const double2* x = static_cast<const double2*>(xv_);
            const double2 p = x[2 * c], q = x[2 * c + 1];
            x0r = p.x; x0i = p.y; x1r = q.x; x1i = q.y;
        } else {
            const float4 p = static_cast<const float4*>(xv_)[c];
            x0r = p.x; x0i = p.y; x1r = p.z; x1i = p.w;
        }
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            if (r < nr) {
                const float4 a = ld_stream(A4 + r * ld2 + c);
                acc[2 * r] = fma((Acc)a.x, x0r, fma(-(Acc)a.y, x0i, acc[2 * r]));
                acc[2 * r + 1] = fma((Acc)a.x, x0i, fma((Acc)a.y, x0r, acc[2 * r + 1]));
                acc[2 * r] = fma((Acc)a.z, x1r, fma(-(Acc)a.w, x1i, acc[2 * r]));
                acc[2 * r + 1] = fma((Acc)a.z, x1i, fma((Acc)a.w, x1r, acc[2 * r + 1]));
            }
        }
    }
    // Odd n: the last column.
    if ((n & 1) && threadIdx.x == 0) {
        const int64_t cl = n - 1;
        Acc xr0, xi0;
        if (X64) {
            const double2 p = static_cast<const double2*>(xv_)[cl];
            xr0 = p.x; xi0 = p.y;
        } else {
            const float2 p = static_cast<const float2*>(xv_)[cl];
            xr0 = p.x; xi0 = p.y;
        }
        for (int r = 0; r < nr; ++r) {
            const float2 a = A[(row0 + r) * lda + cl];
            acc[2 * r] = fma((Acc)a.x, xr0, fma(-(Acc)a.y, xi0, acc[2 * r]));
            acc[2 * r + 1] = fma((Acc)a.x, xi0, fma((Acc)a.y, xr0, acc[2 * r + 1]));
        }
    }
    // Per-thread partial sums (FP32 for the FP32 product) are combined across the block in FP64.
    double accd[2 * ROWS];
#pragma unroll
    for (int r = 0; r < 2 * ROWS; ++r) accd[r] = acc[r];
    block_sum<2 * ROWS, THREADS>(accd, red);
    if (threadIdx.x == 0) {
        double nrm = 0.0;
        for (int r = 0; r < nr; ++r) {
            double vr = accd[2 * r], vi = accd[2 * r + 1];
            if (bv_) {
                if (X64) {
                    const double2 bb = static_cast<const double2*>(bv_)[row0 + r];
                    vr = bb.x - vr;
                    vi = bb.y - vi;
                } else {
                    const float2 bb = static_cast<const float2*>(bv_)[row0 + r];
                    vr = static_cast<double>(bb.x - static_cast<float>(vr));
                    vi = static_cast<double>(bb.y - static_cast<float>(vi));
                }
                nrm += vr * vr + vi * vi;
            }
            if (X64) static_cast<double2*>(yv_)[row0 + r] = make_double2(vr, vi);
            else static_cast<float2*>(yv_)[row0 + r] = make_float2((float)vr, (float)vi);
        }
        if (part) part[blk] = nrm;
    }
}


}  // namespace sb
