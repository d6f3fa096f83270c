// Row-block body of the complex64 matrix-vector product, shared by the single-instance kernel
// (blas.cu) and the batched sweep kernel (batch.cu) (internal).
//
// Reference: DenseMatrix::matvec_into -> gemv_c64 (crates/sonium-solvers/crates/sonium-solvers-core/
// src/dense.rs:416-427) and cublasCgemv (crates/sonium-compute/src/cuda/cublas_blas23.rs:165).
// HBM-bound: each CTA owns ROWS rows, streams them with 128-bit evict-first loads (UNROLL loads in
// flight per row and thread) and reuses each x element across its rows.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "sb_device.cuh"

namespace sb {

// Threads of every matrix-vector product CTA.
constexpr int kGemvThreads = 256;
// Rows per CTA and 16-byte loads in flight per row and thread of the complex64 products, single
// operator and batched (measured at N = 20480 against 4 rows x 2 loads: FP32 vectors 1 x 4, 0.49
// ms against 0.51-0.52 ms; FP64 vectors 2 x 4, 0.49-0.53 ms against 0.55-0.60 ms: their x is
// twice a row's bytes, so two rows share each x load). Few rows and many CTAs keep more loads in
// flight per SM than wide row blocks with their register cost.
constexpr int kGemv64Rows = 1, kGemv64Unroll = 4;
constexpr int kGemvX64Rows = 2, kGemvX64Unroll = 4;

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



// ---------------------------------------------------------------------------------------------
// Complex-half matrix: one uint32 per entry (FP16 real part in the low half, imaginary part in
// the high half), the entries of a complex64 matrix times a power-of-two scale, rows lda entries
// apart (lda a multiple of 4). FP32 vectors and accumulation; results times the inverse scale
// (exact). 4 bytes per entry: half the HBM traffic of the complex64 product.
// ---------------------------------------------------------------------------------------------
// Launch shape of the complex-half products (single operator and batched): 2 rows a CTA, 4 loads
// of 16 bytes in flight per row and thread (measured at N = 20480: 0.244-0.245 ms a launch; 16
// rows x 1 load, which shares each x chunk across 16 rows but needs 128 registers, 2 CTAs per SM,
// 0.250-0.253 ms; 8 x 2 0.291 ms; 16 x 2 0.348 ms; 4 x 4 0.342 ms).
constexpr int kGemv16PRows = 2;
constexpr int kGemv16PUnroll = 4;
// Row blocks of the batched solver's largest-part scan and conversion to the complex-half copy.
constexpr int kGemv16Rows = 16;
constexpr int kHalfThreads = 256;  // threads of the largest-part scan and the conversion

__device__ __forceinline__ float2 half_pair(uint32_t u) {
    __half2 h;
    memcpy(&h, &u, sizeof(h));
    return __half22float2(h);
}

__device__ __forceinline__ void cmac(float& re, float& im, float2 a, float xr, float xi) {
    re = fmaf(a.x, xr, fmaf(-a.y, xi, re));
    im = fmaf(a.x, xi, fmaf(a.y, xr, im));
}

// Rows [blk * ROWS, blk * ROWS + ROWS) of y = (A x) / scale, or b - (A x) / scale with part[blk]
// = the squared norm of those rows; the inverse scale is inv_scale[row] (kRowScale) or
// inv_scale[0]. Called by every thread of a THREADS-wide CTA.
template <int ROWS, int THREADS, int UNROLL, bool kRowScale = false>
__device__ __forceinline__ void gemv_c16_block(const uint32_t* __restrict__ A, int64_t n, int64_t lda,
                                               const float* __restrict__ inv_scale, const float2* __restrict__ x,
                                               float2* __restrict__ y, const float2* __restrict__ b,
                                               double* __restrict__ part, int64_t blk) {
    __shared__ double red[(THREADS / 32) * 2 * ROWS];
    const int64_t row0 = blk * (int64_t)ROWS;
    const int nr = static_cast<int>((n - row0) < ROWS ? (n - row0) : ROWS);
    float acc[2 * ROWS];
#pragma unroll
    for (int r = 0; r < 2 * ROWS; ++r) acc[r] = 0.f;
    const int64_t n4 = n >> 2;    // uint4 = four complex-half entries
    const int64_t ld4 = lda >> 2;  // lda is a multiple of 4: every row starts 16-byte aligned
    const uint4* A4 = reinterpret_cast<const uint4*>(A + row0 * lda);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    int64_t c = threadIdx.x;
    for (; c + (UNROLL - 1) * THREADS < n4; c += UNROLL * THREADS) {
        float4 xa[UNROLL], xb[UNROLL];
        uint4 av[UNROLL][ROWS];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const int64_t cc = c + u * THREADS;
            xa[u] = __ldg(x4 + 2 * cc);
            xb[u] = __ldg(x4 + 2 * cc + 1);
#pragma unroll
            for (int r = 0; r < ROWS; ++r) av[u][r] = (r < nr) ? __ldcs(A4 + r * ld4 + cc) : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(av[u][r].x), xa[u].x, xa[u].y);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(av[u][r].y), xa[u].z, xa[u].w);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(av[u][r].z), xb[u].x, xb[u].y);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(av[u][r].w), xb[u].z, xb[u].w);
            }
    }
    for (; c < n4; c += THREADS) {
        const float4 xa = x4[2 * c], xb = x4[2 * c + 1];
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            if (r < nr) {
                const uint4 a = __ldcs(A4 + r * ld4 + c);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(a.x), xa.x, xa.y);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(a.y), xa.z, xa.w);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(a.z), xb.x, xb.y);
                cmac(acc[2 * r], acc[2 * r + 1], half_pair(a.w), xb.z, xb.w);
            }
        }
    }
    // n not a multiple of 4: the last one to three columns, one thread each.
    {
        const int64_t cl = 4 * n4 + threadIdx.x;
        if (cl < n) {
            const float2 xv = x[cl];
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
                if (r < nr) cmac(acc[2 * r], acc[2 * r + 1], half_pair(A[(row0 + r) * lda + cl]), xv.x, xv.y);
        }
    }
    double accd[2 * ROWS];
#pragma unroll
    for (int r = 0; r < 2 * ROWS; ++r) accd[r] = acc[r];
    block_sum<2 * ROWS, THREADS>(accd, red);
    if (threadIdx.x == 0) {
        double nrm = 0.0;
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            if (r >= nr) break;
            const float inv = kRowScale ? inv_scale[row0 + r] : *inv_scale;
            float vr = static_cast<float>(accd[2 * r]) * inv, vi = static_cast<float>(accd[2 * r + 1]) * inv;
            if (b) {
                const float2 bb = b[row0 + r];
                vr = bb.x - vr;
                vi = bb.y - vi;
                nrm += static_cast<double>(vr) * vr + static_cast<double>(vi) * vi;
            }
            y[row0 + r] = make_float2(vr, vi);
        }
        if (part) part[blk] = nrm;
    }
}

// Largest |re| / |im| over rows row, row + step, ... < row_end of a complex64 matrix (lda even),
// atomically maxed into *out as float bits (non-negative floats order as their bits); a
// non-finite part counts as +inf. Called by every thread of a kHalfThreads-wide CTA.
__device__ __forceinline__ void half_absmax_rows(const float2* __restrict__ A, int64_t n, int64_t lda, int64_t row,
                                                 int64_t row_end, int64_t step, unsigned* __restrict__ out) {
    __shared__ float red[kHalfThreads / 32];
    float m = 0.f;
    const int64_t n2 = n >> 1;
    for (; row < row_end; row += step) {
        const float4* r4 = reinterpret_cast<const float4*>(A + row * lda);
        for (int64_t c = threadIdx.x; c < n2; c += kHalfThreads) {
            const float4 v = __ldcs(r4 + c);
            m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
            if (!(fabsf(v.x) + fabsf(v.y) + fabsf(v.z) + fabsf(v.w) <= 3.4e38f)) m = INFINITY;
        }
        if ((n & 1) && threadIdx.x == 0) {
            const float2 v = A[row * lda + n - 1];
            m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
            if (!(fabsf(v.x) + fabsf(v.y) <= 3.4e38f)) m = INFINITY;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kHalfThreads / 32; ++w) m = fmaxf(m, red[w]);
        atomicMax(out, __float_as_uint(m));
    }
}

// aux[1] = scale = 2^e with the largest part (aux[0]) times scale in [2^13, 2^14): exact to apply
// and undo, a factor 4 below FP16 overflow, and parts 2^24 below the largest still normal.
// aux[2] = 1 / scale. One thread.
__device__ __forceinline__ void half_scale_from_max(unsigned* aux) {
    const float m = __uint_as_float(aux[0]);
    float sc = 1.f;
    if (m > 0.f && m <= 3.4e38f) {
        int e = 13 - ilogbf(m);
        e = e < -120 ? -120 : (e > 120 ? 120 : e);
        sc = ldexpf(1.f, e);
    }
    aux[1] = __float_as_uint(sc);
    aux[2] = __float_as_uint(1.f / sc);
}

// Power-of-two scale of a row (or matrix) whose largest |re|, |im| is m: m times the scale lies in
// [2^13, 2^14) (exact to apply and undo, a factor 4 below FP16 overflow); 1 for m = 0 or non-finite.
__device__ __forceinline__ float half_scale_for(float m) {
    if (!(m > 0.f && m <= 3.4e38f)) return 1.f;
    int e = 13 - ilogbf(m);
    e = e < -120 ? -120 : (e > 120 ? 120 : e);
    return ldexpf(1.f, e);
}

// FP16 (re, im) of v times sc, packed as re | im << 16; *bad |= 1 when a part leaves the FP16 range.
__device__ __forceinline__ uint32_t half_pack(float2 v, float sc, int* bad) {
    const float a = v.x * sc, b = v.y * sc;
    if (!(fabsf(a) <= 65504.f && fabsf(b) <= 65504.f)) *bad = 1;
    const __half2 h = __floats2half2_rn(a, b);
    uint32_t w;
    memcpy(&w, &h, sizeof(w));
    return w;
}

// H[row][c] = FP16(scale A[row][c]) (round to nearest) for c < n, 0 for n <= c < lda16, over rows
// row, row + step, ... < row_end; four entries a thread. Called by a kHalfThreads-wide CTA.
__device__ __forceinline__ void half_convert_rows(const float2* __restrict__ A, int64_t n, int64_t lda32,
                                                  const unsigned* __restrict__ aux, uint32_t* __restrict__ H,
                                                  int64_t lda16, int64_t row, int64_t row_end, int64_t step) {
    const float sc = __uint_as_float(aux[1]);
    const int64_t q = lda16 >> 2;  // chunks of four entries per row
    for (; row < row_end; row += step) {
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
            for (int j = 0; j < 4; ++j) {
                const __half2 h = __floats2half2_rn(v[j].x * sc, v[j].y * sc);
                memcpy(&w[j], &h, sizeof(h));
            }
            __stcs(reinterpret_cast<uint4*>(H + row * lda16 + c), make_uint4(w[0], w[1], w[2], w[3]));
        }
    }
}

}  // namespace sb
