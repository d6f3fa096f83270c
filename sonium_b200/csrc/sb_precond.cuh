// Block-Jacobi preconditioner kernels' bodies (internal), shared by the single-operator solver
// (precond.cu) and the batched solver (batch.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sb {

// Threads of the inversion CTA: the elimination updates BS x BS entries per pivot. Blocks of 128
// (128 KB of shared memory, one CTA per SM) use 1024 threads: the solve with blocks of 128 went
// 26.86 -> 26.59 ms at N = 20480 against 512 threads.
constexpr int bj_threads(int bs) { return bs >= 128 ? 1024 : 256; }

__device__ __forceinline__ float2 bj_cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Entries of the gathered block in FP32, from a complex64 or a complex128 matrix.
__device__ __forceinline__ float2 bj_entry(float2 v) { return v; }
__device__ __forceinline__ float2 bj_entry(double2 v) {
    return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
}

// Blocks of 128 with 1024 threads, in registers: thread (ty, tx) = (tid / 32, tid % 32) holds rows
// 4 ty .. 4 ty + 3 and columns 4 tx .. 4 tx + 3 of the block. Gauss-Jordan with implicit partial
// pivoting: step k takes as pivot p_k the largest |M[i][k]| among rows not yet pivots (the lowest
// index on ties) and exchanges it in place, with no row interchange (a_pk <- 1 / a_pk, a_pj <-
// a_pj / a_pk, a_ik <- -a_ik / a_pk, a_ij <- a_ij - a_ik a_pj / a_pk). Row p_k then holds x_k's
// equation and column c the coefficient of y_{p_c}, so inv[k][m] = M[p_k][c] with p_c = m. Only
// the step's column and scaled pivot row pass through shared memory (double-buffered by the step's
// parity, three barriers per step); a step costs 16 complex updates per thread.
template <class TA>
__device__ __forceinline__ void bj_invert128_reg(const TA* __restrict__ A, int64_t lda, int rows,
                                                 const int32_t* __restrict__ perm, float2* __restrict__ out,
                                                 int* __restrict__ status) {
    constexpr int BS = 128;
    __shared__ float2 s_col[2][BS];
    __shared__ float2 s_row[2][BS];
    __shared__ int s_piv[BS];             // p_k
    __shared__ int s_step[BS];            // the step at which row r was the pivot
    __shared__ unsigned char s_used[BS];
    __shared__ int s_p;
    __shared__ float2 s_inv;
    __shared__ int s_singular;
    const int tid = threadIdx.x, ty = tid >> 5, tx = tid & 31;
    float2 m[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = 4 * ty + a;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int j = 4 * tx + b;
            float2 v = make_float2(i == j ? 1.f : 0.f, 0.f);
            if (i < rows && j < rows) v = bj_entry(A[(int64_t)perm[i] * lda + perm[j]]);
            m[a][b] = v;
        }
    }
    if (tid < BS) s_used[tid] = 0;
    if (tid == 0) s_singular = 0;
    __syncthreads();
    for (int k = 0; k < BS; ++k) {
        const int buf = k & 1, kc = k & 3;
        // the column before the step
        if (tx == (k >> 2)) {
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                float2 v = m[a][0];
#pragma unroll
                for (int b = 1; b < 4; ++b)
                    if (b == kc) v = m[a][b];
                s_col[buf][4 * ty + a] = v;
            }
        }
        __syncthreads();
        // pivot: warp 0
        if (ty == 0) {
            float best = -1.f;
            int bi = BS;
#pragma unroll
            for (int q = 0; q < BS / 32; ++q) {
                const int i = tx + 32 * q;
                if (!s_used[i]) {
                    const float2 v = s_col[buf][i];
                    const float a = v.x * v.x + v.y * v.y;
                    if (a > best) {
                        best = a;
                        bi = i;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (tx == 0) {
                if (!(best > 0.f)) {
                    s_singular = 1;
                } else {
                    s_p = bi;
                    s_piv[k] = bi;
                    s_step[bi] = k;
                    s_used[bi] = 1;
                    const float2 v = s_col[buf][bi];
                    const float d = 1.f / (v.x * v.x + v.y * v.y);
                    s_inv = make_float2(v.x * d, -v.y * d);
                }
            }
        }
        __syncthreads();
        if (s_singular) break;
        const int p = s_p;
        const float2 inv = s_inv;
        // the pivot row, scaled
        if (ty == (p >> 2)) {
            const int pa = p & 3;
#pragma unroll
            for (int a = 0; a < 4; ++a)
                if (a == pa) {
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const float2 nv = (4 * tx + b == k) ? inv : bj_cmul(m[a][b], inv);
                        m[a][b] = nv;
                        s_row[buf][4 * tx + b] = nv;
                    }
                }
        }
        __syncthreads();
        float2 rv[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) rv[b] = s_row[buf][4 * tx + b];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = 4 * ty + a;
            if (i == p) continue;
            const float2 f = s_col[buf][i];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (4 * tx + b == k) {
                    const float2 q = bj_cmul(f, inv);
                    m[a][b] = make_float2(-q.x, -q.y);
                } else {
                    const float2 pr = bj_cmul(f, rv[b]);
                    m[a][b] = make_float2(m[a][b].x - pr.x, m[a][b].y - pr.y);
                }
            }
        }
    }
    if (s_singular) {
        if (tid == 0) atomicOr(status, 1);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int i = 4 * ty + a, j = 4 * tx + b;
                out[j * BS + i] = make_float2(i == j ? 1.f : 0.f, 0.f);
            }
        return;
    }
    // inv^T: out[m][k] = inv[k][m] = M[p_k][c], p_c = m
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int r = 4 * ty + a;
        const int kr = s_step[r];
#pragma unroll
        for (int b = 0; b < 4; ++b) out[s_piv[4 * tx + b] * BS + kr] = m[a][b];
    }
}

// One CTA (THREADS threads, BS * BS float2 of dynamic shared memory at M) per block: gather the
// diagonal block M = A[p_i][p_j], i, j < rows (identity beyond), rounded to complex64 when A is
// complex128, invert it in place (Gauss-Jordan, partial pivoting) and store its transpose at out.
// A zero pivot (a singular block) stores the identity and raises bit 0 of *status.
template <int BS, int THREADS, class TA = float2>
__device__ __forceinline__ void bj_invert_block(const TA* __restrict__ A, int64_t lda, int rows,
                                                const int32_t* __restrict__ perm, float2* __restrict__ out,
                                                int* __restrict__ status, float2* M) {
    if constexpr (BS == 128 && THREADS == 1024) {
        bj_invert128_reg<TA>(A, lda, rows, perm, out, status);
        return;
    }
    __shared__ int piv[BS];
    __shared__ float2 fcol[BS];
    __shared__ int s_p;
    __shared__ float2 s_inv;
    __shared__ int s_singular;
    for (int t = threadIdx.x; t < BS * BS; t += THREADS) {
        const int i = t / BS, j = t % BS;
        float2 v = make_float2(i == j ? 1.f : 0.f, 0.f);
        if (i < rows && j < rows) v = bj_entry(A[(int64_t)perm[i] * lda + perm[j]]);
        M[t] = v;
    }
    if (threadIdx.x == 0) s_singular = 0;
    __syncthreads();
    for (int k = 0; k < BS; ++k) {
        // pivot: the largest |M[i][k]|, i >= k (warp 0)
        if (threadIdx.x < 32) {
            float best = -1.f;
            int bi = k;
            for (int i = k + threadIdx.x; i < BS; i += 32) {
                const float2 v = M[i * BS + k];
                const float a = v.x * v.x + v.y * v.y;
                if (a > best) {
                    best = a;
                    bi = i;
                }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (threadIdx.x == 0) {
                s_p = bi;
                piv[k] = bi;
                if (!(best > 0.f)) s_singular = 1;
            }
        }
        __syncthreads();
        if (s_singular) break;
        const int p = s_p;
        if (p != k)
            for (int j = threadIdx.x; j < BS; j += THREADS) {
                const float2 t = M[k * BS + j];
                M[k * BS + j] = M[p * BS + j];
                M[p * BS + j] = t;
            }
        __syncthreads();
        if (threadIdx.x == 0) {
            const float2 v = M[k * BS + k];
            const float d = 1.f / (v.x * v.x + v.y * v.y);
            s_inv = make_float2(v.x * d, -v.y * d);
        }
        __syncthreads();
        const float2 inv = s_inv;
        // row k /= pivot, with M[k][k] taking 1 / pivot
        for (int j = threadIdx.x; j < BS; j += THREADS) M[k * BS + j] = (j == k) ? inv : bj_cmul(M[k * BS + j], inv);
        __syncthreads();
        // rows i != k: M[i][j] -= M[i][k] M[k][j], with M[i][k] taking -M[i][k] / pivot (column k
        // is read into fcol first: its entries are overwritten in the same pass)
        for (int i = threadIdx.x; i < BS; i += THREADS) fcol[i] = M[i * BS + k];
        __syncthreads();
        for (int t = threadIdx.x; t < BS * BS; t += THREADS) {
            const int i = t / BS, j = t % BS;
            if (i == k) continue;
            const float2 f = fcol[i];
            if (j == k) {
                const float2 q = bj_cmul(f, inv);
                M[t] = make_float2(-q.x, -q.y);
            } else {
                const float2 pr = bj_cmul(f, M[k * BS + j]);
                M[t] = make_float2(M[t].x - pr.x, M[t].y - pr.y);
            }
        }
        __syncthreads();
    }
    if (s_singular) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        for (int t = threadIdx.x; t < BS * BS; t += THREADS) {
            const int i = t / BS, j = t % BS;
            out[t] = make_float2(i == j ? 1.f : 0.f, 0.f);
        }
        return;
    }
    // Undo the row interchanges as column interchanges of the inverse, last first.
    for (int k = BS - 1; k >= 0; --k) {
        const int p = piv[k];
        if (p != k)
            for (int i = threadIdx.x; i < BS; i += THREADS) {
                const float2 t = M[i * BS + k];
                M[i * BS + k] = M[i * BS + p];
                M[i * BS + p] = t;
            }
        __syncthreads();
    }
    // inv^T: out[j][i] = M[i][j]
    for (int t = threadIdx.x; t < BS * BS; t += THREADS) {
        const int j = t / BS, i = t % BS;
        out[t] = M[i * BS + j];
    }
}

// Threads of the apply CTA: kBjSplit threads per row, each summing BS / kBjSplit columns (short
// dependent chains, 4x the parallelism of one thread per row).
constexpr int kBjSplit = 4;

// y[p_i] = sum_j inv[i][j] x[p_j] for one block (BS * kBjSplit threads: thread i + BS q takes
// row i, columns [q BS / kBjSplit, (q + 1) BS / kBjSplit)). The block's x is gathered into shared
// memory before any y is written, so x and y may be the same vector. V is float2 (FP32 vectors
// and arithmetic) or double2 (FP64 vectors; the FP32 inverse entries are exact in FP64 and the
// products are accumulated in FP64, so the preconditioner is the same linear map either way).
template <int BS, class V = float2>
__device__ __forceinline__ void bj_apply_block(const float2* __restrict__ invT, int rows,
                                               const int32_t* __restrict__ perm, const V* x, V* y) {
    using R = decltype(V{}.x);
    __shared__ V xs[BS];
    __shared__ V ps[kBjSplit][BS];
    const int i = threadIdx.x % BS, q = threadIdx.x / BS;
    if (threadIdx.x < BS) xs[i] = i < rows ? x[perm[i]] : V{R(0), R(0)};
    __syncthreads();
    constexpr int kCols = BS / kBjSplit;
    R re = R(0), im = R(0);
#pragma unroll 8
    for (int jj = 0; jj < kCols; ++jj) {
        const int j = q * kCols + jj;
        const float2 a = invT[j * BS + i];
        const V v = xs[j];
        const R ax = static_cast<R>(a.x), ay = static_cast<R>(a.y);
        re = fma(ax, v.x, fma(-ay, v.y, re));
        im = fma(ax, v.y, fma(ay, v.x, im));
    }
    ps[q][i] = V{re, im};
    __syncthreads();
    if (q == 0 && i < rows) {
        V t = ps[0][i];
#pragma unroll
        for (int u = 1; u < kBjSplit; ++u) {
            t.x += ps[u][i].x;
            t.y += ps[u][i].y;
        }
        y[perm[i]] = t;
    }
}

}  // namespace sb
