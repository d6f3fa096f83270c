// FP64-grade residual of a block of right-hand sides on the integer tensor cores: R = B - A X for
// the complex128 matrix A (N x N) and r complex128 vectors, as exact signed-8-bit slice products
// with INT32 accumulation (tcgen05 kind::i8): the Ozaki splitting.
//
// Reference: the block residual of block GMRES, R = B - A X by one apply_block per restart
// (crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:829) and in the true-
// residual check (block_true_metrics, :571-620), i.e. one complex GEMM in FP64
// (DenseMatrix::matmul_into, crates/sonium-solvers/crates/sonium-solvers-core/src/dense.rs:450-490).
//
// Splitting (error-free splitting of Ozaki, Ogita, Oishi and Rump, with integer slices): complex
// row i of A has the power-of-two scale sigma_i > max_j max(|Re a_ij|, |Im a_ij|), right-hand side c
// the scale tau_c > max_j max(|Re x_jc|, |Im x_jc|). A real value v of scale s is written exactly as
//     v / s = sum_{t=1..S} d_t 2^(1-7t) + e,  d_1 = rint(64 v / s), d_t = rint(128 e_{t-1}) (t > 1),
// every digit an integer in [-64, 64] and |e| <= 2^(-7S); S = kSlices = 8 (2^-56 of the scale).
// The product of slice t of A with slice u of X is exact in INT32 (digit products <= 2^12, at most
// 2^15 terms per accumulation, at most 8 products per diagonal: below 2^31). Products are summed
// by diagonal t + u = c, which shares the factor 2^(2-7c); diagonals c = 2 .. S + 1 are kept (36
// products). Per term the dropped diagonals and the two remainders are below 9.05 * 2^-56 of
// sigma_i tau_c, the size of an FP64 rounding of a term near the row's and the vector's largest
// entries; the FP64 epilogue adds a few roundings of the result. Not bit-identical to an FP64 GEMM.
//
// Layout: the slices of A are S int8 planes of the interleaved real matrix Ahat (rows 2i, 2i+1 =
// Re, Im of row i; the 2N x N layout of the BF16 block product), built once per assembled matrix;
// the slices of X are S planes of Xhat (per block of 128 right-hand sides 256 rows: Re x_c, then
// Im x_c), built per call. D = Ahat Xhat^T gives Re y = D[2i][c] - D[2i+1][128+c] and
// Im y = D[2i][128+c] + D[2i+1][c], combined between neighbouring TMEM lanes.
//
// Kernel: one CTA per (128 Ahat rows, 128 right-hand sides, K range), 6 warps. TMEM holds two
// 128 x 256 INT32 accumulators (all 512 columns). The diagonals go in passes of two, (cc, cc + 1)
// for cc = 2, 4, 6, 8: stage k = 1..cc of a K block holds A slice k and X slice cc + 1 - k, so
// diagonal cc + 1 is (stage k's A, stage k's X) and diagonal cc is (stage k - 1's A, stage k's X):
// a stage is released once the next one has been used, 20 stages per K block for 36 products.
// Warp 0 lane 0 issues the TMA loads (8-stage ring of 24 KB: A 128 x 64 and X 256 x 64 bytes,
// 64-byte swizzle), warp 1 lane 0 the MMAs (128 x 256 x 32); after every pass warps 2-5 read both
// accumulators, scale them to FP64 and add them into this CTA's own partial-sum tile (the earlier
// passes' sums loaded together, one latency per 32 columns) while the producer already loads the
// next pass. A last kernel forms R = B - sum of the K-range partials in a fixed order
// (deterministic: no atomics). Every wait is bounded; a timeout records an error in the status
// word, skips the stores, waits for its copies and MMAs in flight and frees TMEM.

#include <cuda.h>

#include <algorithm>

#include "sb_internal.cuh"
#include "sb_profile.cuh"
#include "sb_umma.cuh"

namespace sb {

namespace {

constexpr int kSlices = 8;
constexpr int kOzM = 128;                                // Ahat rows per tile (64 complex rows)
constexpr int kOzRhs = 128;                              // right-hand sides per tile (256 Xhat rows)
#ifndef SB_OZ_K
#define SB_OZ_K 128
#endif
constexpr int kOzK = SB_OZ_K;                            // K per stage: one swizzle row of int8 (128 B)
constexpr int kOzStages = kOzK == 128 ? 4 : 8;
constexpr uint32_t kOzABytes = kOzM * kOzK;              // 16 KB
constexpr uint32_t kOzXBytes = 2 * kOzRhs * kOzK;        // 32 KB
constexpr uint32_t kOzStageBytes = kOzABytes + kOzXBytes;
constexpr uint32_t kOzSmem = kOzStages * kOzStageBytes + 1024;
constexpr uint32_t kOzTmemCols = 512;
constexpr int kOzSegBlocks = (1 << 15) / kOzK;           // K blocks per exact INT32 accumulation
constexpr int kOzMaxPasses = 8;
constexpr int kOzThreads = 192;
constexpr int kOzMaxSplit = 4;

constexpr CUtensorMapSwizzle kOzSwizzle = kOzK == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;

// Shared-memory descriptor of a K-major tile row of kOzK bytes (the TMA box's swizzle).
__device__ __forceinline__ uint64_t oz_desc(uint32_t addr) {
    return kOzK == 128 ? umma::smem_desc_k_sw128(addr) : umma::smem_desc_k_sw64(addr);
}

constexpr int kErrOzProducer = 1;
constexpr int kErrOzMma = 2;
constexpr int kErrOzEpilogue = 4;

struct OzPasses {
    int count;
    int cc[kOzMaxPasses];                          // stage k = 1..cc holds A slice k, X slice cc + 1 - k
    int lo[kOzMaxPasses];                          // diagonal cc into accumulator columns 0..255
    int hi[kOzMaxPasses];                          // diagonal cc + 1 into columns 256..511
    double slo[kOzMaxPasses], shi[kOzMaxPasses];   // 2^(2 - 7 cc), 2^(2 - 7 (cc + 1))
};

OzPasses make_passes() {
    OzPasses p{};
    // diagonals 2 .. kSlices + 1 in pairs (cc, cc + 1); a last odd diagonal d alone as (d - 1, d)
    for (int c = 2; c <= kSlices + 1; c += 2) {
        const int i = p.count++;
        if (c + 1 <= kSlices + 1) {
            p.cc[i] = c;
            p.lo[i] = 1;
            p.hi[i] = 1;
        } else {
            p.cc[i] = c - 1;
            p.lo[i] = 0;
            p.hi[i] = 1;
        }
        p.slo[i] = std::ldexp(1.0, 2 - 7 * p.cc[i]);
        p.shi[i] = std::ldexp(1.0, 2 - 7 * (p.cc[i] + 1));
    }
    return p;
}

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Scale of a row of values with largest magnitude m: 2^e > m (frexp exponent); NaN for a row with a
// non-finite entry or beyond 2^1000; 0 for a row below 2^-1000 (its digits are zero).
__device__ __forceinline__ double slice_scale(double m, bool bad, double* inv) {
    if (bad || !(m < 0x1p1000)) {
        *inv = 0.0;
        return __longlong_as_double(0x7ff8000000000000ll);
    }
    if (m < 0x1p-1000) {
        *inv = 0.0;
        return 0.0;
    }
    int e = 0;
    frexp(m, &e);
    *inv = ldexp(1.0, -e);
    return ldexp(1.0, e);
}

// The kSlices digits of v * inv (|v * inv| < 1), exact.
__device__ __forceinline__ void slice_digits(double v, double inv, int (&d)[kSlices]) {
    double q = v * inv;
    if (!(fabs(q) < 1.0)) q = 0.0;
    q *= 64.0;
    double t = rint(q);
    d[0] = static_cast<int>(t);
    q -= t;
#pragma unroll
    for (int s = 1; s < kSlices; ++s) {
        q *= 128.0;
        t = rint(q);
        d[s] = static_cast<int>(t);
        q -= t;
    }
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
    return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) |
           ((uint32_t)(d & 0xff) << 24);
}

// Largest |Re|, |Im| of `len` complex values and whether any is non-finite, over the whole block.
__device__ double block_max(const double2* __restrict__ v, int64_t len, bool* bad_out) {
    __shared__ double red[32];
    double m = 0.0;
    bool bad = false;
    for (int64_t j = threadIdx.x; j < len; j += blockDim.x) {
        const double2 a = v[j];
        bad |= !isfinite(a.x) || !isfinite(a.y);
        m = fmax(m, fmax(fabs(a.x), fabs(a.y)));
    }
    bad = __syncthreads_or(bad) != 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double x = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (threadIdx.x == 0) red[0] = x;
    }
    __syncthreads();
    m = red[0];
    __syncthreads();
    *bad_out = bad;
    return m;
}

// Slices of `len` complex values v (scale from the whole run) into rows re_row / im_row of every
// plane (plane t at planes + t * plane_bytes, rows ldk bytes apart); 4 values per thread.
__device__ void write_slices(const double2* __restrict__ v, int64_t len, double inv, int8_t* __restrict__ planes,
                             int64_t plane_bytes, int64_t re_row, int64_t im_row, int64_t ldk) {
    for (int64_t j4 = threadIdx.x; j4 * 4 < len; j4 += blockDim.x) {
        int dr[4][kSlices], di[4][kSlices];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t j = j4 * 4 + u;
            const double2 a = j < len ? v[j] : make_double2(0.0, 0.0);
            slice_digits(a.x, inv, dr[u]);
            slice_digits(a.y, inv, di[u]);
        }
#pragma unroll
        for (int s = 0; s < kSlices; ++s) {
            int8_t* p = planes + s * plane_bytes;
            *reinterpret_cast<uint32_t*>(p + re_row * ldk + j4 * 4) = pack4(dr[0][s], dr[1][s], dr[2][s], dr[3][s]);
            *reinterpret_cast<uint32_t*>(p + im_row * ldk + j4 * 4) = pack4(di[0][s], di[1][s], di[2][s], di[3][s]);
        }
    }
}

// Matrix slices: one CTA per complex row i (rows 2i, 2i + 1 of Ahat).
__global__ void __launch_bounds__(256) k_oz_split_matrix(const double2* __restrict__ A, int64_t n, int64_t lda,
                                                          int8_t* __restrict__ planes, int64_t plane_bytes,
                                                          int64_t ldk, double* __restrict__ rowscale) {
    const int64_t i = blockIdx.x;
    const double2* row = A + i * lda;
    bool bad = false;
    const double m = block_max(row, n, &bad);
    double inv = 0.0;
    const double sigma = slice_scale(m, bad, &inv);
    if (threadIdx.x == 0) rowscale[i] = sigma;
    write_slices(row, n, inv, planes, plane_bytes, 2 * i, 2 * i + 1, ldk);
}

// Vector slices: one CTA per right-hand side c (rows 256 b + q and 256 b + 128 + q, c = 128 b + q).
__global__ void __launch_bounds__(256) k_oz_split_vectors(const double2* __restrict__ x, int64_t ldx, int64_t n,
                                                           int8_t* __restrict__ planes, int64_t plane_bytes,
                                                           int64_t ldk, double* __restrict__ colscale) {
    const int64_t c = blockIdx.x;
    const double2* v = x + c * ldx;
    bool bad = false;
    const double m = block_max(v, n, &bad);
    double inv = 0.0;
    const double tau = slice_scale(m, bad, &inv);
    if (threadIdx.x == 0) colscale[c] = tau;
    const int64_t b = c / kOzRhs, q = c % kOzRhs;
    write_slices(v, n, inv, planes, plane_bytes, b * 2 * kOzRhs + q, b * 2 * kOzRhs + kOzRhs + q, ldk);
}

__global__ void __launch_bounds__(kOzThreads, 1)
    k_ozaki_residual(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_x,
                     const OzPasses ps, int arows, int xrows, int nkb_all, int ksplit,
                     const double* __restrict__ rowscale, const double* __restrict__ colscale, int64_t n, int r,
                     double* __restrict__ part, int64_t ldp, int64_t zstride, int* __restrict__ status) {
#if defined(__CUDA_ARCH__)
    using namespace umma;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kOzStages], empty_bar[kOzStages], acc_bar, free_bar, final_bar;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ volatile int consumed;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rblock = blockIdx.x, mtile = blockIdx.y;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const int per = (nkb_all + ksplit - 1) / ksplit;
    const int kb0 = blockIdx.z * per;
    const int nkb = max(0, min(per, nkb_all - kb0));
    const int nseg = (nkb + kOzSegBlocks - 1) / kOzSegBlocks;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kOzStages; ++s) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        mbar_init(smem_u32(&acc_bar), 1);
        mbar_init(smem_u32(&free_bar), 4);
        mbar_init(smem_u32(&final_bar), 1);
        mbar_fence_init();
        abort_flag = 0;
        consumed = 0;
        prefetch_tmap(&tm_a);
        prefetch_tmap(&tm_x);
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), kOzTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tacc = tmem_base;
    int err = 0;
    if (warp == 0) {
        if (lane == 0) {
            // TMA producer: the same (pass, segment, K block, stage) order as the MMA issuer.
            int issued = 0;
            bool stop = false;
            for (int p = 0; p < ps.count && !stop; ++p) {
                const int cc = ps.cc[p];
                for (int sg = 0; sg < nseg && !stop; ++sg) {
                    const int kbs = kb0 + sg * kOzSegBlocks, kbe = kb0 + min(nkb, (sg + 1) * kOzSegBlocks);
                    for (int kb = kbs; kb < kbe && !stop; ++kb) {
                        for (int k = 1; k <= cc; ++k) {
                            const int s = issued % kOzStages, use = issued / kOzStages;
                            if (issued >= kOzStages && !mbar_wait(smem_u32(&empty_bar[s]), (use - 1) & 1)) {
                                err |= kErrOzProducer;
                                abort_flag = 1;
                            }
                            if (abort_flag) {
                                stop = true;
                                break;
                            }
                            const uint32_t st = base + s * kOzStageBytes;
                            const uint32_t fb = smem_u32(&full_bar[s]);
                            mbar_expect_tx(fb, kOzStageBytes);
                            tma_load_2d(st, &tm_a, fb, kb * kOzK, (k - 1) * arows + mtile * kOzM);
                            tma_load_2d(st + kOzABytes, &tm_x, fb, kb * kOzK, (cc - k) * xrows + rblock * 2 * kOzRhs);
                            ++issued;
                        }
                    }
                }
            }
            // Loads still in flight land before the CTA may exit.
            if (abort_flag) {
                __threadfence_block();
                for (int q = consumed; q < issued; ++q)
                    if (!mbar_wait(smem_u32(&full_bar[q % kOzStages]), (q / kOzStages) & 1)) err |= kErrOzProducer;
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            const uint32_t idesc = instr_desc_s8_s32(kOzM, 2 * kOzRhs);
            int g = 0, drains = 0;
            bool stop = false;
            for (int p = 0; p < ps.count && !stop; ++p) {
                const int cc = ps.cc[p], lo = ps.lo[p], hi = ps.hi[p];
                for (int sg = 0; sg < nseg && !stop; ++sg) {
                    // The epilogue has read the previous pass's accumulators.
                    if (drains > 0 && (abort_flag || !mbar_wait(smem_u32(&free_bar), (drains - 1) & 1))) {
                        if (!abort_flag) err |= kErrOzMma;
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    uint32_t acc_lo = 0, acc_hi = 0;
                    const int kbs = kb0 + sg * kOzSegBlocks, kbe = kb0 + min(nkb, (sg + 1) * kOzSegBlocks);
                    for (int kb = kbs; kb < kbe && !stop; ++kb) {
                        for (int k = 1; k <= cc; ++k) {
                            const int s = g % kOzStages;
                            if (abort_flag || !mbar_wait(smem_u32(&full_bar[s]), (g / kOzStages) & 1)) {
                                if (!abort_flag) err |= kErrOzMma;
                                abort_flag = 1;
                                stop = true;
                                break;
                            }
                            consumed = g + 1;
                            tc_fence_after();
                            const int sp = (g + kOzStages - 1) % kOzStages;  // stage k - 1 (k >= 2)
                            const uint32_t sa = base + s * kOzStageBytes, sa_prev = base + sp * kOzStageBytes;
#pragma unroll
                            for (int kk = 0; kk < kOzK / 32; ++kk) {
                                const uint64_t xd = oz_desc(sa + kOzABytes + kk * 32);
                                if (hi) {
                                    mma_s8(tacc + 256, oz_desc(sa + kk * 32), xd, idesc, acc_hi);
                                    acc_hi = 1;
                                }
                                if (lo && k >= 2) {
                                    mma_s8(tacc, oz_desc(sa_prev + kk * 32), xd, idesc, acc_lo);
                                    acc_lo = 1;
                                }
                            }
                            // Stage k is used by the MMAs of stage k (both diagonals) and the
                            // diagonal-cc MMA of stage k + 1 (none after the last stage of the block).
                            if (k >= 2) mma_commit(smem_u32(&empty_bar[sp]));
                            if (k == cc) mma_commit(smem_u32(&empty_bar[s]));
                            ++g;
                        }
                    }
                    // The pass's accumulators are complete (on the error path: the epilogue wakes
                    // and sees the abort flag).
                    mma_commit(smem_u32(&acc_bar));
                    ++drains;
                }
            }
            // Every MMA issued above has completed before tensor memory is released.
            mma_commit(smem_u32(&final_bar));
            if (!mbar_wait(smem_u32(&final_bar), 0)) err |= kErrOzMma;
        }
        __syncwarp();
    } else {
        // Epilogue: warps 2..5; warp w may read TMEM lanes 32 (w % 4) .. + 31.
        const int quad = warp & 3;
        const int t = quad * 32 + lane;                     // accumulator lane = Ahat row in the tile
        const int64_t row = (int64_t)mtile * kOzM + t;
        const int64_t i = row >> 1;
        const int parity = static_cast<int>(row & 1);
        const bool live_row = i < n;
        const double sigma = live_row ? rowscale[i] : 0.0;
        const uint32_t lane_addr = tacc + ((uint32_t)(quad * 32) << 16);
        double* pz = part + (int64_t)blockIdx.z * zstride;
        int drains = 0;
        bool stop = false;
        for (int p = 0; p < ps.count && !stop; ++p) {
            const int lo = ps.lo[p], hi = ps.hi[p];
            const double slo = ps.slo[p], shi = ps.shi[p];
            for (int sg = 0; sg < nseg; ++sg) {
                if (abort_flag) {
                    stop = true;
                    break;
                }
                const bool ok = mbar_wait(smem_u32(&acc_bar), drains & 1);
                if (!ok) {
                    err |= kErrOzEpilogue;
                    abort_flag = 1;
                }
                tc_fence_after();
                // tcgen05.ld is warp-collective: the decision to read is made per warp.
                if (__all_sync(0xffffffffu, ok && !abort_flag)) {
                    const bool first = (p == 0 && sg == 0);
#pragma unroll 1
                    for (int grp = 0; grp < kOzRhs / 32; ++grp) {
                        const int rhs0 = rblock * kOzRhs + grp * 32;
                        double* dst0 = pz + ((int64_t)rhs0 * ldp + i) * 2 + parity;
                        // The partial sums of the earlier passes, loaded together (one latency).
                        double v[32];
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            v[c] = (!first && live_row && rhs0 + c < r) ? dst0[(int64_t)c * ldp * 2] : 0.0;
                        const double tau_l = rhs0 + lane < r ? colscale[rhs0 + lane] : 0.0;
                        uint32_t a[32], b[32];
                        if (lo) {
                            tmem_ld32_raw(lane_addr + grp * 32, a);            // D vs Re x (diagonal cc)
                            tmem_ld32_raw(lane_addr + kOzRhs + grp * 32, b);   // D vs Im x
#pragma unroll
                            for (int c = 0; c < 32; ++c) {
                                const int nb = __shfl_xor_sync(0xffffffffu, (int)b[c], 1);
                                const double da = (double)(int)a[c], dn = (double)nb;
                                const double tau = __shfl_sync(0xffffffffu, tau_l, c);
                                v[c] = fma((parity ? da + dn : da - dn) * slo, sigma * tau, v[c]);
                            }
                        }
                        if (hi) {
                            tmem_ld32_raw(lane_addr + 256 + grp * 32, a);           // diagonal cc + 1
                            tmem_ld32_raw(lane_addr + 256 + kOzRhs + grp * 32, b);
#pragma unroll
                            for (int c = 0; c < 32; ++c) {
                                const int nb = __shfl_xor_sync(0xffffffffu, (int)b[c], 1);
                                const double da = (double)(int)a[c], dn = (double)nb;
                                const double tau = __shfl_sync(0xffffffffu, tau_l, c);
                                v[c] = fma((parity ? da + dn : da - dn) * shi, sigma * tau, v[c]);
                            }
                        }
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (live_row && rhs0 + c < r) dst0[(int64_t)c * ldp * 2] = v[c];
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&free_bar));
                ++drains;
            }
        }
        // A K range with no blocks (more splits than blocks) contributes zeros.
        if (nseg == 0 && live_row) {
            for (int rhs = rblock * kOzRhs; rhs < min(r, (rblock + 1) * kOzRhs); ++rhs)
                pz[((int64_t)rhs * ldp + i) * 2 + parity] = 0.0;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tacc, kOzTmemCols);
    if (err) atomicOr(status, err);
#endif
}

// res_c = b_c - sum_z part_z[c] (z ascending); zstride in complex entries.
__global__ void k_oz_combine(const double2* __restrict__ b, int64_t ldb, const double2* __restrict__ part,
                             int64_t ldp, int64_t zstride, int ks, int64_t n, int r, double2* __restrict__ res,
                             int64_t ldr) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * r) return;
    const int64_t c = t / n, i = t % n;
    double2 s = part[c * ldp + i];
    for (int z = 1; z < ks; ++z) {
        const double2 q = part[z * zstride + c * ldp + i];
        s.x += q.x;
        s.y += q.y;
    }
    const double2 bv = b[c * ldb + i];
    res[c * ldr + i] = make_double2(bv.x - s.x, bv.y - s.y);
}

}  // namespace

// Slices of an operator's complex128 matrix and the per-call vector slices (internal).
struct OzakiWork {
    int64_t n = 0, ldk = 0, arows = 0;
    DevBuf a, rowscale, status;
    CUtensorMap tm_a;
    int rblocks = 0;
    DevBuf x, colscale;
    CUtensorMap tm_x;
    DevBuf part;
};

void ozaki_release(Operator& op) {
    delete static_cast<OzakiWork*>(op.ozaki);
    op.ozaki = nullptr;
}

int ozaki_status(const Operator& op, bool reset) {
    OzakiWork* w = static_cast<OzakiWork*>(op.ozaki);
    if (!w) return 0;
    int v = 0;
    SB_CUDA(cudaMemcpy(&v, w->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (reset && v) memset_sync(w->status.p, 0, sizeof(int));
    return v;
}

static OzakiWork& ozaki_prepare(const Operator& cop, cudaStream_t s) {
    Operator& op = const_cast<Operator&>(cop);
    if (op.ozaki) return *static_cast<OzakiWork*>(op.ozaki);
    SB_REQUIRE(op.A64.p, SB_ERR_INVALID_ARGUMENT, "block residual: the operator holds no complex128 matrix");
    OzakiWork* w = new OzakiWork();
    op.ozaki = w;
    try {
        w->n = op.n;
        w->ldk = cdiv(op.n, kOzK) * kOzK;
        w->arows = cdiv(2 * op.n, kOzM) * kOzM;
        const size_t plane = (size_t)w->arows * w->ldk;
        w->a.alloc(plane * kSlices);
        w->rowscale.alloc(sizeof(double) * op.n);
        w->status.alloc(sizeof(int));
        SB_CUDA(cudaMemsetAsync(w->a.p, 0, plane * kSlices, s));
        SB_CUDA(cudaMemsetAsync(w->status.p, 0, sizeof(int), s));
        k_oz_split_matrix<<<static_cast<unsigned>(op.n), 256, 0, s>>>(op.A64.as<double2>(), op.n, op.n,
                                                                      w->a.as<int8_t>(), (int64_t)plane, w->ldk,
                                                                      w->rowscale.as<double>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        w->tm_a = make_tmap_2d(w->a.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, (int64_t)kSlices * w->arows, w->ldk, kOzK,
                               kOzM, kOzSwizzle);
        SB_CUDA(cudaFuncSetAttribute(k_ozaki_residual, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem));
    } catch (...) {
        ozaki_release(op);
        throw;
    }
    return *w;
}

// K splits: the count (1..4) with the fewest CTA waves per unit of work, every split at least 8
// K blocks; ties to fewer splits.
static int ozaki_splits(int64_t tiles, int nkb, int sms) {
    int best = 1;
    double best_t = 1e300;
    for (int ks = 1; ks <= kOzMaxSplit; ++ks) {
        if (ks > 1 && nkb < 8 * ks) break;
        const double waves = (double)cdiv(tiles * ks, sms) / ks;
        if (waves < best_t - 1e-9) {
            best_t = waves;
            best = ks;
        }
    }
    return best;
}

void ozaki_residual(const Operator& op, const double2* b, int64_t ldb, const double2* x, int64_t ldx, int r,
                    double2* res, int64_t ldr, cudaStream_t s) {
    SB_REQUIRE(r >= 1, SB_ERR_INVALID_ARGUMENT, "block residual: r must be positive");
    SB_REQUIRE(op.n <= ((int64_t)1 << 26), SB_ERR_INVALID_ARGUMENT, "block residual: n too large");
    OzakiWork& w = ozaki_prepare(op, s);
    const int rblocks = static_cast<int>(cdiv(r, kOzRhs));
    if (rblocks > w.rblocks) {
        const int64_t xrows_new = (int64_t)rblocks * 2 * kOzRhs;
        const size_t bytes = (size_t)xrows_new * w.ldk * kSlices;
        w.x.alloc(bytes);
        w.colscale.alloc(sizeof(double) * rblocks * kOzRhs);
        SB_CUDA(cudaMemsetAsync(w.x.p, 0, bytes, s));
        w.rblocks = rblocks;
        w.tm_x = make_tmap_2d(w.x.p, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, (int64_t)kSlices * xrows_new, w.ldk, kOzK,
                              2 * kOzRhs, kOzSwizzle);
    }
    const int64_t xrows = (int64_t)w.rblocks * 2 * kOzRhs;  // rows per plane of the allocated X slices
    const int64_t tiles = (int64_t)rblocks * (w.arows / kOzM);
    const int nkb = static_cast<int>(w.ldk / kOzK);
    const int ks = ozaki_splits(tiles, nkb, device_sm_count(op.device));
    const int64_t ldp = op.n;
    const int64_t zstride = (int64_t)r * ldp;  // complex entries per K-range partial
    const size_t part_bytes = sizeof(double2) * (size_t)zstride * ks;
    if (w.part.bytes < part_bytes) w.part.alloc(part_bytes);
    ProfScope prof(SB_PROF_RESIDUAL, s);
    k_oz_split_vectors<<<static_cast<unsigned>(r), 256, 0, s>>>(x, ldx, op.n, w.x.as<int8_t>(), xrows * w.ldk, w.ldk,
                                                                w.colscale.as<double>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    const dim3 grid(static_cast<unsigned>(rblocks), static_cast<unsigned>(w.arows / kOzM), static_cast<unsigned>(ks));
    k_ozaki_residual<<<grid, kOzThreads, kOzSmem, s>>>(
        w.tm_a, w.tm_x, make_passes(), static_cast<int>(w.arows), static_cast<int>(xrows), nkb, ks,
        w.rowscale.as<double>(), w.colscale.as<double>(), op.n, r, w.part.as<double>(), ldp, 2 * zstride,
        w.status.as<int>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    const int64_t tot = op.n * r;
    k_oz_combine<<<static_cast<unsigned>(cdiv(tot, 256)), 256, 0, s>>>(b, ldb, w.part.as<double2>(), ldp, zstride, ks,
                                                                     op.n, r, res, ldr);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

}  // namespace sb
