// Tensor-core block product for many right-hand sides: Y = A X with the complex matrix A (N x N)
// and R complex vectors X, as real BF16 products on the 5th-generation tensor cores (tcgen05,
// operands staged by TMA, FP32 accumulators in tensor memory).
//
// Reference: the block product of LinearOperator::apply_block (crates/sonium-solvers/crates/
// sonium-solvers-core/src/traits.rs:2949-3120) -> DenseMatrix::matmul_into (dense.rs:450-490),
// which block GMRES (crates/sonium-solvers/crates/sonium-solvers-iterative/src/block_gmres.rs:163)
// calls once per block step; there it is one complex GEMM in FP64.
//
// Arithmetic: each real operand is split into two BF16 terms, a = a_hi + a_lo with
// a_hi = bf16(a) and a_lo = bf16(a - a_hi) (16 significant bits together); a product is
// a_hi b_hi + a_hi b_lo + a_lo b_hi (the a_lo b_lo term, ~2^-16 relative, is dropped), accumulated
// in FP32 on the tensor cores. The complex product is arranged as one real GEMM: the rows of A are
// interleaved as (Re A_i, Im A_i) -> a 2N x N real matrix Ahat; a block of 128 right-hand sides is
// the 256 x N real matrix Xhat = (Re X_c ; Im X_c); D = Ahat Xhat^T gives
//   Re Y_ic = D[2i][c] - D[2i+1][128+c],   Im Y_ic = D[2i][128+c] + D[2i+1][c],
// combined in the epilogue between neighbouring TMEM lanes with one shuffle.
//
// Kernel structure: persistent, one CTA per SM walking the work units (128 Ahat rows, 128
// right-hand sides, K half; right-hand-side block fastest, so the CTAs running side by side read an
// Ahat tile's second use from L2). 6 warps: lane 0 of warp 0 issues the TMA loads of a four-stage
// ring that runs on across units (per stage: Ahat hi/lo 128 x 32 and Xhat hi/lo 256 x 32 BF16
// tiles, 64-byte swizzle, 48 KB), lane 0 of warp 1 issues 6 MMAs (128 x 256 x 16) per stage and
// commits them to the stage's "empty" barrier, and warps 2-5 read the accumulator (tcgen05.ld) and
// write Y. TMEM holds two 128 x 256 FP32 accumulators (all 512 columns) used by alternate units,
// so the epilogue of one unit overlaps the K loop of the next. All waits are bounded; a timeout
// records an error in the status word, skips the stores, waits for its copies and MMAs in flight
// and still releases tensor memory.

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "sb_device.cuh"
#include "sb_internal.cuh"
#include "sb_profile.cuh"
#include "sb_umma.cuh"

namespace sb {

namespace {

constexpr int kTileM = 128;       // Ahat rows per CTA (64 complex rows)
constexpr int kTileRhs = kTensorRhsTile;  // right-hand sides per CTA (256 Xhat rows)
constexpr int kTileK = 32;        // K per stage: one 64-byte swizzle row of BF16
constexpr int kStages = 4;        // stages in flight: three stage times to hide a TMA load
constexpr uint32_t kABytes = kTileM * kTileK * 2;           // 8 KB per term
constexpr uint32_t kXBytes = 2 * kTileRhs * kTileK * 2;     // 16 KB per term
constexpr uint32_t kStageBytes = 2 * kABytes + 2 * kXBytes; // 48 KB
constexpr uint32_t kSmemBytes = kStages * kStageBytes + 1024;
constexpr uint32_t kTmemCols = 2 * kTileRhs;                // 256 FP32 columns

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Status-word codes of the block product.
constexpr int kErrTimeoutProducer = 1;
constexpr int kErrTimeoutMma = 2;
constexpr int kErrTimeoutEpilogue = 4;

// Persistent: grid = one CTA per SM; the CTA walks the work units u = blockIdx.x + t gridDim.x
// (unit = right-hand-side block fastest, then row tile, then K half). 6 warps: warp 0 lane 0 the
// TMA producer (the stage ring runs on across units), warp 1 lane 0 the MMA issuer, warps 2-5 the
// epilogue. Two 256-column accumulators (all 512 TMEM columns) alternate between units, so the
// epilogue of unit t overlaps the K loop of unit t + 1.
constexpr int kPThreads = 192;
constexpr uint32_t kPTmemCols = 2 * kTmemCols;

__device__ __forceinline__ void unit_coords(int64_t u, int rblocks, int mtiles, int& rb, int& mt, int& kz) {
    rb = static_cast<int>(u % rblocks);
    const int64_t rest = u / rblocks;
    mt = static_cast<int>(rest % mtiles);
    kz = static_cast<int>(rest / mtiles);
}

__global__ void __launch_bounds__(kPThreads, 1)
    k_block_bf16x3(const __grid_constant__ CUtensorMap tm_a_hi, const __grid_constant__ CUtensorMap tm_a_lo,
                   const __grid_constant__ CUtensorMap tm_x_hi, const __grid_constant__ CUtensorMap tm_x_lo,
                   int ldk, int64_t n, int r, float* __restrict__ y, int64_t ldy, int* __restrict__ status,
                   const int* __restrict__ block_gate, int ksplit, int rblocks, int mtiles) {
#if defined(__CUDA_ARCH__)
    using namespace umma;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], acc_full[2], acc_empty[2], final_bar;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ volatile int consumed;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const int64_t units = (int64_t)rblocks * mtiles * ksplit;
    const int nkb_all = ldk / kTileK;
    const int per = (nkb_all + ksplit - 1) / ksplit;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 4);
        }
        mbar_init(smem_u32(&final_bar), 1);
        mbar_fence_init();
        abort_flag = 0;
        consumed = 0;
        prefetch_tmap(&tm_a_hi);
        prefetch_tmap(&tm_a_lo);
        prefetch_tmap(&tm_x_hi);
        prefetch_tmap(&tm_x_lo);
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), kPTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tacc = tmem_base;
    int err = 0;
    if (warp == 0) {
        if (lane == 0) {
            // TMA producer: every unit's K blocks, one ring across the units.
            int issued = 0;
            bool stop = false;
            for (int64_t u = blockIdx.x; u < units && !stop; u += gridDim.x) {
                int rb, mt, kz;
                unit_coords(u, rblocks, mtiles, rb, mt, kz);
                if (block_gate && block_gate[rb] == 0) continue;
                const int kb0 = kz * per;
                const int nkb = min(per, nkb_all - kb0);
                for (int kb = 0; kb < nkb; ++kb) {
                    const int s = issued % kStages, use = issued / kStages;
                    if (issued >= kStages && !mbar_wait(smem_u32(&empty_bar[s]), (use - 1) & 1)) {
                        err |= kErrTimeoutProducer;
                        abort_flag = 1;
                    }
                    if (abort_flag) {
                        stop = true;
                        break;
                    }
                    const uint32_t st = base + s * kStageBytes;
                    const uint32_t fb = smem_u32(&full_bar[s]);
                    mbar_expect_tx(fb, kStageBytes);
                    const int kx = (kb0 + kb) * kTileK;
                    tma_load_2d(st, &tm_a_hi, fb, kx, mt * kTileM);
                    tma_load_2d(st + kABytes, &tm_a_lo, fb, kx, mt * kTileM);
                    tma_load_2d(st + 2 * kABytes, &tm_x_hi, fb, kx, rb * 2 * kTileRhs);
                    tma_load_2d(st + 2 * kABytes + kXBytes, &tm_x_lo, fb, kx, rb * 2 * kTileRhs);
                    ++issued;
                }
            }
            // Loads still in flight land before the CTA may exit.
            if (abort_flag) {
                __threadfence_block();
                for (int q = consumed; q < issued; ++q)
                    if (!mbar_wait(smem_u32(&full_bar[q % kStages]), (q / kStages) & 1)) err |= kErrTimeoutProducer;
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: unit t into accumulator t & 1, once the epilogue has read it out.
            const uint32_t idesc = instr_desc_bf16_f32(kTileM, 2 * kTileRhs);
            int g = 0, t = 0;
            bool stop = false;
            for (int64_t u = blockIdx.x; u < units && !stop; u += gridDim.x) {
                int rb, mt, kz;
                unit_coords(u, rblocks, mtiles, rb, mt, kz);
                if (block_gate && block_gate[rb] == 0) continue;
                const int buf = t & 1;
                if (t >= 2 && (abort_flag || !mbar_wait(smem_u32(&acc_empty[buf]), ((t >> 1) - 1) & 1))) {
                    if (!abort_flag) err |= kErrTimeoutMma;
                    abort_flag = 1;
                    mma_commit(smem_u32(&acc_full[buf]));  // the epilogue wakes and sees the flag
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tacc + buf * kTmemCols;
                const int nkb = min(per, nkb_all - kz * per);
                for (int kb = 0; kb < nkb; ++kb) {
                    const int s = g % kStages;
                    if (abort_flag || !mbar_wait(smem_u32(&full_bar[s]), (g / kStages) & 1)) {
                        if (!abort_flag) err |= kErrTimeoutMma;
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    consumed = g + 1;
                    tc_fence_after();
                    const uint32_t st = base + s * kStageBytes;
#pragma unroll
                    for (int kk = 0; kk < kTileK / 16; ++kk) {
                        const uint64_t a_hi = smem_desc_k_sw64(st + kk * 32);
                        const uint64_t a_lo = smem_desc_k_sw64(st + kABytes + kk * 32);
                        const uint64_t x_hi = smem_desc_k_sw64(st + 2 * kABytes + kk * 32);
                        const uint64_t x_lo = smem_desc_k_sw64(st + 2 * kABytes + kXBytes + kk * 32);
                        mma_bf16(acc, a_hi, x_hi, idesc, (kb | kk) != 0 ? 1u : 0u);
                        mma_bf16(acc, a_hi, x_lo, idesc, 1u);
                        mma_bf16(acc, a_lo, x_hi, idesc, 1u);
                    }
                    mma_commit(smem_u32(&empty_bar[s]));
                    ++g;
                }
                // The unit's accumulator is complete (on the error path: the epilogue wakes and
                // sees the abort flag).
                mma_commit(smem_u32(&acc_full[buf]));
                ++t;
            }
            // Every MMA issued above has completed before tensor memory is released.
            mma_commit(smem_u32(&final_bar));
            if (!mbar_wait(smem_u32(&final_bar), 0)) err |= kErrTimeoutMma;
        }
        __syncwarp();
    } else {
        // Epilogue: warps 2..5; warp w reads TMEM lanes 32 (w % 4) .. + 31.
        const int quad = warp & 3;
        const int tl = quad * 32 + lane;  // TMEM lane = Ahat row within the tile
        int t = 0;
        for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
            int rb, mt, kz;
            unit_coords(u, rblocks, mtiles, rb, mt, kz);
            if (block_gate && block_gate[rb] == 0) continue;
            if (abort_flag) break;
            const int buf = t & 1;
            const bool ok = mbar_wait(smem_u32(&acc_full[buf]), (t >> 1) & 1);
            if (!ok) {
                err |= kErrTimeoutEpilogue;
                abort_flag = 1;
            }
            tc_fence_after();
            // tcgen05.ld is warp-collective: the decision to read the accumulator is made per warp.
            if (__all_sync(0xffffffffu, ok && !abort_flag)) {
                const int64_t row = (int64_t)mt * kTileM + tl;
                const int64_t i = row >> 1;
                const int parity = static_cast<int>(row & 1);
                const uint32_t lane_addr = tacc + buf * kTmemCols + ((uint32_t)(quad * 32) << 16);
#pragma unroll 1
                for (int gq = 0; gq < kTileRhs / 32; ++gq) {
                    float a[32], b[32];
                    tmem_ld32(lane_addr + gq * 32, a);              // D[t][c]       (Re X part)
                    tmem_ld32(lane_addr + kTileRhs + gq * 32, b);   // D[t][128 + c] (Im X part)
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const float v = __shfl_xor_sync(0xffffffffu, b[c], 1);
                        const float out = parity ? a[c] + v : a[c] - v;
                        const int rhs = rb * kTileRhs + gq * 32 + c;
                        if (i < n && rhs < r) {
                            float* dst = y + ((int64_t)rhs * ldy + i) * 2 + parity;
                            if (ksplit > 1) atomicAdd(dst, out);
                            else *dst = out;
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&acc_empty[buf]));
            ++t;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tacc, kPTmemCols);
    if (err) atomicOr(status, err);
#endif
}

// Ahat planes from the complex128 matrix: rows (2i, 2i+1) = (Re, Im) of row i, split hi / lo.
__global__ void k_split_matrix64(const double2* __restrict__ A, int64_t n, int64_t lda, __nv_bfloat16* __restrict__ hi,
                                 __nv_bfloat16* __restrict__ lo, int64_t ldk) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    const int64_t i = t / n, j = t % n;
    const double2 a = A[i * lda + j];
    const __nv_bfloat16 hr = __double2bfloat16(a.x), hi_ = __double2bfloat16(a.y);
    hi[(2 * i) * ldk + j] = hr;
    hi[(2 * i + 1) * ldk + j] = hi_;
    lo[(2 * i) * ldk + j] = __double2bfloat16(a.x - (double)__bfloat162float(hr));
    lo[(2 * i + 1) * ldk + j] = __double2bfloat16(a.y - (double)__bfloat162float(hi_));
}
__global__ void k_split_matrix32(const float2* __restrict__ A, int64_t n, int64_t lda, __nv_bfloat16* __restrict__ hi,
                                 __nv_bfloat16* __restrict__ lo, int64_t ldk) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    const int64_t i = t / n, j = t % n;
    const float2 a = A[i * lda + j];
    const __nv_bfloat16 hr = __float2bfloat16_rn(a.x), hi_ = __float2bfloat16_rn(a.y);
    hi[(2 * i) * ldk + j] = hr;
    hi[(2 * i + 1) * ldk + j] = hi_;
    lo[(2 * i) * ldk + j] = __float2bfloat16_rn(a.x - __bfloat162float(hr));
    lo[(2 * i + 1) * ldk + j] = __float2bfloat16_rn(a.y - __bfloat162float(hi_));
}

// Xhat planes of r complex64 vectors (vector c at x + c * ldx): block b of 128 vectors is 256
// rows, (Re x_c) at row c - 128 b and (Im x_c) at row 128 + c - 128 b. Rows of vectors c >= r are
// zero; columns >= n keep the zero fill of the allocation.
__global__ void k_split_vectors(const float2* __restrict__ x, int64_t ldx, int r, int64_t n, int rblocks,
                                __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int64_t ldk) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)rblocks * kTileRhs * n;
    if (t >= total) return;
    const int64_t c = t / n, k = t % n;
    const int64_t b = c / kTileRhs, q = c % kTileRhs;
    const float2 v = c < r ? x[c * ldx + k] : make_float2(0.f, 0.f);
    const int64_t re = (b * 2 * kTileRhs + q) * ldk + k, im = (b * 2 * kTileRhs + kTileRhs + q) * ldk + k;
    const __nv_bfloat16 hr = __float2bfloat16_rn(v.x), hi_ = __float2bfloat16_rn(v.y);
    hi[re] = hr;
    hi[im] = hi_;
    lo[re] = __float2bfloat16_rn(v.x - __bfloat162float(hr));
    lo[im] = __float2bfloat16_rn(v.y - __bfloat162float(hi_));
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        SB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        SB_REQUIRE(p && q == cudaDriverEntryPointSuccess, SB_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// 2-D BF16 tensor map over rows x ldk (row pitch ldk elements), box of box_rows x 32, 64B swizzle.
CUtensorMap make_map(void* base, int64_t rows, int64_t ldk, int box_rows) {
    return make_tmap_2d(base, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, rows, ldk, kTileK, box_rows,
                        CU_TENSOR_MAP_SWIZZLE_64B);
}

}  // namespace

CUtensorMap make_tmap_2d(void* base, CUtensorMapDataType type, int elem_bytes, int64_t rows, int64_t ldk,
                         int box_inner, int box_rows, CUtensorMapSwizzle swizzle) {
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const cuuint64_t dims[2] = {(cuuint64_t)ldk, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ldk * elem_bytes};
    const cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_rows};
    const cuuint32_t elem[2] = {1, 1};
    const CUresult rc = encode_fn()(&m, type, 2, base, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                    swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    SB_REQUIRE(rc == CUDA_SUCCESS, SB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

// Split planes of an operator's matrix and of the right-hand-side blocks (internal).
struct TensorWork {
    uint64_t gen = 0;  // changes whenever a plane (and so a tensor map) is re-allocated
    int64_t n = 0, ldk = 0, rows = 0;
    DevBuf a_hi, a_lo;
    CUtensorMap tm_a_hi, tm_a_lo;
    int rblocks = 0;
    DevBuf x_hi, x_lo, status;
    CUtensorMap tm_x_hi, tm_x_lo;
};

static uint64_t g_tensor_gen = 0;

uint64_t tensor_generation(const Operator& op) {
    const TensorWork* w = static_cast<const TensorWork*>(op.tensor);
    return w ? w->gen : 0;
}

void tensor_release(Operator& op) {
    delete static_cast<TensorWork*>(op.tensor);
    op.tensor = nullptr;
    ozaki_release(op);
}

bool tensor_ready(const Operator& op) { return op.tensor != nullptr; }

void tensor_prepare(Operator& op) {
    SB_REQUIRE(op.A64.p || op.A32.p, SB_ERR_INVALID_ARGUMENT, "operator has no matrix");
    SB_CUDA(cudaSetDevice(op.device));
    tensor_release(op);
    TensorWork* w = new TensorWork();
    op.tensor = w;
    w->gen = ++g_tensor_gen;
    w->n = op.n;
    w->ldk = cdiv(op.n, kTileK) * kTileK;
    w->rows = cdiv(2 * op.n, kTileM) * kTileM;
    const size_t bytes = sizeof(__nv_bfloat16) * w->rows * w->ldk;
    w->a_hi.alloc(bytes);
    w->a_lo.alloc(bytes);
    w->status.alloc(sizeof(int));
    SB_CUDA(cudaMemsetAsync(w->a_hi.p, 0, bytes, op.stream));
    SB_CUDA(cudaMemsetAsync(w->a_lo.p, 0, bytes, op.stream));
    SB_CUDA(cudaMemsetAsync(w->status.p, 0, sizeof(int), op.stream));
    const int64_t tot = op.n * op.n;
    if (op.A64.p)
        k_split_matrix64<<<cdiv(tot, 256), 256, 0, op.stream>>>(op.A64.as<double2>(), op.n, op.n,
                                                               w->a_hi.as<__nv_bfloat16>(), w->a_lo.as<__nv_bfloat16>(),
                                                               w->ldk);
    else
        k_split_matrix32<<<cdiv(tot, 256), 256, 0, op.stream>>>(op.A32.as<float2>(), op.n, op.lda32,
                                                               w->a_hi.as<__nv_bfloat16>(), w->a_lo.as<__nv_bfloat16>(),
                                                               w->ldk);
    count_launch();
    SB_CUDA(cudaGetLastError());
    w->tm_a_hi = make_map(w->a_hi.p, w->rows, w->ldk, kTileM);
    w->tm_a_lo = make_map(w->a_lo.p, w->rows, w->ldk, kTileM);
    SB_CUDA(cudaFuncSetAttribute(k_block_bf16x3, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    SB_CUDA(cudaStreamSynchronize(op.stream));
}

void tensor_reserve(const Operator& op, int r) {
    TensorWork* w = static_cast<TensorWork*>(op.tensor);
    SB_REQUIRE(w, SB_ERR_INVALID_ARGUMENT, "tensor-core block product: call sb_operator_prepare_block_tensor first");
    const int rblocks = static_cast<int>(cdiv(r, kTileRhs));
    if (rblocks <= w->rblocks) return;
    const size_t bytes = sizeof(__nv_bfloat16) * (size_t)rblocks * 2 * kTileRhs * w->ldk;
    w->x_hi.alloc(bytes);
    w->x_lo.alloc(bytes);
    memset_sync(w->x_hi.p, 0, bytes);
    memset_sync(w->x_lo.p, 0, bytes);
    w->rblocks = rblocks;
    w->gen = ++g_tensor_gen;
    w->tm_x_hi = make_map(w->x_hi.p, (int64_t)rblocks * 2 * kTileRhs, w->ldk, 2 * kTileRhs);
    w->tm_x_lo = make_map(w->x_lo.p, (int64_t)rblocks * 2 * kTileRhs, w->ldk, 2 * kTileRhs);
}

// Y (r vectors, vector c at y + c * ldy, complex64) = A X (vector c at x + c * ldx).
void tensor_block_product(const Operator& op, const float2* x, int64_t ldx, int r, float2* y, int64_t ldy,
                          cudaStream_t s, const int* block_gate) {
    TensorWork* w = static_cast<TensorWork*>(op.tensor);
    SB_REQUIRE(w, SB_ERR_INVALID_ARGUMENT, "tensor-core block product: call sb_operator_prepare_block_tensor first");
    SB_REQUIRE(r >= 1, SB_ERR_INVALID_ARGUMENT, "tensor-core block product: r must be positive");
    const int rblocks = static_cast<int>(cdiv(r, kTileRhs));
    if (rblocks > w->rblocks) tensor_reserve(op, r);
    const int64_t tot = (int64_t)rblocks * kTileRhs * w->n;
    {
        ProfScope prof(SB_PROF_OTHER, s);
        k_split_vectors<<<cdiv(tot, 256), 256, 0, s>>>(x, ldx, r, w->n, rblocks, w->x_hi.as<__nv_bfloat16>(),
                                                       w->x_lo.as<__nv_bfloat16>(), w->ldk);
        count_launch();
    }
    SB_CUDA(cudaGetLastError());
    // Two K halves per tile when one pass over the tiles would leave the last wave of SMs mostly
    // idle (fewer than 6 waves of CTAs); every half keeps at least one K block.
    const int64_t ctas = (int64_t)rblocks * (w->rows / kTileM);
    const int nkb = static_cast<int>(w->ldk / kTileK);
    const int ksplit = (ctas < 6 * (int64_t)device_sm_count(op.device) && nkb >= 2) ? 2 : 1;
    if (ksplit > 1)
        SB_CUDA(cudaMemset2DAsync(y, sizeof(float2) * ldy, 0, sizeof(float2) * w->n, r, s));
    ProfScope prof(SB_PROF_TENSOR, s);
    const int mtiles = static_cast<int>(w->rows / kTileM);
    const int64_t units = ctas * ksplit;
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>(units, device_sm_count(op.device)));
    k_block_bf16x3<<<grid, kPThreads, kSmemBytes, s>>>(w->tm_a_hi, w->tm_a_lo, w->tm_x_hi, w->tm_x_lo,
                                                        static_cast<int>(w->ldk), w->n, r, reinterpret_cast<float*>(y),
                                                        ldy, w->status.as<int>(), block_gate, ksplit, rblocks, mtiles);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

int tensor_status(const Operator& op, bool reset) {
    TensorWork* w = static_cast<TensorWork*>(op.tensor);
    if (!w) return 0;
    int v = 0;
    SB_CUDA(cudaMemcpy(&v, w->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (reset && v) memset_sync(w->status.p, 0, sizeof(int));
    return v;
}

}  // namespace sb
