// Batched frequency sweep: many independent TBEM instances (mesh, wavenumber) assembled in one
// persistent launch and solved together by a batched mixed-precision GMRES.
//
// Reference: the frequency sweep re-assembles and solves one frequency after another
// (crates/sonium-bem/src/core/solver/frequency_sweep.rs:541-600, build_tbem_system_stabilized at
// :20); each solve is gmres_core (crates/sonium-solvers/crates/sonium-solvers-iterative/src/
// gmres.rs:631-1047). Here all instances advance in lockstep: every kernel of an Arnoldi step
// covers all instances through a flattened list of row blocks (an instance's blocks are
// contiguous; a block finds its instance by binary search over a prefix array), every instance
// carries its own convergence state, and kernels of an instance whose flag says "done" return at
// once (the per-instance mask). One restart cycle of the whole batch is one CUDA graph. The
// arithmetic per instance is the single-instance mixed solver's (gmres.cu, gmres_mixed_ir): FP32
// inner GMRES on the complex64 matrix, FP64 Hessenberg / Givens, FP64 refinement residual with
// FP64 accumulation, the same stopping rules and statistics.
//
// The same machinery solves many right-hand sides of ONE operator (sb_gmres_multi): the
// instances are the right-hand sides, every vector family is stored right-hand-side-major so a
// step's products for all of them are one block product on the tensor cores (tensor.cu: BF16
// hi/lo split, FP32 accumulation), and the FP64 refinement residual of all of them is one
// integer-slice block residual on the complex128 matrix (ozaki.cu: INT8 slices, exact INT32
// accumulation on the tensor cores, FP64-grade). Each right-hand side keeps its own Krylov basis and
// convergence state (the reference's block_gmres, block_gmres.rs:163, shares one basis instead).


#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>

#include "sb_blas.cuh"
#include "sb_device.cuh"
#include "sb_gemv.cuh"
#include "sb_internal.cuh"
#include "sb_krylov.cuh"
#include "sb_precond.cuh"
#include "sb_profile.cuh"

struct sb_mesh {
    sb::Mesh* m;
};

namespace sb {

// Per-instance device descriptor of the batched solver.
struct BInst {
    const float2* A;  // complex64 matrix, row-major, even leading dimension lda
    int64_t lda, n, ldv;
    int64_t vs;       // distance between consecutive basis vectors
    float2* V;        // Krylov basis: vector i at V + i * vs
    float2* w;
    float2* rb;       // inner right-hand side r / ||r||
    float2* d;        // inner solution
    float2* rq;       // inner residual at restarts
    double2* x;       // FP64 solution
    const double2* b; // FP64 right-hand side
    double2* r;       // FP64 residual b - A x
    KState* st;
    double2 *H, *cs, *sn, *g, *y, *red, *red2, *part;
    double* pnorm;    // per-block / per-chunk squared-norm partials
    double* nrm;      // [0] first Gram-Schmidt |w|^2, [1] second pass, [2] reduced norm^2
    double* scal;     // [0] 1 / ||r||, [1] ||r||, [2] inner beta, [3] inner tolerance, [4] inner ||b||
    int* outer;       // 1 while the instance refines
    int* live;        // 1 while its inner solve runs
    int* brk;         // inner breakdown before the first step
    // Complex-half copy of A for the inner products (SB_INNER_FP16): entries times a power-of-two
    // scale, rows lda16 apart; aux16 = [largest part's bits, scale, 1 / scale].
    const uint32_t* A16;
    int64_t lda16;
    unsigned* aux16;
    // Block-Jacobi right preconditioner of the inner solve (SB_INNER_PRECOND_BLOCK_JACOBI): the
    // transposed block inverses, the Morton permutation, and t = M^-1 of the product's input.
    const float2* bj_inv;
    const int32_t* bj_perm;
    float2* t;
};

namespace {

constexpr int kChunk = 256;  // vector rows per CTA of the vector kernels
constexpr int kBDotVecs = 8;
constexpr int kDotSpan = 32;  // kChunk row slices per CTA of the Gram-Schmidt dots
constexpr int kRowsPerThread = 4;  // rows per thread of the projection and next-vector kernels
constexpr int kWide = kChunk * kRowsPerThread;
constexpr int kScal = 5;

__device__ __forceinline__ int find_inst(const int64_t* __restrict__ pre, int ninst, int64_t unit) {
    // Instances of equal size (every right-hand side of one operator): the proportional guess is
    // the answer, two dependent loads instead of a binary search's log2(ninst).
    const int64_t total = pre[ninst];
    const int guess = static_cast<int>(min((int64_t)ninst - 1, unit * ninst / max(total, (int64_t)1)));
    if (pre[guess] <= unit && unit < pre[guess + 1]) return guess;
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= unit) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Which per-instance flag gates a launch.
enum GateKind { G_NONE = 0, G_OUTER = 1, G_LIVE = 2, G_ACTIVE = 3, G_REORTH = 4, G_RESTART = 5 };
__device__ __forceinline__ bool open_gate(const BInst& I, int gk) {
    switch (gk) {
        case G_OUTER: return *I.outer != 0;
        case G_LIVE: return *I.live != 0;
        case G_ACTIVE: return I.st->active != 0;
        case G_REORTH: return I.st->active != 0 && I.st->reorth != 0;
        case G_RESTART: return *I.live != 0 && I.st->reason == 0;
        default: return true;
    }
}

// The batched FP32-vector complex64 product keeps 4 rows x 2 loads per CTA: at the single
// operator's 1 x 4 the sweep's flattened grid (one CTA per row of every instance) made the
// FP32-inner sweep solve slower (711 against 646 ms for 64 instances).
constexpr int kBGemv64Rows = 4, kBGemv64Unroll = 2;

// Matrix-vector products over the flattened row blocks (kBGemv64Rows rows per CTA).
// mode 0: w = A V_j; mode 1: rq = rb - A d (partial norms); modes 2 / 3: the same with t
// (= M^-1 V_j or M^-1 d under the block-Jacobi preconditioner) in place of V_j / d.
__global__ void __launch_bounds__(kGemvThreads) k_bgemv32(const BInst* __restrict__ inst,
                                                          const int64_t* __restrict__ pre, int ninst, int mode,
                                                          int j, int gk) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t blk = blockIdx.x - pre[b];
    const float2* src = mode == 0 ? I.V + (int64_t)j * I.vs : (mode == 1 ? I.d : I.t);
    if (mode == 0 || mode == 2)
        gemv_c64_block<kBGemv64Rows, kGemvThreads, kBGemv64Unroll, false>(I.A, I.n, I.lda, src, I.w, nullptr,
                                                                           nullptr, blk);
    else
        gemv_c64_block<kBGemv64Rows, kGemvThreads, kBGemv64Unroll, false>(I.A, I.n, I.lda, src, I.rq, I.rb, I.pnorm,
                                                                           blk);
}

// The same products on the complex-half copies (kGemv16PRows rows per CTA).
__global__ void __launch_bounds__(kGemvThreads) k_bgemv16(const BInst* __restrict__ inst,
                                                          const int64_t* __restrict__ pre, int ninst, int mode,
                                                          int j, int gk) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t blk = blockIdx.x - pre[b];
    const float* inv = reinterpret_cast<const float*>(I.aux16 + 2);
    const float2* src = mode == 0 ? I.V + (int64_t)j * I.vs : (mode == 1 ? I.d : I.t);
    if (mode == 0 || mode == 2)
        gemv_c16_block<kGemv16PRows, kGemvThreads, kGemv16PUnroll>(I.A16, I.n, I.lda16, inv, src, I.w, nullptr,
                                                                   nullptr, blk);
    else
        gemv_c16_block<kGemv16PRows, kGemvThreads, kGemv16PUnroll>(I.A16, I.n, I.lda16, inv, src, I.rq, I.rb,
                                                                   I.pnorm, blk);
}

// Block-Jacobi over the flattened blocks of every instance: inverses (one CTA per block) and
// products. apply mode 0: t = M^-1 V_j; 1: t = M^-1 d; 2: d = M^-1 d (in place: a block's inputs
// are gathered before its outputs are written, and blocks are disjoint).
template <int BS>
__global__ void __launch_bounds__(bj_threads(BS)) k_bbj_invert(const BInst* __restrict__ inst,
                                                               const int64_t* __restrict__ pre, int ninst,
                                                               int* __restrict__ status) {
    extern __shared__ float2 Mbj[];
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    const int64_t blk = blockIdx.x - pre[b], base = blk * BS;
    const int rows = static_cast<int>(I.n - base < BS ? I.n - base : BS);
    bj_invert_block<BS, bj_threads(BS)>(I.A, I.lda, rows, I.bj_perm + base,
                                        const_cast<float2*>(I.bj_inv) + blk * BS * BS, status, Mbj);
}
template <int BS>
__global__ void __launch_bounds__(BS * kBjSplit) k_bbj_apply(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                  int ninst, int mode, int j, int gk) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t blk = blockIdx.x - pre[b], base = blk * BS;
    const int rows = static_cast<int>(I.n - base < BS ? I.n - base : BS);
    const float2* src = mode == 0 ? I.V + (int64_t)j * I.vs : I.d;
    float2* dst = mode == 2 ? I.d : I.t;
    bj_apply_block<BS>(I.bj_inv + blk * BS * BS, rows, I.bj_perm + base, src, dst);
}

// Complex-half copies of every instance's complex64 matrix: largest part, scale, conversion,
// over the same kGemv16Rows row blocks.
__global__ void __launch_bounds__(kHalfThreads) k_bhalf_absmax(const BInst* __restrict__ inst,
                                                               const int64_t* __restrict__ pre, int ninst) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    const int64_t r0 = (blockIdx.x - pre[b]) * kGemv16Rows;
    half_absmax_rows(I.A, I.n, I.lda, r0, r0 + kGemv16Rows < I.n ? r0 + kGemv16Rows : I.n, 1, I.aux16);
}
__global__ void k_bhalf_scale(const BInst* __restrict__ inst, int ninst) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < ninst) half_scale_from_max(inst[b].aux16);
}
__global__ void __launch_bounds__(kHalfThreads) k_bhalf_convert(const BInst* __restrict__ inst,
                                                                const int64_t* __restrict__ pre, int ninst) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    const int64_t r0 = (blockIdx.x - pre[b]) * kGemv16Rows;
    half_convert_rows(I.A, I.n, I.lda, I.aux16, const_cast<uint32_t*>(I.A16), I.lda16, r0,
                      r0 + kGemv16Rows < I.n ? r0 + kGemv16Rows : I.n, 1);
}

// r = b - A x with FP64 vectors and FP64 accumulation on the complex64 matrix, partial norms
// (kGemvX64Rows rows per CTA).
__global__ void __launch_bounds__(kGemvThreads) k_bres64(const BInst* __restrict__ inst,
                                                         const int64_t* __restrict__ pre, int ninst, int gk) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    gemv_c64_block<kGemvX64Rows, kGemvThreads, kGemvX64Unroll, true>(I.A, I.n, I.lda, I.x, I.r, I.b, I.pnorm,
                                                                     blockIdx.x - pre[b]);
}

// Per-chunk squared norms: sel 0 = rb, 1 = b, 2 = b - r (= A x), 3 = r.
__global__ void __launch_bounds__(kChunk) k_bvnorm(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                   int ninst, int sel, int gk) {
    __shared__ double red[kChunk / 32];
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t chunk = blockIdx.x - pre[b];
    const int64_t r = chunk * kChunk + threadIdx.x;
    double v[1] = {0.0};
    if (r < I.n) {
        if (sel == 0) {
            const float2 a = I.rb[r];
            v[0] = (double)a.x * a.x + (double)a.y * a.y;
        } else if (sel == 1) {
            const double2 a = I.b[r];
            v[0] = a.x * a.x + a.y * a.y;
        } else if (sel == 2) {
            const double2 a = I.b[r], q = I.r[r];
            const double ar = a.x - q.x, ai = a.y - q.y;
            v[0] = ar * ar + ai * ai;
        } else {
            const double2 q = I.r[r];
            v[0] = q.x * q.x + q.y * q.y;
        }
    }
    block_sum<1, kChunk>(v, red);
    if (threadIdx.x == 0) I.pnorm[chunk] = v[0];
}

// *out = 1 when any instance still runs its Arnoldi cycle (one CTA).
__global__ void __launch_bounds__(256) k_ball_active(const BInst* __restrict__ inst, int ninst, int* __restrict__ out) {
    int on = 0;
    for (int b = threadIdx.x; b < ninst; b += 256) on |= inst[b].st->active ? 1 : 0;
    const int any = __syncthreads_or(on);
    if (threadIdx.x == 0) *out = any;
}

// gate[g] = 1 when any instance of group g (kTensorRhsTile instances) still runs its Arnoldi
// cycle: groups that are all done skip the step's block product.
__global__ void __launch_bounds__(kTensorRhsTile) k_bany_active(const BInst* __restrict__ inst, int ninst,
                                                                int* __restrict__ gate) {
    const int b = blockIdx.x * kTensorRhsTile + threadIdx.x;
    const int on = (b < ninst && inst[b].st->active) ? 1 : 0;
    const int any = __syncthreads_or(on);
    if (threadIdx.x == 0) gate[blockIdx.x] = any;
}

// rq = rb - w (w = A d from a block product), per-chunk squared norms of rq.
__global__ void __launch_bounds__(kChunk) k_bresid_w(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                     int ninst, int gk) {
    __shared__ double red[kChunk / 32];
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t chunk = blockIdx.x - pre[b];
    const int64_t r = chunk * kChunk + threadIdx.x;
    double v[1] = {0.0};
    if (r < I.n) {
        const float2 a = I.rb[r], q = I.w[r];
        const float2 o = make_float2(a.x - q.x, a.y - q.y);
        I.rq[r] = o;
        v[0] = (double)o.x * o.x + (double)o.y * o.y;
    }
    block_sum<1, kChunk>(v, red);
    if (threadIdx.x == 0) I.pnorm[chunk] = v[0];
}

// nrm[slot] = sum of the instance's partials (their count is the instance's span of `pre`).
// One CTA per instance sums its partial norms (up to one per row of its residual product).
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_bsum_partials(const BInst* __restrict__ inst,
                                                               const int64_t* __restrict__ pre, int slot, int gk) {
    __shared__ double red[kSumThreads / 32];
    const BInst& I = inst[blockIdx.x];
    if (!open_gate(I, gk)) return;
    const int64_t cnt = pre[blockIdx.x + 1] - pre[blockIdx.x];
    double s = 0.0;
    for (int64_t c = threadIdx.x; c < cnt; c += kSumThreads) s += I.pnorm[c];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < kSumThreads / 32 ? red[threadIdx.x] : 0.0;
        s = warp_sum(s);
        if (threadIdx.x == 0) I.nrm[slot] = s;
    }
}

// Gram-Schmidt dots over the flattened chunks of kDotSpan * kChunk rows:
// part[chunk * (k + 1) + i] = V_i^H w (i < k), |w|^2 at i = k. A thread takes two adjacent rows per
// 16-byte load (vectors have an even leading dimension; a row at n or beyond counts as zero) and
// sums its kDotSpan / 2 row pairs in FP32 (the vectors are complex64); the CTA sum is FP64.
__global__ void __launch_bounds__(kChunk, 4) k_bdots(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                  int ninst, int k, int gk) {
    __shared__ double red[(kChunk / 32) * 2 * kBDotVecs];
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t chunk = blockIdx.x - pre[b];
    const int i0 = blockIdx.y * kBDotVecs;
    const int64_t n = I.n, vs = I.vs;
    const float4* __restrict__ W = reinterpret_cast<const float4*>(I.w);
    const float2* __restrict__ V = I.V;
    float acc[2 * kBDotVecs];
#pragma unroll
    for (int t = 0; t < 2 * kBDotVecs; ++t) acc[t] = 0.f;
    for (int sl = 0; sl < kDotSpan / 2; ++sl) {
        const int64_t r = (chunk * kDotSpan + 2 * sl) * kChunk + 2 * threadIdx.x;  // rows r, r + 1
        if (r >= n) break;
        const bool two = r + 1 < n;
        float4 wv = W[r >> 1];
        if (!two) wv.z = wv.w = 0.f;
#pragma unroll
        for (int t = 0; t < kBDotVecs; ++t) {
            const int i = i0 + t;
            if (i < k) {
                float4 v = *reinterpret_cast<const float4*>(V + i * vs + r);
                if (!two) v.z = v.w = 0.f;
                acc[2 * t] = fmaf(v.x, wv.x, fmaf(v.y, wv.y, fmaf(v.z, wv.z, fmaf(v.w, wv.w, acc[2 * t]))));
                acc[2 * t + 1] =
                    fmaf(v.x, wv.y, fmaf(-v.y, wv.x, fmaf(v.z, wv.w, fmaf(-v.w, wv.z, acc[2 * t + 1]))));
            } else if (i == k) {
                acc[2 * t] = fmaf(wv.x, wv.x, fmaf(wv.y, wv.y, fmaf(wv.z, wv.z, fmaf(wv.w, wv.w, acc[2 * t]))));
            }
        }
    }
    double accd[2 * kBDotVecs];
#pragma unroll
    for (int t = 0; t < 2 * kBDotVecs; ++t) accd[t] = acc[t];
    block_sum<2 * kBDotVecs, kChunk>(accd, red);
    if (threadIdx.x == 0)
        for (int t = 0; t < kBDotVecs; ++t) {
            const int i = i0 + t;
            if (i <= k) I.part[chunk * (k + 1) + i] = make_double2(accd[2 * t], accd[2 * t + 1]);
        }
}

// red (second = 0) or red2 (second = 1) [i] = sum over the instance's chunks, i <= k.
__global__ void k_breduce(const BInst* __restrict__ inst, const int64_t* __restrict__ pre, int k, int second, int gk) {
    const BInst& I = inst[blockIdx.y];
    if (!open_gate(I, gk)) return;
    const int i = blockIdx.x;
    const int64_t chunks = pre[blockIdx.y + 1] - pre[blockIdx.y];
    double sr = 0.0, si = 0.0;
    for (int64_t c = threadIdx.x; c < chunks; c += 32) {
        const double2 v = I.part[c * (k + 1) + i];
        sr += v.x;
        si += v.y;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if (threadIdx.x == 0) (second ? I.red2 : I.red)[i] = make_double2(sr, si);
}

// w -= sum_{i<k} coeff[i] V_i (coeff = red or red2), partial |w|^2 per chunk of kWide rows
// (kRowsPerThread rows per thread, kChunk apart: every basis load of a warp stays coalesced).
__global__ void __launch_bounds__(kChunk) k_bproject(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                     int ninst, int k, int second, int gk) {
    __shared__ double2 sc[kMaxKrylov + 1];
    __shared__ double red[kChunk / 32];
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const double2* coeff = second ? I.red2 : I.red;
    for (int t = threadIdx.x; t < k; t += kChunk) sc[t] = coeff[t];
    __syncthreads();
    const int64_t chunk = blockIdx.x - pre[b];
    const int64_t n = I.n;
    const float2* __restrict__ V = I.V;
    const int64_t vs = I.vs;
    int64_t rr[kRowsPerThread];
    double ar[kRowsPerThread], ai[kRowsPerThread];
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
        rr[q] = chunk * kWide + q * kChunk + threadIdx.x;
        const float2 w0 = rr[q] < n ? I.w[rr[q]] : make_float2(0.f, 0.f);
        ar[q] = w0.x;
        ai[q] = w0.y;
    }
    for (int i = 0; i < k; ++i) {
        const double2 c = sc[i];
        float2 v[kRowsPerThread];
#pragma unroll
        for (int q = 0; q < kRowsPerThread; ++q) v[q] = rr[q] < n ? V[i * vs + rr[q]] : make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < kRowsPerThread; ++q) {
            ar[q] -= c.x * v[q].x - c.y * v[q].y;
            ai[q] -= c.x * v[q].y + c.y * v[q].x;
        }
    }
    double nr2[1] = {0.0};
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q)
        if (rr[q] < n) {
            const float2 o = make_float2(static_cast<float>(ar[q]), static_cast<float>(ai[q]));
            I.w[rr[q]] = o;
            nr2[0] += (double)o.x * o.x + (double)o.y * o.y;
        }
    block_sum<1, kChunk>(nr2, red);
    if (threadIdx.x == 0) I.pnorm[chunk] = nr2[0];
}

__global__ void k_bafter_first(const BInst* __restrict__ inst, int ninst, int j) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ninst) return;
    const BInst& I = inst[b];
    after_first_dev(I.st, I.red, I.nrm + 0, I.H, j);
}

__global__ void k_bgivens(const BInst* __restrict__ inst, int ninst, int j) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ninst) return;
    const BInst& I = inst[b];
    givens_step_dev(I.st, I.red2, I.nrm + 1, I.H, I.cs, I.sn, I.g, j);
}

// V_{j+1} = w / ||w|| for the instances still running (chunks of kWide rows).
__global__ void __launch_bounds__(kChunk) k_bnext(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                  int ninst, int j) {
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!I.st->active) return;
    const double s = I.st->inv_wn;
    const int64_t n = I.n;
    float2* __restrict__ dst = I.V + (int64_t)(j + 1) * I.vs;
    const int64_t r0 = (blockIdx.x - pre[b]) * kWide + threadIdx.x;
    float2 v[kRowsPerThread];
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
        const int64_t r = r0 + q * kChunk;
        v[q] = r < n ? I.w[r] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
        const int64_t r = r0 + q * kChunk;
        if (r < n) dst[r] = make_float2(static_cast<float>(v[q].x * s), static_cast<float>(v[q].y * s));
    }
}

// Vector updates over the flattened chunks.
enum VecOp {
    OP_B_TO_R = 0,    // r = b, x = 0
    OP_R_TO_RB = 1,   // rb = r / ||r|| (complex64), d = 0
    OP_RB_TO_V0 = 2,  // V_0 = rb / beta (first inner cycle)
    OP_RQ_TO_V0 = 3,  // V_0 = rq / beta (restarts)
    OP_D_UPDATE = 4,  // d += V y (k = jdone)
    OP_X_UPDATE = 5,  // x += ||r|| d
};
__global__ void __launch_bounds__(kChunk) k_bvec(const BInst* __restrict__ inst, const int64_t* __restrict__ pre,
                                                 int ninst, int op, int gk) {
    __shared__ double2 sy[kMaxKrylov + 1];
    const int b = find_inst(pre, ninst, blockIdx.x);
    const BInst& I = inst[b];
    if (!open_gate(I, gk)) return;
    const int64_t r = (blockIdx.x - pre[b]) * kChunk + threadIdx.x;
    if (op == OP_D_UPDATE) {
        const int k = I.st->jdone;
        for (int t = threadIdx.x; t < k; t += kChunk) sy[t] = I.y[t];
        __syncthreads();
        if (r >= I.n) return;
        double sr = 0.0, si = 0.0;
        for (int i = 0; i < k; ++i) {
            const float2 v = I.V[i * I.vs + r];
            sr += sy[i].x * v.x - sy[i].y * v.y;
            si += sy[i].x * v.y + sy[i].y * v.x;
        }
        const float2 d = I.d[r];
        I.d[r] = make_float2(static_cast<float>(d.x + sr), static_cast<float>(d.y + si));
        return;
    }
    if (r >= I.n) return;
    switch (op) {
        case OP_B_TO_R:
            I.r[r] = I.b[r];
            I.x[r] = make_double2(0.0, 0.0);
            break;
        case OP_R_TO_RB: {
            const double s = I.scal[0];
            I.rb[r] = make_float2(static_cast<float>(I.r[r].x * s), static_cast<float>(I.r[r].y * s));
            I.d[r] = make_float2(0.f, 0.f);
            break;
        }
        case OP_RB_TO_V0:
        case OP_RQ_TO_V0: {
            const float2 v = op == OP_RB_TO_V0 ? I.rb[r] : I.rq[r];
            const double s = 1.0 / I.scal[2];
            I.V[r] = make_float2(static_cast<float>(v.x * s), static_cast<float>(v.y * s));
            break;
        }
        case OP_X_UPDATE: {
            const double s = I.scal[1];
            const float2 d = I.d[r];
            I.x[r] = make_double2(I.x[r].x + s * d.x, I.x[r].y + s * d.y);
            break;
        }
        default:
            break;
    }
}

// Cycle start: live instances get H = 0, g = (beta, 0, ...) and an active state; the others an
// inactive state, so every gated kernel of the cycle skips them.
__global__ void k_bcycle_init(const BInst* __restrict__ inst, int m) {
    const BInst& I = inst[blockIdx.x];
    cycle_init_dev(I.st, I.H, I.g, m, 1, I.scal[2], I.scal[4], I.scal[3], threadIdx.x, blockDim.x, *I.live != 0);
}

__global__ void k_bupper(const BInst* __restrict__ inst, int ninst) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ninst) return;
    const BInst& I = inst[b];
    if (!*I.live) return;
    upper_solve_dev(I.st, I.H, I.g, I.y);
}

// Inner-solve control per instance (thread per instance), the decisions gmres_core takes between
// cycles (gmres.rs:790-1047 with the refinement caller's trusted estimate):
// mode 0, inner start: live = outer; beta = ||rb|| (nrm[2]) becomes the inner ||b||; a zero or
//   non-finite beta is a breakdown before the first step.
// mode 1, after a cycle: an estimated convergence or an inner breakdown (reason != 0), or the last
//   allowed cycle, ends the inner solve; otherwise the restart residual norm (nrm[2]) is the next
//   beta, and the solve ends when it meets the inner tolerance or is not finite.
__global__ void k_bcontrol(const BInst* __restrict__ inst, int ninst, int mode, int last) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ninst) return;
    const BInst& I = inst[b];
    if (mode == 0) {
        *I.brk = 0;
        *I.live = *I.outer;
        if (!*I.live) return;
        const double beta = sqrt(I.nrm[2]);
        I.scal[4] = beta < 1e-15 ? 1.0 : beta;
        I.scal[2] = beta;
        if (!isfinite(beta) || beta == 0.0) {
            *I.live = 0;
            *I.brk = 1;
        }
        return;
    }
    if (!*I.live) return;
    if (I.st->reason != 0 || last) {
        *I.live = 0;
        return;
    }
    const double beta = sqrt(I.nrm[2]);
    I.scal[2] = beta;
    if (beta / I.scal[4] < I.scal[3] || !isfinite(beta) || beta == 0.0) *I.live = 0;
}

int64_t cdiv64(int64_t a, int64_t b) { return (a + b - 1) / b; }
size_t round256(size_t v) { return (v + 255) / 256 * 256; }

struct Pinned {
    void* p = nullptr;
    void alloc(size_t n) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        SB_CUDA(cudaMallocHost(&p, n));
    }
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

// ---------------------------------------------------------------------------------------------
// Batch object
// ---------------------------------------------------------------------------------------------
struct Batch {
    int device = 0;
    int ninst = 0;
    int64_t m = 0;  // Krylov dimension the workspace was sized for
    std::vector<int64_t> nvec;  // unknowns per instance
    // Many right-hand sides of one operator: products through `shared` (tensor-core block product
    // for the inner solves, the integer-slice block residual for the FP64 one); vectors stored
    // right-hand-side-major.
    Operator* shared = nullptr;
    float2 *w_all = nullptr, *d_all = nullptr, *v_all = nullptr;
    double2 *x_all = nullptr, *r_all = nullptr, *b_all = nullptr;
    int64_t ld_all = 0;
    std::vector<Mesh*> meshes;
    std::vector<sb_physics> phys;
    std::vector<double2> beta;
    std::vector<BatchAsmInst> asm_h;
    std::vector<double2*> rhs;  // per-instance right-hand side (pool_rhs)
    std::vector<BInst> h;
    std::vector<int64_t> pre64, prex, pre16, pre16p, pre256, predot, prewide;
    DevBuf asm_d, inst_d, pre64_d, prex_d, pre16_d, pre16p_d, pre256_d, predot_d, prewide_d, pre_asm;
    // Inner products on the complex64 matrices (SB_INNER_FP32) or on complex-half copies built
    // after each assembly (SB_INNER_FP16; independent instances only).
    int inner = SB_INNER_FP32;
    bool half_valid = false;
    bool amax_valid = false;  // pool_half_aux[4 b] holds instance b's largest part (streams assembly)
    DevBuf pool_half, pool_half_aux;
    int graph_inner = -1;
    // Block-Jacobi right preconditioner of the inner solves (independent instances only).
    int inner_precond = SB_INNER_PRECOND_NONE;
    int bj_size = 64;
    bool bj_valid = false;
    std::vector<int64_t> prebj;
    DevBuf pool_bj, pool_bj_perm, prebj_d, bj_status;
    int graph_pre = -1;
    DevBuf pool_mat, pool_rhs, pool_f32, pool_f64, pool_small, pool_state;
    DevBuf gate;  // per group of kTensorRhsTile instances: any still in the Arnoldi cycle
    cudaStream_t stream = nullptr;
    // The restart cycle as graph chunks of kBatchChunk steps, launched while any instance is in
    // its cycle (anyact: device flag, chk: its two pinned host copies, ev: their events).
    std::vector<cudaGraph_t> graphs;
    std::vector<cudaGraphExec_t> execs;
    std::vector<int64_t> chunk_kernels;
    DevBuf anyact;
    Pinned chk;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    unsigned graph_prof = 0;
    uint64_t graph_gen = 0;  // tensor-plane generation the captured cycle refers to
    std::vector<ProfPair> prof_pairs;
    Pinned pin;  // host mirror of the per-instance states, norms, scalars and flags
    bool assembled = false, solved = false;
    double last_assembly_ms = 0.0, last_solve_ms = 0.0;
    // Assembly form: SB_BATCH_ASM_AUTO (the autotuner's choice for this batch shape), _PERSISTENT
    // or _STREAMS; the autotuner's two measurements when it ran for this batch.
    int asm_mode = SB_BATCH_ASM_AUTO, asm_chosen = 0;
    // Persistent form: far CTA slots per SM of its split form (0 = one launch); set by the autotuner.
    int asm_split = 3;
    double tune_persistent_ms = 0.0, tune_streams_ms = 0.0;
    double tune_split_ms[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    SideStream side;
    void reset_graph() {
        for (cudaGraphExec_t e : execs)
            if (e) cudaGraphExecDestroy(e);
        for (cudaGraph_t g : graphs)
            if (g) cudaGraphDestroy(g);
        execs.clear();
        graphs.clear();
        chunk_kernels.clear();
        profile_release(prof_pairs);
    }
    ~Batch() {
        reset_graph();
        for (cudaEvent_t& e : ev)
            if (e) cudaEventDestroy(e);
        side.release();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// The device block pool_state and its pinned host mirror share one layout, so one copy moves a
// group of fields for all instances.
struct StateView {
    KState* st;
    double* nrm;   // 3 per instance
    double* scal;  // kScal per instance
    int* outer;
    int* live;
    int* brk;
};
StateView state_view(void* base, int ni) {
    char* p = static_cast<char*>(base);
    StateView v;
    v.st = reinterpret_cast<KState*>(p);
    p += round256(sizeof(KState) * ni);
    v.nrm = reinterpret_cast<double*>(p);
    p += round256(sizeof(double) * 3 * ni);
    v.scal = reinterpret_cast<double*>(p);
    p += round256(sizeof(double) * kScal * ni);
    v.outer = reinterpret_cast<int*>(p);
    p += round256(sizeof(int) * ni);
    v.live = reinterpret_cast<int*>(p);
    p += round256(sizeof(int) * ni);
    v.brk = reinterpret_cast<int*>(p);
    return v;
}
size_t state_bytes(int ni) {
    return round256(sizeof(KState) * ni) + round256(sizeof(double) * 3 * ni) +
           round256(sizeof(double) * kScal * ni) + 3 * round256(sizeof(int) * ni);
}

}  // namespace

// Sizes the solver workspace of every instance for restart m and builds the descriptors.
// Where instance b's complex-half copy and scale live in the batch's half pools (null before the
// pools exist).
static void half_pointers(const Batch& B, int b, BInst& I) {
    I.lda16 = (B.nvec[b] + 3) / 4 * 4;
    if (!B.pool_half.p) {
        I.A16 = nullptr;
        I.aux16 = nullptr;
        return;
    }
    size_t off = 0;
    for (int c = 0; c < b; ++c) off += round256(sizeof(uint32_t) * B.nvec[c] * ((B.nvec[c] + 3) / 4 * 4));
    I.A16 = reinterpret_cast<const uint32_t*>(B.pool_half.as<char>() + off);
    I.aux16 = B.pool_half_aux.as<unsigned>() + 4 * b;
}

// Where instance b's block inverses and permutation live in the batch's pools (null before).
static void bj_pointers(const Batch& B, int b, BInst& I) {
    if (!B.pool_bj.p || !B.pool_bj_perm.p) {
        I.bj_inv = nullptr;
        I.bj_perm = nullptr;
        return;
    }
    int64_t off_perm = 0;
    for (int c = 0; c < b; ++c) off_perm += B.nvec[c];
    I.bj_perm = B.pool_bj_perm.as<int32_t>() + off_perm;
    I.bj_inv = B.pool_bj.as<float2>() + B.prebj[b] * B.bj_size * B.bj_size;
}

template <int BS>
static void bj_invert_launch(Batch& B) {
    const size_t smem = sizeof(float2) * BS * BS;
    SB_CUDA(cudaFuncSetAttribute(k_bbj_invert<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    k_bbj_invert<BS><<<static_cast<unsigned>(B.prebj.back()), bj_threads(BS), smem, B.stream>>>(
        B.inst_d.as<BInst>(), B.prebj_d.as<int64_t>(), B.ninst, B.bj_status.as<int>());
    count_launch();
    SB_CUDA(cudaGetLastError());
}

// Builds every instance's block-Jacobi inverses (after each assembly): Morton permutations once
// per batch, the block layout per block size.
static void batch_bj_prepare(Batch& B) {
    if (B.bj_valid) return;
    const int ni = B.ninst, bs = B.bj_size;
    bool layout = false;
    if (!B.pool_bj_perm.p) {
        int64_t total = 0;
        for (int b = 0; b < ni; ++b) total += B.nvec[b];
        std::vector<int32_t> perm;
        perm.reserve(total);
        for (int b = 0; b < ni; ++b) {
            const std::vector<int32_t> p = element_morton_order(*B.meshes[b]);
            perm.insert(perm.end(), p.begin(), p.end());
        }
        B.pool_bj_perm.alloc(sizeof(int32_t) * total);
        h2d_sync(B.pool_bj_perm.p, perm.data(), sizeof(int32_t) * total);
        layout = true;
    }
    std::vector<int64_t> prebj(ni + 1, 0);
    for (int b = 0; b < ni; ++b) prebj[b + 1] = prebj[b] + cdiv64(B.nvec[b], bs);
    if (layout || prebj != B.prebj || !B.pool_bj.p) {
        B.prebj = prebj;
        B.pool_bj.release();
        B.pool_bj.alloc(sizeof(float2) * prebj.back() * bs * bs);
        B.prebj_d.alloc(sizeof(int64_t) * (ni + 1));
        h2d_sync(B.prebj_d.p, prebj.data(), sizeof(int64_t) * (ni + 1));
        for (int b = 0; b < ni; ++b) bj_pointers(B, b, B.h[b]);
        h2d_sync(B.inst_d.p, B.h.data(), sizeof(BInst) * ni);
    }
    if (!B.bj_status.p) B.bj_status.alloc(sizeof(int));
    ProfScope prof(SB_PROF_OTHER, B.stream);
    SB_CUDA(cudaMemsetAsync(B.bj_status.p, 0, sizeof(int), B.stream));
    switch (bs) {
        case 32: bj_invert_launch<32>(B); break;
        case 96: bj_invert_launch<96>(B); break;
        case 128: bj_invert_launch<128>(B); break;
        default: bj_invert_launch<64>(B); break;
    }
    B.bj_valid = true;
}

// t = M^-1 V_j (mode 0), t = M^-1 d (1) or d = M^-1 d (2) for every instance whose gate is open.
static void batch_bj_apply(Batch& B, int mode, int j, int gk) {
    const unsigned g = static_cast<unsigned>(B.prebj.back());
    const BInst* I = B.inst_d.as<BInst>();
    const int64_t* p = B.prebj_d.as<int64_t>();
    ProfScope prof(SB_PROF_ARNOLDI, B.stream);
    switch (B.bj_size) {
        case 32: k_bbj_apply<32><<<g, 32 * kBjSplit, 0, B.stream>>>(I, p, B.ninst, mode, j, gk); break;
        case 96: k_bbj_apply<96><<<g, 96 * kBjSplit, 0, B.stream>>>(I, p, B.ninst, mode, j, gk); break;
        case 128: k_bbj_apply<128><<<g, 128 * kBjSplit, 0, B.stream>>>(I, p, B.ninst, mode, j, gk); break;
        default: k_bbj_apply<64><<<g, 64 * kBjSplit, 0, B.stream>>>(I, p, B.ninst, mode, j, gk); break;
    }
    count_launch();
    SB_CUDA(cudaGetLastError());
}

// Builds the complex-half copies of every instance's complex64 matrix (after each assembly).
static void batch_half_prepare(Batch& B) {
    if (B.half_valid) return;
    const int ni = B.ninst;
    if (!B.pool_half.p) {
        size_t bytes = 0;
        for (int b = 0; b < ni; ++b) bytes += round256(sizeof(uint32_t) * B.nvec[b] * ((B.nvec[b] + 3) / 4 * 4));
        B.pool_half.alloc(bytes);
        if (!B.pool_half_aux.p) B.pool_half_aux.alloc(sizeof(unsigned) * 4 * ni);
        for (int b = 0; b < ni; ++b) half_pointers(B, b, B.h[b]);
        h2d_sync(B.inst_d.p, B.h.data(), sizeof(BInst) * ni);
    }
    const cudaStream_t s = B.stream;
    const BInst* I = B.inst_d.as<BInst>();
    const unsigned g16 = static_cast<unsigned>(B.pre16.back());
    ProfScope prof(SB_PROF_OTHER, s);
    if (!B.amax_valid) {
        SB_CUDA(cudaMemsetAsync(B.pool_half_aux.p, 0, sizeof(unsigned) * 4 * ni, s));
        k_bhalf_absmax<<<g16, kHalfThreads, 0, s>>>(I, B.pre16_d.as<int64_t>(), ni);
        count_launch();
    }
    k_bhalf_scale<<<static_cast<unsigned>(cdiv64(ni, 64)), 64, 0, s>>>(I, ni);
    k_bhalf_convert<<<g16, kHalfThreads, 0, s>>>(I, B.pre16_d.as<int64_t>(), ni);
    for (int t = 0; t < 2; ++t) count_launch();
    SB_CUDA(cudaGetLastError());
    B.half_valid = true;
}

static void batch_workspace(Batch& B, int64_t m) {
    if (B.m == m) return;
    B.reset_graph();
    B.m = 0;
    B.solved = false;
    const int ni = B.ninst;
    const bool shared = B.shared != nullptr;
    size_t f32 = 0, f64 = 0, small = 0;
    for (int b = 0; b < ni; ++b) {
        const int64_t n = B.nvec[b], ldv = (n + 1) / 2 * 2;
        const int64_t chunks = cdiv64(n, kChunk);
        f32 += round256(sizeof(float2) * (m + 1) * ldv) + 5 * round256(sizeof(float2) * ldv);
        f64 += 2 * round256(sizeof(double2) * ldv);
        small += round256(sizeof(double2) * (m + 1) * m) + 2 * round256(sizeof(double2) * m) +
                 2 * round256(sizeof(double2) * (m + 1)) + 2 * round256(sizeof(double2) * (m + 2)) +
                 round256(sizeof(double2) * chunks * (m + 2)) +
                 round256(sizeof(double) * std::max({cdiv64(n, kBGemv64Rows), cdiv64(n, kGemvX64Rows), cdiv64(n, kGemv16PRows), chunks}));
    }
    B.pool_f32.alloc(f32);
    B.pool_f64.alloc(f64);
    B.pool_small.alloc(small);
    B.pool_state.alloc(state_bytes(ni));
    B.pin.alloc(state_bytes(ni));
    memset_sync(B.pool_state.p, 0, state_bytes(ni));
    std::memset(B.pin.p, 0, state_bytes(ni));
    const StateView dv = state_view(B.pool_state.p, ni);
    char* pf32 = B.pool_f32.as<char>();
    char* pf64 = B.pool_f64.as<char>();
    char* ps = B.pool_small.as<char>();
    auto take = [](char*& pool, size_t bytes) {
        char* p = pool;
        pool += round256(bytes);
        return p;
    };
    B.h.assign(ni, BInst{});
    if (shared) {
        // Right-hand-side-major families, each one block: vector c of a family at base + c * ld_all,
        // basis vector i of right-hand side c at v_all + (i * ninst + c) * ld_all. Zero-filled so the
        // block products never read stale values.
        memset_sync(B.pool_f32.p, 0, f32);
        memset_sync(B.pool_f64.p, 0, f64);
        const int64_t ld = B.ld_all;
        B.v_all = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * (m + 1) * ni * ld));
        B.w_all = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ni * ld));
        float2* rb_all = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ni * ld));
        B.d_all = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ni * ld));
        float2* rq_all = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ni * ld));
        B.x_all = reinterpret_cast<double2*>(take(pf64, sizeof(double2) * ni * ld));
        B.r_all = reinterpret_cast<double2*>(take(pf64, sizeof(double2) * ni * ld));
        for (int b = 0; b < ni; ++b) {
            BInst& I = B.h[b];
            I.V = B.v_all + b * ld;
            I.vs = ni * ld;
            I.w = B.w_all + b * ld;
            I.rb = rb_all + b * ld;
            I.d = B.d_all + b * ld;
            I.rq = rq_all + b * ld;
            I.x = B.x_all + b * ld;
            I.r = B.r_all + b * ld;
        }
    }
    B.pre64.assign(ni + 1, 0);
    B.prex.assign(ni + 1, 0);
    B.pre16.assign(ni + 1, 0);
    B.pre16p.assign(ni + 1, 0);
    B.pre256.assign(ni + 1, 0);
    B.predot.assign(ni + 1, 0);
    B.prewide.assign(ni + 1, 0);
    for (int b = 0; b < ni; ++b) {
        const int64_t n = B.nvec[b], ldv = (n + 1) / 2 * 2;
        const int64_t chunks = cdiv64(n, kChunk);
        BInst& I = B.h[b];
        I.n = n;
        I.ldv = ldv;
        if (!shared) {
            I.A = B.asm_h[b].A32;
            I.lda = B.asm_h[b].lda32;
            half_pointers(B, b, I);
            I.V = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * (m + 1) * ldv));
            I.vs = ldv;
            I.w = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ldv));
            I.rb = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ldv));
            I.d = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ldv));
            I.rq = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ldv));
            I.t = reinterpret_cast<float2*>(take(pf32, sizeof(float2) * ldv));
            bj_pointers(B, b, I);
            I.x = reinterpret_cast<double2*>(take(pf64, sizeof(double2) * ldv));
            I.r = reinterpret_cast<double2*>(take(pf64, sizeof(double2) * ldv));
        }
        I.b = B.rhs[b];
        I.H = reinterpret_cast<double2*>(take(ps, sizeof(double2) * (m + 1) * m));
        I.cs = reinterpret_cast<double2*>(take(ps, sizeof(double2) * m));
        I.sn = reinterpret_cast<double2*>(take(ps, sizeof(double2) * m));
        I.g = reinterpret_cast<double2*>(take(ps, sizeof(double2) * (m + 1)));
        I.y = reinterpret_cast<double2*>(take(ps, sizeof(double2) * (m + 1)));
        I.red = reinterpret_cast<double2*>(take(ps, sizeof(double2) * (m + 2)));
        I.red2 = reinterpret_cast<double2*>(take(ps, sizeof(double2) * (m + 2)));
        I.part = reinterpret_cast<double2*>(take(ps, sizeof(double2) * chunks * (m + 2)));
        I.pnorm = reinterpret_cast<double*>(take(ps, sizeof(double) * std::max({cdiv64(n, kBGemv64Rows), cdiv64(n, kGemvX64Rows), cdiv64(n, kGemv16PRows), chunks})));
        I.st = dv.st + b;
        I.nrm = dv.nrm + 3 * b;
        I.scal = dv.scal + kScal * b;
        I.outer = dv.outer + b;
        I.live = dv.live + b;
        I.brk = dv.brk + b;
        B.pre64[b + 1] = B.pre64[b] + cdiv64(n, kBGemv64Rows);
        B.prex[b + 1] = B.prex[b] + cdiv64(n, kGemvX64Rows);
        B.pre16[b + 1] = B.pre16[b] + cdiv64(n, kGemv16Rows);
        B.pre16p[b + 1] = B.pre16p[b] + cdiv64(n, kGemv16PRows);
        B.pre256[b + 1] = B.pre256[b] + chunks;
        B.predot[b + 1] = B.predot[b] + cdiv64(n, (int64_t)kChunk * kDotSpan);
        B.prewide[b + 1] = B.prewide[b] + cdiv64(n, (int64_t)kWide);
    }
    B.inst_d.alloc(sizeof(BInst) * ni);
    B.pre64_d.alloc(sizeof(int64_t) * (ni + 1));
    B.prex_d.alloc(sizeof(int64_t) * (ni + 1));
    B.pre16_d.alloc(sizeof(int64_t) * (ni + 1));
    B.pre16p_d.alloc(sizeof(int64_t) * (ni + 1));
    B.pre256_d.alloc(sizeof(int64_t) * (ni + 1));
    B.predot_d.alloc(sizeof(int64_t) * (ni + 1));
    h2d_sync(B.predot_d.p, B.predot.data(), sizeof(int64_t) * (ni + 1));
    B.prewide_d.alloc(sizeof(int64_t) * (ni + 1));
    h2d_sync(B.prewide_d.p, B.prewide.data(), sizeof(int64_t) * (ni + 1));
    h2d_sync(B.inst_d.p, B.h.data(), sizeof(BInst) * ni);
    h2d_sync(B.pre64_d.p, B.pre64.data(), sizeof(int64_t) * (ni + 1));
    h2d_sync(B.prex_d.p, B.prex.data(), sizeof(int64_t) * (ni + 1));
    h2d_sync(B.pre16_d.p, B.pre16.data(), sizeof(int64_t) * (ni + 1));
    h2d_sync(B.pre16p_d.p, B.pre16p.data(), sizeof(int64_t) * (ni + 1));
    h2d_sync(B.pre256_d.p, B.pre256.data(), sizeof(int64_t) * (ni + 1));
    B.m = m;
}

// One Arnoldi step of every running instance (every launch gated per instance).
static void batch_step(Batch& B, int j) {
    const BInst* I = B.inst_d.as<BInst>();
    const int ni = B.ninst;
    const unsigned g64 = static_cast<unsigned>(B.pre64.back()), g256 = static_cast<unsigned>(B.pre256.back());
    const int64_t* p64 = B.pre64_d.as<int64_t>();
    const int64_t* p256 = B.pre256_d.as<int64_t>();
    const int k = j + 1;
    const cudaStream_t s = B.stream;
    const unsigned gi = static_cast<unsigned>(cdiv64(ni, 64));
    capture_step(j);
    if (B.shared) {
        // all right-hand sides at once: W = A V_j on the tensor cores, skipping groups whose
        // instances have all left the cycle
        const unsigned groups = static_cast<unsigned>(cdiv64(ni, kTensorRhsTile));
        k_bany_active<<<groups, kTensorRhsTile, 0, s>>>(I, ni, B.gate.as<int>());
        count_launch();
        tensor_block_product(*B.shared, B.v_all + (int64_t)j * ni * B.ld_all, B.ld_all, ni, B.w_all, B.ld_all, s,
                             B.gate.as<int>());
    } else {
        // w = A V_j, or w = A (M^-1 V_j) under the block-Jacobi preconditioner
        const bool bj = B.inner_precond == SB_INNER_PRECOND_BLOCK_JACOBI;
        if (bj) batch_bj_apply(B, 0, j, G_ACTIVE);
        const int mode = bj ? 2 : 0;
        if (B.inner == SB_INNER_FP16) {
            ProfScope prof(SB_PROF_GEMV16, s);
            k_bgemv16<<<static_cast<unsigned>(B.pre16p.back()), kGemvThreads, 0, s>>>(I, B.pre16p_d.as<int64_t>(), ni,
                                                                                      mode, j, G_ACTIVE);
        } else {
            ProfScope prof(SB_PROF_GEMV32, s);
            k_bgemv32<<<g64, kGemvThreads, 0, s>>>(I, p64, ni, mode, j, G_ACTIVE);
        }
        count_launch();
    }
    ProfScope prof(SB_PROF_ARNOLDI, s);
    const int64_t* pdot = B.predot_d.as<int64_t>();
    const dim3 gd(static_cast<unsigned>(B.predot.back()), static_cast<unsigned>(cdiv64(k + 1, kBDotVecs)));
    const dim3 gr(static_cast<unsigned>(k + 1), static_cast<unsigned>(ni));
    k_bdots<<<gd, kChunk, 0, s>>>(I, pdot, ni, k, G_ACTIVE);
    k_breduce<<<gr, 32, 0, s>>>(I, pdot, k, 0, G_ACTIVE);
    const unsigned gw = static_cast<unsigned>(B.prewide.back());
    const int64_t* pw = B.prewide_d.as<int64_t>();
    k_bproject<<<gw, kChunk, 0, s>>>(I, pw, ni, k, 0, G_ACTIVE);
    k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, pw, 0, G_ACTIVE);
    k_bafter_first<<<gi, 64, 0, s>>>(I, ni, j);
    k_bdots<<<gd, kChunk, 0, s>>>(I, pdot, ni, k, G_REORTH);
    k_breduce<<<gr, 32, 0, s>>>(I, pdot, k, 1, G_REORTH);
    k_bproject<<<gw, kChunk, 0, s>>>(I, pw, ni, k, 1, G_REORTH);
    k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, pw, 1, G_REORTH);
    k_bgivens<<<gi, 64, 0, s>>>(I, ni, j);
    k_bnext<<<gw, kChunk, 0, s>>>(I, pw, ni, j);
    for (int t = 0; t < 11; ++t) count_launch();
    (void)g64;
    SB_CUDA(cudaGetLastError());
}

// One restart cycle of the whole batch: m Arnoldi steps captured once into a CUDA graph.
static void batch_cycle(Batch& B) {
    constexpr int kBatchChunk = 4;  // 4 vs 8 steps: sweep 96.2 vs 96.0 solves/s
    const uint64_t gen = B.shared ? tensor_generation(*B.shared) : 0;
    const int pre_key = B.inner_precond * 1024 + B.bj_size;
    const int nch = static_cast<int>((B.m + kBatchChunk - 1) / kBatchChunk);
    if (B.execs.empty() || B.graph_prof != prof_key() || B.graph_gen != gen || B.graph_inner != B.inner ||
        B.graph_pre != pre_key) {
        B.reset_graph();
        capture_begin(&B.prof_pairs);
        for (int c = 0; c < nch; ++c) {
            const int64_t before = kernel_count();
            cudaGraph_t g = nullptr;
            SB_CUDA(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
            try {
                for (int j = c * kBatchChunk; j < std::min<int64_t>(B.m, (c + 1) * kBatchChunk); ++j) batch_step(B, j);
            } catch (...) {
                cudaStreamEndCapture(B.stream, &g);
                if (g) cudaGraphDestroy(g);
                capture_end();
                B.reset_graph();
                throw;
            }
            SB_CUDA(cudaStreamEndCapture(B.stream, &g));
            B.graphs.push_back(g);
            cudaGraphExec_t e = nullptr;
            SB_CUDA(cudaGraphInstantiate(&e, g, 0));
            B.execs.push_back(e);
            B.chunk_kernels.push_back(kernel_count() - before);
            add_kernel_count(-(kernel_count() - before));
        }
        capture_end();
        B.graph_prof = prof_key();
        B.graph_gen = gen;
        B.graph_inner = B.inner;
        B.graph_pre = pre_key;
    }
    if (!B.anyact.p) {
        B.anyact.alloc(sizeof(int));
        B.chk.alloc(2 * sizeof(int));
        for (cudaEvent_t& e : B.ev) SB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    int* hchk = static_cast<int*>(B.chk.p);
    // Chunk c + 1 is queued before the host reads chunk c's flag; launching stops once no instance
    // is left in its cycle (the queued chunk's gated launches return at once).
    auto launch = [&](int c) {
        SB_CUDA(cudaGraphLaunch(B.execs[c], B.stream));
        add_kernel_count(B.chunk_kernels[c]);
        k_ball_active<<<1, 256, 0, B.stream>>>(B.inst_d.as<BInst>(), B.ninst, B.anyact.as<int>());
        count_launch();
        SB_CUDA(cudaMemcpyAsync(hchk + (c & 1), B.anyact.p, sizeof(int), cudaMemcpyDeviceToHost, B.stream));
        SB_CUDA(cudaEventRecord(B.ev[c & 1], B.stream));
    };
    launch(0);
    if (nch > 1) launch(1);
    for (int c = 0; c + 1 < nch; ++c) {
        SB_CUDA(cudaEventSynchronize(B.ev[c & 1]));
        if (!hchk[c & 1]) break;
        if (c + 2 < nch) launch(c + 2);
    }
}

// r = b - A x for every right-hand side of a shared operator: the integer-slice block residual on
// the complex128 matrix (FP64-grade, INT8 tensor cores; ozaki.cu).
static void shared_residual64(Batch& B) {
    const Operator& op = *B.shared;
    ozaki_residual(op, B.b_all, B.ld_all, B.x_all, B.ld_all, B.ninst, B.r_all, B.ld_all, B.stream);
}

// Mixed-precision iterative refinement of every instance in lockstep (gmres_mixed_ir semantics
// per instance, zero initial guess).
static void batch_solve(Batch& B, const sb_ir_config& cfg, sb_gmres_stats* stats) {
    SB_CUDA(cudaSetDevice(B.device));
    batch_workspace(B, cfg.inner_restart);
    const int ni = B.ninst;
    const BInst* I = B.inst_d.as<BInst>();
    const unsigned g64 = static_cast<unsigned>(B.pre64.back()), g256 = static_cast<unsigned>(B.pre256.back());
    const unsigned gi = static_cast<unsigned>(cdiv64(ni, 64));
    const int64_t* p64 = B.pre64_d.as<int64_t>();
    const int64_t* p256 = B.pre256_d.as<int64_t>();
    const cudaStream_t s = B.stream;
    const StateView hv = state_view(B.pin.p, ni);
    const StateView dv = state_view(B.pool_state.p, ni);
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        SB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    };
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        SB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    };
    auto launched = [&](int count) {
        for (int t = 0; t < count; ++t) count_launch();
        SB_CUDA(cudaGetLastError());
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t& a;
        cudaEvent_t& b;
        ~EvGuard() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } evg{e0, e1};
    SB_CUDA(cudaEventRecord(e0, s));
    if (B.inner == SB_INNER_FP16) batch_half_prepare(B);
    if (!B.shared && B.inner_precond == SB_INNER_PRECOND_BLOCK_JACOBI) batch_bj_prepare(B);
    for (int b = 0; b < ni; ++b) stats[b] = sb_gmres_stats{};
    // x = 0, r = b and ||b|| (with a zero initial guess the first residual needs no product).
    k_bvec<<<g256, kChunk, 0, s>>>(I, p256, ni, OP_B_TO_R, G_NONE);
    k_bvnorm<<<g256, kChunk, 0, s>>>(I, p256, ni, 1, G_NONE);
    k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, p256, 2, G_NONE);
    launched(3);
    d2h(hv.nrm, dv.nrm, sizeof(double) * 3 * ni);
    SB_CUDA(cudaStreamSynchronize(s));
    std::vector<double> bnorm(ni), bref(ni), rn(ni), rel(ni, 1.0);
    std::vector<int> status(ni, SB_SOLVER_MAX_ITERATIONS), outer(ni, 1), was_live(ni, 0);
    for (int b = 0; b < ni; ++b) {
        bnorm[b] = std::sqrt(hv.nrm[3 * b + 2]);
        bref[b] = bnorm[b] < 1e-15 ? 1.0 : bnorm[b];
        rn[b] = bnorm[b];
    }
    for (int64_t it = 0; it <= cfg.max_refinements; ++it) {
        if (it > 0) {
            // FP64 residual of the refining instances.
            if (B.shared) {
                shared_residual64(B);
                k_bvnorm<<<g256, kChunk, 0, s>>>(I, p256, ni, 3, G_OUTER);
                k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, p256, 2, G_OUTER);
                launched(2);
            } else {
                {
                    ProfScope prof(SB_PROF_GEMV32, s);
                    k_bres64<<<static_cast<unsigned>(B.prex.back()), kGemvThreads, 0, s>>>(I, B.prex_d.as<int64_t>(),
                                                                                         ni, G_OUTER);
                }
                k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, B.prex_d.as<int64_t>(), 2, G_OUTER);
                launched(2);
            }
            d2h(hv.nrm, dv.nrm, sizeof(double) * 3 * ni);
            SB_CUDA(cudaStreamSynchronize(s));
            for (int b = 0; b < ni; ++b)
                if (outer[b]) {
                    rn[b] = std::sqrt(hv.nrm[3 * b + 2]);
                    ++stats[b].matvecs;
                }
        }
        int refining = 0;
        for (int b = 0; b < ni; ++b) {
            if (outer[b]) {
                rel[b] = rn[b] / bref[b];
                if (rel[b] < cfg.tolerance) {
                    outer[b] = 0;
                    status[b] = SB_SOLVER_CONVERGED;
                } else if (!std::isfinite(rn[b])) {
                    outer[b] = 0;
                    status[b] = SB_SOLVER_NUMERICAL_ERROR;
                } else if (it == cfg.max_refinements) {
                    outer[b] = 0;
                } else {
                    ++refining;
                    hv.scal[kScal * b + 0] = 1.0 / rn[b];
                    hv.scal[kScal * b + 1] = rn[b];
                    // The inner solve need not go further than the outer target asks.
                    hv.scal[kScal * b + 3] = std::max(cfg.inner_tolerance, 0.5 * cfg.tolerance / rel[b]);
                }
            }
            hv.outer[b] = outer[b];
        }
        if (!refining) break;
        // The pinned mirror is modified only after a synchronisation that follows its last copy.
        h2d(dv.outer, hv.outer, sizeof(int) * ni);
        h2d(dv.scal, hv.scal, sizeof(double) * kScal * ni);
        // Inner FP32 solves of A d = r / ||r||, in lockstep.
        k_bvec<<<g256, kChunk, 0, s>>>(I, p256, ni, OP_R_TO_RB, G_OUTER);
        k_bvnorm<<<g256, kChunk, 0, s>>>(I, p256, ni, 0, G_OUTER);
        k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, p256, 2, G_OUTER);
        k_bcontrol<<<gi, 64, 0, s>>>(I, ni, 0, 0);
        launched(4);
        for (int b = 0; b < ni; ++b) was_live[b] = outer[b];
        for (int64_t cyc = 0; cyc < cfg.inner_max_iterations; ++cyc) {
            const bool last = cyc + 1 == cfg.inner_max_iterations;
            k_bvec<<<g256, kChunk, 0, s>>>(I, p256, ni, cyc == 0 ? OP_RB_TO_V0 : OP_RQ_TO_V0, G_LIVE);
            k_bcycle_init<<<ni, 256, 0, s>>>(I, static_cast<int>(B.m));
            launched(2);
            batch_cycle(B);
            k_bupper<<<gi, 64, 0, s>>>(I, ni);
            k_bvec<<<g256, kChunk, 0, s>>>(I, p256, ni, OP_D_UPDATE, G_LIVE);
            launched(2);
            if (!last) {
                // restart residual rq = rb - A d of the instances that completed m steps
                if (B.shared) {
                    tensor_block_product(*B.shared, B.d_all, B.ld_all, ni, B.w_all, B.ld_all, s);
                    k_bresid_w<<<g256, kChunk, 0, s>>>(I, p256, ni, G_RESTART);
                    k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, p256, 2, G_RESTART);
                    launched(2);
                } else {
                    // rq = rb - A d, or rb - A (M^-1 d) under the block-Jacobi preconditioner
                    const bool bj = B.inner_precond == SB_INNER_PRECOND_BLOCK_JACOBI;
                    if (bj) batch_bj_apply(B, 1, 0, G_RESTART);
                    const int mode = bj ? 3 : 1;
                    if (B.inner == SB_INNER_FP16) {
                        {
                            ProfScope prof(SB_PROF_GEMV16, s);
                            k_bgemv16<<<static_cast<unsigned>(B.pre16p.back()), kGemvThreads, 0, s>>>(
                                I, B.pre16p_d.as<int64_t>(), ni, mode, 0, G_RESTART);
                        }
                        k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, B.pre16p_d.as<int64_t>(), 2, G_RESTART);
                    } else {
                        {
                            ProfScope prof(SB_PROF_GEMV32, s);
                            k_bgemv32<<<g64, kGemvThreads, 0, s>>>(I, p64, ni, mode, 0, G_RESTART);
                        }
                        k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, p64, 2, G_RESTART);
                    }
                    launched(2);
                }
            }
            d2h(hv.st, dv.st, sizeof(KState) * ni);
            k_bcontrol<<<gi, 64, 0, s>>>(I, ni, 1, last ? 1 : 0);
            launched(1);
            d2h(hv.live, dv.live, sizeof(int) * ni);
            d2h(hv.brk, dv.brk, sizeof(int) * ni);
            SB_CUDA(cudaStreamSynchronize(s));
            int steps_max = 0, running = 0;
            for (int b = 0; b < ni; ++b) {
                if (!was_live[b]) continue;
                const KState& st = hv.st[b];
                steps_max = std::max(steps_max, st.jdone);
                stats[b].iterations += st.jdone;
                stats[b].matvecs += st.jdone;
                stats[b].matvecs_fp32 += st.jdone;
                if (st.reason == 0) {
                    ++stats[b].restarts;
                    if (!last) {
                        ++stats[b].matvecs;
                        ++stats[b].matvecs_fp32;
                    }
                }
                was_live[b] = hv.live[b];
                running += hv.live[b];
            }
            profile_account(B.prof_pairs, steps_max);
            if (!running) break;
        }
        // x += ||r|| d (d = M^-1 y under the block-Jacobi preconditioner)
        if (!B.shared && B.inner_precond == SB_INNER_PRECOND_BLOCK_JACOBI) batch_bj_apply(B, 2, 0, G_OUTER);
        k_bvec<<<g256, kChunk, 0, s>>>(I, p256, ni, OP_X_UPDATE, G_OUTER);
        launched(1);
        for (int b = 0; b < ni; ++b) {
            if (!outer[b]) continue;
            ++stats[b].refinements;
            if (hv.brk[b]) {  // breakdown before the first inner step: x is unchanged, r stays valid
                outer[b] = 0;
                status[b] = SB_SOLVER_BREAKDOWN;
            }
        }
    }
    // Every instance stopped right after its residual was formed, so r = b - A x is current:
    // ||A x|| = ||b - r|| gives the backward error without another product.
    k_bvnorm<<<g256, kChunk, 0, s>>>(I, p256, ni, 2, G_NONE);
    k_bsum_partials<<<ni, kSumThreads, 0, s>>>(I, p256, 0, G_NONE);
    launched(2);
    d2h(hv.nrm, dv.nrm, sizeof(double) * 3 * ni);
    SB_CUDA(cudaEventRecord(e1, s));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    B.last_solve_ms = ms;
    B.solved = true;
    for (int b = 0; b < ni; ++b) {
        sb_gmres_stats& st = stats[b];
        const double axn = std::sqrt(hv.nrm[3 * b + 0]);
        st.estimated_residual = rel[b];
        st.device_ms = ms;
        if (!std::isfinite(rn[b]) || !std::isfinite(axn)) {
            st.status = SB_SOLVER_NUMERICAL_ERROR;
            st.converged = 0;
            st.residual = INFINITY;
            st.backward_error = INFINITY;
            continue;
        }
        st.converged = status[b] == SB_SOLVER_CONVERGED ? 1 : 0;
        st.status = status[b];
        st.residual = bnorm[b] > 0 ? rn[b] / bnorm[b] : rn[b];
        st.backward_error = rn[b] / std::max(axn + bnorm[b], 2.2250738585072014e-308);
    }
}

// ---------------------------------------------------------------------------------------------
// Many right-hand sides of one operator
// ---------------------------------------------------------------------------------------------
static Batch& multi_batch(Operator& op, int r) {
    Batch* B = static_cast<Batch*>(op.multi);
    if (B && B->ninst == r) return *B;
    delete B;
    op.multi = nullptr;
    B = new Batch();
    op.multi = B;
    B->device = op.device;
    B->ninst = r;
    B->shared = &op;
    B->nvec.assign(r, op.n);
    B->ld_all = (op.n + 1) / 2 * 2;
    SB_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    B->gate.alloc(sizeof(int) * cdiv64(r, kTensorRhsTile));
    B->pool_rhs.alloc(sizeof(double2) * r * B->ld_all);
    memset_sync(B->pool_rhs.p, 0, sizeof(double2) * r * B->ld_all);
    B->b_all = B->pool_rhs.as<double2>();
    for (int c = 0; c < r; ++c) B->rhs.push_back(B->b_all + (int64_t)c * B->ld_all);
    B->assembled = true;
    return *B;
}

void multi_release(Operator& op) {
    delete static_cast<Batch*>(op.multi);
    op.multi = nullptr;
}

// Solve A x_c = b_c for r right-hand sides given right-hand-side-major on the device (b_c at
// b + c * ldb, x_c at x + c * ldx, complex128).
void multi_solve_device(Operator& op, const double2* b, int64_t ldb, int r, double2* x, int64_t ldx,
                        const sb_ir_config& cfg, sb_gmres_stats* stats) {
    SB_REQUIRE(op.A64.p, SB_ERR_INVALID_ARGUMENT,
               "multi-RHS solve: the FP64 refinement needs the complex128 matrix (SB_PRECISION_FP64 or "
               "SB_PRECISION_FP64_FP32)");
    SB_CUDA(cudaSetDevice(op.device));
    if (!tensor_ready(op)) tensor_prepare(op);
    tensor_reserve(op, r);
    Batch& B = multi_batch(op, r);
    batch_workspace(B, cfg.inner_restart);
    SB_CUDA(cudaStreamSynchronize(op.stream));
    SB_CUDA(cudaMemcpy2DAsync(B.b_all, sizeof(double2) * B.ld_all, b, sizeof(double2) * ldb, sizeof(double2) * op.n,
                              r, cudaMemcpyDeviceToDevice, B.stream));
    batch_solve(B, cfg, stats);
    SB_REQUIRE(tensor_status(op, true) == 0, SB_ERR_DEVICE_CHECK,
               "multi-RHS solve: a pipeline wait of the tensor-core kernel timed out");
    SB_REQUIRE(ozaki_status(op, true) == 0, SB_ERR_DEVICE_CHECK,
               "multi-RHS solve: a pipeline wait of the block-residual kernel timed out");
    SB_CUDA(cudaMemcpy2DAsync(x, sizeof(double2) * ldx, B.x_all, sizeof(double2) * B.ld_all, sizeof(double2) * op.n,
                              r, cudaMemcpyDeviceToDevice, B.stream));
    SB_CUDA(cudaStreamSynchronize(B.stream));
}

}  // namespace sb

using namespace sb;

struct sb_batch {
    sb::Batch* b;
};

namespace {

template <class F>
int guarded_batch(F&& f) {
    return abi_guard(std::forward<F>(f));
}

}  // namespace

extern "C" {

SB_API int sb_batch_create(int64_t count, sb_mesh* const* meshes, const sb_physics* physics,
                           const sb_complex* betas, sb_batch** out) {
    return guarded_batch([&] {
        SB_REQUIRE(out, SB_ERR_INVALID_ARGUMENT, "batch: null output handle");
        *out = nullptr;
        SB_REQUIRE(meshes && physics && betas && count >= 1, SB_ERR_INVALID_ARGUMENT,
                   "batch: need at least one instance with mesh, physics and beta");
        SB_REQUIRE(count <= 4096, SB_ERR_INVALID_ARGUMENT, "batch: at most 4096 instances");
        Batch* B = new Batch();
        try {
            B->ninst = static_cast<int>(count);
            for (int64_t i = 0; i < count; ++i) {
                SB_REQUIRE(meshes[i] && meshes[i]->m, SB_ERR_INVALID_ARGUMENT, "batch: null mesh");
                SB_REQUIRE(!meshes[i]->m->quad, SB_ERR_UNSUPPORTED_ELEMENT, "batch: Tri3 meshes only");
                SB_REQUIRE(sb_physics_validate(&physics[i]) == SB_OK, SB_ERR_INVALID_ARGUMENT,
                           "batch: invalid physics parameters");
                SB_REQUIRE(std::isfinite(betas[i].re) && std::isfinite(betas[i].im), SB_ERR_INVALID_ARGUMENT,
                           "batch: beta must be finite");
                Mesh* m = meshes[i]->m;
                if (i == 0) B->device = m->device;
                SB_REQUIRE(m->device == B->device, SB_ERR_INVALID_ARGUMENT, "batch: all meshes on one device");
                SB_CUDA(cudaSetDevice(B->device));
                if (!m->bc_kind.p) mesh_set_bc(*m, nullptr, nullptr, nullptr, nullptr);
                SB_REQUIRE(!m->any_bc_value, SB_ERR_INVALID_ARGUMENT,
                           "batch: meshes with prescribed boundary values are not batched (rigid or "
                           "admittance surfaces only)");
                B->meshes.push_back(m);
                B->nvec.push_back(m->n);
                B->phys.push_back(physics[i]);
                B->beta.push_back(make_double2(betas[i].re, betas[i].im));
            }
            SB_CUDA(cudaSetDevice(B->device));
            ensure_tables(B->device);
            SB_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
            // complex64 matrices, coefficient arrays and diagonals in one pool, right-hand sides
            // in another (they survive workspace re-sizing).
            size_t mat = 0, cof = 0, dg = 0, rhs = 0;
            for (Mesh* m : B->meshes) {
                const int64_t lda = (m->n + 1) / 2 * 2;
                mat += round256(sizeof(float2) * m->n * lda);
                cof += round256(sizeof(double) * coefficient_fields() * m->ld);
                dg += round256(sizeof(double2) * m->n);
                rhs += round256(sizeof(double2) * ((m->n + 1) / 2 * 2));
            }
            B->pool_mat.alloc(mat + cof + dg);
            B->pool_rhs.alloc(rhs);
            memset_sync(B->pool_rhs.p, 0, rhs);
            char* pm = B->pool_mat.as<char>();
            char* pc = pm + mat;
            char* pd = pc + cof;
            char* pr = B->pool_rhs.as<char>();
            for (int i = 0; i < B->ninst; ++i) {
                Mesh* m = B->meshes[i];
                BatchAsmInst A;
                A.elem = m->elem.as<double>();
                A.qp32 = m->qp32.as<float>();
                A.coord_bound = m->coord_bound;
                A.n = m->n;
                A.ld = m->ld;
                A.n_tiles = m->n_tiles;
                A.lda32 = (m->n + 1) / 2 * 2;
                A.A32 = reinterpret_cast<float2*>(pm);
                pm += round256(sizeof(float2) * m->n * A.lda32);
                A.coef = reinterpret_cast<double*>(pc);
                pc += round256(sizeof(double) * coefficient_fields() * m->ld);
                A.diag = reinterpret_cast<double2*>(pd);
                pd += round256(sizeof(double2) * m->n);
                A.k = B->phys[i].harmonic_factor * B->phys[i].wave_number;
                A.near_ptr = m->near_ptr.as<int64_t>();
                A.near_col = m->near_col.as<int32_t>();
                A.near_row = m->near_row.as<int32_t>();
                A.nnz = m->nnz;
                A.amax = nullptr;
                A.mesh = m;
                B->asm_h.push_back(A);
                B->rhs.push_back(reinterpret_cast<double2*>(pr));
                pr += round256(sizeof(double2) * ((m->n + 1) / 2 * 2));
            }
            B->asm_d.alloc(sizeof(BatchAsmInst) * B->ninst);
            SB_CUDA(cudaMemcpy(B->asm_d.p, B->asm_h.data(), sizeof(BatchAsmInst) * B->ninst,
                               cudaMemcpyHostToDevice)); SB_CUDA(cudaStreamSynchronize(0));
        } catch (...) {
            delete B;
            throw;
        }
        *out = new sb_batch{B};
    });
}

SB_API int sb_batch_destroy(sb_batch* batch) {
    if (!batch) return SB_OK;
    if (batch->b) {
        cudaSetDevice(batch->b->device);
        delete batch->b;
    }
    delete batch;
    return SB_OK;
}

// Autotuner memory: batch shape (device, per-instance unknowns and near pairs) -> assembly form.
static std::mutex g_tune_mu;
static std::map<std::vector<int64_t>, int> g_tune;

static std::vector<int64_t> batch_shape_key(const Batch& B) {
    std::vector<int64_t> key{B.device};
    for (const BatchAsmInst& I : B.asm_h) {
        key.push_back(I.n);
        key.push_back(I.nnz);
    }
    return key;
}

// The remembered choice of a batch shape: form + 16 * (far CTA slots per SM of the split
// persistent form, 0 = its single launch).
static int tuned_assembly_form(const Batch& B, int* split) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(batch_shape_key(B));
    if (it == g_tune.end()) return SB_BATCH_ASM_AUTO;
    *split = it->second / 16;
    return it->second % 16;
}

static void remember_assembly_form(const Batch& B, int form, int split) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[batch_shape_key(B)] = form + 16 * split;
}

SB_API int sb_batch_set_assembly_mode(sb_batch* batch, int mode) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null handle");
        SB_REQUIRE(mode == SB_BATCH_ASM_AUTO || mode == SB_BATCH_ASM_PERSISTENT || mode == SB_BATCH_ASM_STREAMS,
                   SB_ERR_INVALID_ARGUMENT, "batch: unknown assembly mode");
        batch->b->asm_mode = mode;
    });
}

SB_API int sb_batch_assembly_split(const sb_batch* batch, int* far_slots_per_sm, double* layout_ms) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null handle");
        const Batch& B = *batch->b;
        if (far_slots_per_sm) *far_slots_per_sm = B.asm_split;
        if (layout_ms)
            for (int t = 0; t < 5; ++t) layout_ms[t] = B.tune_split_ms[t];
    });
}

SB_API int sb_batch_assembly_tuning(const sb_batch* batch, int* chosen, double* persistent_ms, double* streams_ms) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null handle");
        const Batch& B = *batch->b;
        if (chosen) *chosen = B.asm_chosen;
        if (persistent_ms) *persistent_ms = B.tune_persistent_ms;
        if (streams_ms) *streams_ms = B.tune_streams_ms;
    });
}

SB_API int sb_batch_assemble(sb_batch* batch) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null handle");
        Batch& B = *batch->b;
        SB_CUDA(cudaSetDevice(B.device));
        maybe_inject(SB_INJECT_LAUNCH);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        SB_CUDA(cudaEventCreate(&e0));
        SB_CUDA(cudaEventCreate(&e1));
        struct EvGuard {
            cudaEvent_t a, b;
            ~EvGuard() {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } evg{e0, e1};
        auto run = [&](int form, int split) -> double {
            SB_CUDA(cudaEventRecord(e0, B.stream));
            for (int i = 0; i < B.ninst; ++i)
                coefficients_for(*B.meshes[i], B.phys[i], B.beta[i].x, B.beta[i].y,
                                 const_cast<double*>(B.asm_h[i].coef), B.stream);
            // With complex-half inner products the kernels also record each matrix's largest part.
            const bool track = B.inner == SB_INNER_FP16;
            if (track && !B.pool_half_aux.p) B.pool_half_aux.alloc(sizeof(unsigned) * 4 * B.ninst);
            if (form == SB_BATCH_ASM_PERSISTENT) {
                unsigned* aux = track ? B.pool_half_aux.as<unsigned>() : nullptr;
                bool changed = false;
                for (int i = 0; i < B.ninst; ++i) {
                    unsigned* want = aux ? aux + 4 * i : nullptr;
                    if (B.asm_h[i].amax != want) {
                        B.asm_h[i].amax = want;
                        changed = true;
                    }
                }
                if (changed) {
                    SB_CUDA(cudaStreamSynchronize(B.stream));  // no earlier launch still reads the descriptors
                    h2d_sync(B.asm_d.p, B.asm_h.data(), sizeof(BatchAsmInst) * B.ninst);
                }
                if (aux) SB_CUDA(cudaMemsetAsync(aux, 0, sizeof(unsigned) * 4 * B.ninst, B.stream));
                assemble_batch(B.asm_h, B.asm_d.as<BatchAsmInst>(), B.pre_asm, B.stream, B.device, &B.side, split);
                B.amax_valid = track;
            } else {
                assemble_batch_streams(B.asm_h, B.stream, B.side, track ? B.pool_half_aux.as<unsigned>() : nullptr);
                B.amax_valid = track;
            }
            SB_CUDA(cudaEventRecord(e1, B.stream));
            SB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            return ms;
        };
        int form = B.asm_mode, split = B.asm_split;
        if (form == SB_BATCH_ASM_AUTO) form = tuned_assembly_form(B, &split);
        if (form == SB_BATCH_ASM_AUTO) {
            // Autotune, after one untimed assembly (first touches): the persistent form as one launch
            // and as two launches (far tiles on 4, 3 or 2 CTA slots per SM), and the per-instance
            // streams form,
            // each once (every run writes the complete matrices); the fastest is kept for every
            // batch of this shape on this device.
            run(SB_BATCH_ASM_STREAMS, 0);
            double best = 1e300;
            for (int sp : {0, 4, 3, 2}) {
                const double t = run(SB_BATCH_ASM_PERSISTENT, sp);
                B.tune_split_ms[sp] = t;
                if (t < best) {
                    best = t;
                    split = sp;
                }
            }
            B.tune_persistent_ms = best;
            B.tune_streams_ms = run(SB_BATCH_ASM_STREAMS, 0);
            form = B.tune_streams_ms < B.tune_persistent_ms ? SB_BATCH_ASM_STREAMS : SB_BATCH_ASM_PERSISTENT;
            remember_assembly_form(B, form, split);
            B.last_assembly_ms = std::min(B.tune_persistent_ms, B.tune_streams_ms);
        } else {
            B.last_assembly_ms = run(form, split);
        }
        B.asm_split = split;
        B.asm_chosen = form;
        B.assembled = true;
        B.half_valid = false;
        B.bj_valid = false;
    });
}

SB_API int sb_batch_set_inner_preconditioner(sb_batch* batch, int kind, int block_size) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        SB_REQUIRE(kind == SB_INNER_PRECOND_NONE || kind == SB_INNER_PRECOND_BLOCK_JACOBI, SB_ERR_INVALID_ARGUMENT,
                   "inner preconditioner must be SB_INNER_PRECOND_NONE or SB_INNER_PRECOND_BLOCK_JACOBI");
        Batch& B = *batch->b;
        if (kind == SB_INNER_PRECOND_BLOCK_JACOBI) {
            SB_REQUIRE(block_size == 32 || block_size == 64 || block_size == 96 || block_size == 128,
                       SB_ERR_INVALID_ARGUMENT, "block_size must be 32, 64, 96 or 128");
            if (block_size != B.bj_size) B.bj_valid = false;
            B.bj_size = block_size;
        }
        B.inner_precond = kind;
    });
}

SB_API int sb_batch_set_inner_precision(sb_batch* batch, int inner) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        SB_REQUIRE(inner == SB_INNER_FP32 || inner == SB_INNER_FP16, SB_ERR_INVALID_ARGUMENT,
                   "inner precision must be SB_INNER_FP32 or SB_INNER_FP16");
        Batch& B = *batch->b;
        B.inner = inner;
        if (inner == SB_INNER_FP32 && B.pool_half.p) {
            // Drop the copies and the instance descriptors' pointers to them.
            B.pool_half.release();
            B.pool_half_aux.release();
            B.half_valid = false;
            B.amax_valid = false;
            if (!B.h.empty()) {
                SB_CUDA(cudaSetDevice(B.device));
                for (int b = 0; b < B.ninst; ++b) half_pointers(B, b, B.h[b]);
                h2d_sync(B.inst_d.p, B.h.data(), sizeof(BInst) * B.ninst);
            }
        }
    });
}

SB_API int sb_batch_set_rhs_plane_wave(sb_batch* batch, const double* direction) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b && direction, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        Batch& B = *batch->b;
        const double dn = std::sqrt(direction[0] * direction[0] + direction[1] * direction[1] +
                                    direction[2] * direction[2]);
        SB_REQUIRE(std::isfinite(dn) && dn > 0, SB_ERR_INVALID_ARGUMENT, "batch: direction must be nonzero");
        SB_CUDA(cudaSetDevice(B.device));
        for (int i = 0; i < B.ninst; ++i)
            incident_plane_wave(*B.meshes[i], B.phys[i], B.beta[i].x, B.beta[i].y, direction, nullptr, 1, B.rhs[i],
                                B.stream, false);
        SB_CUDA(cudaStreamSynchronize(B.stream));
    });
}

SB_API int sb_batch_set_rhs(sb_batch* batch, int64_t index, const sb_complex* b) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b && b, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        Batch& B = *batch->b;
        SB_REQUIRE(index >= 0 && index < B.ninst, SB_ERR_INVALID_ARGUMENT, "batch: index out of range");
        const int64_t n = B.meshes[index]->n;
        for (int64_t i = 0; i < n; ++i)
            SB_REQUIRE(std::isfinite(b[i].re) && std::isfinite(b[i].im), SB_ERR_NOT_FINITE,
                       "batch: non-finite right-hand side");
        SB_CUDA(cudaSetDevice(B.device));
        SB_CUDA(cudaStreamSynchronize(B.stream));
        h2d_sync(B.rhs[index], b, sizeof(double2) * n);
    });
}

SB_API int sb_batch_solve(sb_batch* batch, const sb_ir_config* cfg, sb_gmres_stats* stats) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b && cfg && stats, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        SB_REQUIRE(cfg->max_refinements >= 0 && cfg->inner_restart > 0 && cfg->inner_restart <= kMaxKrylov &&
                       cfg->inner_max_iterations > 0 && cfg->tolerance > 0 && cfg->inner_tolerance > 0,
                   SB_ERR_INVALID_ARGUMENT, "batch: invalid refinement configuration");
        Batch& B = *batch->b;
        SB_REQUIRE(B.assembled, SB_ERR_INVALID_ARGUMENT, "batch: assemble before solving");
        maybe_inject(SB_INJECT_LAUNCH);
        batch_solve(B, *cfg, stats);
    });
}

SB_API int sb_batch_solution(const sb_batch* batch, int64_t index, sb_complex* x) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b && x, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        Batch& B = *batch->b;
        SB_REQUIRE(index >= 0 && index < B.ninst, SB_ERR_INVALID_ARGUMENT, "batch: index out of range");
        SB_REQUIRE(B.solved, SB_ERR_INVALID_ARGUMENT, "batch: no solution yet");
        SB_CUDA(cudaSetDevice(B.device));
        SB_CUDA(cudaStreamSynchronize(B.stream));
        SB_CUDA(cudaMemcpy(x, B.h[index].x, sizeof(double2) * B.h[index].n, cudaMemcpyDeviceToHost));
    });
}

SB_API int sb_batch_matrix_c64(const sb_batch* batch, int64_t index, sb_complex32* matrix) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b && matrix, SB_ERR_INVALID_ARGUMENT, "batch: null argument");
        Batch& B = *batch->b;
        SB_REQUIRE(index >= 0 && index < B.ninst, SB_ERR_INVALID_ARGUMENT, "batch: index out of range");
        SB_REQUIRE(B.assembled, SB_ERR_INVALID_ARGUMENT, "batch: not assembled");
        const BatchAsmInst& A = B.asm_h[index];
        SB_CUDA(cudaSetDevice(B.device));
        SB_CUDA(cudaStreamSynchronize(B.stream));
        SB_CUDA(cudaMemcpy2D(matrix, sizeof(float2) * A.n, A.A32, sizeof(float2) * A.lda32, sizeof(float2) * A.n,
                             A.n, cudaMemcpyDeviceToHost));
    });
}

SB_API int sb_batch_timings(const sb_batch* batch, double* assembly_ms, double* solve_ms) {
    return guarded_batch([&] {
        SB_REQUIRE(batch && batch->b, SB_ERR_INVALID_ARGUMENT, "batch: null handle");
        if (assembly_ms) *assembly_ms = batch->b->last_assembly_ms;
        if (solve_ms) *solve_ms = batch->b->last_solve_ms;
    });
}

}  // extern "C"
