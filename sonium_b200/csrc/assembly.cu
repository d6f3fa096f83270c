// Dense Burton-Miller TBEM assembly on sm_100a: mesh precompute, near-pair classification and
// the far / near / self kernels.
//
// Reference (paths relative to the sonium workspace root):
//   build_tbem_system_with_beta_parallel  crates/sonium-bem/src/core/assembly/tbem.rs:1284-1466
//   regular_integration                   crates/sonium-bem/src/core/integration/regular.rs:124-321
//   generate_subelements                  crates/sonium-bem/src/core/integration/singular.rs:1372-1540
//   singular_integration                  crates/sonium-bem/src/core/integration/singular.rs:297-614
//
// Work split. A pair (source i, field j) whose level-0 subdivision test passes
// (dist(centre_j, x_i) >= 3 sqrt(area_j)) is a single 13-point leaf: the far kernel evaluates
// those with field-element quadrature points staged in shared memory by a bulk async copy and
// one thread per (row, column) so that the complex stores of a warp are contiguous. Pairs that
// may fail the test (a superset with a 1e-9 relative margin, decided with correctly rounded
// operations so every kernel agrees) go to the near kernel, one warp per pair, which replays
// the reference subdivision tree exactly (level order, the 15-split and 110-leaf limits) and
// reduces the leaf points with warp shuffles. The diagonal goes to the self kernel, one warp per
// element (regularised edge integral + Duffy sub-triangles).

#include <mutex>

#include "sb_device.cuh"
#include "sb_gemv.cuh"
#include "sb_internal.cuh"
#include "sb_profile.cuh"

namespace sb {

// ---------------------------------------------------------------------------------------------
// Quadrature tables
// ---------------------------------------------------------------------------------------------
__constant__ double c_gl_x[kGLTotal];
__constant__ double c_gl_w[kGLTotal];
__constant__ double c_tri_xi[kTriTotal];
__constant__ double c_tri_eta[kTriTotal];
__constant__ double c_tri_w[kTriTotal];
__constant__ int c_tri_off[kTriOrders];
__constant__ int c_tri_cnt[kTriOrders];
// (cos, sin)(m pi / 64), m = 0..127: the pair phase of the FP32 far field is a table angle plus a
// remainder below pi / 128 (global memory, read through the read-only cache: the lanes of a warp
// read different entries).
constexpr int kPhaseTab = 128;
__device__ float2 g_phase_tab[kPhaseTab];

// Gauss-Legendre on [-1, 1] by Newton iteration on the Legendre three-term recurrence.
void host_gauss_legendre(int n, double* x, double* w) {
    const int half = (n + 1) / 2;
    const double nf = n;
    for (int i = 0; i < half; ++i) {
        double root = std::cos(3.14159265358979323846 * (i + 0.75) / (nf + 0.5));
        for (int it = 0; it < 32; ++it) {
            double p0 = 1.0, p1 = root;
            for (int d = 2; d <= n; ++d) {
                double p2 = ((2 * d - 1) * root * p1 - (d - 1) * p0) / d;
                p0 = p1;
                p1 = p2;
            }
            double dp = nf * (root * p1 - p0) / (root * root - 1.0);
            double next = root - p1 / dp;
            bool done = std::fabs(next - root) <= 8.9e-16 * std::fmax(std::fabs(next), 1.0);
            root = next;
            if (done) break;
        }
        double p0 = 1.0, p1 = root;
        for (int d = 2; d <= n; ++d) {
            double p2 = ((2 * d - 1) * root * p1 - (d - 1) * p0) / d;
            p0 = p1;
            p1 = p2;
        }
        double dp = nf * (root * p1 - p0) / (root * root - 1.0);
        double wt = 2.0 / ((1.0 - root * root) * dp * dp);
        if (n == 1) {
            root = 0.0;
            wt = 2.0;
        }
        x[i] = -root;
        x[n - 1 - i] = root;
        w[i] = wt;
        w[n - 1 - i] = wt;
    }
}

// The published 13-point degree-7 symmetric triangle rule on the unit simplex, with the
// 15-digit constants the reference table carries (crates/sonium-bem/src/core/integration/
// gauss.rs:524-538) so that leaf quadratures agree with it to rounding.
static const double kRule13[13][3] = {
    {0.333333333333333, 0.333333333333333, -0.149570044467682},
    {0.260345966079040, 0.260345966079040, 0.175615257433208},
    {0.260345966079040, 0.479308067841920, 0.175615257433208},
    {0.479308067841920, 0.260345966079040, 0.175615257433208},
    {0.065130102902216, 0.065130102902216, 0.053347235608838},
    {0.065130102902216, 0.869739794195568, 0.053347235608838},
    {0.869739794195568, 0.065130102902216, 0.053347235608838},
    {0.638444188569810, 0.048690315425316, 0.077113760890257},
    {0.048690315425316, 0.638444188569810, 0.077113760890257},
    {0.638444188569810, 0.312865496004874, 0.077113760890257},
    {0.312865496004874, 0.638444188569810, 0.077113760890257},
    {0.048690315425316, 0.312865496004874, 0.077113760890257},
    {0.312865496004874, 0.048690315425316, 0.077113760890257}};

// triangle_quadrature (gauss.rs:110-156) for leaf orders 4..7: order 4 is the 13-point rule,
// higher orders the Duffy-collapsed Gauss-Legendre product; weights sum to 0.5.
int host_triangle_rule(int order, double* xi, double* eta, double* w) {
    if (order == 4) {
        for (int i = 0; i < 13; ++i) {
            xi[i] = kRule13[i][0];
            eta[i] = kRule13[i][1];
            w[i] = kRule13[i][2] * 0.5;
        }
        return 13;
    }
    double gx[16], gw[16];
    host_gauss_legendre(order, gx, gw);
    int c = 0;
    for (int a = 0; a < order; ++a) {
        double u = 0.5 * (gx[a] + 1.0), uw = 0.5 * gw[a];
        for (int b = 0; b < order; ++b) {
            double v = 0.5 * (gx[b] + 1.0), vw = 0.5 * gw[b];
            xi[c] = u;
            eta[c] = (1.0 - u) * v;
            w[c] = uw * vw * (1.0 - u);
            ++c;
        }
    }
    return c;
}

void ensure_tables(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    SB_REQUIRE(device >= 0 && device < 64, SB_ERR_INVALID_ARGUMENT, "device index out of range");
    if (done[device]) return;
    double gx[kGLTotal], gw[kGLTotal];
    for (int n = 1; n <= kMaxGL; ++n) host_gauss_legendre(n, gx + n * (n - 1) / 2, gw + n * (n - 1) / 2);
    double tx[kTriTotal], te[kTriTotal], tw[kTriTotal];
    int off[kTriOrders], cnt[kTriOrders], c = 0;
    for (int o = 4; o <= 7; ++o) {
        off[o - 4] = c;
        cnt[o - 4] = host_triangle_rule(o, tx + c, te + c, tw + c);
        c += cnt[o - 4];
    }
    SB_CUDA(cudaMemcpyToSymbol(c_gl_x, gx, sizeof(gx)));
    SB_CUDA(cudaMemcpyToSymbol(c_gl_w, gw, sizeof(gw)));
    SB_CUDA(cudaMemcpyToSymbol(c_tri_xi, tx, sizeof(tx)));
    SB_CUDA(cudaMemcpyToSymbol(c_tri_eta, te, sizeof(te)));
    SB_CUDA(cudaMemcpyToSymbol(c_tri_w, tw, sizeof(tw)));
    SB_CUDA(cudaMemcpyToSymbol(c_tri_off, off, sizeof(off)));
    SB_CUDA(cudaMemcpyToSymbol(c_tri_cnt, cnt, sizeof(cnt)));
    float2 ph[kPhaseTab];
    for (int m = 0; m < kPhaseTab; ++m)
        ph[m] = make_float2(static_cast<float>(std::cos(m * (M_PI / 64.0))), static_cast<float>(std::sin(m * (M_PI / 64.0))));
    SB_CUDA(cudaMemcpyToSymbol(g_phase_tab, ph, sizeof(ph)));
    SB_CUDA(cudaDeviceSynchronize());  // tables in place before kernels on any stream read them
    done[device] = true;
}

// ---------------------------------------------------------------------------------------------
// Mesh precompute
// ---------------------------------------------------------------------------------------------
#define E(f, e) elem[(int64_t)(f) * ld + (e)]

// compute_element_geometry (generators.rs:771-830) and the level-0 subdivision centre
// local_to_global(1/3, 1/3) (singular.rs:1409-1418, 1580-1606), with explicitly rounded
// operations so the host-visible geometry does not depend on multiply-add contraction.
__global__ void k_element_geometry(const double* __restrict__ nodes,
                                   const uint32_t* __restrict__ tris, int64_t n, int64_t ld,
                                   double* __restrict__ elem) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ld) return;
    if (e >= n) {
        for (int f = 0; f < EFIELDS; ++f) E(f, e) = 0.0;
        return;
    }
    double v[3][3];
    for (int a = 0; a < 3; ++a) {
        uint32_t t = tris[3 * e + a];
        for (int j = 0; j < 3; ++j) v[a][j] = nodes[3 * (int64_t)t + j];
    }
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 3; ++j) E(EV0X + 3 * a + j, e) = v[a][j];
    for (int j = 0; j < 3; ++j) {
        double s = __dadd_rn(__dadd_rn(__dadd_rn(0.0, v[0][j]), v[1][j]), v[2][j]);
        E(ECX + j, e) = __ddiv_rn(s, 3.0);
    }
    double a1[3], a2[3];
    for (int j = 0; j < 3; ++j) {
        a1[j] = __dsub_rn(v[1][j], v[0][j]);
        a2[j] = __dsub_rn(v[2][j], v[0][j]);
    }
    double c0 = __dsub_rn(__dmul_rn(a1[1], a2[2]), __dmul_rn(a1[2], a2[1]));
    double c1 = __dsub_rn(__dmul_rn(a1[2], a2[0]), __dmul_rn(a1[0], a2[2]));
    double c2 = __dsub_rn(__dmul_rn(a1[0], a2[1]), __dmul_rn(a1[1], a2[0]));
    double len = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(c0, c0), __dmul_rn(c1, c1)), __dmul_rn(c2, c2)));
    E(EAREA, e) = __ddiv_rn(len, 2.0);
    E(EJAC, e) = len;
    if (len > 1e-15) {
        E(ENX, e) = __ddiv_rn(c0, len);
        E(ENY, e) = __ddiv_rn(c1, len);
        E(ENZ, e) = __ddiv_rn(c2, len);
    } else {
        E(ENX, e) = E(ENY, e) = E(ENZ, e) = 0.0;
    }
    const double third = __ddiv_rn(1.0, 3.0);
    const double sf0 = __dsub_rn(__dsub_rn(1.0, third), third);
    for (int j = 0; j < 3; ++j) {
        double g = __dadd_rn(0.0, __dmul_rn(sf0, v[0][j]));
        g = __dadd_rn(g, __dmul_rn(third, v[1][j]));
        g = __dadd_rn(g, __dmul_rn(third, v[2][j]));
        E(EGX + j, e) = g;
    }
    E(ESQA, e) = __dsqrt_rn(E(EAREA, e));
}

// Far-field leaf points of every element: position of the 13-point rule on the flat triangle
// (compute_parameters, regular.rs:636-714) and weight * Jacobian, in tile-blocked SoA
// qp[((tile * 13 + q) * 4 + c) * kFarTile + lane] so one contiguous block feeds a column tile.
__global__ void k_far_points(const double* __restrict__ elem, int64_t n, int64_t ld,
                             double* __restrict__ qp) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ld) return;
    const int64_t tile = e / kFarTile;
    const int lane = static_cast<int>(e % kFarTile);
    const int o = c_tri_off[0];
    for (int q = 0; q < kFarPoints; ++q) {
        double* dst = qp + ((tile * kFarPoints + q) * 4) * kFarTile + lane;
        if (e >= n) {
            dst[0] = dst[kFarTile] = dst[2 * kFarTile] = dst[3 * kFarTile] = 0.0;
            continue;
        }
        const double s = c_tri_xi[o + q], t = c_tri_eta[o + q];
        const double sf0 = 1.0 - s - t;
        for (int j = 0; j < 3; ++j)
            dst[j * kFarTile] = sf0 * E(EV0X + j, e) + s * E(EV1X + j, e) + t * E(EV2X + j, e);
        dst[3 * kFarTile] = c_tri_w[o + q] * E(EJAC, e);
    }
}

// Superset of the reference's level-0 "must subdivide" test ratdis < 3 (singular.rs:1431):
// dist^2 < 9 (1 + 1e-9) area, evaluated with correctly rounded operations so that the
// classifier and the far kernel make bitwise-identical decisions.
__device__ __forceinline__ bool near_superset(double gx, double gy, double gz, double thr,
                                              double x, double y, double z) {
    double dx = __dsub_rn(gx, x), dy = __dsub_rn(gy, y), dz = __dsub_rn(gz, z);
    double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return d2 < thr;
}
__device__ __forceinline__ double near_threshold(double area) {
    return __dmul_rn(9.000000009, area);
}

constexpr int kNearRows = 32;
constexpr int kNearCols = 256;  // columns per chunk of the classifier, one per thread

// Bounds of every chunk of kNearCols columns: box[8 t + 0..2] the lower and [8 t + 3..5] the upper
// corner of the chunk's level-0 subdivision centres, [8 t + 6] its largest near threshold.
__global__ void __launch_bounds__(kNearCols) k_near_chunk_bounds(const double* __restrict__ elem, int64_t n,
                                                                 int64_t ld, double* __restrict__ box) {
    __shared__ double red[kNearCols / 32][7];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t j = blockIdx.x * (int64_t)kNearCols + tid;
    double v[7];
    if (j < n) {
        v[0] = v[3] = E(EGX, j);
        v[1] = v[4] = E(EGY, j);
        v[2] = v[5] = E(EGZ, j);
        v[6] = near_threshold(E(EAREA, j));
    } else {
        v[0] = v[1] = v[2] = INFINITY;
        v[3] = v[4] = v[5] = v[6] = -INFINITY;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = fmin(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
#pragma unroll
        for (int c = 3; c < 7; ++c) v[c] = fmax(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
    }
    if (lane == 0)
        for (int c = 0; c < 7; ++c) red[warp][c] = v[c];
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kNearCols / 32; ++w) {
            for (int c = 0; c < 3; ++c) v[c] = fmin(v[c], red[w][c]);
            for (int c = 3; c < 7; ++c) v[c] = fmax(v[c], red[w][c]);
        }
        for (int c = 0; c < 7; ++c) box[8 * blockIdx.x + c] = v[c];
        box[8 * blockIdx.x + 7] = 0.0;
    }
}

// Near-pair classification, one CTA per 32 source rows. pass 0 counts per row, pass 1 writes
// the column indices in increasing order and the row of every pair (row_ptr from the scan). A
// chunk of columns whose box lies farther from the box of the CTA's rows than its largest
// threshold allows is skipped: every pair in it would test far (the 1e-9 margin covers the
// rounding of both squared distances), so both passes and the decisions stay those of the full
// test.
__global__ void __launch_bounds__(kNearCols) k_near_pass(const double* __restrict__ elem, int64_t n,
                                                         int64_t ld, int pass, const double* __restrict__ box,
                                                         int64_t* __restrict__ counts,
                                                         const int64_t* __restrict__ row_ptr,
                                                         int32_t* __restrict__ cols, int32_t* __restrict__ rows) {
    __shared__ double sx[kNearRows][3];
    __shared__ double srb[6];
    __shared__ unsigned sball[kNearCols / 32][kNearRows];
    __shared__ int64_t sbase[kNearRows];
    __shared__ int scount[kNearRows];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t row0 = blockIdx.x * (int64_t)kNearRows;
    if (tid < kNearRows) {
        int64_t i = row0 + tid;
        for (int c = 0; c < 3; ++c) sx[tid][c] = (i < n) ? E(ECX + c, i) : 1e300;
        scount[tid] = 0;
        sbase[tid] = (pass == 1 && i < n) ? row_ptr[i] : 0;
    }
    __syncthreads();
    if (tid == 0) {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int r = 0; r < kNearRows && row0 + r < n; ++r)
            for (int c = 0; c < 3; ++c) {
                lo[c] = fmin(lo[c], sx[r][c]);
                hi[c] = fmax(hi[c], sx[r][c]);
            }
        for (int c = 0; c < 3; ++c) {
            srb[c] = lo[c];
            srb[3 + c] = hi[c];
        }
    }
    __syncthreads();
    for (int64_t c0 = 0; c0 < n; c0 += kNearCols) {
        const double* B = box + 8 * (c0 / kNearCols);
        double gap2 = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double g = fmax(0.0, fmax(B[c] - srb[3 + c], srb[c] - B[3 + c]));
            gap2 += g * g;
        }
        if (gap2 > B[6] * (1.0 + 1e-9)) continue;  // the same decision in every thread
        const int64_t j = c0 + tid;
        double gx = 0, gy = 0, gz = 0, thr = -1.0;
        if (j < n) {
            gx = E(EGX, j);
            gy = E(EGY, j);
            gz = E(EGZ, j);
            thr = near_threshold(E(EAREA, j));
        }
        for (int r = 0; r < kNearRows; ++r) {
            const int64_t i = row0 + r;
            bool p = (j < n) && (i < n) && (j != i) &&
                     near_superset(gx, gy, gz, thr, sx[r][0], sx[r][1], sx[r][2]);
            unsigned b = __ballot_sync(0xffffffffu, p);
            if (pass == 0) {
                if (lane == 0 && b) atomicAdd(&scount[r], __popc(b));
            } else {
                if (lane == 0) sball[warp][r] = b;
            }
        }
        if (pass == 1) {
            __syncthreads();
            for (int r = 0; r < kNearRows; ++r) {
                const unsigned b = sball[warp][r];
                if (b & (1u << lane)) {
                    int64_t pos = sbase[r];
                    for (int w = 0; w < warp; ++w) pos += __popc(sball[w][r]);
                    pos += __popc(b & ((1u << lane) - 1u));
                    cols[pos] = static_cast<int32_t>(j);
                    rows[pos] = static_cast<int32_t>(row0 + r);
                }
            }
            __syncthreads();
            if (tid < kNearRows) {
                int64_t t = 0;
                for (int w = 0; w < kNearCols / 32; ++w) t += __popc(sball[w][tid]);
                sbase[tid] += t;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (pass == 0 && tid < kNearRows && row0 + tid < n) counts[row0 + tid] = scount[tid];
}

// Exclusive scan of the per-row pair counts into the CSR row pointers (one CTA): ptr[n] = *total
// = the number of pairs.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) k_scan_counts(const int64_t* __restrict__ counts, int64_t n,
                                                              int64_t* __restrict__ ptr, long long* __restrict__ total) {
    __shared__ long long wsum[kScanThreads / 32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t per = (n + kScanThreads - 1) / kScanThreads;
    const int64_t b = min(n, tid * per), e = min(n, b + per);
    long long s = 0;
    for (int64_t i = b; i < e; ++i) s += counts[i];
    long long incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        long long w = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        wsum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    long long run = incl - s + (warp ? wsum[warp - 1] : 0);
    for (int64_t i = b; i < e; ++i) {
        ptr[i] = run;
        run += counts[i];
    }
    if (tid == kScanThreads - 1) {
        ptr[n] = run;
        *total = run;
    }
}

// ---------------------------------------------------------------------------------------------
// Per-assembly element coefficients
// ---------------------------------------------------------------------------------------------
// coef[f * ld + e], f: 0-7 = (cG, cH, cHt, cE) complex matrix weights of the field element,
// 8-15 = (dG, dH, dHt, dE) complex RHS weights (nonzero only for a nonzero prescribed value),
// 16-17 = diagonal free term, 18-19 = RHS free term. From the coefficient / RHS formulas of
// build_tbem_system_with_beta_parallel (tbem.rs:1344-1358, 1404-1444) with gamma = 1.
enum { CF_CG = 0, CF_CH = 2, CF_CHT = 4, CF_CE = 6, CF_DG = 8, CF_DH = 10, CF_DHT = 12,
       CF_DE = 14, CF_DIAG = 16, CF_RHS = 18, CF_FIELDS = 20 };

__global__ void k_coefficients(int64_t n, int64_t ld, const int32_t* __restrict__ kind,
                               const double2* __restrict__ value,
                               const uint8_t* __restrict__ has_adm,
                               const double2* __restrict__ adm, double tau, double pf,
                               double2 beta, double* __restrict__ coef) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ld) return;
    double2 out[10];
    for (int f = 0; f < 10; ++f) out[f] = make_double2(0.0, 0.0);
    if (e < n) {
        const int k = kind ? kind[e] : 0;
        const double2 v = value ? value[e] : make_double2(0.0, 0.0);
        const bool hv = sqrt(v.x * v.x + v.y * v.y) > 1e-15;  // has_nonzero_bc, tbem.rs:1239
        const bool ha = has_adm && has_adm[e];
        const double2 Y = (ha && adm) ? adm[e] : make_double2(0.0, 0.0);
        const double2 gt = make_double2(tau, 0.0);   // gamma * tau
        const double2 iwr = make_double2(0.0, pf);   // i omega rho
        const double2 bt = cscale(beta, tau);        // beta * tau
        if (k == SB_BC_VELOCITY) {
            out[1] = gt;    // H
            out[3] = beta;  // E
            if (ha) {
                const double2 yi = cmul(Y, iwr);
                out[0] = make_double2(-cmul(gt, yi).x, -cmul(gt, yi).y);
                out[2] = make_double2(-cmul(beta, yi).x, -cmul(beta, yi).y);
            }
            if (hv) {
                const double2 vi = cmul(v, iwr);
                out[4] = cmul(gt, vi);
                out[6] = cmul(beta, vi);
            }
            double2 d = make_double2(-0.5, 0.0);
            if (ha) {
                const double2 t = cscale(cmul(cmul(Y, iwr), bt), 0.5);
                d = make_double2(d.x - t.x, d.y - t.y);
            }
            out[8] = d;
            out[9] = cscale(cmul(cmul(v, iwr), bt), 0.5);
        } else if (k == SB_BC_PRESSURE) {
            out[0] = make_double2(-gt.x, -gt.y);
            out[2] = make_double2(-beta.x, -beta.y);
            if (hv) {
                out[5] = cmul(gt, v);
                out[7] = cmul(beta, v);
            }
            out[8] = cscale(bt, 0.5);
            out[9] = make_double2(-0.5 * v.x, -0.5 * v.y);
        }
    }
    for (int f = 0; f < 10; ++f) {
        coef[(int64_t)(2 * f) * ld + e] = out[f].x;
        coef[(int64_t)(2 * f + 1) * ld + e] = out[f].y;
    }
}

// ---------------------------------------------------------------------------------------------
// Channel accumulation shared by all kernels: one quadrature point of regular.rs:229-281.
// ---------------------------------------------------------------------------------------------
struct Acc {
    double gr = 0, gi = 0, hr = 0, hi = 0, tr = 0, ti = 0, er = 0, ei = 0;
};

// Adds the (G, H, H^T, E) contribution of a point at offset d = y - x (distance r, inverse
// rinv) with weight * Jacobian `wga`, field normal ny and source normal nx.
__device__ __forceinline__ void point_channels(Acc& a, double dx, double dy, double dz,
                                               double r, double rinv, double wga, double nyx,
                                               double nyy, double nyz, double nxx, double nxy,
                                               double nxz, double k, double k2) {
    double s, c;
    sb_sincos(k * r, &s, &c);
    const double gs = wga * kInv4Pi * rinv;
    const double g_r = c * gs, g_i = s * gs;
    const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
    const double rny = ux * nyx + uy * nyy + uz * nyz;
    const double rnx = -(ux * nxx + uy * nxy + uz * nxz);
    // zhh_base = G * (-1/r + i k)
    const double b_r = -g_r * rinv - g_i * k;
    const double b_i = g_r * k - g_i * rinv;
    a.gr += g_r;
    a.gi += g_i;
    a.hr = fma(b_r, rny, a.hr);
    a.hi = fma(b_i, rny, a.hi);
    a.tr = fma(b_r, rnx, a.tr);
    a.ti = fma(b_i, rnx, a.ti);
    const double rq = rny * rnx;
    const double nxny = nxx * nyx + nxy * nyy + nxz * nyz;
    const double ri2 = rinv * rinv;
    const double f_r = (3.0 * ri2 - k2) * rq + nxny * ri2;
    const double f_i = -k * rinv * (3.0 * rq + nxny);
    a.er += g_r * f_r - g_i * f_i;
    a.ei += g_r * f_i + g_i * f_r;
}

__device__ __forceinline__ double2 combine(const Acc& a, const double* __restrict__ coef,
                                           int64_t ld, int64_t j, int base) {
    const double cgr = coef[(int64_t)(base + 0) * ld + j], cgi = coef[(int64_t)(base + 1) * ld + j];
    const double chr = coef[(int64_t)(base + 2) * ld + j], chi = coef[(int64_t)(base + 3) * ld + j];
    const double ctr = coef[(int64_t)(base + 4) * ld + j], cti = coef[(int64_t)(base + 5) * ld + j];
    const double cer = coef[(int64_t)(base + 6) * ld + j], cei = coef[(int64_t)(base + 7) * ld + j];
    double2 v;
    v.x = a.gr * cgr - a.gi * cgi + a.hr * chr - a.hi * chi + a.tr * ctr - a.ti * cti + a.er * cer - a.ei * cei;
    v.y = a.gr * cgi + a.gi * cgr + a.hr * chi + a.hi * chr + a.tr * cti + a.ti * ctr + a.er * cei + a.ei * cer;
    return v;
}

// ---------------------------------------------------------------------------------------------
// Far kernel
// ---------------------------------------------------------------------------------------------
constexpr int kFarRows = 32;
constexpr int kQpTileDoubles = kFarPoints * 4 * kFarTile;
constexpr long kWaitLimit = 1L << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded wait on an mbarrier phase. Returns false when the iteration limit is hit.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <bool kWithRhs, bool kWithF32>
__global__ void __launch_bounds__(kFarTile) k_far(const double* __restrict__ qp,
                                                  const double* __restrict__ elem, int64_t n,
                                                  int64_t ld, const double* __restrict__ coef,
                                                  double k, double2* __restrict__ A64,
                                                  float2* __restrict__ A32, int64_t lda32,
                                                  double2* __restrict__ far_part,
                                                  int64_t n_tiles, int* __restrict__ status) {
    extern __shared__ __align__(128) double smem[];
    double* sq = smem;                              // [13][4][kFarTile]
    double* sr = smem + kQpTileDoubles;             // [kFarRows][6]
    __shared__ __align__(8) uint64_t bar;
    __shared__ double sred[kFarTile / 32][2];
    const int tid = threadIdx.x;
    const int64_t tile = blockIdx.x;
    const int64_t j = tile * kFarTile + tid;
    const int64_t row0 = blockIdx.y * (int64_t)kFarRows;
    const double k2 = k * k;

    // Stage this column tile's quadrature points with one bulk async copy (TMA engine).
    const uint32_t bar_a = smem_addr(&bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = kQpTileDoubles * sizeof(double);
        const double* src = qp + tile * (int64_t)kQpTileDoubles;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(sq)),
            "l"(src), "r"(bytes), "r"(bar_a)
            : "memory");
    }
    // Source rows (collocation point and normal) with plain loads meanwhile.
    for (int t = tid; t < kFarRows * 6; t += kFarTile) {
        const int r = t / 6, f = t % 6;
        const int64_t i = row0 + r;
        sr[t] = (i < n) ? E(ECX + f, i) : 0.0;  // ECX..ECZ then ENX..ENZ are contiguous fields
    }
    // Column constants in registers.
    double nyx = 0, nyy = 0, nyz = 0, gx = 0, gy = 0, gz = 0, thr = -1;
    if (j < n) {
        nyx = E(ENX, j);
        nyy = E(ENY, j);
        nyz = E(ENZ, j);
        gx = E(EGX, j);
        gy = E(EGY, j);
        gz = E(EGZ, j);
        thr = near_threshold(E(EAREA, j));
    }
    const bool ok = mbar_wait(bar_a, 0);
    if (__syncthreads_or(!ok)) {
        // Timed out: report, skip the tile, and stay resident for a second bounded wait so that
        // the bulk copy this CTA issued lands before its shared memory can pass to another CTA.
        // (If that wait also runs out, the copy may still land late; the status word tells the
        // host to discard the whole assembly either way.)
        if (tid == 0) atomicExch(status, 1);
        mbar_wait(bar_a, 0);
        __syncthreads();
        return;
    }

    const int64_t rows_here = (n - row0 < kFarRows) ? (n - row0) : kFarRows;
    for (int r = 0; r < rows_here; ++r) {
        const int64_t i = row0 + r;
        const double xx = sr[r * 6 + 0], xy = sr[r * 6 + 1], xz = sr[r * 6 + 2];
        const double nxx = sr[r * 6 + 3], nxy = sr[r * 6 + 4], nxz = sr[r * 6 + 5];
        const bool active = (j < n) && (j != i) && !near_superset(gx, gy, gz, thr, xx, xy, xz);
        double2 rhs_c = make_double2(0.0, 0.0);
        if (active) {
            Acc a;
#pragma unroll
            for (int q = 0; q < kFarPoints; ++q) {
                const double* p = sq + q * 4 * kFarTile + tid;
                const double dx = p[0] - xx, dy = p[kFarTile] - xy, dz = p[2 * kFarTile] - xz;
                const double w = p[3 * kFarTile];
                const double d2 = dx * dx + dy * dy + dz * dz;
                const double rinv = sb_rsqrt2(d2);
                point_channels(a, dx, dy, dz, d2 * rinv, rinv, w, nyx, nyy, nyz, nxx, nxy, nxz, k, k2);
            }
            const double2 v = combine(a, coef, ld, j, CF_CG);
            A64[i * n + j] = v;
            if (kWithF32) A32[i * lda32 + j] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
            if (kWithRhs) rhs_c = combine(a, coef, ld, j, CF_DG);
        }
        if (kWithRhs) {
            double sx = warp_sum(rhs_c.x), sy = warp_sum(rhs_c.y);
            if ((tid & 31) == 0) {
                sred[tid >> 5][0] = sx;
                sred[tid >> 5][1] = sy;
            }
            __syncthreads();
            if (tid == 0) {
                double tx = 0, ty = 0;
                for (int w = 0; w < kFarTile / 32; ++w) {
                    tx += sred[w][0];
                    ty += sred[w][1];
                }
                far_part[i * n_tiles + tile] = make_double2(tx, ty);
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Mixed-precision far kernel (SB_PRECISION_FP32): the phase argument k r stays in FP64, the rest
// of the 13-point leaf in FP32.
//
// Per pair the centroid offset d_c = c_j - x_i, r_c = |d_c| and exp(i k r_c) come from FP64
// (k r_c reduced modulo 2 pi in FP64, the reduced angle's sin / cos in FP32). Per point, with
// delta_q = y_q - c_j precomputed per element, the distance change is formed without
// cancellation as r_q - r_c = (2 d_c . delta_q + |delta_q|^2) / (r_q + r_c) and its small phase
// k (r_q - r_c) rotates exp(i k r_c). Everything else (G, H, H^T, E factors and the sums) is
// FP32; the near and self pairs keep the FP64 kernels. (N = 20480, k = 10: per-entry error
// against the FP64 matrix median 2e-7; the mixed solution within 3e-8 of the FP64 one.)
// ---------------------------------------------------------------------------------------------
// A flat triangle's quadrature points lie in its plane, so each offset delta_q = y_q - c_j is
// two in-plane coordinates (a_q, b_q) on the element's orthonormal frame (e1, e2), e1 along the
// first edge and e2 = n_y x e1: d_c . delta_q = a_q (d_c . e1) + b_q (d_c . e2), delta_q . n_x =
// a_q (e1 . n_x) + b_q (e2 . n_x) and delta_q . n_y = 0, so r . n_y = d_c . n_y is one value per
// pair. The point data per element is (a, b, |delta|^2, w J / 4 pi); the frame follows it.
constexpr int kQ32 = 4;                              // per point: a, b, |delta|^2, w * J / (4 pi)
constexpr int kQ32Frame = kFarPoints * kQ32;         // then e1 x, y, z, e2 x, y, z
constexpr int kQ32Fields = kQ32Frame + 6;

// Element point data for the FP32 far kernel: qp32[(q * kQ32 + c) * ld + e], frame at
// qp32[(kQ32Frame + c) * ld + e].
__global__ void k_far_points32(const double* __restrict__ elem, int64_t n, int64_t ld,
                               float* __restrict__ qp32) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ld) return;
    if (e >= n) {
        for (int c = 0; c < kQ32Fields; ++c) qp32[(int64_t)c * ld + e] = 0.f;
        return;
    }
    double e1[3], e2[3];
    const double nx = E(ENX, e), ny = E(ENY, e), nz = E(ENZ, e);
    for (int j = 0; j < 3; ++j) e1[j] = E(EV1X + j, e) - E(EV0X + j, e);
    const double l1 = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    for (int j = 0; j < 3; ++j) e1[j] /= l1;
    e2[0] = ny * e1[2] - nz * e1[1];
    e2[1] = nz * e1[0] - nx * e1[2];
    e2[2] = nx * e1[1] - ny * e1[0];
    const int o = c_tri_off[0];
    for (int q = 0; q < kFarPoints; ++q) {
        float* dst = qp32 + (int64_t)(q * kQ32) * ld + e;
        const double s = c_tri_xi[o + q], t = c_tri_eta[o + q];
        const double sf0 = 1.0 - s - t;
        double dl[3];
        for (int j = 0; j < 3; ++j)
            dl[j] = sf0 * E(EV0X + j, e) + s * E(EV1X + j, e) + t * E(EV2X + j, e) - E(ECX + j, e);
        dst[0] = static_cast<float>(dl[0] * e1[0] + dl[1] * e1[1] + dl[2] * e1[2]);
        dst[ld] = static_cast<float>(dl[0] * e2[0] + dl[1] * e2[1] + dl[2] * e2[2]);
        dst[2 * ld] = static_cast<float>(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
        dst[3 * ld] = static_cast<float>(c_tri_w[o + q] * E(EJAC, e) * kInv4Pi);
    }
    for (int j = 0; j < 3; ++j) {
        qp32[(int64_t)(kQ32Frame + j) * ld + e] = static_cast<float>(e1[j]);
        qp32[(int64_t)(kQ32Frame + 3 + j) * ld + e] = static_cast<float>(e2[j]);
    }
}

// sin / cos in FP32 for |x| <= pi: quadrant reduction by pi/2 and Taylor series to x^9 / x^10
// on |r| <= pi/4 (truncation below 2e-9).
__device__ __forceinline__ void sincos_f32(float x, float* so, float* co) {
    // x 2/pi rounded to the nearest integer by adding 1.5 * 2^23 (one rounding, ties to even, as
    // rintf), which also leaves the integer's low bits in the sum's mantissa: no conversion
    // instructions on the special-function unit.
    const float y = fmaf(x, 0.636619772f, 12582912.0f);
    const float q = y - 12582912.0f;
    float r = fmaf(-q, 1.57079637f, x);
    r = fmaf(-q, -4.37113883e-8f, r);
    const float r2 = r * r;
    float ps = 2.75573192e-6f;
    ps = fmaf(ps, r2, -1.98412698e-4f);
    ps = fmaf(ps, r2, 8.33333333e-3f);
    ps = fmaf(ps, r2, -1.66666667e-1f);
    const float sn = fmaf(ps * r2, r, r);
    float pc = -2.75573192e-7f;
    pc = fmaf(pc, r2, 2.48015873e-5f);
    pc = fmaf(pc, r2, -1.38888889e-3f);
    pc = fmaf(pc, r2, 4.16666667e-2f);
    pc = fmaf(pc, r2, -0.5f);
    const float cs = fmaf(pc, r2, 1.0f);
    const int quad = __float_as_int(y) & 3;
    float sv = sn, cv = cs;
    if (quad & 1) {
        sv = cs;
        cv = -sn;
    }
    if (quad & 2) {
        sv = -sv;
        cv = -cv;
    }
    *so = sv;
    *co = cv;
}

constexpr int kFar32Rows = 64;

// Packed FP32 pairs: sm_100 executes one f32x2 add / multiply / fma for two lanes in one issue
// slot, so the far field evaluates two quadrature points per instruction (points 2p, 2p + 1 in
// the .x / .y lanes of pair p; the 13th point runs alone).
constexpr int kFarPairs = kFarPoints / 2;
// The columns' k |delta|^2 and weights sit in shared memory (each thread reads only its own
// column), their in-plane coordinates in registers: 128 registers, 4 CTAs per SM (N = 20480:
// 9.17 ms per assembly; capped at 96 registers for 5 CTAs per SM the loop spills, 9.55 ms).
constexpr bool kFar32SmemCols = true;
constexpr int kFar32MinBlocks = kFar32SmemCols ? 4 : 3;
static_assert(kFarPoints == 2 * kFarPairs + 1, "the packed far loop pairs all points but the last");
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Channel sums of one far pair in the pair-phase frame (see far32_tile).
struct Far32Sums {
    float gr, gi, hr, hi, tr, ti, er, ei;
};

// FP32 constants of one far pair (row i, column j; d_c = c_j - x_i, column frame e1, e2, row
// normal n_x, column normal n_y).
struct Far32Pair {
    float a2k, b2k;  // 2 k d_c . e1, 2 k d_c . e2
    float rc2, rc;   // |d_c|^2, |d_c|
    float ea, eb;    // -e1 . n_x, -e2 . n_x
    float fnx;       // -d_c . n_x
    float fny;       // d_c . n_y (= r_q n_y . r_hat for every point of the flat element)
    float nxny;      // n_x . n_y
};

// FP32 margin test: true when the pair is certainly beyond the near-pair threshold, g = (level-0
// centre of the column in FP32, thr_hi). thr_hi bounds (sqrt(thr) + the FP32 rounding of the
// coordinates) squared from above (far32_col_threshold), so a pair this test calls far is far for
// the correctly rounded FP64 test too; the FP64 test decides every pair this one does not.
__device__ __forceinline__ bool far_by_margin(float4 g, float4 x) {
    const float dx = g.x - x.x, dy = g.y - x.y, dz = g.z - x.z;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > g.w;
}

// thr_hi of a column: (1 + 1e-6) (sqrt(thr) + 5e-7 R)^2 rounded up, R bounding every |coordinate|.
// Per coordinate the FP32 difference of the rounded values is within 4.1 * 2^-24 R of the exact
// difference, the FP32 distance within 4.3e-7 R of the exact one, and the FP32 square of it
// (three roundings) within a factor 1 + 3 * 2^-24.
__device__ __forceinline__ float far32_col_threshold(double thr, double bound) {
    const double s = sqrt(fmax(thr, 0.0)) + 5e-7 * bound;
    return __double2float_ru((1.0 + 1e-6) * s * s);
}

// One quadrature point (a, b, k |delta|^2, w J / 4 pi) of a far pair, scalar (the point left over
// by the packed pairs). t = k (r_q - r_c) = k (2 d_c . delta + |delta|^2) / (r_q + r_c).
template <bool kChecked>
__device__ __forceinline__ void far32_point(Far32Sums& s, float pa, float pb, float pdk, float pw,
                                            const Far32Pair& c, float kf, float invk, float k2f) {
    const float numk = fmaf(c.a2k, pa, fmaf(c.b2k, pb, pdk));
    const float rq2 = fmaf(numk, invk, c.rc2);
    const float rinv = rsqrtf(rq2);
    const float t = numk * rcp_approx(fmaf(rq2, rinv, c.rc));
    float st, ct;
    if (!kChecked || fabsf(t) <= 3.14159265f) {
        __sincosf(t, &st, &ct);
    } else {
        sincos_f32(t, &st, &ct);
    }
    const float gs = pw * rinv;
    const float g_r = ct * gs, g_i = st * gs;
    const float rny = c.fny * rinv;
    const float rnx = fmaf(pb, c.eb, fmaf(pa, c.ea, c.fnx)) * rinv;
    const float b_r = -fmaf(g_r, rinv, g_i * kf);
    const float b_i = fmaf(g_r, kf, -g_i * rinv);
    s.gr += g_r;
    s.gi += g_i;
    s.hr = fmaf(b_r, rny, s.hr);
    s.hi = fmaf(b_i, rny, s.hi);
    s.tr = fmaf(b_r, rnx, s.tr);
    s.ti = fmaf(b_i, rnx, s.ti);
    const float rqq = rny * rnx;
    const float s3 = fmaf(3.f, rqq, c.nxny);
    const float f_r = fmaf(rinv * rinv, s3, -k2f * rqq);
    const float f_i = -kf * rinv * s3;
    s.er = fmaf(g_r, f_r, fmaf(-g_i, f_i, s.er));
    s.ei = fmaf(g_r, f_i, fmaf(g_i, f_r, s.ei));
}

// The 12 packed points of a far pair (the 13th is far32_point). kChecked: test every pair's
// phase offsets against pi and take the quadrant-reduced sine / cosine beyond it; without it the
// caller has shown |t| <= k max |delta| < 3 for every point of the column (|r_q - r_c| <= |delta|).
template <bool kChecked, bool kSmemCols>
__device__ __forceinline__ Far32Sums far32_pairs(const Far32Pair& c, const float2 (&PA)[kFarPairs],
                                                 const float2 (&PB)[kFarPairs], const float4* sPDW,
                                                 const float4 (&PDW)[kSmemCols ? 1 : kFarPairs], int tid, float kf,
                                                 float invk, float k2f) {
    // Points in pairs. With u = g_r / r + g_i k and nbi = g_i / r - g_r k (b = g (-1/r + i k) =
    // -(u + i nbi)), r.n_y = fny / r and q1 = (3 r.n_y r.(-n_x) + n_x.n_y) / r:
    //   H = -fny sum (u + i nbi) / r,  H^T = -sum (u + i nbi) r.(-n_x),
    //   E = sum q1 (u + i nbi) - k^2 fny sum g r.(-n_x) / r,
    // so every channel is a lane sum of one fma per point.
    const float2 A2K = bc2(c.a2k), B2K = bc2(c.b2k), RC2 = bc2(c.rc2), RC = bc2(c.rc);
    const float2 EA = bc2(c.ea), EB = bc2(c.eb), FNX = bc2(c.fnx), FNY3 = bc2(3.f * c.fny);
    const float2 NXNY = bc2(c.nxny), KK = bc2(kf), NK = bc2(-kf), INVK = bc2(invk);
    float2 AGR, AGI, SHR, SHI, NATR, NATI, AER, AEI, GQR, GQI;  // set by the first pair
#pragma unroll
    for (int p = 0; p < kFarPairs; ++p) {
        float4 dw;
        if constexpr (kSmemCols) dw = sPDW[p * kFarTile + tid]; else dw = PDW[p];
        const float2 numk = pfma(A2K, PA[p], pfma(B2K, PB[p], make_float2(dw.x, dw.y)));
        const float2 rq2 = pfma(numk, INVK, RC2);
        const float2 rinv = make_float2(rsqrtf(rq2.x), rsqrtf(rq2.y));
        const float2 den = pfma(rq2, rinv, RC);
        const float2 t = pmul(numk, make_float2(rcp_approx(den.x), rcp_approx(den.y)));
        // Special-function sine / cosine while both phase offsets are within one element
        // size (|t| <= pi, every resolved mesh), else the quadrant-reduced version.
        float2 S, C;
        if (!kChecked || fmaxf(fabsf(t.x), fabsf(t.y)) <= 3.14159265f) {
            __sincosf(t.x, &S.x, &C.x);
            __sincosf(t.y, &S.y, &C.y);
        } else {
            sincos_f32(t.x, &S.x, &C.x);
            sincos_f32(t.y, &S.y, &C.y);
        }
        const float2 gs = pmul(make_float2(dw.z, dw.w), rinv);
        const float2 gr = pmul(C, gs), gi = pmul(S, gs);
        const float2 rnx = pmul(pfma(PB[p], EB, pfma(PA[p], EA, FNX)), rinv);
        const float2 u = pfma(gr, rinv, pmul(gi, KK));
        const float2 nbi = pfma(gi, rinv, pmul(gr, NK));
        const float2 rq1 = pmul(rnx, rinv);
        const float2 q1 = pmul(rinv, pfma(FNY3, rq1, NXNY));
        if (p == 0) {
            AGR = gr;
            AGI = gi;
            SHR = pmul(u, rinv);
            SHI = pmul(nbi, rinv);
            NATR = pmul(u, rnx);
            NATI = pmul(nbi, rnx);
            AER = pmul(q1, u);
            AEI = pmul(q1, nbi);
            GQR = pmul(gr, rq1);
            GQI = pmul(gi, rq1);
        } else {
            AGR = padd(AGR, gr);
            AGI = padd(AGI, gi);
            SHR = pfma(u, rinv, SHR);
            SHI = pfma(nbi, rinv, SHI);
            NATR = pfma(u, rnx, NATR);
            NATI = pfma(nbi, rnx, NATI);
            AER = pfma(q1, u, AER);
            AEI = pfma(q1, nbi, AEI);
            GQR = pfma(gr, rq1, GQR);
            GQI = pfma(gi, rq1, GQI);
        }
    }
    const float kfny = k2f * c.fny;
    return Far32Sums{AGR.x + AGR.y,
                     AGI.x + AGI.y,
                     -c.fny * (SHR.x + SHR.y),
                     -c.fny * (SHI.x + SHI.y),
                     -(NATR.x + NATR.y),
                     -(NATI.x + NATI.y),
                     (AER.x + AER.y) - kfny * (GQR.x + GQR.y),
                     (AEI.x + AEI.y) - kfny * (GQI.x + GQI.y)};
}

// Shared memory of one FP32 far tile (the persistent batched kernel overlays it with the near
// pairs' subdivision buffers).
struct Far32Smem {
    float shs[kFar32Rows];        // rows: complex-half scales (with A16)
    double sx[kFar32Rows][3];     // rows: collocation points
    float4 sxf[kFar32Rows];       // rows: collocation points in FP32 (margin test)
    float snx[kFar32Rows][3];     // rows: negated normals -n_x
    float4 sgf[kFarTile];         // column: level-0 centre in FP32, thr_hi
    float4 scf[2][kFarTile];      // column: matrix weights (cG, cH | cHt, cE)
    float4 sfa[kFarTile];         // column: e1 x, y, z, e2 x
    float2 sfb[kFarTile];         // column: e2 y, z
    double sred[kFarTile / 32][2];
    float4 sPDW[kFarPairs * kFarTile];  // (k |delta|^2, w J / 4 pi) of points 2p, 2p + 1 at [p * kFarTile + tid]
};

// One (128-column tile, 64-row block) of the FP32 far field; all 128 threads of the CTA call it.
template <bool kWithRhs, bool kSmemCols = true>
__device__ __forceinline__ void far32_tile(const float* __restrict__ qp32, const double* __restrict__ elem,
                                           int64_t n, int64_t ld, const double* __restrict__ coef, double k,
                                           double coord_bound, float2* __restrict__ A32, int64_t lda32,
                                           double2* __restrict__ far_part, int64_t n_tiles, int64_t tile,
                                           int64_t row0, unsigned* __restrict__ amax = nullptr,
                                           uint32_t* __restrict__ A16 = nullptr, int64_t lda16 = 0,
                                           const float* __restrict__ hscale = nullptr,
                                           int* __restrict__ hflag = nullptr, Far32Smem* smem = nullptr) {
    Far32Smem& S = *smem;
    auto& shs = S.shs;
    auto& sx = S.sx;
    auto& sxf = S.sxf;
    auto& snx = S.snx;
    auto& sgf = S.sgf;
    auto& scf = S.scf;
    auto& sfa = S.sfa;
    auto& sfb = S.sfb;
    auto& sred = S.sred;
    const int tid = threadIdx.x;
    const int64_t j = tile * kFarTile + tid;
    __syncthreads();  // a previous tile of a persistent CTA may still read the shared arrays
    for (int t = tid; t < kFar32Rows * 3; t += kFarTile) {
        const int r = t / 3, c = t % 3;
        const int64_t i = row0 + r;
        sx[r][c] = (i < n) ? E(ECX + c, i) : 0.0;
        snx[r][c] = (i < n) ? -static_cast<float>(E(ENX + c, i)) : 0.f;
    }
    for (int r = tid; r < kFar32Rows; r += kFarTile) {
        const int64_t i = row0 + r;
        sxf[r] = (i < n) ? make_float4(static_cast<float>(E(ECX, i)), static_cast<float>(E(ECY, i)),
                                       static_cast<float>(E(ECZ, i)), 0.f)
                         : make_float4(0.f, 0.f, 0.f, 0.f);
        if (A16) shs[r] = (i < n) ? hscale[i] : 1.f;
    }
    const float kf = static_cast<float>(k), k2f = kf * kf, invk = 1.f / kf;
    // The column's 13 points: in-plane coordinates in registers (points 2p, 2p + 1 in the lanes of
    // pair p, the 13th alone); k |delta|^2 and the weights in shared memory with kSmemCols, else in
    // registers.
    float2 PA[kFarPairs], PB[kFarPairs];
    constexpr int kR = kSmemCols ? 1 : kFarPairs;
    float4* sPDW = nullptr;  // (k |delta|^2, w J / 4 pi) of points 2p, 2p + 1 at [p * kFarTile + tid]
    if constexpr (kSmemCols) sPDW = S.sPDW;
    float4 PDW[kR];
    float la, lb, lpdk, lw;
    double cx = 0, cy = 0, cz = 0;
    float nyx = 0, nyy = 0, nyz = 0;
    const int64_t jj = j < n ? j : 0;
    // |t| = k |r_q - r_c| <= k |delta| for every point: a column with k max |delta| below 3 needs no
    // per-point range test of the special-function sine / cosine (decided per warp).
    float dmax2 = 0.f;
#pragma unroll
    for (int p = 0; p < kFarPairs; ++p) {
        const float* s0 = qp32 + (int64_t)(2 * p * kQ32) * ld + jj;
        const float* s1 = s0 + (int64_t)kQ32 * ld;
        PA[p] = make_float2(s0[0], s1[0]);
        PB[p] = make_float2(s0[ld], s1[ld]);
        dmax2 = fmaxf(dmax2, fmaxf(s0[2 * ld], s1[2 * ld]));
        const float4 v = make_float4(kf * s0[2 * ld], kf * s1[2 * ld], s0[3 * ld], s1[3 * ld]);
        if constexpr (kSmemCols) sPDW[p * kFarTile + tid] = v; else PDW[p] = v;
    }
    {
        const float* sl = qp32 + (int64_t)((kFarPoints - 1) * kQ32) * ld + jj;
        la = sl[0];
        lb = sl[ld];
        lpdk = kf * sl[2 * ld];
        lw = sl[3 * ld];
        dmax2 = sl[2 * ld];
        const float* fr = qp32 + (int64_t)kQ32Frame * ld + jj;
        sfa[tid] = make_float4(fr[0], fr[ld], fr[2 * ld], fr[3 * ld]);
        sfb[tid] = make_float2(fr[4 * ld], fr[5 * ld]);
    }
    if (j < n) {
        cx = E(ECX, j); cy = E(ECY, j); cz = E(ECZ, j);
        nyx = static_cast<float>(E(ENX, j));
        nyy = static_cast<float>(E(ENY, j));
        nyz = static_cast<float>(E(ENZ, j));
        sgf[tid] = make_float4(static_cast<float>(E(EGX, j)), static_cast<float>(E(EGY, j)),
                               static_cast<float>(E(EGZ, j)),
                               far32_col_threshold(near_threshold(E(EAREA, j)), coord_bound));
        float cw[8];
        for (int f = 0; f < 8; ++f) cw[f] = static_cast<float>(coef[(int64_t)(CF_CG + f) * ld + j]);
        scf[0][tid] = make_float4(cw[0], cw[1], cw[2], cw[3]);
        scf[1][tid] = make_float4(cw[4], cw[5], cw[6], cw[7]);
    } else {
        sgf[tid] = make_float4(0.f, 0.f, 0.f, INFINITY);
        scf[0][tid] = scf[1][tid] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const bool warp_fast = __all_sync(0xffffffffu, kf * kf * dmax2 < 9.f);
    __syncthreads();
    const int64_t rows_here = (n - row0 < kFar32Rows) ? (n - row0) : kFar32Rows;
    float vmax = 0.f;  // largest |re|, |im| this thread wrote (+inf for a non-finite part)
    int hbad = 0;      // a complex-half entry this thread wrote left the FP16 range
    for (int r = 0; r < rows_here; ++r) {
        const int64_t i = row0 + r;
        bool active = (j < n) && (j != i);
        // the rare pairs the margin test leaves open: the FP64 test on the column's global data
        if (active && !far_by_margin(sgf[tid], sxf[r]))
            active = !near_superset(E(EGX, j), E(EGY, j), E(EGZ, j), near_threshold(E(EAREA, j)), sx[r][0], sx[r][1],
                                    sx[r][2]);
        double2 rhs_c = make_double2(0.0, 0.0);
        if (active) {
            // FP64: centroid offset, distance and the reduced phase k r_c mod 2 pi.
            const double dcx = cx - sx[r][0], dcy = cy - sx[r][1], dcz = cz - sx[r][2];
            const double rc2 = dcx * dcx + dcy * dcy + dcz * dcz;
            const double rc = rc2 * sb_rsqrt1(rc2);
            const double ph = k * rc;
            // exp(i k r_c): k r_c = m pi / 64 + b with m the nearest integer (found by adding
            // 1.5 * 2^52, which leaves m in the low mantissa bits), |b| <= pi / 128 from an FP64 fma
            // (pi / 64 rounded to FP64: m times its error stays below 1e-13 for k r_c < 1e3), then
            // the table entry rotated by b's sine and cosine (Taylor to b^3 and b^4, truncation
            // below 1e-10); error about 1e-7 from the FP32 table.
            const double y = fma(ph, 0x1.45f306dc9c883p+4, 0x1.8p52);  // 64 / pi
            const double nq = y - 0x1.8p52;
            const int m = __double2loint(y) & (kPhaseTab - 1);
            const float b = static_cast<float>(fma(-nq, 0x1.921fb54442d18p-5, ph));  // pi / 64
            const float b2 = b * b;
            const float sb = fmaf(b * b2, -1.f / 6.f, b);
            const float cb = fmaf(b2, fmaf(b2, 1.f / 24.f, -0.5f), 1.f);
            const float2 tab = __ldg(&g_phase_tab[m]);
            const float cc = tab.x * cb - tab.y * sb, sc = tab.y * cb + tab.x * sb;
            const float fx = static_cast<float>(dcx), fy = static_cast<float>(dcy), fz = static_cast<float>(dcz);
            const float nnx = snx[r][0], nny = snx[r][1], nnz = snx[r][2];
            const float4 fa = sfa[tid];
            const float2 fb = sfb[tid];
            Far32Pair c;
            c.a2k = 2.f * kf * (fx * fa.x + fy * fa.y + fz * fa.z);
            c.b2k = 2.f * kf * (fx * fa.w + fy * fb.x + fz * fb.y);
            c.rc2 = static_cast<float>(rc2);
            c.rc = static_cast<float>(rc);
            c.ea = fa.x * nnx + fa.y * nny + fa.z * nnz;
            c.eb = fa.w * nnx + fb.x * nny + fb.y * nnz;
            c.fnx = fx * nnx + fy * nny + fz * nnz;
            c.fny = fx * nyx + fy * nyy + fz * nyz;
            c.nxny = -(nnx * nyx + nny * nyy + nnz * nyz);
            Far32Sums sm = warp_fast ? far32_pairs<false, kSmemCols>(c, PA, PB, sPDW, PDW, tid, kf, invk, k2f)
                                     : far32_pairs<true, kSmemCols>(c, PA, PB, sPDW, PDW, tid, kf, invk, k2f);
            if (warp_fast)
                far32_point<false>(sm, la, lb, lpdk, lw, c, kf, invk, k2f);
            else
                far32_point<true>(sm, la, lb, lpdk, lw, c, kf, invk, k2f);
            const float4 w0 = scf[0][tid], w1 = scf[1][tid];  // (cG, cH), (cHt, cE)
            const float ur = sm.gr * w0.x - sm.gi * w0.y + sm.hr * w0.z - sm.hi * w0.w + sm.tr * w1.x -
                             sm.ti * w1.y + sm.er * w1.z - sm.ei * w1.w;
            const float ui = sm.gr * w0.y + sm.gi * w0.x + sm.hr * w0.w + sm.hi * w0.z + sm.tr * w1.y +
                             sm.ti * w1.x + sm.er * w1.w + sm.ei * w1.z;
            // rotate by the pair phase exp(i k r_c) = (cc, sc)
            const float2 v = make_float2(ur * cc - ui * sc, ur * sc + ui * cc);
            A32[i * lda32 + j] = v;
            const float av = fmaxf(fabsf(v.x), fabsf(v.y));
            vmax = (av <= 3.4e38f) ? fmaxf(vmax, av) : INFINITY;
            if (A16) A16[i * lda16 + j] = half_pack(v, shs[r], &hbad);
            if (kWithRhs) {
                Acc a;
                a.gr = sm.gr * cc - sm.gi * sc; a.gi = sm.gr * sc + sm.gi * cc;
                a.hr = sm.hr * cc - sm.hi * sc; a.hi = sm.hr * sc + sm.hi * cc;
                a.tr = sm.tr * cc - sm.ti * sc; a.ti = sm.tr * sc + sm.ti * cc;
                a.er = sm.er * cc - sm.ei * sc; a.ei = sm.er * sc + sm.ei * cc;
                rhs_c = combine(a, coef, ld, j, CF_DG);
            }
        }
        if (kWithRhs) {
            double sxr = warp_sum(rhs_c.x), syr = warp_sum(rhs_c.y);
            if ((tid & 31) == 0) {
                sred[tid >> 5][0] = sxr;
                sred[tid >> 5][1] = syr;
            }
            __syncthreads();
            if (tid == 0) {
                double tx = 0, ty = 0;
                for (int w = 0; w < kFarTile / 32; ++w) {
                    tx += sred[w][0];
                    ty += sred[w][1];
                }
                far_part[i * n_tiles + tile] = make_double2(tx, ty);
            }
            __syncthreads();
        }
    }
    // The largest part written, for the scale of the complex-half copy (one atomic per warp
    // whose maximum exceeds the running one).
    if (amax) {
#pragma unroll
        for (int o = 16; o; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if ((tid & 31) == 0 && __float_as_uint(vmax) > *reinterpret_cast<volatile unsigned*>(amax))
            atomicMax(amax, __float_as_uint(vmax));
    }
    if (A16 && __any_sync(0xffffffffu, hbad) && (tid & 31) == 0) atomicOr(hflag, 1);
}

template <bool kWithRhs>
__global__ void __launch_bounds__(kFarTile, kFar32MinBlocks) k_far32(const float* __restrict__ qp32,
                                                    const double* __restrict__ elem, int64_t n,
                                                    int64_t ld, const double* __restrict__ coef,
                                                    double k, double coord_bound, float2* __restrict__ A32,
                                                    int64_t lda32, double2* __restrict__ far_part, int64_t n_tiles,
                                                    unsigned* __restrict__ amax, uint32_t* __restrict__ A16,
                                                    int64_t lda16, const float* __restrict__ hscale,
                                                    int* __restrict__ hflag) {
    __shared__ Far32Smem fs;
    far32_tile<kWithRhs, kFar32SmemCols>(qp32, elem, n, ld, coef, k, coord_bound, A32, lda32, far_part, n_tiles,
                                         blockIdx.x, blockIdx.y * (int64_t)kFar32Rows, amax, A16, lda16, hscale,
                                         hflag, &fs);
}

// Complex-half copy during the FP32 assembly (after the near and self kernels): each row's scale
// from its near and diagonal entries (the largest of a row on resolved meshes), then those
// entries' FP16 values; the far kernel converts the rest with the same scales. Thread per row.
__global__ void __launch_bounds__(256) k_near_row_scale(const float2* __restrict__ A32, int64_t lda32, int64_t n,
                                                        const int64_t* __restrict__ near_ptr,
                                                        const int32_t* __restrict__ near_col, float* __restrict__ s,
                                                        float* __restrict__ inv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float m = 0.f;
    for (int64_t p = near_ptr[i]; p <= near_ptr[i + 1]; ++p) {
        const int64_t j = p < near_ptr[i + 1] ? near_col[p] : i;
        const float2 v = A32[i * lda32 + j];
        const float av = fmaxf(fabsf(v.x), fabsf(v.y));
        m = (av <= 3.4e38f) ? fmaxf(m, av) : INFINITY;
    }
    const float sc = half_scale_for(m);
    s[i] = sc;
    inv[i] = 1.f / sc;
}
__global__ void __launch_bounds__(256) k_near_to_half(const float2* __restrict__ A32, int64_t lda32, int64_t n,
                                                      const int64_t* __restrict__ near_ptr,
                                                      const int32_t* __restrict__ near_col,
                                                      const float* __restrict__ s, uint32_t* __restrict__ A16,
                                                      int64_t lda16, int* __restrict__ hflag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float sc = s[i];
    int bad = 0;
    for (int64_t p = near_ptr[i]; p <= near_ptr[i + 1]; ++p) {
        const int64_t j = p < near_ptr[i + 1] ? near_col[p] : i;
        A16[i * lda16 + j] = half_pack(A32[i * lda32 + j], sc, &bad);
    }
    if (bad) atomicOr(hflag, 1);
}

// Largest |re|, |im| of the near-pair and diagonal entries of the complex64 matrix (the far
// kernel covers the rest), atomically maxed into *amax as float bits.
__global__ void __launch_bounds__(256) k_near_absmax(const float2* __restrict__ A32, int64_t lda32, int64_t n,
                                                     const int64_t* __restrict__ near_ptr,
                                                     const int32_t* __restrict__ near_col, unsigned* __restrict__ amax) {
    float m = 0.f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        for (int64_t p = near_ptr[i]; p <= near_ptr[i + 1]; ++p) {
            const int64_t j = p < near_ptr[i + 1] ? near_col[p] : i;
            const float2 v = A32[i * lda32 + j];
            const float av = fmaxf(fabsf(v.x), fabsf(v.y));
            m = (av <= 3.4e38f) ? fmaxf(m, av) : INFINITY;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(amax, __float_as_uint(m));
}

// ---------------------------------------------------------------------------------------------
// Near kernel: one warp per near pair, exact replay of generate_subelements + regular leaves.
// ---------------------------------------------------------------------------------------------
constexpr int kNearWarps = 4;
constexpr int kMaxNse = 60;
constexpr int kMaxLeaves = 110;

struct NearWarpSmem {
    double xs[2][kMaxNse][3];
    double es[2][kMaxNse][3];
    double lv[kMaxNse][6];   // kept leaves of the current level: local vertices
    int lorder[kMaxNse];
    int loff[kMaxNse + 1];
};

// compute_gauss_order (singular.rs:1543-1573).
__device__ __forceinline__ int gauss_order(double disfac) {
    for (int o = 4; o <= 7; ++o) {
        const double b = disfac / (2.0 * o + 1.0);
        double p = 1.0;
        for (int t = 0; t < 2 * o + 1; ++t) p *= b;
        const double eg = p, eh = p * b, ee = p * b * b;
        if (eg < 0.0005 && eh < 0.0005 && ee < 0.0005) return o;
    }
    return 7;
}

// Adds one quadrature point's (G, H, H^T, E) to NB basis-weighted channel sums (weights nb[b]).
template <int NB>
__device__ __forceinline__ void point_channels_w(Acc* a, const double* nb, double dx, double dy, double dz,
                                                 double r, double rinv, double wga, double nyx, double nyy,
                                                 double nyz, double nxx, double nxy, double nxz, double k,
                                                 double k2) {
    double s, c;
    sb_sincos(k * r, &s, &c);
    const double gs = wga * kInv4Pi * rinv;
    const double g_r = c * gs, g_i = s * gs;
    const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
    const double rny = ux * nyx + uy * nyy + uz * nyz;
    const double rnx = -(ux * nxx + uy * nxy + uz * nxz);
    const double b_r = -g_r * rinv - g_i * k;
    const double b_i = g_r * k - g_i * rinv;
    const double rq = rny * rnx;
    const double nxny = nxx * nyx + nxy * nyy + nxz * nyz;
    const double ri2 = rinv * rinv;
    const double f_r = (3.0 * ri2 - k2) * rq + nxny * ri2;
    const double f_i = -k * rinv * (3.0 * rq + nxny);
    const double e_r = g_r * f_r - g_i * f_i, e_i = g_r * f_i + g_i * f_r;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const double w = nb[b];
        a[b].gr = fma(g_r, w, a[b].gr);
        a[b].gi = fma(g_i, w, a[b].gi);
        a[b].hr = fma(b_r * rny, w, a[b].hr);
        a[b].hi = fma(b_i * rny, w, a[b].hi);
        a[b].tr = fma(b_r * rnx, w, a[b].tr);
        a[b].ti = fma(b_i * rnx, w, a[b].ti);
        a[b].er = fma(e_r, w, a[b].er);
        a[b].ei = fma(e_i, w, a[b].ei);
    }
}

// Discontinuous Tri3 panel bases (basis_values, crates/sonium-bem/src/core/mesh/element.rs:
// 229-262): NB = 3 the linear basis 2 lambda_b - 1/3, NB = 6 the quadratic one (vertex functions
// lambda (2 lambda - 1), then 4 lambda0 lambda1, 4 lambda1 lambda2, 4 lambda2 lambda0).
template <int NB>
__device__ __forceinline__ void panel_basis(double s, double t, double* nb) {
    const double l0 = 1.0 - s - t;
    if constexpr (NB == 3) {
        nb[0] = 2.0 * l0 - 1.0 / 3.0;
        nb[1] = 2.0 * s - 1.0 / 3.0;
        nb[2] = 2.0 * t - 1.0 / 3.0;
    } else {
        nb[0] = l0 * (2.0 * l0 - 1.0);
        nb[1] = s * (2.0 * s - 1.0);
        nb[2] = t * (2.0 * t - 1.0);
        nb[3] = 4.0 * l0 * s;
        nb[4] = 4.0 * s * t;
        nb[5] = 4.0 * t * l0;
    }
}

// Reference-coordinate derivatives (d/ds, d/dt) of the panel basis (panel_basis_gradients,
// integration/singular.rs:1180-1195).
template <int NB>
__device__ __forceinline__ void panel_basis_deriv(double s, double t, double (*d)[2]) {
    if constexpr (NB == 3) {
        d[0][0] = -2.0; d[0][1] = -2.0;
        d[1][0] = 2.0; d[1][1] = 0.0;
        d[2][0] = 0.0; d[2][1] = 2.0;
    } else {
        const double l = 1.0 - s - t;
        d[0][0] = 1.0 - 4.0 * l; d[0][1] = 1.0 - 4.0 * l;
        d[1][0] = 4.0 * s - 1.0; d[1][1] = 0.0;
        d[2][0] = 0.0; d[2][1] = 4.0 * t - 1.0;
        d[3][0] = 4.0 * (l - s); d[3][1] = -4.0 * s;
        d[4][0] = 4.0 * t; d[4][1] = 4.0 * s;
        d[5][0] = -4.0 * t; d[5][1] = 4.0 * (l - t);
    }
}

// One kept leaf of a near pair's subdivision: its vertices in the field element's reference
// coordinates (s, t of each of the three), its Gauss order, and the leaves its subdivision level
// kept (low 16 bits; bit 16 set at level 0, the element itself), the same in every leaf of a level.
struct NearLeaf {
    double lv[6];
    int order, group;
};

// The points of the kept leaves of one subdivision level (lvs / lorder, keep of them) into the
// lane-partial sums: lane 0 lays out the leaves' point offsets, the lanes stride over the points.
// iforie: the level-0 leaf, the element itself (its reference coordinates are the points').
template <int NB>
__device__ __forceinline__ void near_eval_kept(Acc* a, const double (*lvs)[6], const int* lorder, int* loff,
                                               int keep, bool iforie,
                                               const double (&V)[3][3], double x0, double x1, double x2,
                                               double nxx, double nxy, double nxz, double nyx, double nyy,
                                               double nyz, double jac, double k, double k2, int lane) {
    // Point offsets of the kept leaves (serial scan by lane 0: at most 60 leaves).
    if (lane == 0) {
        int o = 0;
        for (int l = 0; l < keep; ++l) {
            loff[l] = o;
            o += c_tri_cnt[lorder[l] - 4];
        }
        loff[keep] = o;
    }
    __syncwarp();
    const int npts = loff[keep];
    for (int f = lane; f < npts; f += 32) {
        int lo = 0, hi = keep - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (loff[mid] <= f) lo = mid; else hi = mid - 1;
        }
        const int l = lo;
        const int q = f - loff[l];
        const int ti = c_tri_off[lorder[l] - 4] + q;
        const double xi = c_tri_xi[ti], et = c_tri_eta[ti], wq = c_tri_w[ti];
        double xio, eto, weih2;
        if (iforie) {
            xio = xi;
            eto = et;
            weih2 = wq;
        } else {
            const double* lv = lvs[l];
            const double lam = 1.0 - xi - et;
            xio = lv[0] * lam + lv[2] * xi + lv[4] * et;
            eto = lv[1] * lam + lv[3] * xi + lv[5] * et;
            const double det = fabs((lv[2] - lv[0]) * (lv[5] - lv[1]) - (lv[4] - lv[0]) * (lv[3] - lv[1]));
            weih2 = wq * det;
        }
        const double sf0 = 1.0 - xio - eto;
        const double px = sf0 * V[0][0] + xio * V[1][0] + eto * V[2][0];
        const double py = sf0 * V[0][1] + xio * V[1][1] + eto * V[2][1];
        const double pz = sf0 * V[0][2] + xio * V[1][2] + eto * V[2][2];
        const double dx = px - x0, dy = py - x1, dz = pz - x2;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 >= 1e-30)) continue;  // dis < 1e-15 (normalize, element.rs:304-311)
        const double rinv = sb_rsqrt2(d2);
        const double dis = d2 * rinv;
        if constexpr (NB == 1) {
            point_channels(a[0], dx, dy, dz, dis, rinv, weih2 * jac, nyx, nyy, nyz, nxx, nxy, nxz, k, k2);
        } else {
            double nb[NB];
            panel_basis<NB>(xio, eto, nb);
            point_channels_w<NB>(a, nb, dx, dy, dz, dis, rinv, weih2 * jac, nyx, nyy, nyz, nxx, nxy, nxz, k,
                                 k2);
        }
    }
}

// Evaluates the regular-integration channels of field element j seen from the point x with
// normal nx into lane-partial sums: NB = 1 the constant basis, NB = 3 / 6 the discontinuous
// linear / quadratic basis weights.
// kMode 0 evaluates as it subdivides; kMode 1 only counts the kept leaves (returned by lane 0's
// call, the others return the same); kMode 2 writes them, level by level, to plan[0 .. count).
template <int NB, int kMode = 0>
__device__ int near_channels_at(Acc* a, NearWarpSmem& S, const double* __restrict__ elem, int64_t ld,
                                double x0, double x1, double x2, double nxx, double nxy, double nxz,
                                int64_t j, double k, double k2, int lane, NearLeaf* __restrict__ plan = nullptr) {
    double V[3][3];
    for (int t = 0; t < 3; ++t)
        for (int c = 0; c < 3; ++c) V[t][c] = E(EV0X + 3 * t + c, j);
    const double nyx = E(ENX, j), nyy = E(ENY, j), nyz = E(ENZ, j);
    const double area = E(EAREA, j), jac = E(EJAC, j);

    if (lane == 0) {
        S.xs[0][0][0] = 0.0; S.xs[0][0][1] = 1.0; S.xs[0][0][2] = 0.0;
        S.es[0][0][0] = 0.0; S.es[0][0][1] = 0.0; S.es[0][0][2] = 1.0;
    }
    __syncwarp();
    int cur = 0, nsel = 1, total = 0;
    double faclin = 2.0;
    const unsigned lt = (1u << lane) - 1u;
    for (int level = 0; level < 64; ++level) {
        faclin *= 0.5;
        const double arels = __dmul_rn(__dmul_rn(area, faclin), faclin);
        const double sqa = __dsqrt_rn(arels);
        bool sub[2] = {false, false};
        double rat[2] = {0.0, 0.0};
        for (int h = 0; h < 2; ++h) {
            const int s = lane + 32 * h;
            if (s < nsel) {
                const double* xp = S.xs[cur][s];
                const double* ep = S.es[cur][s];
                const double sc = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(0.0, xp[0]), xp[1]), xp[2]), 3.0);
                const double tc = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(0.0, ep[0]), ep[1]), ep[2]), 3.0);
                const double sf0 = __dsub_rn(__dsub_rn(1.0, sc), tc);
                double g[3];
                for (int c = 0; c < 3; ++c) {
                    double v = __dadd_rn(0.0, __dmul_rn(sf0, V[0][c]));
                    v = __dadd_rn(v, __dmul_rn(sc, V[1][c]));
                    v = __dadd_rn(v, __dmul_rn(tc, V[2][c]));
                    g[c] = v;
                }
                const double dx = __dsub_rn(g[0], x0), dy = __dsub_rn(g[1], x1), dz = __dsub_rn(g[2], x2);
                const double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                rat[h] = __ddiv_rn(dist, sqa);
                sub[h] = rat[h] < 3.0;
            }
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, sub[0]);
        const unsigned m1 = __ballot_sync(0xffffffffu, sub[1]);
        const int nsub = __popc(m0) + __popc(m1);
        // Position of the 16th subdivision, which ends the level (singular.rs:1432-1436).
        int breakpos = nsel;
        if (nsub >= 16) {
            if (__popc(m0) >= 16) {
                unsigned m = m0;
                for (int t = 0; t < 15; ++t) m &= m - 1;
                breakpos = __ffs(m) - 1;
            } else {
                unsigned m = m1;
                for (int t = 0; t < 15 - __popc(m0); ++t) m &= m - 1;
                breakpos = 32 + __ffs(m) - 1;
            }
        }
        const unsigned valid0 = breakpos >= 32 ? 0xffffffffu : ((1u << breakpos) - 1u);
        const unsigned valid1 = breakpos >= 64 ? 0xffffffffu : (breakpos <= 32 ? 0u : ((1u << (breakpos - 32)) - 1u));
        const unsigned nsel0 = nsel >= 32 ? 0xffffffffu : ((1u << nsel) - 1u);
        const unsigned nsel1 = nsel >= 64 ? 0xffffffffu : (nsel <= 32 ? 0u : ((1u << (nsel - 32)) - 1u));
        const unsigned l0 = ~m0 & valid0 & nsel0;
        const unsigned l1 = ~m1 & valid1 & nsel1;
        const int nleaf = __popc(l0) + __popc(l1);
        const int keep = min(nleaf, kMaxLeaves - total);
        const int nxt = cur ^ 1;
        // Kept leaves and children of this level.
        for (int h = 0; h < 2; ++h) {
            const int s = lane + 32 * h;
            if (s >= nsel) continue;
            const unsigned lm = h == 0 ? l0 : l1;
            if (lm & (1u << lane)) {
                const int rank = (h == 0) ? __popc(l0 & lt) : __popc(l0) + __popc(l1 & lt);
                if (rank < keep) {
                    for (int t = 0; t < 3; ++t) {
                        S.lv[rank][2 * t] = S.xs[cur][s][t];
                        S.lv[rank][2 * t + 1] = S.es[cur][s][t];
                    }
                    S.lorder[rank] = gauss_order(0.5 / rat[h]);
                }
            }
            const unsigned sm = h == 0 ? m0 : m1;
            if (sm & (1u << lane)) {
                const int rank = (h == 0) ? __popc(m0 & lt) : __popc(m0) + __popc(m1 & lt);
                if (rank < 15) {
                    const double* xp = S.xs[cur][s];
                    const double* ep = S.es[cur][s];
                    double xm[6], em[6];
                    for (int t = 0; t < 3; ++t) {
                        const int t1 = (t + 1) % 3;
                        xm[t] = xp[t];
                        xm[t + 3] = (xp[t] + xp[t1]) / 2.0;
                        em[t] = ep[t];
                        em[t + 3] = (ep[t] + ep[t1]) / 2.0;
                    }
                    const int b = 4 * rank;
                    for (int t = 0; t < 3; ++t) {
                        const int t2 = (t == 0) ? 5 : t + 2;
                        S.xs[nxt][b + t][0] = xm[t];
                        S.xs[nxt][b + t][1] = xm[t + 3];
                        S.xs[nxt][b + t][2] = xm[t2];
                        S.es[nxt][b + t][0] = em[t];
                        S.es[nxt][b + t][1] = em[t + 3];
                        S.es[nxt][b + t][2] = em[t2];
                    }
                    S.xs[nxt][b + 3][0] = xm[3];
                    S.xs[nxt][b + 3][1] = xm[4];
                    S.xs[nxt][b + 3][2] = xm[5];
                    S.es[nxt][b + 3][0] = em[3];
                    S.es[nxt][b + 3][1] = em[4];
                    S.es[nxt][b + 3][2] = em[5];
                }
            }
        }
        __syncwarp();
        if constexpr (kMode == 0) {
            near_eval_kept<NB>(a, S.lv, S.lorder, S.loff, keep, fabs(fabs(faclin) - 1.0) < 1e-10, V, x0, x1, x2, nxx,
                               nxy, nxz, nyx, nyy, nyz, jac, k, k2, lane);
        } else if constexpr (kMode == 2) {
            for (int l = lane; l < keep; l += 32) {
                NearLeaf& o = plan[total + l];
                for (int t = 0; t < 6; ++t) o.lv[t] = S.lv[l][t];
                o.order = S.lorder[l];
                o.group = keep | (level == 0 ? 1 << 16 : 0);
            }
        }
        total += keep;
        __syncwarp();
        if (total >= kMaxLeaves || nsub == 0) break;
        nsel = min(nsub, 15) * 4;
        cur = nxt;
    }
    return total;
}

// The constant basis: pair (i, j) seen from the centroid of element i.
__device__ __forceinline__ void near_pair_channels(Acc& a, NearWarpSmem& S, const double* __restrict__ elem,
                                                   int64_t ld, int64_t i, int64_t j, double k, double k2,
                                                   int lane) {
    near_channels_at<1>(&a, S, elem, ld, E(ECX, i), E(ECY, i), E(ECZ, i), E(ENX, i), E(ENY, i), E(ENZ, i), j, k,
                        k2, lane);
}

__device__ __forceinline__ Acc warp_reduce(const Acc& a) {
    Acc r;
    r.gr = warp_sum(a.gr); r.gi = warp_sum(a.gi);
    r.hr = warp_sum(a.hr); r.hi = warp_sum(a.hi);
    r.tr = warp_sum(a.tr); r.ti = warp_sum(a.ti);
    r.er = warp_sum(a.er); r.ei = warp_sum(a.ei);
    return r;
}

// 5 resident CTAs (20 warps) per SM: 96 registers; more warps hide the FP64 latency of the
// subdivision replay (N = 20480: 2.88 -> 2.56 ms; 6 CTAs 2.83 ms). The grid holds what is
// resident and each warp strides over the pairs, so that the uneven trees (52 to over 400
// points per pair) do not leave CTAs held by one slow warp.
constexpr int kNearMinBlocks = 5;
__global__ void __launch_bounds__(32 * kNearWarps, kNearMinBlocks) k_near(const double* __restrict__ elem,
                                                          int64_t n, int64_t ld,
                                                          const int32_t* __restrict__ rows,
                                                          const int32_t* __restrict__ cols,
                                                          int64_t nnz,
                                                          const double* __restrict__ coef,
                                                          double k, double2* __restrict__ A64,
                                                          float2* __restrict__ A32, int64_t lda32,
                                                          double2* __restrict__ near_rhs) {
    __shared__ NearWarpSmem smem[kNearWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kNearWarps;
    for (int64_t p = blockIdx.x * (int64_t)kNearWarps + warp; p < nnz; p += stride) {
        const int64_t i = rows[p], j = cols[p];
        Acc a;
        near_pair_channels(a, smem[warp], elem, ld, i, j, k, k * k, lane);
        const Acc t = warp_reduce(a);
        if (lane == 0) {
            const double2 v = combine(t, coef, ld, j, CF_CG);
            if (A64) A64[i * n + j] = v;
            if (A32) A32[i * lda32 + j] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
            if (near_rhs) near_rhs[p] = combine(t, coef, ld, j, CF_DG);
        }
        __syncwarp();  // the warp's shared replay state is reused by its next pair
    }
}

// The near pairs' subdivision plan of a mesh. Which leaves a pair keeps depends on the geometry
// alone (the collocation point, the field element), not on the wave number, so a mesh records them
// once and later assemblies evaluate the recorded leaves (k_near_cached) instead of repeating the
// subdivision tests. kPass 0 counts each pair's kept leaves into counts[p]; kPass 1 writes them,
// level by level in the order k_near keeps them, to plan[off[p] .. off[p + 1]).
template <int kPass>
__global__ void __launch_bounds__(32 * kNearWarps, kNearMinBlocks) k_near_plan(
    const double* __restrict__ elem, int64_t n, int64_t ld, const int32_t* __restrict__ rows,
    const int32_t* __restrict__ cols, int64_t nnz, int64_t* __restrict__ counts, const int64_t* __restrict__ off,
    NearLeaf* __restrict__ plan) {
    __shared__ NearWarpSmem smem[kNearWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kNearWarps;
    for (int64_t p = blockIdx.x * (int64_t)kNearWarps + warp; p < nnz; p += stride) {
        const int64_t i = rows[p], j = cols[p];
        if constexpr (kPass == 0) {
            const int t = near_channels_at<1, 1>(nullptr, smem[warp], elem, ld, E(ECX, i), E(ECY, i), E(ECZ, i),
                                                 E(ENX, i), E(ENY, i), E(ENZ, i), j, 0.0, 0.0, lane);
            if (lane == 0) counts[p] = t;
        } else {
            near_channels_at<1, 2>(nullptr, smem[warp], elem, ld, E(ECX, i), E(ECY, i), E(ECZ, i), E(ENX, i),
                                   E(ENY, i), E(ENZ, i), j, 0.0, 0.0, lane, plan + off[p]);
        }
        __syncwarp();
    }
}

// Shared memory of one warp of k_near_cached: a pair's whole recorded leaf list and the point
// offsets of the level being evaluated.
struct NearPlanSmem {
    double lv[kMaxLeaves][6];
    int lorder[kMaxLeaves];
    int group[kMaxLeaves];
    int loff[kMaxNse + 1];
};
static_assert(sizeof(NearLeaf) == 7 * sizeof(double), "a leaf is seven 8-byte words");

// k_near from a recorded plan: the same leaves, levels and per-lane point order as the
// subdividing kernel, so the same sums bit for bit. The warp reads the pair's leaves into shared
// memory in one coalesced pass, then evaluates them level by level.
__global__ void __launch_bounds__(32 * kNearWarps, kNearMinBlocks) k_near_cached(
    const double* __restrict__ elem, int64_t n, int64_t ld, const int32_t* __restrict__ rows,
    const int32_t* __restrict__ cols, int64_t nnz, const int64_t* __restrict__ off,
    const NearLeaf* __restrict__ plan, const double* __restrict__ coef, double k, double2* __restrict__ A64,
    float2* __restrict__ A32, int64_t lda32, double2* __restrict__ near_rhs) {
    __shared__ NearPlanSmem smem[kNearWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    NearPlanSmem& S = smem[warp];
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kNearWarps;
    const double k2 = k * k;
    const uint64_t* __restrict__ words = reinterpret_cast<const uint64_t*>(plan);
    for (int64_t p = blockIdx.x * (int64_t)kNearWarps + warp; p < nnz; p += stride) {
        const int64_t i = rows[p], j = cols[p];
        const int64_t o0 = off[p];
        const int64_t cnt64 = off[p + 1] - o0;
        const int cnt = static_cast<int>(cnt64 < kMaxLeaves ? cnt64 : kMaxLeaves);
        for (int w = lane; w < 7 * cnt; w += 32) {
            const int l = w / 7, c = w - 7 * l;
            const uint64_t v = __ldg(words + (o0 + l) * 7 + c);
            if (c < 6) {
                S.lv[l][c] = __longlong_as_double(static_cast<long long>(v));
            } else {
                S.lorder[l] = static_cast<int>(static_cast<uint32_t>(v));
                S.group[l] = static_cast<int>(static_cast<uint32_t>(v >> 32));
            }
        }
        double V[3][3];
        for (int t = 0; t < 3; ++t)
            for (int c = 0; c < 3; ++c) V[t][c] = E(EV0X + 3 * t + c, j);
        const double nyx = E(ENX, j), nyy = E(ENY, j), nyz = E(ENZ, j), jac = E(EJAC, j);
        const double x0 = E(ECX, i), x1 = E(ECY, i), x2 = E(ECZ, i);
        const double nxx = E(ENX, i), nxy = E(ENY, i), nxz = E(ENZ, i);
        Acc a;
        __syncwarp();
        for (int g = 0; g < cnt;) {
            const int grp = S.group[g];
            // a level keeps 1 to kMaxNse leaves; the bounds only guard the loop against a bad plan
            const int room = cnt - g < kMaxNse ? cnt - g : kMaxNse;
            const int keep = (grp & 0xffff) < room ? (grp & 0xffff) : room;
            if (keep <= 0) break;
            near_eval_kept<1>(&a, S.lv + g, S.lorder + g, S.loff, keep, (grp >> 16) != 0, V, x0, x1, x2, nxx, nxy,
                              nxz, nyx, nyy, nyz, jac, k, k2, lane);
            __syncwarp();  // the level's offsets are read before the next level replaces them
            g += keep;
        }
        const Acc t = warp_reduce(a);
        if (lane == 0) {
            const double2 v = combine(t, coef, ld, j, CF_CG);
            if (A64) A64[i * n + j] = v;
            if (A32) A32[i * lda32 + j] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
            if (near_rhs) near_rhs[p] = combine(t, coef, ld, j, CF_DG);
        }
        __syncwarp();  // the pair's leaves are read before the next pair's replace them
    }
}

// Grid of k_near for nnz pairs: what is resident (kNearMinBlocks CTAs per SM), or fewer.
static unsigned near_grid(int64_t nnz, int device) {
    const int64_t need = (nnz + kNearWarps - 1) / kNearWarps;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(kNearMinBlocks) *
                                                                                  device_sm_count(device))));
}

// ---------------------------------------------------------------------------------------------
// Self kernel: one warp per element (singular_integration_with_params_mode, singular.rs:297-614).
// ---------------------------------------------------------------------------------------------
// Channel sums of the self pair of element i, partial per lane (reduce with warp_reduce).
__device__ __forceinline__ void self_channels(Acc& a, const double* __restrict__ elem, int64_t ld, int64_t i,
                                              double k, int lane) {
    const double k2 = k * k;
    const double x0 = E(ECX, i), x1 = E(ECY, i), x2 = E(ECZ, i);
    const double nxx = E(ENX, i), nxy = E(ENY, i), nxz = E(ENZ, i);
    const double nyx = nxx, nyy = nxy, nyz = nxz;
    const double jac = E(EJAC, i);
    double V[3][3];
    for (int t = 0; t < 3; ++t)
        for (int c = 0; c < 3; ++c) V[t][c] = E(EV0X + 3 * t + c, i);
    // QuadratureParams::for_ka with estimate_element_size = max(sqrt(area), 1e-10).
    const double ka = k * fmax(sqrt(E(EAREA, i)), 1e-10);
    int ngpo1, nsub, nsec1, nsec2;
    if (ka < 0.3) { ngpo1 = 3; nsub = 4; nsec1 = 4; nsec2 = 2; }
    else if (ka < 1.0) { ngpo1 = 4; nsub = 5; nsec1 = 6; nsec2 = 2; }
    else if (ka < 2.0) { ngpo1 = 5; nsub = 6; nsec1 = 8; nsec2 = 3; }
    else { ngpo1 = 6; nsub = 7; nsec1 = 10; nsec2 = 4; }
    const int ego = ngpo1 * (ngpo1 - 1) / 2, sgo = nsub * (nsub - 1) / 2;
    const int n_edge = nsec1 * ngpo1, n_bulk = nsec2 * nsub * nsub;
    const int per_edge = n_edge + n_bulk;
    const double csi6[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    const double eta6[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
    double edge_r = 0.0, edge_i = 0.0;
    for (int f = lane; f < 3 * per_edge; f += 32) {
        const int ieg = f / per_edge, rem = f % per_edge;
        const int ig1 = (ieg + 1) % 3, ig2 = ieg + 3;
        if (rem < n_edge) {
            // Regularised hypersingular edge term: ((grad G x t) . n_x) w.
            const int isec = rem / ngpo1, ig = rem % ngpo1;
            double dp[3], leneg = 0.0;
            for (int c = 0; c < 3; ++c) {
                dp[c] = V[ig1][c] - V[ieg][c];
                leneg += dp[c] * dp[c];
            }
            leneg = sqrt(leneg);
            const double to0 = dp[0] / leneg, to1 = dp[1] / leneg, to2 = dp[2] / leneg;
            const double leneg_scaled = leneg / (2.0 * nsec1);
            const double delsec = 2.0 / nsec1;
            double secmid = -1.0 - delsec / 2.0;
            for (int s = 0; s <= isec; ++s) secmid += delsec;
            const double sga = secmid + c_gl_x[ego + ig] / nsec1;
            const double wga = c_gl_w[ego + ig] * leneg_scaled;
            const double dx = V[ieg][0] + dp[0] * (sga + 1.0) / 2.0 - x0;
            const double dy = V[ieg][1] + dp[1] * (sga + 1.0) / 2.0 - x1;
            const double dz = V[ieg][2] + dp[2] * (sga + 1.0) / 2.0 - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            double s, c;
            sb_sincos(k * dis, &s, &c);
            const double g_r = c * kInv4Pi * rinv, g_i = s * kInv4Pi * rinv;
            const double f_r = -g_r * rinv - g_i * k, f_i = g_r * k - g_i * rinv;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            // (u x t) . n_x
            const double cr = (uy * to2 - uz * to1) * nxx + (uz * to0 - ux * to2) * nxy +
                              (ux * to1 - uy * to0) * nxz;
            edge_r += f_r * cr * wga;
            edge_i += f_i * cr * wga;
        } else {
            // Duffy sub-triangle (centroid, vertex, edge midpoint) with an nsub x nsub GL rule.
            const int r2 = rem - n_edge;
            const int isec = r2 / (nsub * nsub), ab = r2 % (nsub * nsub);
            const int ia = ab / nsub, ib = ab % nsub;
            const double aresub = 1.0 / 24.0 / nsec2;
            double ss[3], ts[3];
            ss[0] = ts[0] = 1.0 / 3.0;
            if (isec == 0) {
                ss[1] = csi6[ieg]; ss[2] = csi6[ig2]; ts[1] = eta6[ieg]; ts[2] = eta6[ig2];
            } else {
                ss[1] = csi6[ig2]; ss[2] = csi6[ig1]; ts[1] = eta6[ig2]; ts[2] = eta6[ig1];
            }
            const double sga = c_gl_x[sgo + ia], tga = c_gl_x[sgo + ib];
            const double wei = c_gl_w[sgo + ia] * c_gl_w[sgo + ib];
            const double sgg = 0.5 * (1.0 - sga) * ss[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
            const double tgg = 0.5 * (1.0 - sga) * ts[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
            const double sf0 = 1.0 - sgg - tgg;
            const double dx = sf0 * V[0][0] + sgg * V[1][0] + tgg * V[2][0] - x0;
            const double dy = sf0 * V[0][1] + sgg * V[1][1] + tgg * V[2][1] - x1;
            const double dz = sf0 * V[0][2] + sgg * V[1][2] + tgg * V[2][2] - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            const double wga = wei * (1.0 + sga) * aresub * jac;
            double s, c;
            sb_sincos(k * dis, &s, &c);
            const double gs = wga * kInv4Pi * rinv;
            const double g_r = c * gs, g_i = s * gs;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            const double rny = ux * nyx + uy * nyy + uz * nyz;
            const double rnx = -(ux * nxx + uy * nxy + uz * nxz);
            const double b_r = -g_r * rinv - g_i * k, b_i = g_r * k - g_i * rinv;
            a.gr += g_r; a.gi += g_i;
            a.hr += b_r * rny; a.hi += b_i * rny;
            a.tr += b_r * rnx; a.ti += b_i * rnx;
            const double nd = nxx * nyx + nxy * nyy + nxz * nyz;
            a.er += g_r * k2 * nd;
            a.ei += g_i * k2 * nd;
        }
    }
    a.er += edge_r;
    a.ei += edge_i;
}

__device__ __forceinline__ void self_store(const Acc& t, const double* __restrict__ coef, int64_t ld, int64_t n,
                                           int64_t i, double2* __restrict__ A64, float2* __restrict__ A32,
                                           int64_t lda32, double2* __restrict__ self_rhs,
                                           double2* __restrict__ diag) {
    double2 v = combine(t, coef, ld, i, CF_CG);
    v.x += coef[(int64_t)(CF_DIAG) * ld + i];
    v.y += coef[(int64_t)(CF_DIAG + 1) * ld + i];
    if (A64) A64[i * n + i] = v;
    if (A32) A32[i * lda32 + i] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    diag[i] = v;
    double2 r = make_double2(coef[(int64_t)(CF_RHS) * ld + i], coef[(int64_t)(CF_RHS + 1) * ld + i]);
    if (self_rhs) {
        const double2 c = combine(t, coef, ld, i, CF_DG);
        r.x += c.x;
        r.y += c.y;
        self_rhs[i] = r;
    }
}

__global__ void __launch_bounds__(128) k_self(const double* __restrict__ elem, int64_t n,
                                              int64_t ld, const double* __restrict__ coef,
                                              double k, double2* __restrict__ A64,
                                              float2* __restrict__ A32, int64_t lda32,
                                              double2* __restrict__ self_rhs,
                                              double2* __restrict__ diag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + warp;
    if (i >= n) return;
    Acc a;
    self_channels(a, elem, ld, i, k, lane);
    const Acc t = warp_reduce(a);
    if (lane == 0) self_store(t, coef, ld, n, i, A64, A32, lda32, self_rhs, diag);
}

// =============================================================================================
// Discontinuous Tri3 bases (build_tbem_system_linear, crates/sonium-bem/src/core/assembly/
// tbem.rs:1490-1620; build_tbem_system_discontinuous_stabilized, :2810-2990): element e carries
// NB DOFs (3 linear, 6 quadratic), DOF NB e + c collocated at local point c of the basis's
// interior points (mesh/element.rs:91-123) with the element's flat normal; the row of that DOF
// holds, for every field element j, the NB basis-weighted integrals in columns NB j + b. FP64
// throughout (complex128 matrix).
// =============================================================================================
__constant__ double c_lin_coll[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
__constant__ double c_quad_coll[6][2] = {{0.0915762135097715, 0.0915762135097715},
                                         {0.8168475729804585, 0.0915762135097715},
                                         {0.0915762135097715, 0.8168475729804585},
                                         {0.445948490915965, 0.445948490915965},
                                         {0.445948490915965, 0.108103018168070},
                                         {0.108103018168070, 0.445948490915965}};
constexpr int kLinRows = 32;

template <int NB>
__device__ __forceinline__ void coll_local(int q, double& s, double& t) {
    if constexpr (NB == 3) {
        s = c_lin_coll[q][0];
        t = c_lin_coll[q][1];
    } else {
        s = c_quad_coll[q][0];
        t = c_quad_coll[q][1];
    }
}

// Collocation points of the NB n rows (local_to_global, element.rs:65-76) and their (flat
// element) normals, SoA: cp[c * n3 + r], cn[c * n3 + r].
template <int NB>
__global__ void k_lin_points(const double* __restrict__ elem, int64_t n, int64_t ld, double* __restrict__ cp,
                             double* __restrict__ cn) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n3 = NB * n;
    if (r >= n3) return;
    const int64_t e = r / NB;
    const int q = static_cast<int>(r % NB);
    double s, t;
    coll_local<NB>(q, s, t);
    const double sf[3] = {1.0 - s - t, s, t};
    for (int c = 0; c < 3; ++c) {
        double v = 0.0;
        for (int a = 0; a < 3; ++a) v += sf[a] * E(EV0X + 3 * a + c, e);
        cp[c * n3 + r] = v;
        cn[c * n3 + r] = E(ENX + c, e);
    }
}

// Incident plane-wave right-hand side at arbitrary collocation points (IncidentField::
// compute_rhs_with_beta, incident.rs:807-833): points / normals SoA with stride `st`.
__global__ void k_plane_wave_at(const double* __restrict__ pts, const double* __restrict__ nrm, int64_t np,
                                int64_t st, const double* __restrict__ dirs, const double2* __restrict__ amps,
                                int64_t r, double k, double hf, double tau, double2 beta,
                                double2* __restrict__ rhs) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= np * r) return;
    const int64_t i = t / r, q = t % r;
    const double d0 = dirs[3 * q], d1 = dirs[3 * q + 1], d2 = dirs[3 * q + 2];
    const double2 A = amps ? amps[q] : make_double2(1.0, 0.0);
    const double kdx = hf * k * (d0 * pts[i] + d1 * pts[st + i] + d2 * pts[2 * st + i]);
    const double kdn = hf * k * (d0 * nrm[i] + d1 * nrm[st + i] + d2 * nrm[2 * st + i]);
    double s, c;
    sb_sincos(kdx, &s, &c);
    const double2 p = cmul(A, make_double2(c, s));
    const double2 dpdn = make_double2(-kdn * p.y, kdn * p.x);  // i kdn p
    const double2 bt = cscale(beta, tau);
    rhs[t] = make_double2(-(p.x + bt.x * dpdn.x - bt.y * dpdn.y), -(p.y + bt.x * dpdn.y + bt.y * dpdn.x));
}

// Near-pair classification of the NB n collocation rows against the n elements (the element's
// own row block excluded): pass 0 counts, pass 1 writes the columns in increasing order.
template <int NB>
__global__ void __launch_bounds__(256) k_lin_near_pass(const double* __restrict__ elem, int64_t n, int64_t ld,
                                                       const double* __restrict__ cp, int pass,
                                                       int64_t* __restrict__ counts,
                                                       const int64_t* __restrict__ row_ptr,
                                                       int32_t* __restrict__ cols) {
    __shared__ double sx[kNearRows][3];
    __shared__ unsigned sball[8][kNearRows];
    __shared__ int64_t sbase[kNearRows];
    __shared__ int scount[kNearRows];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t n3 = NB * n;
    const int64_t row0 = blockIdx.x * (int64_t)kNearRows;
    if (tid < kNearRows) {
        const int64_t r = row0 + tid;
        for (int c = 0; c < 3; ++c) sx[tid][c] = (r < n3) ? cp[c * n3 + r] : 1e300;
        scount[tid] = 0;
        sbase[tid] = (pass == 1 && r < n3) ? row_ptr[r] : 0;
    }
    __syncthreads();
    for (int64_t c0 = 0; c0 < n; c0 += 256) {
        const int64_t j = c0 + tid;
        double gx = 0, gy = 0, gz = 0, thr = -1.0;
        if (j < n) {
            gx = E(EGX, j);
            gy = E(EGY, j);
            gz = E(EGZ, j);
            thr = near_threshold(E(EAREA, j));
        }
        for (int rr = 0; rr < kNearRows; ++rr) {
            const int64_t r = row0 + rr;
            const bool p = (j < n) && (r < n3) && (j != r / NB) &&
                           near_superset(gx, gy, gz, thr, sx[rr][0], sx[rr][1], sx[rr][2]);
            const unsigned b = __ballot_sync(0xffffffffu, p);
            if (pass == 0) {
                if (lane == 0 && b) atomicAdd(&scount[rr], __popc(b));
            } else {
                if (lane == 0) sball[warp][rr] = b;
            }
        }
        if (pass == 1) {
            __syncthreads();
            for (int rr = 0; rr < kNearRows; ++rr) {
                const unsigned b = sball[warp][rr];
                if (b & (1u << lane)) {
                    int before = __popc(b & ((1u << lane) - 1u));
                    for (int w = 0; w < warp; ++w) before += __popc(sball[w][rr]);
                    cols[sbase[rr] + scount[rr] + before] = static_cast<int32_t>(j);
                }
            }
            __syncthreads();
            if (tid < kNearRows) {
                int add = 0;
                for (int w = 0; w < 8; ++w) add += __popc(sball[w][tid]);
                scount[tid] += add;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (pass == 0 && tid < kNearRows && row0 + tid < n3) counts[row0 + tid] = scount[tid];
}

// Far field of the discontinuous bases: one thread per field element (128-column tiles), 32 rows
// per CTA; the element's 13-point leaf (the reference's single far leaf) staged in shared memory,
// the NB basis values of each point from the rule's reference coordinates.
template <int NB>
__global__ void __launch_bounds__(kFarTile) k_lin_far(const double* __restrict__ qp, const double* __restrict__ elem,
                                                      int64_t n, int64_t ld, const double* __restrict__ cp,
                                                      const double* __restrict__ coef, double k,
                                                      double2* __restrict__ A) {
    extern __shared__ __align__(128) double smem[];
    double* sq = smem;                   // [13][4][kFarTile]
    double* sr = smem + kQpTileDoubles;  // [kLinRows][6]
    const int tid = threadIdx.x;
    const int64_t tile = blockIdx.x;
    const int64_t j = tile * kFarTile + tid;
    const int64_t n3 = NB * n;
    const int64_t row0 = blockIdx.y * (int64_t)kLinRows;
    const double k2 = k * k;
    const double* src = qp + tile * (int64_t)kQpTileDoubles;
    for (int t = tid; t < kQpTileDoubles; t += kFarTile) sq[t] = src[t];
    for (int t = tid; t < kLinRows * 6; t += kFarTile) {
        const int rr = t / 6, f = t % 6;
        const int64_t r = row0 + rr;
        double v = 0.0;
        if (r < n3) v = f < 3 ? cp[f * n3 + r] : E(ENX + (f - 3), r / NB);
        sr[t] = v;
    }
    double nyx = 0, nyy = 0, nyz = 0, gx = 0, gy = 0, gz = 0, thr = -1;
    if (j < n) {
        nyx = E(ENX, j);
        nyy = E(ENY, j);
        nyz = E(ENZ, j);
        gx = E(EGX, j);
        gy = E(EGY, j);
        gz = E(EGZ, j);
        thr = near_threshold(E(EAREA, j));
    }
    __syncthreads();
    const int64_t rows_here = (n3 - row0 < kLinRows) ? (n3 - row0) : kLinRows;
    for (int rr = 0; rr < rows_here; ++rr) {
        const int64_t r = row0 + rr;
        const double xx = sr[rr * 6 + 0], xy = sr[rr * 6 + 1], xz = sr[rr * 6 + 2];
        const double nxx = sr[rr * 6 + 3], nxy = sr[rr * 6 + 4], nxz = sr[rr * 6 + 5];
        const bool active = (j < n) && (j != r / NB) && !near_superset(gx, gy, gz, thr, xx, xy, xz);
        if (!active) continue;
        Acc a[NB];
        for (int q = 0; q < kFarPoints; ++q) {
            const double* p = sq + q * 4 * kFarTile + tid;
            const double dx = p[0] - xx, dy = p[kFarTile] - xy, dz = p[2 * kFarTile] - xz;
            const double w = p[3 * kFarTile];
            const double d2 = dx * dx + dy * dy + dz * dz;
            const double rinv = sb_rsqrt2(d2);
            double nb[NB];
            panel_basis<NB>(c_tri_xi[c_tri_off[0] + q], c_tri_eta[c_tri_off[0] + q], nb);  // the 13-point leaf
            point_channels_w<NB>(a, nb, dx, dy, dz, d2 * rinv, rinv, w, nyx, nyy, nyz, nxx, nxy, nxz, k, k2);
        }
        for (int b = 0; b < NB; ++b) A[r * n3 + NB * j + b] = combine(a[b], coef, ld, j, CF_CG);
    }
}

__device__ __forceinline__ Acc lin_reduce(const Acc& a) { return warp_reduce(a); }

// Near pairs of the discontinuous bases: one warp per (collocation row, field element) pair.
template <int NB>
__global__ void __launch_bounds__(32 * kNearWarps) k_lin_near(const double* __restrict__ elem, int64_t n, int64_t ld,
                                                              const double* __restrict__ cp,
                                                              const int64_t* __restrict__ row_ptr,
                                                              const int32_t* __restrict__ cols, int64_t nnz,
                                                              const double* __restrict__ coef, double k,
                                                              double2* __restrict__ A) {
    __shared__ NearWarpSmem sm[kNearWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t p = blockIdx.x * (int64_t)kNearWarps + warp;
    if (p >= nnz) return;
    const int64_t n3 = NB * n;
    int64_t lo = 0, hi = n3 - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (row_ptr[mid] <= p) lo = mid; else hi = mid - 1;
    }
    const int64_t r = lo, j = cols[p], e = r / NB;
    Acc a[NB];
    near_channels_at<NB>(a, sm[warp], elem, ld, cp[r], cp[n3 + r], cp[2 * n3 + r], E(ENX, e), E(ENY, e), E(ENZ, e),
                        j, k, k * k, lane);
    Acc t[NB];
    for (int b = 0; b < NB; ++b) t[b] = lin_reduce(a[b]);
    if (lane == 0)
        for (int b = 0; b < NB; ++b) A[r * n3 + NB * j + b] = combine(t[b], coef, ld, j, CF_CG);
}
// Self element of the discontinuous bases (singular_integration_linear_with_params_mode, integration/
// singular.rs:868-1170): one warp per collocation row. The regularised edge integral of E is
// weighted by the basis at the edge point; the centroid-centred Duffy sub-triangles give G, H,
// H^T and the area part of E, k^2 (n_x . n_y) G N_b plus the basis-gradient term
// (-(n_x . n_y)(grad N_b . r_hat) + (r_hat . n_y)(grad N_b . n_x)) times G (-1/r + i k). The
// free term of the row's element goes on the diagonal.
template <int NB>
__global__ void __launch_bounds__(128) k_lin_self(const double* __restrict__ elem, int64_t n, int64_t ld,
                                                  const double* __restrict__ cp, const double* __restrict__ coef,
                                                  double k, double2* __restrict__ A, double2* __restrict__ diag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t n3 = NB * n;
    const int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + warp;
    if (r >= n3) return;
    const int64_t i = r / NB;
    const double k2 = k * k;
    const double x0 = cp[r], x1 = cp[n3 + r], x2 = cp[2 * n3 + r];
    const double nxx = E(ENX, i), nxy = E(ENY, i), nxz = E(ENZ, i);
    const double nyx = nxx, nyy = nxy, nyz = nxz;
    const double jac = E(EJAC, i);
    double V[3][3];
    for (int t = 0; t < 3; ++t)
        for (int c = 0; c < 3; ++c) V[t][c] = E(EV0X + 3 * t + c, i);
    // panel_basis_gradients (singular.rs:1173-1258): the surface gradient of N_b is
    // a ts + b tt with the panel's tangents and metric (constant over a flat panel).
    double tan_s[3], tan_t[3];
    for (int c = 0; c < 3; ++c) {
        tan_s[c] = -V[0][c] + V[1][c] + 0.0 * V[2][c];
        tan_t[c] = -V[0][c] + 0.0 * V[1][c] + V[2][c];
    }
    double gss = 0, gtt = 0, gst = 0;
    for (int c = 0; c < 3; ++c) {
        gss += tan_s[c] * tan_s[c];
        gtt += tan_t[c] * tan_t[c];
        gst += tan_s[c] * tan_t[c];
    }
    const double gdet = gss * gtt - gst * gst;
    const double ka = k * fmax(sqrt(E(EAREA, i)), 1e-10);
    int ngpo1, nsub, nsec1, nsec2;
    if (ka < 0.3) { ngpo1 = 3; nsub = 4; nsec1 = 4; nsec2 = 2; }
    else if (ka < 1.0) { ngpo1 = 4; nsub = 5; nsec1 = 6; nsec2 = 2; }
    else if (ka < 2.0) { ngpo1 = 5; nsub = 6; nsec1 = 8; nsec2 = 3; }
    else { ngpo1 = 6; nsub = 7; nsec1 = 10; nsec2 = 4; }
    const int ego = ngpo1 * (ngpo1 - 1) / 2, sgo = nsub * (nsub - 1) / 2;
    const int n_edge = nsec1 * ngpo1, n_bulk = nsec2 * nsub * nsub;
    const int per_edge = n_edge + n_bulk;
    const double csi6[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    const double eta6[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
    Acc a[NB];
    for (int f = lane; f < 3 * per_edge; f += 32) {
        const int ieg = f / per_edge, rem = f % per_edge;
        const int ig1 = (ieg + 1) % 3, ig2 = ieg + 3;
        if (rem < n_edge) {
            const int isec = rem / ngpo1, ig = rem % ngpo1;
            double dp[3], leneg = 0.0;
            for (int c = 0; c < 3; ++c) {
                dp[c] = V[ig1][c] - V[ieg][c];
                leneg += dp[c] * dp[c];
            }
            leneg = sqrt(leneg);
            const double to0 = dp[0] / leneg, to1 = dp[1] / leneg, to2 = dp[2] / leneg;
            const double leneg_scaled = leneg / (2.0 * nsec1);
            const double delsec = 2.0 / nsec1;
            double secmid = -1.0 - delsec / 2.0;
            for (int sct = 0; sct <= isec; ++sct) secmid += delsec;
            const double sga = secmid + c_gl_x[ego + ig] / nsec1;
            const double wga = c_gl_w[ego + ig] * leneg_scaled;
            const double dx = V[ieg][0] + dp[0] * (sga + 1.0) / 2.0 - x0;
            const double dy = V[ieg][1] + dp[1] * (sga + 1.0) / 2.0 - x1;
            const double dz = V[ieg][2] + dp[2] * (sga + 1.0) / 2.0 - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            double sn, cs;
            sb_sincos(k * dis, &sn, &cs);
            const double g_r = cs * kInv4Pi * rinv, g_i = sn * kInv4Pi * rinv;
            const double f_r = -g_r * rinv - g_i * k, f_i = g_r * k - g_i * rinv;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            const double cr = (uy * to2 - uz * to1) * nxx + (uz * to0 - ux * to2) * nxy + (ux * to1 - uy * to0) * nxz;
            const double te = (sga + 1.0) / 2.0;
            double nb[NB];
            panel_basis<NB>(csi6[ieg] * (1.0 - te) + csi6[ig1] * te, eta6[ieg] * (1.0 - te) + eta6[ig1] * te, nb);
            for (int b = 0; b < NB; ++b) {
                a[b].er += f_r * cr * wga * nb[b];
                a[b].ei += f_i * cr * wga * nb[b];
            }
        } else {
            const int r2 = rem - n_edge;
            const int isec = r2 / (nsub * nsub), ab = r2 % (nsub * nsub);
            const int ia = ab / nsub, ib = ab % nsub;
            const double aresub = 1.0 / 24.0 / nsec2;
            double ss[3], ts[3];
            ss[0] = ts[0] = 1.0 / 3.0;
            if (isec == 0) {
                ss[1] = csi6[ieg]; ss[2] = csi6[ig2]; ts[1] = eta6[ieg]; ts[2] = eta6[ig2];
            } else {
                ss[1] = csi6[ig2]; ss[2] = csi6[ig1]; ts[1] = eta6[ig2]; ts[2] = eta6[ig1];
            }
            const double sga = c_gl_x[sgo + ia], tga = c_gl_x[sgo + ib];
            const double wei = c_gl_w[sgo + ia] * c_gl_w[sgo + ib];
            const double sgg = 0.5 * (1.0 - sga) * ss[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
            const double tgg = 0.5 * (1.0 - sga) * ts[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
            const double sf0 = 1.0 - sgg - tgg;
            const double dx = sf0 * V[0][0] + sgg * V[1][0] + tgg * V[2][0] - x0;
            const double dy = sf0 * V[0][1] + sgg * V[1][1] + tgg * V[2][1] - x1;
            const double dz = sf0 * V[0][2] + sgg * V[1][2] + tgg * V[2][2] - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            const double wga = wei * (1.0 + sga) * aresub * jac;
            double sn, cs;
            sb_sincos(k * dis, &sn, &cs);
            const double gs = wga * kInv4Pi * rinv;
            const double g_r = cs * gs, g_i = sn * gs;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            const double rny = ux * nyx + uy * nyy + uz * nyz;
            const double rnx = -(ux * nxx + uy * nxy + uz * nxz);
            const double b_r = -g_r * rinv - g_i * k, b_i = g_r * k - g_i * rinv;
            const double nd = nxx * nyx + nxy * nyy + nxz * nyz;
            double nb[NB], der[NB][2];
            panel_basis<NB>(sgg, tgg, nb);
            panel_basis_deriv<NB>(sgg, tgg, der);
            for (int b = 0; b < NB; ++b) {
                const double w = nb[b];
                a[b].gr += g_r * w; a[b].gi += g_i * w;
                a[b].hr += b_r * rny * w; a[b].hi += b_i * rny * w;
                a[b].tr += b_r * rnx * w; a[b].ti += b_i * rnx * w;
                const double ga = (gtt * der[b][0] - gst * der[b][1]) / gdet;
                const double gb = (gss * der[b][1] - gst * der[b][0]) / gdet;
                const double grad0 = ga * tan_s[0] + gb * tan_t[0], grad1 = ga * tan_s[1] + gb * tan_t[1];
                const double grad2 = ga * tan_s[2] + gb * tan_t[2];
                const double gr = grad0 * ux + grad1 * uy + grad2 * uz;
                const double gsn = grad0 * nxx + grad1 * nxy + grad2 * nxz;
                const double gf = -nd * gr + rny * gsn;
                a[b].er += g_r * k2 * nd * w + b_r * gf;
                a[b].ei += g_i * k2 * nd * w + b_i * gf;
            }
        }
    }
    Acc t[NB];
    for (int b = 0; b < NB; ++b) t[b] = warp_reduce(a[b]);
    if (lane == 0) {
        const int c = static_cast<int>(r % NB);
        for (int b = 0; b < NB; ++b) {
            double2 v = combine(t[b], coef, ld, i, CF_CG);
            if (b == c) {
                v.x += coef[(int64_t)(CF_DIAG) * ld + i];
                v.y += coef[(int64_t)(CF_DIAG + 1) * ld + i];
                diag[r] = v;
            }
            A[r * n3 + NB * i + b] = v;
        }
    }
}

// =============================================================================================
// Quad4 constant panels (the ElementType::Quad4 branches of the constant path): bilinear geometry
// on [-1, 1]^2 with vertices (1, 1), (-1, 1), (-1, -1), (1, -1) (compute_parameters,
// integration/regular.rs:636-714), tensor Gauss-Legendre rules (quad_quadrature,
// integration/gauss.rs:159-170), four-quad subdivision about the subelement centre
// (generate_subelements, integration/singular.rs:1372-1540), the Quad4 self term
// (singular.rs:297-614). FP64, complex128 output.
// =============================================================================================
__constant__ double c_csi8[8] = {1.0, -1.0, -1.0, 1.0, 0.0, -1.0, 0.0, 1.0};
__constant__ double c_eta8[8] = {1.0, 1.0, -1.0, -1.0, 1.0, 0.0, -1.0, 0.0};
constexpr int kQuadTile = 64;   // columns per far-kernel CTA
constexpr int kQuadRows = 32;   // rows per far-kernel CTA
constexpr int kQuadFar = 16;    // far leaf: the 4 x 4 rule

// Position, Jacobian and unit normal of the bilinear map at (s, t), correctly rounded operations
// in the reference's order (the subdivision decisions depend on the positions).
__device__ __forceinline__ void quad_params(const double V[4][3], double s, double t, double pos[3], double& jac,
                                            double nrm[3]) {
    const double s1 = __dmul_rn(0.25, __dadd_rn(s, 1.0)), s2 = __dmul_rn(0.25, __dsub_rn(s, 1.0));
    const double t1 = __dadd_rn(t, 1.0), t2 = __dsub_rn(t, 1.0);
    const double sf[4] = {__dmul_rn(s1, t1), -__dmul_rn(s2, t1), __dmul_rn(s2, t2), -__dmul_rn(s1, t2)};
    const double a = __dmul_rn(0.25, __dadd_rn(t, 1.0)), b = __dmul_rn(0.25, __dsub_rn(t, 1.0));
    const double sds[4] = {a, -a, b, -b};
    const double c = __dmul_rn(0.25, __dadd_rn(s, 1.0)), d = __dmul_rn(0.25, __dsub_rn(1.0, s));
    const double sdt[4] = {c, d, __dmul_rn(0.25, __dsub_rn(s, 1.0)), -c};
    double dxs[3] = {0.0, 0.0, 0.0}, dxt[3] = {0.0, 0.0, 0.0};
    pos[0] = pos[1] = pos[2] = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 3; ++j) {
            pos[j] = __dadd_rn(pos[j], __dmul_rn(sf[i], V[i][j]));
            dxs[j] = __dadd_rn(dxs[j], __dmul_rn(sds[i], V[i][j]));
            dxt[j] = __dadd_rn(dxt[j], __dmul_rn(sdt[i], V[i][j]));
        }
    const double n0 = __dsub_rn(__dmul_rn(dxs[1], dxt[2]), __dmul_rn(dxs[2], dxt[1]));
    const double n1 = __dsub_rn(__dmul_rn(dxs[2], dxt[0]), __dmul_rn(dxs[0], dxt[2]));
    const double n2 = __dsub_rn(__dmul_rn(dxs[0], dxt[1]), __dmul_rn(dxs[1], dxt[0]));
    jac = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(n0, n0), __dmul_rn(n1, n1)), __dmul_rn(n2, n2)));
    if (jac > 1e-15) {
        nrm[0] = __ddiv_rn(n0, jac);
        nrm[1] = __ddiv_rn(n1, jac);
        nrm[2] = __ddiv_rn(n2, jac);
    } else {
        nrm[0] = nrm[1] = nrm[2] = 0.0;
    }
}

__device__ __forceinline__ void quad_vertices(const double* __restrict__ elem, int64_t ld, int64_t e,
                                              double V[4][3]) {
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) V[a][c] = E(EV0X + 3 * a + c, e);
    for (int c = 0; c < 3; ++c) V[3][c] = E(EV3X + c, e);
}

// compute_element_geometry (mesh/generators.rs:771-850) for Quad4: centre = node average,
// normal from the diagonal cross product (p2 - p0) x (p3 - p1), area = compute_element_area
// (mesh/element.rs:326-362, mean of both diagonal splits); level-0 subdivision centre =
// the bilinear map at (0, 0).
__global__ void k_quad_geometry(const double* __restrict__ nodes, const uint32_t* __restrict__ quads, int64_t n,
                                int64_t ld, double* __restrict__ elem) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ld) return;
    if (e >= n) {
        for (int f = 0; f < EFIELDS; ++f) E(f, e) = 0.0;
        return;
    }
    double V[4][3];
    for (int a = 0; a < 4; ++a)
        for (int j = 0; j < 3; ++j) V[a][j] = nodes[3 * (int64_t)quads[4 * e + a] + j];
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 3; ++j) E(EV0X + 3 * a + j, e) = V[a][j];
    for (int j = 0; j < 3; ++j) E(EV3X + j, e) = V[3][j];
    for (int j = 0; j < 3; ++j) {
        const double sm = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(0.0, V[0][j]), V[1][j]), V[2][j]), V[3][j]);
        E(ECX + j, e) = __ddiv_rn(sm, 4.0);
    }
    auto cross_len = [](const double* a, const double* b) {
        const double c0 = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
        const double c1 = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
        const double c2 = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
        return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(c0, c0), __dmul_rn(c1, c1)), __dmul_rn(c2, c2)));
    };
    double d1[3], d2[3];
    for (int j = 0; j < 3; ++j) {
        d1[j] = __dsub_rn(V[2][j], V[0][j]);
        d2[j] = __dsub_rn(V[3][j], V[1][j]);
    }
    const double c0 = __dsub_rn(__dmul_rn(d1[1], d2[2]), __dmul_rn(d1[2], d2[1]));
    const double c1 = __dsub_rn(__dmul_rn(d1[2], d2[0]), __dmul_rn(d1[0], d2[2]));
    const double c2 = __dsub_rn(__dmul_rn(d1[0], d2[1]), __dmul_rn(d1[1], d2[0]));
    const double len = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(c0, c0), __dmul_rn(c1, c1)), __dmul_rn(c2, c2)));
    if (len > 1e-15) {
        E(ENX, e) = __ddiv_rn(c0, len);
        E(ENY, e) = __ddiv_rn(c1, len);
        E(ENZ, e) = __ddiv_rn(c2, len);
    } else {
        E(ENX, e) = E(ENY, e) = E(ENZ, e) = 0.0;
    }
    double v1[3], v2[3], v3[3], v4[3], v5[3], v6[3];
    for (int j = 0; j < 3; ++j) {
        v1[j] = __dsub_rn(V[1][j], V[0][j]);
        v2[j] = __dsub_rn(V[2][j], V[0][j]);
        v3[j] = __dsub_rn(V[3][j], V[0][j]);
        v4[j] = __dsub_rn(V[2][j], V[1][j]);
        v5[j] = __dsub_rn(V[3][j], V[1][j]);
        v6[j] = __dsub_rn(V[0][j], V[1][j]);
    }
    const double a1 = __dmul_rn(0.5, cross_len(v1, v2)), a2 = __dmul_rn(0.5, cross_len(v2, v3));
    const double a3 = __dmul_rn(0.5, cross_len(v4, v5)), a4 = __dmul_rn(0.5, cross_len(v5, v6));
    E(EAREA, e) = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dadd_rn(a1, a2), a3), a4));
    E(EJAC, e) = 0.0;
    double g[3], jac, nrm[3];
    quad_params(V, 0.0, 0.0, g, jac, nrm);
    for (int j = 0; j < 3; ++j) E(EGX + j, e) = g[j];
    E(ESQA, e) = __dsqrt_rn(E(EAREA, e));
}

// Far points of every element: the 4 x 4 Gauss-Legendre rule (quad_quadrature(4)) mapped by the
// bilinear map, weight * Jacobian and the local normal: qq[(q * 7 + f) * ld + e].
__global__ void k_quad_points(const double* __restrict__ elem, int64_t n, int64_t ld, double* __restrict__ qq) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ld) return;
    double V[4][3];
    if (e < n) quad_vertices(elem, ld, e, V);
    const int o = 4 * 3 / 2;  // Gauss-Legendre order 4 in the triangular GL table
    for (int q = 0; q < kQuadFar; ++q) {
        double v[7] = {0, 0, 0, 0, 0, 0, 0};
        if (e < n) {
            const int a = q / 4, b = q % 4;
            double pos[3], jac, nrm[3];
            quad_params(V, c_gl_x[o + a], c_gl_x[o + b], pos, jac, nrm);
            v[0] = pos[0];
            v[1] = pos[1];
            v[2] = pos[2];
            v[3] = c_gl_w[o + a] * c_gl_w[o + b] * jac;
            v[4] = nrm[0];
            v[5] = nrm[1];
            v[6] = nrm[2];
        }
        for (int f = 0; f < 7; ++f) qq[(int64_t)(q * 7 + f) * ld + e] = v[f];
    }
}

// Far pairs of a Quad4 mesh: one thread per field element (64-column tiles), 32 rows per CTA,
// the column tile's 16 far points (position, weight * Jacobian, normal) in shared memory.
__global__ void __launch_bounds__(kQuadTile) k_quad_far(const double* __restrict__ qq,
                                                        const double* __restrict__ elem, int64_t n, int64_t ld,
                                                        const double* __restrict__ coef, double k,
                                                        double2* __restrict__ A) {
    extern __shared__ __align__(16) double smem[];
    double* sq = smem;                                 // [16 * 7][kQuadTile]
    double* sr = smem + kQuadFar * 7 * kQuadTile;      // [kQuadRows][6]
    const int tid = threadIdx.x;
    const int64_t j0 = blockIdx.x * (int64_t)kQuadTile;
    const int64_t j = j0 + tid;
    const int64_t row0 = blockIdx.y * (int64_t)kQuadRows;
    const double k2 = k * k;
    for (int f = 0; f < kQuadFar * 7; ++f) sq[f * kQuadTile + tid] = (j < ld) ? qq[(int64_t)f * ld + j] : 0.0;
    for (int t = tid; t < kQuadRows * 6; t += kQuadTile) {
        const int rr = t / 6, f = t % 6;
        const int64_t i = row0 + rr;
        sr[t] = (i < n) ? E(ECX + f, i) : 0.0;
    }
    double gx = 0, gy = 0, gz = 0, thr = -1;
    if (j < n) {
        gx = E(EGX, j);
        gy = E(EGY, j);
        gz = E(EGZ, j);
        thr = near_threshold(E(EAREA, j));
    }
    __syncthreads();
    const int64_t rows_here = (n - row0 < kQuadRows) ? (n - row0) : kQuadRows;
    for (int rr = 0; rr < rows_here; ++rr) {
        const int64_t i = row0 + rr;
        const double xx = sr[rr * 6 + 0], xy = sr[rr * 6 + 1], xz = sr[rr * 6 + 2];
        const double nxx = sr[rr * 6 + 3], nxy = sr[rr * 6 + 4], nxz = sr[rr * 6 + 5];
        const bool active = (j < n) && (j != i) && !near_superset(gx, gy, gz, thr, xx, xy, xz);
        if (!active) continue;
        Acc a;
        for (int q = 0; q < kQuadFar; ++q) {
            const double* p = sq + q * 7 * kQuadTile + tid;
            const double dx = p[0] - xx, dy = p[kQuadTile] - xy, dz = p[2 * kQuadTile] - xz;
            const double d2 = dx * dx + dy * dy + dz * dz;
            const double rinv = sb_rsqrt2(d2);
            point_channels(a, dx, dy, dz, d2 * rinv, rinv, p[3 * kQuadTile], p[4 * kQuadTile], p[5 * kQuadTile],
                           p[6 * kQuadTile], nxx, nxy, nxz, k, k2);
        }
        A[i * n + j] = combine(a, coef, ld, j, CF_CG);
    }
}

struct QuadWarpSmem {
    double xs[2][kMaxNse][4];
    double es[2][kMaxNse][4];
    double lc[kMaxNse][3];  // kept leaves of the current level: centre (s, t) and edge factor
    int lorder[kMaxNse];
    int loff[kMaxNse + 1];
};

// Regular-integration channels of Quad4 element j seen from x (normal nx), lane-partial sums:
// the level-by-level replay of generate_subelements with the subelements of a level spread
// over the lanes, ballots for the split decisions (the 16th split ends the level), the 110-leaf
// cap, each kept leaf's order x order Gauss-Legendre points spread over the lanes.
__device__ void quad_near_channels(Acc& a, QuadWarpSmem& S, const double* __restrict__ elem, int64_t ld,
                                   double x0, double x1, double x2, double nxx, double nxy, double nxz, int64_t j,
                                   double k, double k2, int lane) {
    double V[4][3];
    quad_vertices(elem, ld, j, V);
    const double area = E(EAREA, j);
    if (lane == 0) {
        for (int v = 0; v < 4; ++v) {
            S.xs[0][0][v] = c_csi8[v];
            S.es[0][0][v] = c_eta8[v];
        }
    }
    __syncwarp();
    int cur = 0, nsel = 1, total = 0;
    double faclin = 2.0;
    const unsigned lt = (1u << lane) - 1u;
    for (int level = 0; level < 64; ++level) {
        faclin *= 0.5;
        const double arels = __dmul_rn(__dmul_rn(area, faclin), faclin);
        const double sqa = __dsqrt_rn(arels);
        bool sub[2] = {false, false};
        double rat[2] = {0.0, 0.0}, scs[2] = {0.0, 0.0}, tcs[2] = {0.0, 0.0};
        for (int h = 0; h < 2; ++h) {
            const int s = lane + 32 * h;
            if (s < nsel) {
                const double* xp = S.xs[cur][s];
                const double* ep = S.es[cur][s];
                const double sc = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(0.0, xp[0]), xp[1]), xp[2]), xp[3]), 4.0);
                const double tc = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(0.0, ep[0]), ep[1]), ep[2]), ep[3]), 4.0);
                double g[3], jac, nrm[3];
                quad_params(V, sc, tc, g, jac, nrm);
                const double dx = __dsub_rn(g[0], x0), dy = __dsub_rn(g[1], x1), dz = __dsub_rn(g[2], x2);
                const double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                rat[h] = __ddiv_rn(dist, sqa);
                sub[h] = rat[h] < 3.0;
                scs[h] = sc;
                tcs[h] = tc;
            }
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, sub[0]);
        const unsigned m1 = __ballot_sync(0xffffffffu, sub[1]);
        const int nsub = __popc(m0) + __popc(m1);
        int breakpos = nsel;
        if (nsub >= 16) {
            if (__popc(m0) >= 16) {
                unsigned m = m0;
                for (int t = 0; t < 15; ++t) m &= m - 1;
                breakpos = __ffs(m) - 1;
            } else {
                unsigned m = m1;
                for (int t = 0; t < 15 - __popc(m0); ++t) m &= m - 1;
                breakpos = 32 + __ffs(m) - 1;
            }
        }
        const unsigned valid0 = breakpos >= 32 ? 0xffffffffu : ((1u << breakpos) - 1u);
        const unsigned valid1 = breakpos >= 64 ? 0xffffffffu : (breakpos <= 32 ? 0u : ((1u << (breakpos - 32)) - 1u));
        const unsigned nsel0 = nsel >= 32 ? 0xffffffffu : ((1u << nsel) - 1u);
        const unsigned nsel1 = nsel >= 64 ? 0xffffffffu : (nsel <= 32 ? 0u : ((1u << (nsel - 32)) - 1u));
        const unsigned l0 = ~m0 & valid0 & nsel0;
        const unsigned l1 = ~m1 & valid1 & nsel1;
        const int nleaf = __popc(l0) + __popc(l1);
        const int keep = min(nleaf, kMaxLeaves - total);
        const int nxt = cur ^ 1;
        for (int h = 0; h < 2; ++h) {
            const int s = lane + 32 * h;
            if (s >= nsel) continue;
            const unsigned lm = h == 0 ? l0 : l1;
            if (lm & (1u << lane)) {
                const int rank = (h == 0) ? __popc(l0 & lt) : __popc(l0) + __popc(l1 & lt);
                if (rank < keep) {
                    S.lc[rank][0] = scs[h];
                    S.lc[rank][1] = tcs[h];
                    S.lc[rank][2] = faclin;
                    S.lorder[rank] = gauss_order(0.5 / rat[h]);
                }
            }
            const unsigned sm = h == 0 ? m0 : m1;
            if (sm & (1u << lane)) {
                const int rank = (h == 0) ? __popc(m0 & lt) : __popc(m0) + __popc(m1 & lt);
                if (rank < 15) {
                    const double* xp = S.xs[cur][s];
                    const double* ep = S.es[cur][s];
                    double xm[8], em[8];
                    for (int t = 0; t < 4; ++t) {
                        const int t1 = (t + 1) % 4;
                        xm[t] = xp[t];
                        xm[t + 4] = (xp[t] + xp[t1]) / 2.0;
                        em[t] = ep[t];
                        em[t + 4] = (ep[t] + ep[t1]) / 2.0;
                    }
                    const int b = 4 * rank;
                    for (int t = 0; t < 4; ++t) {
                        const int t2 = (t == 0) ? 7 : t + 3;
                        S.xs[nxt][b + t][0] = xm[t];
                        S.xs[nxt][b + t][1] = xm[t + 4];
                        S.xs[nxt][b + t][2] = scs[h];
                        S.xs[nxt][b + t][3] = xm[t2];
                        S.es[nxt][b + t][0] = em[t];
                        S.es[nxt][b + t][1] = em[t + 4];
                        S.es[nxt][b + t][2] = tcs[h];
                        S.es[nxt][b + t][3] = em[t2];
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) {
            int o = 0;
            for (int l = 0; l < keep; ++l) {
                S.loff[l] = o;
                o += S.lorder[l] * S.lorder[l];
            }
            S.loff[keep] = o;
        }
        __syncwarp();
        const int npts = S.loff[keep];
        for (int f = lane; f < npts; f += 32) {
            int lo = 0, hi = keep - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (S.loff[mid] <= f) lo = mid; else hi = mid - 1;
            }
            const int l = lo, ord = S.lorder[l];
            const int q = f - S.loff[l];
            const int go = ord * (ord - 1) / 2;
            const double csi = c_gl_x[go + q / ord], eta = c_gl_x[go + q % ord];
            const double wq = c_gl_w[go + q / ord] * c_gl_w[go + q % ord];
            const double fac = S.lc[l][2];
            const bool iforie = fabs(fabs(fac) - 1.0) < 1e-10;
            double xio, eto, weih2;
            if (iforie) {
                xio = csi;
                eto = eta;
                weih2 = wq;
            } else {
                xio = S.lc[l][0] + csi * fac;
                eto = S.lc[l][1] + eta * fac;
                weih2 = wq * (fac * fac);
            }
            double pos[3], jac, ny[3];
            quad_params(V, xio, eto, pos, jac, ny);
            const double dx = pos[0] - x0, dy = pos[1] - x1, dz = pos[2] - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            point_channels(a, dx, dy, dz, dis, rinv, weih2 * jac, ny[0], ny[1], ny[2], nxx, nxy, nxz, k, k2);
        }
        total += keep;
        __syncwarp();
        if (total >= kMaxLeaves || nsub == 0) break;
        nsel = min(nsub, 15) * 4;
        cur = nxt;
    }
}

__global__ void __launch_bounds__(32 * kNearWarps) k_quad_near(const double* __restrict__ elem, int64_t n, int64_t ld,
                                                               const int64_t* __restrict__ row_ptr,
                                                               const int32_t* __restrict__ cols, int64_t nnz,
                                                               const double* __restrict__ coef, double k,
                                                               double2* __restrict__ A) {
    __shared__ QuadWarpSmem sm[kNearWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t p = blockIdx.x * (int64_t)kNearWarps + warp;
    if (p >= nnz) return;
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (row_ptr[mid] <= p) lo = mid; else hi = mid - 1;
    }
    const int64_t i = lo, j = cols[p];
    Acc a;
    quad_near_channels(a, sm[warp], elem, ld, E(ECX, i), E(ECY, i), E(ECZ, i), E(ENX, i), E(ENY, i), E(ENZ, i), j, k,
                       k * k, lane);
    const Acc t = warp_reduce(a);
    if (lane == 0) A[i * n + j] = combine(t, coef, ld, j, CF_CG);
}

// Self term of a Quad4 element (the Quad4 branch of singular_integration_with_params_mode,
// singular.rs:297-614): four edges, sub-triangles fanned from the centre (0, 0) over each edge's
// two halves (area weight 1/4 / nsec2), the bilinear map's Jacobian and normal per point; the
// quadrature parameters from estimate_element_size (singular.rs:1641-1676: sqrt of the two
// triangles split along the diagonal 0-2).
__global__ void __launch_bounds__(128) k_quad_self(const double* __restrict__ elem, int64_t n, int64_t ld,
                                                   const double* __restrict__ coef, double k,
                                                   double2* __restrict__ A, double2* __restrict__ diag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + warp;
    if (i >= n) return;
    const double k2 = k * k;
    const double x0 = E(ECX, i), x1 = E(ECY, i), x2 = E(ECZ, i);
    const double nxx = E(ENX, i), nxy = E(ENY, i), nxz = E(ENZ, i);
    double V[4][3];
    quad_vertices(elem, ld, i, V);
    double size;
    {
        double v1[3], v2[3], v3[3];
        for (int c = 0; c < 3; ++c) {
            v1[c] = V[1][c] - V[0][c];
            v2[c] = V[2][c] - V[0][c];
            v3[c] = V[3][c] - V[0][c];
        }
        const double c10 = v1[1] * v2[2] - v1[2] * v2[1], c11 = v1[2] * v2[0] - v1[0] * v2[2],
                     c12 = v1[0] * v2[1] - v1[1] * v2[0];
        const double c20 = v2[1] * v3[2] - v2[2] * v3[1], c21 = v2[2] * v3[0] - v2[0] * v3[2],
                     c22 = v2[0] * v3[1] - v2[1] * v3[0];
        const double a1 = 0.5 * sqrt(c10 * c10 + c11 * c11 + c12 * c12);
        const double a2 = 0.5 * sqrt(c20 * c20 + c21 * c21 + c22 * c22);
        size = fmax(sqrt(a1 + a2), 1e-10);
    }
    const double ka = k * size;
    int ngpo1, nsub, nsec1, nsec2;
    if (ka < 0.3) { ngpo1 = 3; nsub = 4; nsec1 = 4; nsec2 = 2; }
    else if (ka < 1.0) { ngpo1 = 4; nsub = 5; nsec1 = 6; nsec2 = 2; }
    else if (ka < 2.0) { ngpo1 = 5; nsub = 6; nsec1 = 8; nsec2 = 3; }
    else { ngpo1 = 6; nsub = 7; nsec1 = 10; nsec2 = 4; }
    const int ego = ngpo1 * (ngpo1 - 1) / 2, sgo = nsub * (nsub - 1) / 2;
    const int n_edge = nsec1 * ngpo1, n_bulk = nsec2 * nsub * nsub;
    const int per_edge = n_edge + n_bulk;
    Acc a;
    double edge_r = 0.0, edge_i = 0.0;
    for (int f = lane; f < 4 * per_edge; f += 32) {
        const int ieg = f / per_edge, rem = f % per_edge;
        const int ig1 = (ieg + 1) % 4, ig2 = ieg + 4;
        if (rem < n_edge) {
            const int isec = rem / ngpo1, ig = rem % ngpo1;
            double dp[3], leneg = 0.0;
            for (int c = 0; c < 3; ++c) {
                dp[c] = V[ig1][c] - V[ieg][c];
                leneg += dp[c] * dp[c];
            }
            leneg = sqrt(leneg);
            const double to0 = dp[0] / leneg, to1 = dp[1] / leneg, to2 = dp[2] / leneg;
            const double leneg_scaled = leneg / (2.0 * nsec1);
            const double delsec = 2.0 / nsec1;
            double secmid = -1.0 - delsec / 2.0;
            for (int sct = 0; sct <= isec; ++sct) secmid += delsec;
            const double sga = secmid + c_gl_x[ego + ig] / nsec1;
            const double wga = c_gl_w[ego + ig] * leneg_scaled;
            const double dx = V[ieg][0] + dp[0] * (sga + 1.0) / 2.0 - x0;
            const double dy = V[ieg][1] + dp[1] * (sga + 1.0) / 2.0 - x1;
            const double dz = V[ieg][2] + dp[2] * (sga + 1.0) / 2.0 - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            double sn, cs;
            sb_sincos(k * dis, &sn, &cs);
            const double g_r = cs * kInv4Pi * rinv, g_i = sn * kInv4Pi * rinv;
            const double f_r = -g_r * rinv - g_i * k, f_i = g_r * k - g_i * rinv;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            const double cr = (uy * to2 - uz * to1) * nxx + (uz * to0 - ux * to2) * nxy + (ux * to1 - uy * to0) * nxz;
            edge_r += f_r * cr * wga;
            edge_i += f_i * cr * wga;
        } else {
            const int r2 = rem - n_edge;
            const int isec = r2 / (nsub * nsub), ab = r2 % (nsub * nsub);
            const int ia = ab / nsub, ib = ab % nsub;
            const double aresub = 0.25 / nsec2;
            double ss[3] = {0.0, 0.0, 0.0}, ts[3] = {0.0, 0.0, 0.0};
            if (isec == 0) {
                ss[1] = c_csi8[ieg]; ss[2] = c_csi8[ig2]; ts[1] = c_eta8[ieg]; ts[2] = c_eta8[ig2];
            } else {
                ss[1] = c_csi8[ig2]; ss[2] = c_csi8[ig1]; ts[1] = c_eta8[ig2]; ts[2] = c_eta8[ig1];
            }
            const double sga = c_gl_x[sgo + ia], tga = c_gl_x[sgo + ib];
            const double wei = c_gl_w[sgo + ia] * c_gl_w[sgo + ib];
            const double sgg = 0.5 * (1.0 - sga) * ss[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
            const double tgg = 0.5 * (1.0 - sga) * ts[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
            double pos[3], jac, ny[3];
            quad_params(V, sgg, tgg, pos, jac, ny);
            const double dx = pos[0] - x0, dy = pos[1] - x1, dz = pos[2] - x2;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dis >= 1e-15)) continue;
            const double rinv = 1.0 / dis;
            const double wga = wei * (1.0 + sga) * aresub * jac;
            double sn, cs;
            sb_sincos(k * dis, &sn, &cs);
            const double gs = wga * kInv4Pi * rinv;
            const double g_r = cs * gs, g_i = sn * gs;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            const double rny = ux * ny[0] + uy * ny[1] + uz * ny[2];
            const double rnx = -(ux * nxx + uy * nxy + uz * nxz);
            const double b_r = -g_r * rinv - g_i * k, b_i = g_r * k - g_i * rinv;
            a.gr += g_r; a.gi += g_i;
            a.hr += b_r * rny; a.hi += b_i * rny;
            a.tr += b_r * rnx; a.ti += b_i * rnx;
            const double nd = nxx * ny[0] + nxy * ny[1] + nxz * ny[2];
            a.er += g_r * k2 * nd;
            a.ei += g_i * k2 * nd;
        }
    }
    a.er += edge_r;
    a.ei += edge_i;
    const Acc t = warp_reduce(a);
    if (lane == 0) self_store(t, coef, ld, n, i, A, nullptr, 0, nullptr, diag);
}

// ---------------------------------------------------------------------------------------------
// Persistent batched assembly: every instance of a frequency sweep in one launch. The work list
// is [far tiles of all instances | near pairs (4 per item) | self elements (4 per item)]; each CTA
// walks it with a grid stride, so instances of any size share the SMs. Complex64 output
// (SB_PRECISION_FP32 numerics); instances have no prescribed boundary values.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int find_instance(const int64_t* __restrict__ pre, int ninst, int64_t item) {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Shared memory of the persistent kernel: a CTA works on one item at a time, so the far tile's
// arrays and the near pairs' subdivision buffers share the same bytes.
union BatchAsmSmem {
    Far32Smem far;
    NearWarpSmem near[kNearWarps];
};

// Largest |re|, |im| of the entries a warp wrote for one instance, kept in registers while the
// warp's items stay in that instance and merged into the instance's word when it moves on.
struct WarpAmax {
    unsigned* dst = nullptr;
    float m = 0.f;
    __device__ __forceinline__ void add(unsigned* to, float v) {
        if (to != dst) {
            flush();
            dst = to;
        }
        m = (v <= 3.4e38f) ? fmaxf(m, v) : INFINITY;
    }
    __device__ __forceinline__ void flush() {
        if (dst && m > 0.f) atomicMax(dst, __float_as_uint(m));
        m = 0.f;
    }
};

constexpr int kBatchPerWarp = 4;  // near pairs / self elements per warp and item of the persistent kernel

// kPart: 0 = every item (far tiles alternating with near / self items), 1 = the far tiles only,
// 2 = the near pairs and self elements only.
template <int kPart>
__global__ void __launch_bounds__(kFarTile, 4) k_assemble_batch(const BatchAsmInst* __restrict__ inst, int ninst,
                                                             const int64_t* __restrict__ pre, int near_per_far) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    BatchAsmSmem& sm = *reinterpret_cast<BatchAsmSmem*>(batch_smem);
    // The loop state is the same for the whole CTA and lives in shared memory, so no register holds
    // it across a far tile (whose packed loop uses all 128).
    __shared__ int64_t st_fi, st_qi;
    __shared__ int st_bf, st_bn, st_bs, st_npf;
    const int64_t* fpre = pre;
    const int64_t* npre = pre + (ninst + 1);
    const int64_t* spre = pre + 2 * (ninst + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        st_fi = kPart == 2 ? fpre[ninst] : blockIdx.x;
        st_qi = kPart == 1 ? npre[ninst] + spre[ninst] : blockIdx.x;
        st_bf = st_bn = st_bs = 0;
        st_npf = near_per_far;
    }
    __syncthreads();
    // Each CTA alternates one far tile with near_per_far near / self items (both lists walked with
    // the grid stride), so the far tiles and the FP64 near pairs share the SMs for the whole
    // launch. Items only move forward, so each list's instance is kept and advanced, not searched.
    for (;;) {
        const int64_t nf = fpre[ninst], nq = npre[ninst] + spre[ninst];
        if (st_fi >= nf && st_qi >= nq) break;
        if (kPart != 2 && st_fi < nf) {
            const int64_t fi = st_fi;
            int bf = st_bf;
            while (fpre[bf + 1] <= fi) ++bf;
            const BatchAsmInst& I = inst[bf];
            // column tiles fastest, as the per-instance launch's grid: the CTAs running side by side
            // write neighbouring column blocks of the same rows
            const int64_t local = fi - fpre[bf];
            far32_tile<false, true>(I.qp32, I.elem, I.n, I.ld, I.coef, I.k, I.coord_bound, I.A32, I.lda32, nullptr,
                                    I.n_tiles, local % I.n_tiles, (local / I.n_tiles) * kFar32Rows, I.amax, nullptr,
                                    0, nullptr, nullptr, &sm.far);
            // every warp is done with the tile before the next item reuses its shared memory
            __syncthreads();
            if (threadIdx.x == 0) {
                st_fi = fi + gridDim.x;
                st_bf = bf;
            }
            __syncthreads();
        }
        if (kPart != 1) {
            const int64_t nn = npre[ninst];
            int64_t qi = st_qi;
            int bn = st_bn, bs = st_bs;
            const int npf = st_npf;
            WarpAmax wam;  // lane 0's running maximum of the near and self entries
            for (int rep = 0; rep < npf && qi < nq; ++rep, qi += gridDim.x) {
                if (qi < nn) {
                    while (npre[bn + 1] <= qi) ++bn;
                    const BatchAsmInst& I = inst[bn];
                    const int64_t p0 = (qi - npre[bn]) * (kNearWarps * kBatchPerWarp) + warp * kBatchPerWarp;
                    for (int u = 0; u < kBatchPerWarp; ++u) {
                        const int64_t p = p0 + u;
                        if (p >= I.nnz) break;
                        const int64_t i = I.near_row[p], j = I.near_col[p];
                        Acc a;
                        near_pair_channels(a, sm.near[warp], I.elem, I.ld, i, j, I.k, I.k * I.k, lane);
                        const Acc t = warp_reduce(a);
                        if (lane == 0) {
                            const double2 v = combine(t, I.coef, I.ld, j, CF_CG);
                            const float2 f = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
                            I.A32[i * I.lda32 + j] = f;
                            if (I.amax) wam.add(I.amax, fmaxf(fabsf(f.x), fabsf(f.y)));
                        }
                    }
                } else {
                    const int64_t it = qi - nn;
                    while (spre[bs + 1] <= it) ++bs;
                    const BatchAsmInst& I = inst[bs];
                    const int64_t e0 = (it - spre[bs]) * (kNearWarps * kBatchPerWarp) + warp * kBatchPerWarp;
                    for (int u = 0; u < kBatchPerWarp; ++u) {
                        const int64_t e = e0 + u;
                        if (e >= I.n) break;
                        Acc a;
                        self_channels(a, I.elem, I.ld, e, I.k, lane);
                        const Acc t = warp_reduce(a);
                        if (lane == 0) {
                            self_store(t, I.coef, I.ld, I.n, e, nullptr, I.A32, I.lda32, nullptr, I.diag);
                            if (I.amax) {
                                const float2 f = I.A32[e * I.lda32 + e];
                                wam.add(I.amax, fmaxf(fabsf(f.x), fabsf(f.y)));
                            }
                        }
                    }
                }
            }
            if (lane == 0) wam.flush();
            __syncthreads();  // every warp read the state and finished its items
            if (threadIdx.x == 0) {
                st_qi = qi;
                st_bn = bn;
                st_bs = bs;
                if (st_fi >= nf) st_npf = 1 << 30;  // far list done: the rest of the near / self list
            }
            __syncthreads();
        }
    }
}

// rhs_i = free term + self + far tiles + near pairs (BC-induced RHS of tbem.rs:1421-1444).
__global__ void k_rhs_reduce(int64_t n, int64_t ld, const double* __restrict__ coef,
                             const double2* __restrict__ self_rhs,
                             const double2* __restrict__ far_part, int64_t n_tiles,
                             const int64_t* __restrict__ row_ptr,
                             const double2* __restrict__ near_rhs, double2* __restrict__ rhs) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!self_rhs) {
        rhs[i] = make_double2(coef[(int64_t)CF_RHS * ld + i], coef[(int64_t)(CF_RHS + 1) * ld + i]);
        return;
    }
    double2 r = self_rhs[i];
    for (int64_t t = 0; t < n_tiles; ++t) r = cadd(r, far_part[i * n_tiles + t]);
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) r = cadd(r, near_rhs[p]);
    rhs[i] = r;
}

// ---------------------------------------------------------------------------------------------
// Incident plane-wave RHS (incident.rs:216-245, 315-331, 807-833).
// ---------------------------------------------------------------------------------------------
__global__ void k_plane_wave(const double* __restrict__ elem, int64_t n, int64_t ld,
                             const double* __restrict__ dirs, const double2* __restrict__ amps,
                             int64_t r, double k, double hf, double tau, double2 beta,
                             double2* __restrict__ rhs, int accumulate) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * r) return;
    const int64_t i = t / r, q = t % r;
    const double d0 = dirs[3 * q], d1 = dirs[3 * q + 1], d2 = dirs[3 * q + 2];
    const double2 A = amps ? amps[q] : make_double2(1.0, 0.0);
    const double kdx = hf * k * (d0 * E(ECX, i) + d1 * E(ECY, i) + d2 * E(ECZ, i));
    const double kdn = hf * k * (d0 * E(ENX, i) + d1 * E(ENY, i) + d2 * E(ENZ, i));
    double s, c;
    sb_sincos(kdx, &s, &c);
    const double2 p = cmul(A, make_double2(c, s));
    const double2 dpdn = make_double2(-kdn * p.y, kdn * p.x);  // i kdn p
    const double2 bt = cscale(beta, tau);
    const double2 v = make_double2(-(p.x + bt.x * dpdn.x - bt.y * dpdn.y),
                                   -(p.y + bt.x * dpdn.y + bt.y * dpdn.x));
    if (accumulate) {
        rhs[t] = cadd(rhs[t], v);
    } else {
        rhs[t] = v;
    }
}

__global__ void k_sincos(const double* __restrict__ x, int64_t n, double* __restrict__ s,
                         double* __restrict__ c) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) sb_sincos(x[i], s + i, c + i);
}

#undef E

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
static inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Area of a triangle as compute_element_geometry (generators.rs:771-830) takes it: half the
// length of the cross product of the two edges from the first vertex (host input validation).
static double host_triangle_area(const double* nodes, const uint32_t* t) {
    double a1[3], a2[3];
    for (int j = 0; j < 3; ++j) {
        a1[j] = nodes[3 * t[1] + j] - nodes[3 * t[0] + j];
        a2[j] = nodes[3 * t[2] + j] - nodes[3 * t[0] + j];
    }
    const double c0 = a1[1] * a2[2] - a1[2] * a2[1];
    const double c1 = a1[2] * a2[0] - a1[0] * a2[2];
    const double c2 = a1[0] * a2[1] - a1[1] * a2[0];
    return std::sqrt(c0 * c0 + c1 * c1 + c2 * c2) / 2.0;
}

// Near-pair CSR of a mesh built on the device: chunk bounds, per-row counts, the scan (the pair
// count is the one value read back), then the columns (increasing) and the row of every pair.
static void build_near_csr(Mesh& m) {
    const int64_t nchunk = cdiv(m.n, kNearCols);
    const int64_t nblk = cdiv(m.n, kNearRows);
    DevBuf box, counts, total;
    box.alloc(sizeof(double) * 8 * nchunk);
    counts.alloc(sizeof(int64_t) * m.n);
    total.alloc(sizeof(long long));
    k_near_chunk_bounds<<<nchunk, kNearCols>>>(m.elem.as<double>(), m.n, m.ld, box.as<double>()); count_launch();
    SB_CUDA(cudaGetLastError());
    k_near_pass<<<nblk, kNearCols>>>(m.elem.as<double>(), m.n, m.ld, 0, box.as<double>(), counts.as<int64_t>(),
                                     nullptr, nullptr, nullptr); count_launch();
    SB_CUDA(cudaGetLastError());
    m.near_ptr.alloc(sizeof(int64_t) * (m.n + 1));
    k_scan_counts<<<1, kScanThreads>>>(counts.as<int64_t>(), m.n, m.near_ptr.as<int64_t>(), total.as<long long>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    long long nnz = 0;
    SB_CUDA(cudaMemcpy(&nnz, total.p, sizeof(nnz), cudaMemcpyDeviceToHost));
    m.nnz = nnz;
    m.near_col.alloc(sizeof(int32_t) * std::max<int64_t>(m.nnz, 1));
    m.near_row.alloc(sizeof(int32_t) * std::max<int64_t>(m.nnz, 1));
    k_near_pass<<<nblk, kNearCols>>>(m.elem.as<double>(), m.n, m.ld, 1, box.as<double>(), nullptr,
                                     m.near_ptr.as<int64_t>(), m.near_col.as<int32_t>(), m.near_row.as<int32_t>());
    count_launch();
    SB_CUDA(cudaGetLastError());
}

const std::vector<double>& mesh_host_elem(const Mesh& m) {
    std::lock_guard<std::mutex> lock(m.h_elem_mu);
    if (m.h_elem.empty()) {
        std::vector<double> h(static_cast<size_t>(EFIELDS) * m.ld);
        SB_CUDA(cudaSetDevice(m.device));
        SB_CUDA(cudaMemcpy(h.data(), m.elem.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
        m.h_elem.swap(h);
    }
    return m.h_elem;
}

Mesh* mesh_create(const double* nodes, int64_t n_nodes, const uint32_t* tris, int64_t n_tris,
                  int device) {
    SB_REQUIRE(nodes && tris, SB_ERR_INVALID_ARGUMENT, "mesh: null nodes or connectivity");
    SB_REQUIRE(n_nodes >= 3 && n_tris >= 1, SB_ERR_INVALID_ARGUMENT, "mesh: empty mesh");
    SB_REQUIRE(n_tris < (int64_t(1) << 31), SB_ERR_INVALID_ARGUMENT, "mesh: too many elements");
    for (int64_t a = 0; a < 3 * n_nodes; ++a)
        SB_REQUIRE(std::isfinite(nodes[a]), SB_ERR_INVALID_ARGUMENT, "mesh: non-finite node coordinate");
    for (int64_t a = 0; a < 3 * n_tris; ++a)
        SB_REQUIRE(tris[a] < static_cast<uint64_t>(n_nodes), SB_ERR_INVALID_ARGUMENT,
                   "mesh: connectivity index out of range");
    for (int64_t e = 0; e < n_tris; ++e) {
        const double ar = host_triangle_area(nodes, tris + 3 * e);
        SB_REQUIRE(ar > 1e-300 && std::isfinite(ar), SB_ERR_UNSUPPORTED_ELEMENT,
                   "mesh: degenerate triangle " + std::to_string(e));
    }
    int ndev = 0;
    SB_CUDA(cudaGetDeviceCount(&ndev));
    SB_REQUIRE(device >= 0 && device < ndev, SB_ERR_CUDA, "mesh: CUDA device not available");
    SB_CUDA(cudaSetDevice(device));
    ensure_tables(device);
    maybe_inject(SB_INJECT_ALLOC);
    Mesh* m = new Mesh();
    try {
        m->device = device;
        m->n = n_tris;
        m->n_nodes = n_nodes;
        m->n_tiles = cdiv(n_tris, kFarTile);
        m->ld = m->n_tiles * kFarTile;
        m->h_nodes.assign(nodes, nodes + 3 * n_nodes);
        m->h_tris.assign(tris, tris + 3 * n_tris);
        for (int64_t a = 0; a < 3 * n_nodes; ++a) m->coord_bound = std::max(m->coord_bound, std::fabs(nodes[a]));
        m->nodes.alloc(sizeof(double) * 3 * n_nodes);
        m->tris.alloc(sizeof(uint32_t) * 3 * n_tris);
        m->elem.alloc(sizeof(double) * EFIELDS * m->ld);
        m->qp.alloc(sizeof(double) * kQpTileDoubles * m->n_tiles);
        m->qp32.alloc(sizeof(float) * kQ32Fields * m->ld);
        h2d_sync(m->nodes.p, nodes, sizeof(double) * 3 * n_nodes);
        h2d_sync(m->tris.p, tris, sizeof(uint32_t) * 3 * n_tris);
        const int64_t nb = cdiv(m->ld, 256);
        k_element_geometry<<<nb, 256>>>(m->nodes.as<double>(), m->tris.as<uint32_t>(), m->n, m->ld, m->elem.as<double>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        k_far_points<<<nb, 256>>>(m->elem.as<double>(), m->n, m->ld, m->qp.as<double>()); count_launch();
        SB_CUDA(cudaGetLastError());
        k_far_points32<<<nb, 256>>>(m->elem.as<double>(), m->n, m->ld, m->qp32.as<float>()); count_launch();
        SB_CUDA(cudaGetLastError());
        build_near_csr(*m);
        SB_CUDA(cudaDeviceSynchronize());
        m->h_bc_kind.assign(m->n, SB_BC_VELOCITY);
        m->h_bc_value.assign(2 * m->n, 0.0);
        m->h_adm.assign(2 * m->n, 0.0);
        m->h_has_adm.assign(m->n, 0);
    } catch (...) {
        delete m;
        throw;
    }
    return m;
}

// A Quad4 mesh (constant panels): geometry and far points on the device, the same near-pair
// classifier as triangle meshes (it needs only the centres, level-0 centres and areas).
Mesh* mesh_create_quad(const double* nodes, int64_t n_nodes, const uint32_t* quads, int64_t n_quads, int device) {
    SB_REQUIRE(nodes && quads, SB_ERR_INVALID_ARGUMENT, "mesh: null nodes or connectivity");
    SB_REQUIRE(n_nodes >= 4 && n_quads >= 1, SB_ERR_INVALID_ARGUMENT, "mesh: empty mesh");
    SB_REQUIRE(n_quads < (int64_t(1) << 31), SB_ERR_INVALID_ARGUMENT, "mesh: too many elements");
    for (int64_t a = 0; a < 3 * n_nodes; ++a)
        SB_REQUIRE(std::isfinite(nodes[a]), SB_ERR_INVALID_ARGUMENT, "mesh: non-finite node coordinate");
    for (int64_t a = 0; a < 4 * n_quads; ++a)
        SB_REQUIRE(quads[a] < static_cast<uint64_t>(n_nodes), SB_ERR_INVALID_ARGUMENT,
                   "mesh: connectivity index out of range");
    int ndev = 0;
    SB_CUDA(cudaGetDeviceCount(&ndev));
    SB_REQUIRE(device >= 0 && device < ndev, SB_ERR_CUDA, "mesh: CUDA device not available");
    SB_CUDA(cudaSetDevice(device));
    ensure_tables(device);
    maybe_inject(SB_INJECT_ALLOC);
    Mesh* m = new Mesh();
    try {
        m->device = device;
        m->quad = true;
        m->n = n_quads;
        m->n_nodes = n_nodes;
        m->n_tiles = cdiv(n_quads, kFarTile);
        m->ld = m->n_tiles * kFarTile;
        m->h_nodes.assign(nodes, nodes + 3 * n_nodes);
        m->h_tris.assign(quads, quads + 4 * n_quads);
        m->nodes.alloc(sizeof(double) * 3 * n_nodes);
        m->tris.alloc(sizeof(uint32_t) * 4 * n_quads);
        m->elem.alloc(sizeof(double) * EFIELDS * m->ld);
        m->qq.alloc(sizeof(double) * kQuadFar * 7 * m->ld);
        h2d_sync(m->nodes.p, nodes, sizeof(double) * 3 * n_nodes);
        h2d_sync(m->tris.p, quads, sizeof(uint32_t) * 4 * n_quads);
        const int64_t nb = cdiv(m->ld, 256);
        k_quad_geometry<<<nb, 256>>>(m->nodes.as<double>(), m->tris.as<uint32_t>(), m->n, m->ld, m->elem.as<double>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        k_quad_points<<<nb, 256>>>(m->elem.as<double>(), m->n, m->ld, m->qq.as<double>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        m->h_elem.resize(static_cast<size_t>(EFIELDS) * m->ld);
        SB_CUDA(cudaMemcpy(m->h_elem.data(), m->elem.p, sizeof(double) * m->h_elem.size(), cudaMemcpyDeviceToHost));
        for (int64_t e = 0; e < m->n; ++e) {
            const double ar = m->h_elem[static_cast<size_t>(EAREA) * m->ld + e];
            SB_REQUIRE(ar > 1e-300 && std::isfinite(ar), SB_ERR_UNSUPPORTED_ELEMENT,
                       "mesh: degenerate quadrilateral " + std::to_string(e));
        }
        build_near_csr(*m);
        SB_CUDA(cudaDeviceSynchronize());
        m->h_bc_kind.assign(m->n, SB_BC_VELOCITY);
        m->h_bc_value.assign(2 * m->n, 0.0);
        m->h_adm.assign(2 * m->n, 0.0);
        m->h_has_adm.assign(m->n, 0);
    } catch (...) {
        delete m;
        throw;
    }
    return m;
}

// The constant-panel system of a Quad4 mesh (complex128): coefficients, far pairs, near pairs,
// self terms (rigid, zero-pressure or admittance surfaces).
void assemble_quad(Operator& op, const sb_physics& ph, double beta_re, double beta_im) {
    Mesh& m = *op.mesh;
    SB_CUDA(cudaSetDevice(m.device));
    SB_REQUIRE(!m.any_bc_value, SB_ERR_INVALID_ARGUMENT,
               "Quad4 mesh: prescribed boundary values are not supported (rigid, zero-pressure or admittance "
               "surfaces)");
    SB_REQUIRE(op.A64.p && !op.A32.p, SB_ERR_INVALID_ARGUMENT, "Quad4 mesh: only SB_PRECISION_FP64 is supported");
    maybe_inject(SB_INJECT_LAUNCH);
    const int64_t n = m.n, ld = m.ld;
    const cudaStream_t s = op.stream;
    if (!op.coef.p) op.coef.alloc(sizeof(double) * CF_FIELDS * ld);
    if (!op.diag.p) op.diag.alloc(sizeof(double2) * n);
    if (!op.rhs.p) {
        op.rhs.alloc(sizeof(double2) * n);
        SB_CUDA(cudaMemsetAsync(op.rhs.p, 0, sizeof(double2) * n, s));
    }
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, s));
    k_coefficients<<<cdiv(ld, 256), 256, 0, s>>>(n, ld, m.bc_kind.as<int32_t>(), m.bc_value.as<double2>(),
                                                 m.has_adm.as<uint8_t>(), m.adm.as<double2>(), ph.tau,
                                                 ph.pressure_factor, make_double2(beta_re, beta_im),
                                                 op.coef.as<double>());
    count_launch();
    const double k = ph.harmonic_factor * ph.wave_number;
    double2* A = op.A64.as<double2>();
    {
        ProfScope prof(SB_PROF_FAR, s);
        const size_t sm = sizeof(double) * (kQuadFar * 7 * kQuadTile + kQuadRows * 6);
        SB_CUDA(cudaFuncSetAttribute(k_quad_far, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
        dim3 grid(static_cast<unsigned>(cdiv(n, kQuadTile)), static_cast<unsigned>(cdiv(n, kQuadRows)));
        k_quad_far<<<grid, kQuadTile, sm, s>>>(m.qq.as<double>(), m.elem.as<double>(), n, ld, op.coef.as<double>(), k,
                                               A);
        count_launch();
        SB_CUDA(cudaGetLastError());
    }
    if (m.nnz > 0) {
        ProfScope prof(SB_PROF_NEAR, s);
        k_quad_near<<<cdiv(m.nnz, kNearWarps), 32 * kNearWarps, 0, s>>>(m.elem.as<double>(), n, ld,
                                                                       m.near_ptr.as<int64_t>(),
                                                                       m.near_col.as<int32_t>(), m.nnz,
                                                                       op.coef.as<double>(), k, A);
        count_launch();
        SB_CUDA(cudaGetLastError());
    }
    {
        ProfScope prof(SB_PROF_SELF, s);
        k_quad_self<<<cdiv(n, 4), 128, 0, s>>>(m.elem.as<double>(), n, ld, op.coef.as<double>(), k, A,
                                               op.diag.as<double2>());
        count_launch();
        SB_CUDA(cudaGetLastError());
    }
    SB_CUDA(cudaEventRecord(e1, s));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    op.last_assembly_ms = ms;
    op.phys = ph;
    op.beta_re = beta_re;
    op.beta_im = beta_im;
}

void mesh_set_bc(Mesh& m, const int32_t* kind, const sb_complex* value, const uint8_t* has_adm,
                 const sb_complex* adm) {
    if (!kind && !value && !has_adm && !adm) {
        // The default (rigid: velocity 0, no admittance everywhere): every field is zero.
        static_assert(SB_BC_VELOCITY == 0, "the rigid default is the zero kind");
        SB_CUDA(cudaSetDevice(m.device));
        m.any_bc_value = false;
        m.any_adm = false;
        m.h_bc_kind.assign(m.n, SB_BC_VELOCITY);
        m.h_bc_value.assign(2 * m.n, 0.0);
        m.h_has_adm.assign(m.n, 0);
        m.h_adm.assign(2 * m.n, 0.0);
        if (!m.bc_kind.p) {
            m.bc_kind.alloc(sizeof(int32_t) * m.n);
            m.bc_value.alloc(sizeof(double2) * m.n);
            m.has_adm.alloc(m.n);
            m.adm.alloc(sizeof(double2) * m.n);
        }
        SB_CUDA(cudaMemset(m.bc_kind.p, 0, sizeof(int32_t) * m.n));
        SB_CUDA(cudaMemset(m.bc_value.p, 0, sizeof(double2) * m.n));
        SB_CUDA(cudaMemset(m.has_adm.p, 0, m.n));
        memset_sync(m.adm.p, 0, sizeof(double2) * m.n);
        return;
    }
    for (int64_t e = 0; e < m.n; ++e) {
        const int k = kind ? kind[e] : SB_BC_VELOCITY;
        SB_REQUIRE(k == SB_BC_VELOCITY || k == SB_BC_PRESSURE, SB_ERR_INVALID_ARGUMENT,
                   "bc: kind must be velocity (0) or pressure (1)");
        if (value) SB_REQUIRE(std::isfinite(value[e].re) && std::isfinite(value[e].im),
                              SB_ERR_INVALID_ARGUMENT, "bc: non-finite value");
        if (adm && has_adm && has_adm[e])
            SB_REQUIRE(std::isfinite(adm[e].re) && std::isfinite(adm[e].im),
                       SB_ERR_INVALID_ARGUMENT, "bc: non-finite admittance");
    }
    SB_CUDA(cudaSetDevice(m.device));
    m.any_bc_value = false;
    m.any_adm = false;
    for (int64_t e = 0; e < m.n; ++e) {
        m.h_bc_kind[e] = kind ? kind[e] : SB_BC_VELOCITY;
        m.h_bc_value[2 * e] = value ? value[e].re : 0.0;
        m.h_bc_value[2 * e + 1] = value ? value[e].im : 0.0;
        m.h_has_adm[e] = (has_adm && has_adm[e]) ? 1 : 0;
        m.h_adm[2 * e] = (adm && m.h_has_adm[e]) ? adm[e].re : 0.0;
        m.h_adm[2 * e + 1] = (adm && m.h_has_adm[e]) ? adm[e].im : 0.0;
        if (std::hypot(m.h_bc_value[2 * e], m.h_bc_value[2 * e + 1]) > 1e-15) m.any_bc_value = true;
        if (m.h_has_adm[e]) m.any_adm = true;
    }
    if (!m.bc_kind.p) {
        m.bc_kind.alloc(sizeof(int32_t) * m.n);
        m.bc_value.alloc(sizeof(double2) * m.n);
        m.has_adm.alloc(m.n);
        m.adm.alloc(sizeof(double2) * m.n);
    }
    h2d_sync(m.bc_kind.p, m.h_bc_kind.data(), sizeof(int32_t) * m.n);
    h2d_sync(m.bc_value.p, m.h_bc_value.data(), sizeof(double2) * m.n);
    h2d_sync(m.has_adm.p, m.h_has_adm.data(), m.n);
    h2d_sync(m.adm.p, m.h_adm.data(), sizeof(double2) * m.n);
}

// The near pairs' subdivision plan (k_near_plan): recorded on the second near-pair assembly of a
// mesh (one assembly of a new mesh keeps the subdividing kernel, which costs less than recording
// and evaluating), and only while the device keeps 2 GiB free beside it. Runs on `st`, reads the
// leaf count back once and waits for the plan before marking it ready, so that an assembly of
// another operator of the same mesh on another stream finds it complete.
static void near_plan_prepare(Mesh& m, int device, cudaStream_t st) {
    std::lock_guard<std::mutex> lock(m.near_plan_mu);
    if (m.near_plan_ready || m.near_plan_declined || m.quad || ++m.near_assemblies < 2) return;
    const unsigned grid = near_grid(m.nnz, device);
    DevBuf counts, total;
    counts.alloc(sizeof(int64_t) * m.nnz);
    total.alloc(sizeof(long long));
    m.near_plan_off.alloc(sizeof(int64_t) * (m.nnz + 1));
    k_near_plan<0><<<grid, 32 * kNearWarps, 0, st>>>(m.elem.as<double>(), m.n, m.ld, m.near_row.as<int32_t>(),
                                                     m.near_col.as<int32_t>(), m.nnz, counts.as<int64_t>(), nullptr,
                                                     nullptr);
    count_launch();
    k_scan_counts<<<1, kScanThreads, 0, st>>>(counts.as<int64_t>(), m.nnz, m.near_plan_off.as<int64_t>(),
                                              total.as<long long>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    long long leaves = 0;
    SB_CUDA(cudaMemcpyAsync(&leaves, total.p, sizeof(leaves), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    const size_t bytes = sizeof(NearLeaf) * static_cast<size_t>(std::max<long long>(leaves, 1));
    size_t free_b = 0, total_b = 0;
    SB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (free_b < bytes + (size_t(2) << 30)) {
        m.near_plan_off.release();
        m.near_plan_declined = true;
        return;
    }
    m.near_plan.alloc(bytes);
    k_near_plan<1><<<grid, 32 * kNearWarps, 0, st>>>(m.elem.as<double>(), m.n, m.ld, m.near_row.as<int32_t>(),
                                                     m.near_col.as<int32_t>(), m.nnz, nullptr,
                                                     m.near_plan_off.as<int64_t>(), m.near_plan.as<NearLeaf>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(st));
    m.near_plan_ready = true;
}

void assemble(Operator& op, const sb_physics& ph, double beta_re, double beta_im) {
    if (op.mesh->quad) {
        assemble_quad(op, ph, beta_re, beta_im);
        return;
    }
    Mesh& m = *op.mesh;
    SB_CUDA(cudaSetDevice(m.device));
    maybe_inject(SB_INJECT_LAUNCH);
    const int64_t n = m.n, ld = m.ld;
    const bool with_rhs = m.any_bc_value;
    if (!op.coef.p) op.coef.alloc(sizeof(double) * CF_FIELDS * ld);
    if (with_rhs) {
        if (!op.far_part.p) op.far_part.alloc(sizeof(double2) * n * m.n_tiles);
        if (!op.near_rhs.p) op.near_rhs.alloc(sizeof(double2) * std::max<int64_t>(m.nnz, 1));
        if (!op.self_rhs.p) op.self_rhs.alloc(sizeof(double2) * n);
    }
    if (!op.rhs.p) op.rhs.alloc(sizeof(double2) * n);
    if (!op.diag.p) op.diag.alloc(sizeof(double2) * n);
    if (!op.status.p) op.status.alloc(sizeof(int));
    DevBuf& status = op.status;
    SB_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int), op.stream));
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, op.stream));
    const double2 beta = make_double2(beta_re, beta_im);
    k_coefficients<<<cdiv(ld, 256), 256, 0, op.stream>>>(
        n, ld, m.bc_kind.as<int32_t>(), m.bc_value.as<double2>(), m.has_adm.as<uint8_t>(),
        m.adm.as<double2>(), ph.tau, ph.pressure_factor, beta, op.coef.as<double>()); count_launch();
    SB_CUDA(cudaGetLastError());
    const double k = ph.harmonic_factor * ph.wave_number;
    const bool mixed = op.precision == SB_PRECISION_FP32;
    const bool f32 = op.precision == SB_PRECISION_FP64_FP32;
    double2* A64 = mixed ? nullptr : op.A64.as<double2>();
    float2* A32 = (f32 || mixed) ? op.A32.as<float2>() : nullptr;
    // Near pairs and self terms write entries disjoint from the far tiles. With the FP64 far kernel
    // they run on the side stream, concurrently with it (N = 20480: 38.9 -> 37.3 ms per assembly);
    // the FP32 far kernel fills every SM's register file (4 CTAs x 128 threads x 128 registers),
    // so a concurrent near kernel only time-shares with it, and they run before it on the
    // operator's stream. The right-hand-side reduction waits for both.
    const bool overlap = !mixed;
    if (overlap) {
        op.side.ensure();
        op.side.begin(op.stream);
    }
    auto near_and_self = [&](cudaStream_t st) {
        if (m.nnz > 0) {
            near_plan_prepare(m, op.device, st);
            ProfScope prof(SB_PROF_NEAR, st);
            bool cached;
            {
                std::lock_guard<std::mutex> lock(m.near_plan_mu);
                cached = m.near_plan_ready;
            }
            if (cached)
                k_near_cached<<<near_grid(m.nnz, op.device), 32 * kNearWarps, 0, st>>>(
                    m.elem.as<double>(), n, ld, m.near_row.as<int32_t>(), m.near_col.as<int32_t>(), m.nnz,
                    m.near_plan_off.as<int64_t>(), m.near_plan.as<NearLeaf>(), op.coef.as<double>(), k, A64, A32,
                    op.lda32, with_rhs ? op.near_rhs.as<double2>() : nullptr);
            else
                k_near<<<near_grid(m.nnz, op.device), 32 * kNearWarps, 0, st>>>(
                    m.elem.as<double>(), n, ld, m.near_row.as<int32_t>(), m.near_col.as<int32_t>(), m.nnz,
                    op.coef.as<double>(), k, A64, A32, op.lda32, with_rhs ? op.near_rhs.as<double2>() : nullptr);
            count_launch();
            SB_CUDA(cudaGetLastError());
        }
        ProfScope prof(SB_PROF_SELF, st);
        k_self<<<cdiv(n, 4), 128, 0, st>>>(m.elem.as<double>(), n, ld, op.coef.as<double>(), k, A64, A32, op.lda32,
                                           with_rhs ? op.self_rhs.as<double2>() : nullptr, op.diag.as<double2>());
        count_launch();
        SB_CUDA(cudaGetLastError());
    };
    if (overlap) near_and_self(op.side.s);
    if (mixed) {
        // Near pairs and self terms first; with complex-half inner products the rows' scales come
        // from those entries and the far kernel writes the copy as it writes the matrix.
        near_and_self(op.stream);
        const bool half = op.inner == SB_INNER_FP16;
        uint32_t* A16 = nullptr;
        float* hs = nullptr;
        int* hflag = nullptr;
        if (half) {
            half_alloc(op);
            A16 = op.A16.as<uint32_t>();
            hs = op.half_scale.as<float>();
            hflag = op.half_flag.as<int>();
            SB_CUDA(cudaMemsetAsync(hflag, 0, sizeof(int), op.stream));
            ProfScope prof(SB_PROF_OTHER, op.stream);
            k_near_row_scale<<<cdiv(n, 256), 256, 0, op.stream>>>(A32, op.lda32, n, m.near_ptr.as<int64_t>(),
                                                                  m.near_col.as<int32_t>(), hs, hs + n);
            count_launch();
        }
        {
            ProfScope prof(SB_PROF_FAR, op.stream);
            dim3 grid(static_cast<unsigned>(m.n_tiles), static_cast<unsigned>(cdiv(n, kFar32Rows)));
            if (with_rhs)
                k_far32<true><<<grid, kFarTile, 0, op.stream>>>(m.qp32.as<float>(), m.elem.as<double>(), n, ld,
                                                                 op.coef.as<double>(), k, m.coord_bound, A32, op.lda32,
                                                                 op.far_part.as<double2>(), m.n_tiles, nullptr, A16,
                                                                 op.lda16, hs, hflag);
            else
                k_far32<false><<<grid, kFarTile, 0, op.stream>>>(m.qp32.as<float>(), m.elem.as<double>(), n, ld,
                                                                  op.coef.as<double>(), k, m.coord_bound, A32,
                                                                  op.lda32, nullptr,
                                                                  m.n_tiles, nullptr, A16, op.lda16, hs, hflag);
            count_launch();
            SB_CUDA(cudaGetLastError());
        }
        if (half) {
            ProfScope prof(SB_PROF_OTHER, op.stream);
            k_near_to_half<<<cdiv(n, 256), 256, 0, op.stream>>>(A32, op.lda32, n, m.near_ptr.as<int64_t>(),
                                                                m.near_col.as<int32_t>(), hs, A16, op.lda16, hflag);
            count_launch();
            SB_CUDA(cudaGetLastError());
            op.half_valid = true;
            op.half_check = true;
        }
    } else {
        ProfScope prof(SB_PROF_FAR, op.stream);
        dim3 grid(static_cast<unsigned>(m.n_tiles), static_cast<unsigned>(cdiv(n, kFarRows)));
        const size_t sm = sizeof(double) * (kQpTileDoubles + kFarRows * 6);
        auto launch = [&](auto kern) {
            SB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
            kern<<<grid, kFarTile, sm, op.stream>>>(m.qp.as<double>(), m.elem.as<double>(), n, ld,
                                                    op.coef.as<double>(), k, A64, A32, op.lda32,
                                                    with_rhs ? op.far_part.as<double2>() : nullptr,
                                                    m.n_tiles, status.as<int>()); count_launch();
        };
        if (with_rhs) {
            if (f32) launch(k_far<true, true>); else launch(k_far<true, false>);
        } else {
            if (f32) launch(k_far<false, true>); else launch(k_far<false, false>);
        }
        SB_CUDA(cudaGetLastError());
    }
    if (overlap) op.side.end(op.stream);
    k_rhs_reduce<<<cdiv(n, 256), 256, 0, op.stream>>>(n, ld, op.coef.as<double>(),
                                                       with_rhs ? op.self_rhs.as<double2>() : nullptr,
                                                       with_rhs ? op.far_part.as<double2>() : nullptr,
                                                       m.n_tiles, m.near_ptr.as<int64_t>(),
                                                       with_rhs ? op.near_rhs.as<double2>() : nullptr,
                                                       op.rhs.as<double2>()); count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaEventRecord(e1, op.stream));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    op.last_assembly_ms = ms;
    int st = 0;
    SB_CUDA(cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, op.stream));
    SB_CUDA(cudaStreamSynchronize(op.stream));
    SB_REQUIRE(st == 0, SB_ERR_DEVICE_CHECK, "assembly: shared-memory staging did not complete");
    op.phys = ph;
    op.beta_re = beta_re;
    op.beta_im = beta_im;
}

// Scales the per-element coefficients (matrix weights, RHS weights, free terms) by `sign`: every
// entry of the stabilised discontinuous systems is sign times the unsigned one
// (build_tbem_system_discontinuous_stabilized, tbem.rs:2810-2990).
__global__ void k_scale_coef(double* __restrict__ coef, int64_t count, double sign) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < count) coef[t] *= sign;
}

template <int NB>
static void assemble_disc_nb(Operator& op, const sb_physics& ph, double beta_re, double beta_im) {
    Mesh& m = *op.mesh;
    const int64_t n = m.n, ld = m.ld, n3 = NB * n;
    const cudaStream_t s = op.stream;
    if (!op.coef.p) op.coef.alloc(sizeof(double) * CF_FIELDS * ld);
    if (!op.diag.p) op.diag.alloc(sizeof(double2) * n3);
    if (!op.rhs.p) {
        op.rhs.alloc(sizeof(double2) * n3);
        SB_CUDA(cudaMemsetAsync(op.rhs.p, 0, sizeof(double2) * n3, s));
    }
    if (!op.lin_cp.p) {
        op.lin_cp.alloc(sizeof(double) * 3 * n3);
        op.lin_cn.alloc(sizeof(double) * 3 * n3);
        k_lin_points<NB><<<cdiv(n3, 256), 256, 0, s>>>(m.elem.as<double>(), n, ld, op.lin_cp.as<double>(),
                                                       op.lin_cn.as<double>());
        count_launch();
        DevBuf counts;
        counts.alloc(sizeof(int64_t) * (n3 + 1));
        const int64_t nblk = cdiv(n3, kNearRows);
        k_lin_near_pass<NB><<<nblk, 256, 0, s>>>(m.elem.as<double>(), n, ld, op.lin_cp.as<double>(), 0,
                                                 counts.as<int64_t>(), nullptr, nullptr);
        count_launch();
        SB_CUDA(cudaGetLastError());
        std::vector<int64_t> cnt(n3), ptr(n3 + 1);
        SB_CUDA(cudaMemcpyAsync(cnt.data(), counts.p, sizeof(int64_t) * n3, cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        ptr[0] = 0;
        for (int64_t r = 0; r < n3; ++r) ptr[r + 1] = ptr[r] + cnt[r];
        op.lin_nnz = ptr[n3];
        op.lin_ptr.alloc(sizeof(int64_t) * (n3 + 1));
        SB_CUDA(cudaMemcpyAsync(op.lin_ptr.p, ptr.data(), sizeof(int64_t) * (n3 + 1), cudaMemcpyHostToDevice, s));
        op.lin_col.alloc(sizeof(int32_t) * std::max<int64_t>(op.lin_nnz, 1));
        k_lin_near_pass<NB><<<nblk, 256, 0, s>>>(m.elem.as<double>(), n, ld, op.lin_cp.as<double>(), 1, nullptr,
                                                 op.lin_ptr.as<int64_t>(), op.lin_col.as<int32_t>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        SB_CUDA(cudaStreamSynchronize(s));
    }
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, s));
    k_coefficients<<<cdiv(ld, 256), 256, 0, s>>>(n, ld, m.bc_kind.as<int32_t>(), m.bc_value.as<double2>(),
                                                 m.has_adm.as<uint8_t>(), m.adm.as<double2>(), ph.tau,
                                                 ph.pressure_factor, make_double2(beta_re, beta_im),
                                                 op.coef.as<double>());
    count_launch();
    if (op.sign != 1.0) {
        k_scale_coef<<<cdiv(CF_FIELDS * ld, 256), 256, 0, s>>>(op.coef.as<double>(), CF_FIELDS * ld, op.sign);
        count_launch();
    }
    const double k = ph.harmonic_factor * ph.wave_number;
    double2* A = op.A64.as<double2>();
    {
        ProfScope prof(SB_PROF_FAR, s);
        const size_t sm = sizeof(double) * (kQpTileDoubles + kLinRows * 6);
        SB_CUDA(cudaFuncSetAttribute(k_lin_far<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(sm)));
        dim3 grid(static_cast<unsigned>(m.n_tiles), static_cast<unsigned>(cdiv(n3, kLinRows)));
        k_lin_far<NB><<<grid, kFarTile, sm, s>>>(m.qp.as<double>(), m.elem.as<double>(), n, ld,
                                                 op.lin_cp.as<double>(), op.coef.as<double>(), k, A);
        count_launch();
        SB_CUDA(cudaGetLastError());
    }
    if (op.lin_nnz > 0) {
        ProfScope prof(SB_PROF_NEAR, s);
        k_lin_near<NB><<<cdiv(op.lin_nnz, kNearWarps), 32 * kNearWarps, 0, s>>>(
            m.elem.as<double>(), n, ld, op.lin_cp.as<double>(), op.lin_ptr.as<int64_t>(), op.lin_col.as<int32_t>(),
            op.lin_nnz, op.coef.as<double>(), k, A);
        count_launch();
        SB_CUDA(cudaGetLastError());
    }
    {
        ProfScope prof(SB_PROF_SELF, s);
        k_lin_self<NB><<<cdiv(n3, 4), 128, 0, s>>>(m.elem.as<double>(), n, ld, op.lin_cp.as<double>(),
                                                  op.coef.as<double>(), k, A, op.diag.as<double2>());
        count_launch();
        SB_CUDA(cudaGetLastError());
    }
    SB_CUDA(cudaEventRecord(e1, s));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    op.last_assembly_ms = ms;
}

// build_tbem_system_linear / build_tbem_system_discontinuous_stabilized on the device: collocation
// points and the near-pair CSR of the NB n rows once per operator, then coefficients (times the
// operator's sign), far tiles, near pairs and self rows per assembly.
void assemble_discontinuous(Operator& op, const sb_physics& ph, double beta_re, double beta_im) {
    Mesh& m = *op.mesh;
    SB_CUDA(cudaSetDevice(m.device));
    SB_REQUIRE(!m.any_bc_value, SB_ERR_INVALID_ARGUMENT,
               "discontinuous bases: prescribed boundary values are not supported (rigid, pressure-release "
               "with zero value, or admittance surfaces)");
    maybe_inject(SB_INJECT_LAUNCH);
    if (op.basis == SB_BASIS_QUADRATIC)
        assemble_disc_nb<6>(op, ph, beta_re, beta_im);
    else
        assemble_disc_nb<3>(op, ph, beta_re, beta_im);
    op.phys = ph;
    op.beta_re = beta_re;
    op.beta_im = beta_im;
}

void lin_collocation(const Mesh& m, int basis, double* cp_dev, double* cn_dev) {
    SB_CUDA(cudaSetDevice(m.device));
    if (basis == SB_BASIS_QUADRATIC)
        k_lin_points<6><<<cdiv(6 * m.n, 256), 256>>>(m.elem.as<double>(), m.n, m.ld, cp_dev, cn_dev);
    else
        k_lin_points<3><<<cdiv(3 * m.n, 256), 256>>>(m.elem.as<double>(), m.n, m.ld, cp_dev, cn_dev);
    count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaDeviceSynchronize());
}

void incident_plane_wave_at(int device, const double* pts_dev, const double* nrm_dev, int64_t np, int64_t stride,
                            const sb_physics& ph, double beta_re, double beta_im, const double* dirs_host,
                            const double* amps_host, int64_t r, double2* rhs_dev, cudaStream_t s) {
    SB_CUDA(cudaSetDevice(device));
    DevBuf dd, da;
    dd.alloc(sizeof(double) * 3 * r);
    SB_CUDA(cudaMemcpyAsync(dd.p, dirs_host, sizeof(double) * 3 * r, cudaMemcpyHostToDevice, s));
    if (amps_host) {
        da.alloc(sizeof(double2) * r);
        SB_CUDA(cudaMemcpyAsync(da.p, amps_host, sizeof(double2) * r, cudaMemcpyHostToDevice, s));
    }
    ProfScope prof(SB_PROF_OTHER, s);
    k_plane_wave_at<<<cdiv(np * r, 256), 256, 0, s>>>(pts_dev, nrm_dev, np, stride, dd.as<double>(),
                                                      amps_host ? da.as<double2>() : nullptr, r, ph.wave_number,
                                                      ph.harmonic_factor, ph.tau, make_double2(beta_re, beta_im),
                                                      rhs_dev);
    count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(s));
}

void assemble_batch(const std::vector<BatchAsmInst>& h_inst, const BatchAsmInst* d_inst, DevBuf& pre_buf,
                    cudaStream_t s, int device, SideStream* side, int far_per_sm) {
    const int ninst = static_cast<int>(h_inst.size());
    std::vector<int64_t> pre(3 * (ninst + 1), 0);
    for (int b = 0; b < ninst; ++b) {
        const BatchAsmInst& I = h_inst[b];
        pre[b + 1] = pre[b] + I.n_tiles * cdiv(I.n, kFar32Rows);
        pre[(ninst + 1) + b + 1] = pre[(ninst + 1) + b] + cdiv(I.nnz, kNearWarps * kBatchPerWarp);
        pre[2 * (ninst + 1) + b + 1] = pre[2 * (ninst + 1) + b] + cdiv(I.n, kNearWarps * kBatchPerWarp);
    }
    if (pre_buf.bytes < sizeof(int64_t) * pre.size()) pre_buf.alloc(sizeof(int64_t) * pre.size());
    SB_CUDA(cudaMemcpyAsync(pre_buf.p, pre.data(), sizeof(int64_t) * pre.size(), cudaMemcpyHostToDevice, s));
    const int smem = static_cast<int>(sizeof(BatchAsmSmem));
    for (auto kern : {k_assemble_batch<0>, k_assemble_batch<1>, k_assemble_batch<2>})
        SB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_assemble_batch<0>, kFarTile, smem));
    per_sm = std::max(per_sm, 1);
    const int64_t sms = device_sm_count(device);
    const int64_t nf = pre[ninst], nq = pre[2 * (ninst + 1) - 1] + pre[3 * (ninst + 1) - 1];
    const int64_t* d_pre = pre_buf.as<int64_t>();
    if (!side || far_per_sm <= 0) {
        // one launch: every CTA alternates far tiles with near / self items (both lists end together)
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(nf + nq, per_sm * sms));
        const int near_per_far = static_cast<int>(std::max<int64_t>(1, nf > 0 ? cdiv(nq, nf) : 1));
        ProfScope prof(SB_PROF_FAR, s);
        k_assemble_batch<0><<<static_cast<unsigned>(grid), kFarTile, smem, s>>>(d_inst, ninst, d_pre, near_per_far);
        count_launch();
        SB_CUDA(cudaGetLastError());
        return;
    }
    // Two persistent launches: the far tiles of every instance on far_per_sm CTA slots per SM, the
    // near pairs and self elements on the remaining slots (on the high-priority side stream; with
    // far_per_sm = all of them, its CTAs take the slots the far launch's CTAs free at its end). A
    // CTA of a persistent launch keeps its slot to the end, so the split is fixed.
    const int far_slots = std::min(far_per_sm, per_sm);
    const int near_slots = far_slots < per_sm ? per_sm - far_slots : per_sm;
    side->ensure();
    side->begin(s);
    {
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(nf, far_slots * sms));
        ProfScope prof(SB_PROF_FAR, s);
        k_assemble_batch<1><<<static_cast<unsigned>(grid), kFarTile, smem, s>>>(d_inst, ninst, d_pre, 1);
        count_launch();
    }
    {
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(nq, near_slots * sms));
        ProfScope prof(SB_PROF_NEAR, side->s);
        k_assemble_batch<2><<<static_cast<unsigned>(grid), kFarTile, smem, side->s>>>(d_inst, ninst, d_pre, 1);
        count_launch();
    }
    SB_CUDA(cudaGetLastError());
    side->end(s);
}

void assemble_batch_streams(const std::vector<BatchAsmInst>& h_inst, cudaStream_t s, SideStream& side,
                            unsigned* amax) {
    if (amax) SB_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned) * 4 * h_inst.size(), s));
    side.ensure();
    side.begin(s);
    int dev = 0;
    SB_CUDA(cudaGetDevice(&dev));
    const int sms = device_sm_count(dev);
    for (size_t b = 0; b < h_inst.size(); ++b) {
        const BatchAsmInst& I = h_inst[b];
        if (I.nnz > 0) {
            bool cached = false;
            if (I.mesh) {
                near_plan_prepare(*I.mesh, dev, side.s);
                std::lock_guard<std::mutex> lock(I.mesh->near_plan_mu);
                cached = I.mesh->near_plan_ready;
            }
            ProfScope prof(SB_PROF_NEAR, side.s);
            if (cached)
                k_near_cached<<<near_grid(I.nnz, dev), 32 * kNearWarps, 0, side.s>>>(
                    I.elem, I.n, I.ld, I.near_row, I.near_col, I.nnz, I.mesh->near_plan_off.as<int64_t>(),
                    I.mesh->near_plan.as<NearLeaf>(), I.coef, I.k, nullptr, I.A32, I.lda32, nullptr);
            else
                k_near<<<near_grid(I.nnz, dev), 32 * kNearWarps, 0, side.s>>>(I.elem, I.n, I.ld, I.near_row,
                                                                            I.near_col, I.nnz, I.coef, I.k, nullptr,
                                                                            I.A32, I.lda32, nullptr);
            count_launch();
        }
        ProfScope prof(SB_PROF_SELF, side.s);
        k_self<<<cdiv(I.n, 4), 128, 0, side.s>>>(I.elem, I.n, I.ld, I.coef, I.k, nullptr, I.A32, I.lda32, nullptr,
                                                I.diag);
        count_launch();
        if (amax) {
            const unsigned g = static_cast<unsigned>(std::min<int64_t>(cdiv(I.n, 256), 4 * sms));
            k_near_absmax<<<g, 256, 0, side.s>>>(I.A32, I.lda32, I.n, I.near_ptr, I.near_col, amax + 4 * b);
            count_launch();
        }
    }
    SB_CUDA(cudaGetLastError());
    for (size_t b = 0; b < h_inst.size(); ++b) {
        const BatchAsmInst& I = h_inst[b];
        ProfScope prof(SB_PROF_FAR, s);
        dim3 grid(static_cast<unsigned>(I.n_tiles), static_cast<unsigned>(cdiv(I.n, kFar32Rows)));
        k_far32<false><<<grid, kFarTile, 0, s>>>(I.qp32, I.elem, I.n, I.ld, I.coef, I.k, I.coord_bound, I.A32,
                                                 I.lda32, nullptr,
                                                 I.n_tiles, amax ? amax + 4 * b : nullptr, nullptr, 0, nullptr,
                                                 nullptr);
        count_launch();
    }
    SB_CUDA(cudaGetLastError());
    side.end(s);
}

void SideStream::ensure() {
    if (s) return;
    int least = 0, greatest = 0;
    SB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    SB_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest));
    SB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    SB_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
}

void SideStream::release() {
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (s) cudaStreamDestroy(s);
    s = nullptr;
    fork = join = nullptr;
}

void SideStream::begin(cudaStream_t main) {
    SB_CUDA(cudaEventRecord(fork, main));
    SB_CUDA(cudaStreamWaitEvent(s, fork, 0));
}

void SideStream::end(cudaStream_t main) {
    SB_CUDA(cudaEventRecord(join, s));
    SB_CUDA(cudaStreamWaitEvent(main, join, 0));
}

void coefficients_for(const Mesh& m, const sb_physics& ph, double beta_re, double beta_im, double* coef,
                      cudaStream_t s) {
    k_coefficients<<<cdiv(m.ld, 256), 256, 0, s>>>(m.n, m.ld, m.bc_kind.as<int32_t>(), m.bc_value.as<double2>(),
                                                   m.has_adm.as<uint8_t>(), m.adm.as<double2>(), ph.tau,
                                                   ph.pressure_factor, make_double2(beta_re, beta_im), coef);
    count_launch();
    SB_CUDA(cudaGetLastError());
}

int coefficient_fields() { return CF_FIELDS; }

void incident_plane_wave(const Mesh& m, const sb_physics& ph, double beta_re, double beta_im,
                         const double* dirs_host, const double* amps_host, int64_t r,
                         double2* rhs_dev, cudaStream_t s, bool accumulate) {
    SB_CUDA(cudaSetDevice(m.device));
    DevBuf dd, da;
    dd.alloc(sizeof(double) * 3 * r);
    SB_CUDA(cudaMemcpyAsync(dd.p, dirs_host, sizeof(double) * 3 * r, cudaMemcpyHostToDevice, s));
    if (amps_host) {
        da.alloc(sizeof(double2) * r);
        SB_CUDA(cudaMemcpyAsync(da.p, amps_host, sizeof(double2) * r, cudaMemcpyHostToDevice, s));
    }
    const int64_t tot = m.n * r;
    ProfScope prof(SB_PROF_OTHER, s);
    k_plane_wave<<<cdiv(tot, 256), 256, 0, s>>>(m.elem.as<double>(), m.n, m.ld, dd.as<double>(),
                                                 amps_host ? da.as<double2>() : nullptr, r,
                                                 ph.wave_number, ph.harmonic_factor, ph.tau,
                                                 make_double2(beta_re, beta_im), rhs_dev, accumulate ? 1 : 0); count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(s));
}

void device_sincos(int device, const double* x, int64_t n, double* s, double* c) {
    SB_CUDA(cudaSetDevice(device));
    DevBuf dx, ds, dc;
    dx.alloc(sizeof(double) * n);
    ds.alloc(sizeof(double) * n);
    dc.alloc(sizeof(double) * n);
    h2d_sync(dx.p, x, sizeof(double) * n);
    k_sincos<<<cdiv(n, 256), 256>>>(dx.as<double>(), n, ds.as<double>(), dc.as<double>()); count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaMemcpy(s, ds.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    SB_CUDA(cudaMemcpy(c, dc.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
}

}  // namespace sb
