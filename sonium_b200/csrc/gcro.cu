// GCRO-DR: Krylov subspace recycling for a sequence of related systems (consecutive frequencies
// of a sweep), FP64 on the device.
//
// Reference: gcro_dr_core (crates/sonium-solvers/crates/sonium-solvers-iterative/src/gcro_dr.rs:
// 339-760), build_c_r (:769-850), solve_upper_triangular_dense (:853-870), unapply_givens_local
// (:874-900), update_recycled_subspace (:922-1050), solve_with_g_top_h (:1057-1090); the
// subspace object GcroDrSubspace (:65-110). The algorithm is Parks, de Sturler, Mackey, Johnson,
// Maiti, "Recycling Krylov subspaces for sequences of linear systems", SIAM J. Sci. Comput. 28(5)
// (2006), in the reference's form: the recycled basis U is kept across solves, C = orth(M^-1 A U)
// (M^-1 A U = C R) is rebuilt for every new operator, every Arnoldi vector is projected against C
// twice (unconditionally) before the CGS + DGKS pass against the cycle's basis, and U is replaced
// by harmonic Ritz vectors of the augmented (k + m) problem when a solve ends.
//
// Layout: U, C and the cycle basis V are column blocks of complex128 vectors with an even leading
// dimension (16-byte aligned rows for vector loads). One restart cycle is captured as a CUDA graph
// (like the GMRES driver) with every launch gated by the cycle's `active` flag; the k-column
// coupling block B (k x m) is filled on the device. The small dense algebra (k x k triangular
// solves, the harmonic-Ritz eigenproblem of order k + m) runs on the host in FP64.

#include <algorithm>
#include <complex>
#include <numeric>

#include "sb_blas.cuh"
#include "sb_internal.cuh"
#include "sb_krylov.cuh"
#include "sb_profile.cuh"

namespace sb {

using cd = std::complex<double>;

// ---------------------------------------------------------------------------------------------
// Small dense complex algebra (host, FP64).
// ---------------------------------------------------------------------------------------------
namespace dense {

struct CMat {
    int r = 0, c = 0;
    std::vector<cd> a;
    CMat() = default;
    CMat(int r_, int c_) : r(r_), c(c_), a(static_cast<size_t>(r_) * c_, cd(0.0, 0.0)) {}
    cd& operator()(int i, int j) { return a[static_cast<size_t>(i) * c + j]; }
    const cd& operator()(int i, int j) const { return a[static_cast<size_t>(i) * c + j]; }
};

// LU factorisation with partial pivoting and solve of A x = b (b overwritten by x). Fails when a
// pivot is at or below eps * n * max|u_ii| (the singularity rule of the reference's LU,
// crates/sonium-solvers/crates/sonium-solvers-direct/src/lu.rs:760-769).
bool lu_solve(CMat A, std::vector<cd>& b) {
    const int n = A.r;
    std::vector<int> piv(n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = std::abs(A(k, k));
        for (int i = k + 1; i < n; ++i)
            if (std::abs(A(i, k)) > best) {
                best = std::abs(A(i, k));
                p = i;
            }
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(A(k, j), A(p, j));
        if (best == 0.0) continue;
        const cd inv = 1.0 / A(k, k);
        for (int i = k + 1; i < n; ++i) {
            const cd l = A(i, k) * inv;
            A(i, k) = l;
            if (l != cd(0.0, 0.0))
                for (int j = k + 1; j < n; ++j) A(i, j) -= l * A(k, j);
        }
    }
    double scale = 0.0;
    for (int i = 0; i < n; ++i) scale = std::max(scale, std::abs(A(i, i)));
    const double tol = 2.220446049250313e-16 * std::max(n, 1) * std::max(scale, 2.2250738585072014e-308);
    for (int i = 0; i < n; ++i)
        if (!(std::abs(A(i, i)) > tol)) return false;
    for (int k = 0; k < n; ++k)
        if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) b[i] -= A(i, j) * b[j];
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) b[i] -= A(i, j) * b[j];
        b[i] /= A(i, i);
    }
    for (const cd& v : b)
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) return false;
    return true;
}

// Unitary reduction to upper Hessenberg form, A = Q H Q^H, with complex Householder reflectors
// (alpha = -e^{i arg x0} ||x||, which maps the column exactly onto e1 for complex data).
void hessenberg(CMat& H, CMat& Q) {
    const int n = H.r;
    Q = CMat(n, n);
    for (int i = 0; i < n; ++i) Q(i, i) = 1.0;
    std::vector<cd> v(n);
    for (int j = 0; j + 2 < n; ++j) {
        double xn2 = 0.0;
        for (int i = j + 1; i < n; ++i) xn2 += std::norm(H(i, j));
        const double xn = std::sqrt(xn2);
        if (xn < 1e-300) continue;
        const cd x0 = H(j + 1, j);
        const double ax0 = std::abs(x0);
        const cd phase = ax0 > 0.0 ? x0 / ax0 : cd(1.0, 0.0);
        const cd alpha = -phase * xn;
        double vn2 = 0.0;
        for (int i = j + 1; i < n; ++i) {
            v[i] = H(i, j) - (i == j + 1 ? alpha : cd(0.0, 0.0));
            vn2 += std::norm(v[i]);
        }
        if (vn2 < 1e-300) continue;
        const double beta = 2.0 / vn2;
        for (int k = j; k < n; ++k) {  // H <- P H
            cd d = 0.0;
            for (int i = j + 1; i < n; ++i) d += std::conj(v[i]) * H(i, k);
            d *= beta;
            for (int i = j + 1; i < n; ++i) H(i, k) -= v[i] * d;
        }
        for (int k = 0; k < n; ++k) {  // H <- H P, Q <- Q P  (P is Hermitian)
            cd d = 0.0, e = 0.0;
            for (int i = j + 1; i < n; ++i) {
                d += H(k, i) * v[i];
                e += Q(k, i) * v[i];
            }
            d *= beta;
            e *= beta;
            for (int i = j + 1; i < n; ++i) {
                H(k, i) -= d * std::conj(v[i]);
                Q(k, i) -= e * std::conj(v[i]);
            }
        }
        H(j + 1, j) = alpha;
        for (int i = j + 2; i < n; ++i) H(i, j) = 0.0;
    }
}

// Eigenvalue of the 2 x 2 block [[a, b], [c, d]] closest to d (Wilkinson shift).
cd wilkinson(cd a, cd b, cd c, cd d) {
    const cd tr = 0.5 * (a + d);
    const cd disc = std::sqrt(0.25 * (a - d) * (a - d) + b * c);
    const cd l1 = tr + disc, l2 = tr - disc;
    return std::abs(l1 - d) < std::abs(l2 - d) ? l1 : l2;
}

// Eigen-decomposition of a general complex matrix: Hessenberg reduction, then single-shift QR
// iterations with Givens rotations (Wilkinson shifts, exceptional shifts every 10 sweeps without
// deflation) down to the complex Schur form T = Z^H A Z, eigenvectors of T by back substitution,
// mapped back by Z. Returns false if the iteration limit was hit (the values are then those of
// the partly converged form).
bool eig(const CMat& A, std::vector<cd>& lam, CMat& vecs) {
    const int n = A.r;
    CMat T = A, Z;
    hessenberg(T, Z);
    bool ok = true;
    int hi = n - 1, its = 0, total_its = 0;
    const double eps = 2.220446049250313e-16;
    while (hi > 0) {
        int l = hi;
        for (; l > 0; --l) {
            const double s = std::abs(T(l - 1, l - 1)) + std::abs(T(l, l));
            if (std::abs(T(l, l - 1)) <= eps * (s > 0.0 ? s : 1.0)) {
                T(l, l - 1) = 0.0;
                break;
            }
        }
        if (l == hi) {
            --hi;
            its = 0;
            continue;
        }
        if (++total_its > 60 * n) {
            ok = false;
            break;
        }
        ++its;
        cd sigma;
        if (its % 10 == 0) {
            sigma = T(hi, hi) + std::abs(T(hi, hi - 1).real()) +
                    (hi >= 2 ? std::abs(T(hi - 1, hi - 2).real()) : 0.0);
        } else {
            sigma = wilkinson(T(hi - 1, hi - 1), T(hi - 1, hi), T(hi, hi - 1), T(hi, hi));
        }
        // QR step on the unreduced block [l, hi]: T - sigma I = G R, T <- R G + sigma I.
        std::vector<cd> gc(hi - l), gs(hi - l);
        for (int i = l; i <= hi; ++i) T(i, i) -= sigma;
        for (int i = l; i < hi; ++i) {
            const cd a = T(i, i), b = T(i + 1, i);
            const double r = std::sqrt(std::norm(a) + std::norm(b));
            cd c = 1.0, s = 0.0;
            if (r > 0.0) {
                c = a / r;
                s = b / r;
            }
            gc[i - l] = c;
            gs[i - l] = s;
            for (int k = i; k < n; ++k) {  // rows i, i+1 <- G^H rows
                const cd x = T(i, k), y = T(i + 1, k);
                T(i, k) = std::conj(c) * x + std::conj(s) * y;
                T(i + 1, k) = -s * x + c * y;
            }
        }
        for (int i = l; i < hi; ++i) {
            const cd c = gc[i - l], s = gs[i - l];
            const int rmax = std::min(hi, i + 2);
            for (int k = 0; k <= rmax; ++k) {  // columns i, i+1 <- columns G
                const cd x = T(k, i), y = T(k, i + 1);
                T(k, i) = x * c + y * s;
                T(k, i + 1) = -x * std::conj(s) + y * std::conj(c);
            }
            for (int k = 0; k < n; ++k) {
                const cd x = Z(k, i), y = Z(k, i + 1);
                Z(k, i) = x * c + y * s;
                Z(k, i + 1) = -x * std::conj(s) + y * std::conj(c);
            }
        }
        for (int i = l; i <= hi; ++i) T(i, i) += sigma;
    }
    lam.resize(n);
    for (int i = 0; i < n; ++i) lam[i] = T(i, i);
    double tnorm = 0.0;
    for (const cd& v : T.a) tnorm = std::max(tnorm, std::abs(v));
    const double small = eps * std::max(tnorm, 1e-300);
    CMat S(n, n);  // eigenvectors of T (upper triangular back substitution)
    for (int j = 0; j < n; ++j) {
        S(j, j) = 1.0;
        for (int i = j - 1; i >= 0; --i) {
            cd sum = 0.0;
            for (int l2 = i + 1; l2 <= j; ++l2) sum += T(i, l2) * S(l2, j);
            cd d = T(i, i) - T(j, j);
            if (std::abs(d) < small) d = small;
            S(i, j) = -sum / d;
        }
    }
    vecs = CMat(n, n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            cd s = 0.0;
            for (int l2 = 0; l2 <= j; ++l2) s += Z(i, l2) * S(l2, j);
            vecs(i, j) = s;
        }
    return ok;
}

}  // namespace dense

// ---------------------------------------------------------------------------------------------
// Device workspace and the recycled subspace.
// ---------------------------------------------------------------------------------------------
namespace {

// B[i * m + j] = c1[i] + c2[i]: the two C-projection coefficient passes of Arnoldi step j.
__global__ void k_bcol(const KState* __restrict__ st, const double2* __restrict__ c1, const double2* __restrict__ c2,
                       double2* __restrict__ B, int k, int m, int j) {
    if (!st->active) return;
    for (int i = threadIdx.x; i < k; i += blockDim.x) B[(int64_t)i * m + j] = cadd_(c1[i], c2[i]);
}

__global__ void k_gcro_cycle_init(KState* __restrict__ st, double2* __restrict__ H, double2* __restrict__ g,
                                  double2* __restrict__ B, int kb, int m, double beta, double pbnorm, double tol) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
    cycle_init_dev(st, H, g, m, 1, beta, pbnorm, tol, tid, nth, true);
    for (int64_t t = tid; t < (int64_t)kb * m; t += nth) B[t] = make_double2(0.0, 0.0);
}

__global__ void k_gcro_after_first(KState* __restrict__ st, const double2* __restrict__ red,
                                   const double* __restrict__ nrm, double2* __restrict__ H, int j) {
    after_first_dev(st, red, nrm, H, j);
}

__global__ void k_gcro_givens(KState* __restrict__ st, const double2* __restrict__ red2,
                              const double* __restrict__ nrm2, double2* __restrict__ H, double2* __restrict__ cs,
                              double2* __restrict__ sn, double2* __restrict__ g, int j) {
    givens_step_dev(st, red2, nrm2, H, cs, sn, g, j);
}

__global__ void k_gcro_upper_solve(const KState* __restrict__ st, const double2* __restrict__ H,
                                   const double2* __restrict__ g, double2* __restrict__ y) {
    upper_solve_dev(st, H, g, y);
}

}  // namespace

struct RecycleSpace {
    int device = 0;
    int64_t target = 0;  // vectors kept at the end of a solve (GcroDrSubspace::k)
    int64_t count = 0;   // vectors held now
    int64_t n = 0, ld = 0;
    DevBuf U, Unew;      // target x ld complex128 each

    // Solver workspace of the last solve (buffers for n, m, k; the captured cycle graph).
    int64_t wn = 0, wm = 0, wk = 0;
    DevBuf V, C, w, opb, part, red, red2, redc, redc2, nrm, ydev, zdev, H, cs, sn, g, B, st;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // Everything the captured cycle bakes in besides the subspace's own buffers: the operator's
    // matrices and Jacobi diagonal (a later operator may reuse the same addresses for other roles).
    const void* key_A = nullptr;
    const void* key_A32 = nullptr;
    const void* key_jac = nullptr;
    int64_t key_lda = -1;
    int key_jacobi = -1, key_k = -1;
    unsigned key_prof = 0;
    std::vector<ProfPair> prof_pairs;
    int64_t graph_kernels = 0;

    void reset_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        profile_release(prof_pairs);
    }
    ~RecycleSpace() {
        cudaSetDevice(device);
        reset_graph();
    }
    void ensure_vectors(int64_t n_) {
        if (n_ == n && U.p) return;
        n = n_;
        ld = (n + 1) / 2 * 2;
        count = 0;
        if (target > 0) {
            U.alloc(sizeof(double2) * target * ld);
            Unew.alloc(sizeof(double2) * target * ld);
        }
    }
    void ensure_work(int64_t n_, int64_t m_, int64_t k_) {
        if (n_ == wn && m_ == wm && k_ <= wk && V.p) return;
        reset_graph();
        wn = n_;
        wm = m_;
        wk = std::max<int64_t>(k_, 1);
        const int64_t l = (wn + 1) / 2 * 2;
        V.alloc(sizeof(double2) * (wm + 1) * l);
        C.alloc(sizeof(double2) * wk * l);
        w.alloc(sizeof(double2) * l);
        opb.alloc(sizeof(double2) * l);
        const int64_t kk = std::max(wm, wk) + 2;
        part.alloc(sizeof(double2) * std::max<int64_t>(arnoldi_dot_chunks(wn) * kk, (wn + 255) / 256 + gemv_partials(wn)));
        red.alloc(sizeof(double2) * kk);
        red2.alloc(sizeof(double2) * kk);
        redc.alloc(sizeof(double2) * kk);
        redc2.alloc(sizeof(double2) * kk);
        nrm.alloc(sizeof(double) * 8);
        ydev.alloc(sizeof(double2) * (wm + 1));
        zdev.alloc(sizeof(double2) * (wm + wk + 2));
        H.alloc(sizeof(double2) * (wm + 1) * wm);
        cs.alloc(sizeof(double2) * wm);
        sn.alloc(sizeof(double2) * wm);
        g.alloc(sizeof(double2) * (wm + 1));
        B.alloc(sizeof(double2) * wk * wm);
        st.alloc(sizeof(KState));
    }
};

RecycleSpace* recycle_create(int device, int64_t k) {
    RecycleSpace* s = new RecycleSpace();
    s->device = device;
    s->target = k;
    return s;
}
void recycle_destroy(RecycleSpace* s) { delete s; }
void recycle_reset(RecycleSpace& s) { s.count = 0; }
void recycle_info(const RecycleSpace& s, int64_t* count, int64_t* target, int64_t* n) {
    if (count) *count = s.count;
    if (target) *target = s.target;
    if (n) *n = s.count ? s.n : 0;
}
void recycle_get(const RecycleSpace& s, double2* host) {
    if (!s.count) return;
    SB_CUDA(cudaSetDevice(s.device));
    SB_CUDA(cudaDeviceSynchronize());
    SB_CUDA(cudaMemcpy2D(host, sizeof(double2) * s.n, s.U.p, sizeof(double2) * s.ld, sizeof(double2) * s.n, s.count,
                         cudaMemcpyDeviceToHost));
}
void recycle_set(RecycleSpace& s, int64_t count, int64_t n, const double2* host) {
    SB_REQUIRE(count >= 0 && count <= s.target, SB_ERR_INVALID_ARGUMENT,
               "recycled subspace: more vectors than the target size");
    SB_CUDA(cudaSetDevice(s.device));
    if (count == 0) {
        s.count = 0;
        return;
    }
    SB_REQUIRE(n > 0, SB_ERR_INVALID_ARGUMENT, "recycled subspace: vector length must be positive");
    s.ensure_vectors(n);
    SB_CUDA(cudaMemcpy2D(s.U.p, sizeof(double2) * s.ld, host, sizeof(double2) * n, sizeof(double2) * n, count,
                         cudaMemcpyHostToDevice));
    SB_CUDA(cudaStreamSynchronize(0));  // the copy lands before kernels on the solver's stream read it
    s.count = count;
}

// ---------------------------------------------------------------------------------------------
// The solver.
// ---------------------------------------------------------------------------------------------
namespace {

// One restart cycle: m Arnoldi steps of M^-1 A, each projected against C twice (coefficients
// into column j of B) and then against V with CGS + DGKS; every launch gated by st->active.
void gcro_launch_cycle(const Operator& op, RecycleSpace& S, const double2* jac, int k, int64_t m) {
    const int64_t n = op.n, l = (n + 1) / 2 * 2;
    const cudaStream_t s = op.stream;
    KState* st = S.st.as<KState>();
    const Gate ga{&st->active, nullptr}, gb{&st->active, &st->reorth};
    double2* V = S.V.as<double2>();
    double2* C = S.C.as<double2>();
    double2* w = S.w.as<double2>();
    double2* part = S.part.as<double2>();
    double* partd = S.part.as<double>();
    double* nrm = S.nrm.as<double>();
    for (int64_t j = 0; j < m; ++j) {
        capture_step(static_cast<int>(j));
        if (jac) {
            op_gemv64(op, V + j * l, S.opb.as<double2>(), ga);
            jacobi_apply<double2>(jac, S.opb.as<double2>(), w, n, s, ga);
        } else {
            op_gemv64(op, V + j * l, w, ga);
        }
        if (k > 0) {
            arnoldi_dots<double2>(C, l, k, w, n, part, S.redc.as<double2>(), s, ga);
            arnoldi_project<double2>(C, l, k, S.redc.as<double2>(), w, n, partd, nrm + 3, s, ga);
            arnoldi_dots<double2>(C, l, k, w, n, part, S.redc2.as<double2>(), s, ga);
            arnoldi_project<double2>(C, l, k, S.redc2.as<double2>(), w, n, partd, nrm + 3, s, ga);
            k_bcol<<<1, 128, 0, s>>>(st, S.redc.as<double2>(), S.redc2.as<double2>(), S.B.as<double2>(), k,
                                     static_cast<int>(m), static_cast<int>(j));
            count_launch();
        }
        const int kv = static_cast<int>(j + 1);
        arnoldi_dots<double2>(V, l, kv, w, n, part, S.red.as<double2>(), s, ga);
        arnoldi_project<double2>(V, l, kv, S.red.as<double2>(), w, n, partd, nrm, s, ga);
        k_gcro_after_first<<<1, 1, 0, s>>>(st, S.red.as<double2>(), nrm, S.H.as<double2>(), static_cast<int>(j));
        count_launch();
        arnoldi_dots<double2>(V, l, kv, w, n, part, S.red2.as<double2>(), s, gb);
        arnoldi_project<double2>(V, l, kv, S.red2.as<double2>(), w, n, partd, nrm + 1, s, gb);
        k_gcro_givens<<<1, 1, 0, s>>>(st, S.red2.as<double2>(), nrm + 1, S.H.as<double2>(), S.cs.as<double2>(),
                                      S.sn.as<double2>(), S.g.as<double2>(), static_cast<int>(j));
        count_launch();
        scale_vec<double2, double2>(w, 0.0, &st->inv_wn, V + (j + 1) * l, n, s, ga);
    }
    SB_CUDA(cudaGetLastError());
}

// Replays the captured cycle, capturing it first when the operator, k or profiling changed.
void gcro_run_cycle(const Operator& op, RecycleSpace& S, const double2* jac, int k, int64_t m) {
    const void* key_A = op.A64.p;
    const int kj = jac ? 1 : 0;
    if (!S.exec || S.key_A != key_A || S.key_A32 != op.A32.p || S.key_lda != op.lda32 || S.key_jac != jac ||
        S.key_jacobi != kj || S.key_k != k || S.key_prof != prof_key()) {
        S.reset_graph();
        const int64_t before = kernel_count();
        capture_begin(&S.prof_pairs);
        SB_CUDA(cudaStreamBeginCapture(op.stream, cudaStreamCaptureModeThreadLocal));
        try {
            gcro_launch_cycle(op, S, jac, k, m);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(op.stream, &g);
            if (g) cudaGraphDestroy(g);
            capture_end();
            throw;
        }
        SB_CUDA(cudaStreamEndCapture(op.stream, &S.graph));
        capture_end();
        SB_CUDA(cudaGraphInstantiate(&S.exec, S.graph, 0));
        S.graph_kernels = kernel_count() - before;
        add_kernel_count(-S.graph_kernels);
        S.key_A = key_A;
        S.key_A32 = op.A32.p;
        S.key_lda = op.lda32;
        S.key_jac = jac;
        S.key_jacobi = kj;
        S.key_k = k;
        S.key_prof = prof_key();
    }
    SB_CUDA(cudaGraphLaunch(S.exec, op.stream));
    add_kernel_count(S.graph_kernels);
}

// solve_upper_triangular_dense (gcro_dr.rs:853-870): k x k, entries with |r_ii| <= 1e-30 give 0.
std::vector<cd> upper_solve(const std::vector<cd>& R, int64_t ldr, const std::vector<cd>& g, int k) {
    std::vector<cd> y(k, cd(0.0, 0.0));
    for (int i = k - 1; i >= 0; --i) {
        cd sum = g[i];
        for (int j = i + 1; j < k; ++j) sum -= R[i * ldr + j] * y[j];
        const cd d = R[i * ldr + i];
        if (std::abs(d) > 1e-30) y[i] = sum / d;
    }
    return y;
}

struct Ctx {
    const Operator& op;
    RecycleSpace& S;
    const double2* jac;
    cudaStream_t s;
    int64_t n, l;
    int64_t matvecs = 0;

    Ctx(const Operator& o, RecycleSpace& sp, const double2* j)
        : op(o), S(sp), jac(j), s(o.stream), n(o.n), l((o.n + 1) / 2 * 2) {}

    void sync() { SB_CUDA(cudaStreamSynchronize(s)); }
    template <class T>
    void to_host(T* h, const void* d, size_t count) {
        SB_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * count, cudaMemcpyDeviceToHost, s));
    }
    template <class T>
    void to_dev(void* d, const T* h, size_t count) {
        SB_CUDA(cudaMemcpyAsync(d, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    }
    // out = M^-1 A x
    void apply(const double2* x, double2* out) {
        if (jac) {
            op_gemv64(op, x, S.opb.as<double2>(), Gate{});
            jacobi_apply<double2>(jac, S.opb.as<double2>(), out, n, s);
        } else {
            op_gemv64(op, x, out, Gate{});
        }
        ++matvecs;
    }
    double norm(const double2* v) {
        arnoldi_dots<double2>(v, l, 0, v, n, S.part.as<double2>(), S.red2.as<double2>(), s);
        double2 h;
        to_host(&h, S.red2.p, 1);
        sync();
        return std::sqrt(h.x);
    }
    // ||b - A x|| (residual vector left in opb)
    double residual(const double2* x, const double2* b) {
        op_residual64(op, x, b, S.opb.as<double2>(), S.part.as<double>());
        sum_real(S.part.as<double>(), op_residual64_partials(op), S.nrm.as<double>() + 2, s);
        double h;
        to_host(&h, S.nrm.as<double>() + 2, 1);
        sync();
        ++matvecs;
        return std::sqrt(h);
    }
    // x += sum_i y_i U_i
    void add_u(const std::vector<cd>& y, int k, double2* x) {
        if (k == 0) return;
        to_dev(S.zdev.p, reinterpret_cast<const double2*>(y.data()), k);
        basis_update<double2, double2>(S.U.as<double2>(), S.ld, k, nullptr, S.zdev.as<double2>(), 1.0, x, n, s);
    }
};

// build_c_r (gcro_dr.rs:769-850): C = orth(M^-1 A U) by CGS with an unconditional second pass,
// R (k x k, leading dimension ldr) with M^-1 A U = C R; stops at the first column whose
// projected norm is below 1e-12. Returns the number of columns built.
int build_c_r(Ctx& c, std::vector<cd>& R, int64_t ldr, int k_in) {
    int cc = 0;
    double2* C = c.S.C.as<double2>();
    std::vector<double2> c1(k_in + 1), c2(k_in + 1);
    for (int j = 0; j < k_in; ++j) {
        double2* z = C + cc * c.l;
        c.apply(c.S.U.as<double2>() + j * c.S.ld, z);
        double nz2;
        if (cc > 0) {
            arnoldi_dots<double2>(C, c.l, cc, z, c.n, c.S.part.as<double2>(), c.S.redc.as<double2>(), c.s);
            arnoldi_project<double2>(C, c.l, cc, c.S.redc.as<double2>(), z, c.n, c.S.part.as<double>(),
                                     c.S.nrm.as<double>() + 4, c.s);
            arnoldi_dots<double2>(C, c.l, cc, z, c.n, c.S.part.as<double2>(), c.S.redc2.as<double2>(), c.s);
            arnoldi_project<double2>(C, c.l, cc, c.S.redc2.as<double2>(), z, c.n, c.S.part.as<double>(),
                                     c.S.nrm.as<double>() + 4, c.s);
            c.to_host(c1.data(), c.S.redc.p, cc);
            c.to_host(c2.data(), c.S.redc2.p, cc);
            c.to_host(&nz2, c.S.nrm.as<double>() + 4, 1);
            c.sync();
            for (int i = 0; i < cc; ++i) R[i * ldr + j] = cd(c1[i].x, c1[i].y) + cd(c2[i].x, c2[i].y);
        } else {
            arnoldi_dots<double2>(z, c.l, 0, z, c.n, c.S.part.as<double2>(), c.S.redc.as<double2>(), c.s);
            c.to_host(c1.data(), c.S.redc.p, 1);
            c.sync();
            nz2 = c1[0].x;
        }
        const double nz = std::sqrt(nz2);
        if (!(nz >= 1e-12)) break;
        R[j * ldr + j] = nz;
        scale_vec<double2, double2>(z, 1.0 / nz, nullptr, z, c.n, c.s);
        ++cc;
    }
    return cc;
}

// update_recycled_subspace (gcro_dr.rs:922-1050): harmonic Ritz vectors of M^-1 A on
// range([U V_m]) from the augmented matrix G_top = [[R, B], [0, H]] (un-rotated Hessenberg),
// (G_top + |rho|^2 G_top^-H e_l e_l^H) y = theta y; the take = min(target, k + steps) values of
// smallest |theta| give psi = U y_u + V y_v, orthonormalised by modified Gram-Schmidt (vectors
// whose norm falls to 1e-12 are dropped). `nrot` rotations of the last cycle are valid.
void update_subspace(Ctx& c, const std::vector<cd>& R, int64_t ldr, const std::vector<cd>& Bh, int k_in, int steps,
                     int nrot, int64_t m) {
    RecycleSpace& S = c.S;
    if (S.target == 0 || steps == 0) return;
    const int total = k_in + steps;
    std::vector<double2> Hd((m + 1) * m), csd(m), snd(m);
    c.to_host(Hd.data(), S.H.p, (m + 1) * m);
    c.to_host(csd.data(), S.cs.p, m);
    c.to_host(snd.data(), S.sn.p, m);
    c.sync();
    auto H = [&](int i, int j) -> cd& { return *reinterpret_cast<cd*>(&Hd[i * m + j]); };
    // unapply_givens_local (gcro_dr.rs:874-900)
    for (int j = steps - 1; j >= 0; --j) {
        if (j >= nrot) continue;
        const cd cj(csd[j].x, csd[j].y), sj(snd[j].x, snd[j].y);
        for (int col = j; col < steps; ++col) {
            const cd hj = H(j, col), hj1 = H(j + 1, col);
            H(j, col) = cj * hj - std::conj(sj) * hj1;
            H(j + 1, col) = std::conj(sj) * hj + std::conj(cj) * hj1;
        }
    }
    const cd rho = H(steps, steps - 1);
    dense::CMat G(total, total);
    for (int i = 0; i < k_in; ++i) {
        for (int j = 0; j < k_in; ++j) G(i, j) = R[i * ldr + j];
        for (int j = 0; j < steps; ++j) G(i, k_in + j) = Bh[(size_t)i * m + j];
    }
    for (int i = 0; i < steps; ++i)
        for (int j = 0; j < steps; ++j) G(k_in + i, k_in + j) = H(i, j);
    // solve_with_g_top_h (gcro_dr.rs:1057-1090): G_top^H w = e_l by LU, damped once if singular.
    dense::CMat Gh(total, total);
    for (int i = 0; i < total; ++i)
        for (int j = 0; j < total; ++j) Gh(i, j) = std::conj(G(j, i));
    std::vector<cd> e(total, cd(0.0, 0.0));
    e[total - 1] = 1.0;
    std::vector<cd> wv = e;
    if (!dense::lu_solve(Gh, wv)) {
        for (int i = 0; i < total; ++i) Gh(i, i) += 1e-12;
        wv = e;
        if (!dense::lu_solve(Gh, wv)) wv = e;
    }
    const double rho2 = std::norm(rho);
    dense::CMat M = G;
    for (int i = 0; i < total; ++i) M(i, total - 1) += rho2 * wv[i];
    std::vector<cd> lam;
    dense::CMat Y;
    dense::eig(M, lam, Y);
    std::vector<int> idx(total);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return std::abs(lam[a]) < std::abs(lam[b]); });
    const int take = static_cast<int>(std::min<int64_t>(S.target, total));
    double2* Un = S.Unew.as<double2>();
    int acc = 0;
    std::vector<cd> ycol(total);
    for (int t = 0; t < take; ++t) {
        for (int i = 0; i < total; ++i) ycol[i] = Y(i, idx[t]);
        double2* psi = Un + acc * S.ld;
        SB_CUDA(cudaMemsetAsync(psi, 0, sizeof(double2) * S.ld, c.s));
        c.to_dev(S.zdev.p, reinterpret_cast<const double2*>(ycol.data()), total);
        if (k_in > 0)
            basis_update<double2, double2>(S.U.as<double2>(), S.ld, k_in, nullptr, S.zdev.as<double2>(), 1.0, psi,
                                           c.n, c.s);
        basis_update<double2, double2>(S.V.as<double2>(), c.l, steps, nullptr, S.zdev.as<double2>() + k_in, 1.0, psi,
                                       c.n, c.s);
        for (int p = 0; p < acc; ++p) {  // modified Gram-Schmidt against the accepted vectors
            const double2* prev = Un + p * S.ld;
            arnoldi_dots<double2>(prev, S.ld, 1, psi, c.n, S.part.as<double2>(), S.redc.as<double2>(), c.s);
            arnoldi_project<double2>(prev, S.ld, 1, S.redc.as<double2>(), psi, c.n, S.part.as<double>(),
                                     S.nrm.as<double>() + 5, c.s);
        }
        const double nrm = c.norm(psi);
        if (nrm > 1e-12) {
            scale_vec<double2, double2>(psi, 1.0 / nrm, nullptr, psi, c.n, c.s);
            ++acc;
        }
    }
    if (acc > 0) {
        S.U.swap(S.Unew);
        S.count = acc;
    }
}

}  // namespace

// gcro_dr_core (gcro_dr.rs:339-760) on the device; b, x device vectors of op.n complex128.
void gcro_dr(const Operator& op, const double2* b, double2* x, bool x0_given, RecycleSpace& sp,
             const sb_gmres_config& cfg, int precond, sb_gmres_stats& st) {
    SB_CUDA(cudaSetDevice(op.device));
    SB_REQUIRE(op.device == sp.device, SB_ERR_INVALID_ARGUMENT,
               "gcro_dr: the operator and the recycled subspace are on different devices");
    SB_REQUIRE(cfg.restart > 0 && cfg.restart < kMaxKrylov && cfg.max_iterations > 0, SB_ERR_INVALID_ARGUMENT,
               "gcro_dr: restart must be in 1..126 and max_iterations positive");
    const int64_t n = op.n, m = cfg.restart;
    const cudaStream_t s = op.stream;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    SB_CUDA(cudaEventCreate(&ev0));
    SB_CUDA(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evg{ev0, ev1};
    SB_CUDA(cudaEventRecord(ev0, s));
    st = sb_gmres_stats{};
    auto finish = [&](int status, bool conv, double res, double est) {
        st.status = status;
        st.converged = conv ? 1 : 0;
        st.residual = res;
        st.backward_error = res;
        st.estimated_residual = est;
        SB_CUDA(cudaEventRecord(ev1, s));
        SB_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.f;
        SB_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        st.device_ms = ms;
    };
    if (!x0_given) SB_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, s));
    if (sp.count > 0 && sp.n != n) {  // recycled vectors of another length (gcro_dr.rs:370-372)
        finish(SB_SOLVER_NUMERICAL_ERROR, false, INFINITY, INFINITY);
        return;
    }
    sp.ensure_work(n, m, sp.target);
    if (sp.count == 0) sp.ensure_vectors(n);
    Ctx c(op, sp, precond == SB_PRECOND_JACOBI ? op.diag.as<double2>() : nullptr);
    const double2* pb = b;
    if (c.jac) {
        jacobi_apply<double2>(c.jac, b, sp.w.as<double2>(), n, s);
        pb = sp.w.as<double2>();
    }
    const double b_norm = c.norm(pb);
    const double true_b_norm = c.jac ? c.norm(b) : b_norm;
    const double public_b_norm = true_b_norm < 1e-15 ? 1.0 : true_b_norm;
    const double tol = cfg.tolerance;
    if (b_norm < 1e-15) {
        finish(SB_SOLVER_CONVERGED, true, 0.0, 0.0);
        return;
    }
    // C and R for the current operator; a failed build empties the subspace.
    const int64_t ldr = std::max<int64_t>(sp.target, 1);
    std::vector<cd> R(ldr * ldr, cd(0.0, 0.0));
    int k = 0;
    if (sp.count > 0) {
        k = build_c_r(c, R, ldr, static_cast<int>(sp.count));
        sp.count = k;
    }
    std::vector<double2> Bh(std::max<int64_t>(k, 1) * m), yh(m + 1), alpha(k + 1);
    std::vector<cd> a(k), by(k);
    KState hst{};
    int64_t total_it = 0, restarts = 0;
    int last_steps = 0;
    double2* V = sp.V.as<double2>();
    for (int64_t outer = 0; outer < cfg.max_iterations; ++outer) {
        // w = M^-1 (b - A x), its C component absorbed into x through U R^-1.
        c.residual(x, b);
        double2* src = sp.opb.as<double2>();
        if (c.jac) {
            jacobi_apply<double2>(c.jac, sp.opb.as<double2>(), sp.w.as<double2>(), n, s);
            src = sp.w.as<double2>();
        }
        double beta;
        if (k > 0) {
            arnoldi_dots<double2>(sp.C.as<double2>(), c.l, k, src, n, sp.part.as<double2>(), sp.redc.as<double2>(), s);
            arnoldi_project<double2>(sp.C.as<double2>(), c.l, k, sp.redc.as<double2>(), src, n, sp.part.as<double>(),
                                     sp.nrm.as<double>() + 6, s);
            double nb2;
            c.to_host(alpha.data(), sp.redc.p, k);
            c.to_host(&nb2, sp.nrm.as<double>() + 6, 1);
            c.sync();
            for (int i = 0; i < k; ++i) a[i] = cd(alpha[i].x, alpha[i].y);
            c.add_u(upper_solve(R, ldr, a, k), k, x);
            beta = std::sqrt(nb2);
        } else {
            beta = c.norm(src);
        }
        const double rel0 = beta / b_norm;
        if (!std::isfinite(beta)) {
            st.iterations = total_it;
            st.restarts = restarts;
            st.matvecs = c.matvecs;
            finish(SB_SOLVER_NUMERICAL_ERROR, false, INFINITY, INFINITY);
            return;
        }
        if (rel0 < tol) {
            const double tr = c.residual(x, b) / public_b_norm;
            if (tr < tol || tr < 1e-20) {
                st.iterations = total_it;
                st.restarts = restarts;
                st.matvecs = c.matvecs;
                finish(SB_SOLVER_CONVERGED, true, tr, rel0);
                return;
            }
        }
        // V_0 = w / beta, then one captured cycle.
        scale_vec<double2, double2>(src, 1.0 / beta, nullptr, V, n, s);
        k_gcro_cycle_init<<<8, 256, 0, s>>>(sp.st.as<KState>(), sp.H.as<double2>(), sp.g.as<double2>(),
                                            sp.B.as<double2>(), k, static_cast<int>(m), beta, b_norm, tol);
        count_launch();
        SB_CUDA(cudaGetLastError());
        gcro_run_cycle(op, sp, c.jac, k, m);
        k_gcro_upper_solve<<<1, 1, 0, s>>>(sp.st.as<KState>(), sp.H.as<double2>(), sp.g.as<double2>(),
                                           sp.ydev.as<double2>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        basis_update<double2, double2>(V, c.l, 0, &sp.st.as<KState>()->jdone, sp.ydev.as<double2>(), 1.0, x, n, s);
        c.to_host(&hst, sp.st.p, 1);
        if (k > 0) {
            c.to_host(yh.data(), sp.ydev.p, m);
            c.to_host(Bh.data(), sp.B.p, k * m);
        }
        c.sync();
        profile_account(sp.prof_pairs, hst.jdone);
        const int steps = hst.jdone;
        last_steps = steps;
        total_it += steps;
        c.matvecs += steps;
        if (k > 0 && steps > 0) {  // cancel the C coupling -B y_v of the V correction
            for (int i = 0; i < k; ++i) {
                cd sacc(0.0, 0.0);
                for (int jj = 0; jj < steps; ++jj)
                    sacc += cd(Bh[i * m + jj].x, Bh[i * m + jj].y) * cd(yh[jj].x, yh[jj].y);
                by[i] = -sacc;
            }
            c.add_u(upper_solve(R, ldr, by, k), k, x);
        }
        const double rel_after = steps == 0 ? 0.0 : hst.relres;
        const bool stopped = hst.reason != 0;
        const bool inner = stopped && hst.inv_wn == 0.0;
        if (stopped || rel_after < tol) {
            const double tr = c.residual(x, b) / public_b_norm;
            if (tr < tol || tr < 1e-20) {
                std::vector<cd> Bc(Bh.size());
                for (size_t i = 0; i < Bh.size(); ++i) Bc[i] = cd(Bh[i].x, Bh[i].y);
                update_subspace(c, R, ldr, Bc, k, steps, steps, m);
                st.iterations = total_it;
                st.restarts = restarts;
                st.matvecs = c.matvecs;
                finish(SB_SOLVER_CONVERGED, true, tr, rel_after);
                return;
            }
            if (inner) {
                st.iterations = total_it;
                st.restarts = restarts;
                st.matvecs = c.matvecs;
                finish(SB_SOLVER_BREAKDOWN, false, tr, rel_after);
                return;
            }
        }
        ++restarts;
    }
    // Not converged: refresh the subspace from the last cycle all the same (gcro_dr.rs:724-726).
    {
        std::vector<cd> Bc(Bh.size());
        for (size_t i = 0; i < Bh.size(); ++i) Bc[i] = cd(Bh[i].x, Bh[i].y);
        update_subspace(c, R, ldr, Bc, k, static_cast<int>(m), last_steps, m);
    }
    const double tr = c.residual(x, b) / public_b_norm;
    st.iterations = total_it;
    st.restarts = restarts;
    st.matvecs = c.matvecs;
    finish(SB_SOLVER_MAX_ITERATIONS, false, tr, tr);
}

}  // namespace sb
