// Restarted GMRES and mixed-precision iterative refinement drivers (host side, device vectors).
//
// Reference: gmres_core (crates/sonium-solvers/crates/sonium-solvers-iterative/src/gmres.rs:631-1047)
// with finalize_gmres_solution (gmres.rs:159-247), givens_rotation / solve_upper_triangular
// (gmres_common.rs:91-127) and the CGS + DGKS (0.707) orthogonalisation of cgs_orth.rs:180-300.
// The Krylov basis, the matvec and the Gram-Schmidt passes stay on the device; the (m+1) x m
// Hessenberg matrix, the Givens rotations and the triangular solve stay on the host in FP64, fed
// by one small device-to-host copy per Arnoldi step.

#include <complex>
#include <functional>

#include "sb_blas.cuh"
#include "sb_internal.cuh"

namespace sb {

using cd = std::complex<double>;

namespace {

struct PinnedBuf {
    void* p = nullptr;
    explicit PinnedBuf(size_t bytes) { SB_CUDA(cudaMallocHost(&p, bytes)); }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

void givens(cd a, cd b, cd& c, cd& s) {
    const double tol = 1e-30;
    if (std::abs(b) < tol) {
        c = 1.0;
        s = 0.0;
        return;
    }
    if (std::abs(a) < tol) {
        c = 0.0;
        s = 1.0;
        return;
    }
    const double r = std::sqrt(std::norm(a) + std::norm(b));
    c = a * (1.0 / r);
    s = b * (1.0 / r);
}

std::vector<cd> upper_solve(const std::vector<cd>& h, int64_t ld, const std::vector<cd>& g, int64_t k) {
    std::vector<cd> y(k, cd(0, 0));
    for (int64_t i = k - 1; i >= 0; --i) {
        cd s = g[i];
        for (int64_t j = i + 1; j < k; ++j) s -= h[i * ld + j] * y[j];
        if (std::abs(h[i * ld + i]) > 1e-30) y[i] = s * (1.0 / h[i * ld + i]);
    }
    return y;
}

// Device operator callbacks of one GMRES instance.
template <class T>
struct Problem {
    int64_t n = 0;
    std::function<void(const T*, T*)> apply;                    // y = A x
    std::function<double(const T*, const T*, T*)> residual;     // r = b - A x, returns ||r||
    const double2* jacobi = nullptr;                            // diagonal for Jacobi, or null
    cudaStream_t stream = nullptr;
};

struct CoreResult {
    int64_t iterations = 0, restarts = 0, matvecs = 0;
    double residual = 1.0, estimated = 1.0;
    bool converged = false;
    int status = SB_SOLVER_MAX_ITERATIONS;
};

// gmres_core (gmres.rs:631-1047) with an identity or Jacobi left preconditioner.
template <class T>
CoreResult gmres_core(const Problem<T>& P, const T* b, T* x, int64_t max_it, int64_t m,
                      double tol, int64_t check_interval) {
    const int64_t n = P.n;
    const cudaStream_t s = P.stream;
    CoreResult R;
    DevBuf V, w, opb, r, part, red, red2, nrm, ydev;
    // Even leading dimension: every basis vector starts 16-byte aligned, which the vectorised
    // complex64 matvec needs for its two-entry loads of x.
    const int64_t ldv = (n + 1) / 2 * 2;
    V.alloc(sizeof(T) * (m + 1) * ldv);
    w.alloc(sizeof(T) * n);
    opb.alloc(sizeof(T) * n);
    r.alloc(sizeof(T) * n);
    const int64_t dchunks = arnoldi_dot_chunks(n);
    part.alloc(sizeof(double2) * std::max<int64_t>(dchunks * (m + 2), (n + 255) / 256 + gemv_partials(n)));
    red.alloc(sizeof(double2) * (m + 2));
    red2.alloc(sizeof(double2) * (m + 2));
    nrm.alloc(sizeof(double) * 2);
    ydev.alloc(sizeof(double2) * (m + 1));
    PinnedBuf host(sizeof(double2) * (m + 4));
    double2* hbuf = host.as<double2>();
    T* Vp = V.as<T>();
    auto Vj = [&](int64_t j) { return Vp + j * ldv; };

    auto norm_of = [&](const T* v) -> double {
        arnoldi_dots<T>(v, n, 0, v, n, part.as<double2>(), red2.as<double2>(), s);
        SB_CUDA(cudaMemcpyAsync(hbuf, red2.p, sizeof(double2), cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        return std::sqrt(hbuf[0].x);
    };
    auto precond = [&](const T* in, T* out) {
        if (P.jacobi) jacobi_apply<T>(P.jacobi, in, out, n, s);
        else if (in != out) SB_CUDA(cudaMemcpyAsync(out, in, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
    };
    auto true_rel = [&](double bnorm) {
        ++R.matvecs;
        return P.residual(x, b, r.as<T>()) / bnorm;
    };
    auto update_x = [&](const std::vector<cd>& y) {
        for (size_t i = 0; i < y.size(); ++i) hbuf[i] = make_double2(y[i].real(), y[i].imag());
        SB_CUDA(cudaMemcpyAsync(ydev.p, hbuf, sizeof(double2) * y.size(), cudaMemcpyHostToDevice, s));
        basis_update<T, T>(Vp, ldv, static_cast<int>(y.size()), ydev.as<double2>(), 1.0, x, n, s);
        SB_CUDA(cudaStreamSynchronize(s));
    };

    const double raw_bn = norm_of(b);
    const bool rhs_zero = raw_bn < 1e-15;
    const double bnorm = rhs_zero ? 1.0 : raw_bn;
    double pbnorm = bnorm;
    if (P.jacobi) {
        precond(b, w.as<T>());
        const double raw_pb = norm_of(w.as<T>());
        if (!rhs_zero && raw_pb < 1e-15) {
            R.status = SB_SOLVER_BREAKDOWN;
            return R;
        }
        pbnorm = rhs_zero ? 1.0 : raw_pb;
    }
    std::vector<cd> H((m + 1) * m), cs, sn, g(m + 1);
    for (int64_t outer = 0; outer < max_it; ++outer) {
        ++R.matvecs;
        const double rn = P.residual(x, b, opb.as<T>());
        const double trel = rn / bnorm;
        double beta = rn;
        if (P.jacobi) {
            precond(opb.as<T>(), w.as<T>());
            beta = norm_of(w.as<T>());
        } else {
            SB_CUDA(cudaMemcpyAsync(w.p, opb.p, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        }
        const double rel = beta / pbnorm;
        if (rel < tol && trel < tol) {
            R.converged = true;
            R.status = SB_SOLVER_CONVERGED;
            R.estimated = rel;
            R.residual = trel;
            return R;
        }
        if (!std::isfinite(beta) || beta == 0.0) {
            R.status = SB_SOLVER_BREAKDOWN;
            R.estimated = rel;
            R.residual = trel;
            return R;
        }
        scale_vec<T, T>(w.as<T>(), 1.0 / beta, Vj(0), n, s);
        std::fill(H.begin(), H.end(), cd(0, 0));
        cs.clear();
        sn.clear();
        std::fill(g.begin(), g.end(), cd(0, 0));
        g[0] = beta;
        bool restart_now = false;
        for (int64_t j = 0; j < m; ++j) {
            ++R.iterations;
            ++R.matvecs;
            if (P.jacobi) {
                P.apply(Vj(j), opb.as<T>());
                precond(opb.as<T>(), w.as<T>());
            } else {
                P.apply(Vj(j), w.as<T>());
            }
            const int k = static_cast<int>(j + 1);
            arnoldi_dots<T>(Vp, ldv, k, w.as<T>(), n, part.as<double2>(), red.as<double2>(), s);
            arnoldi_project<T>(Vp, ldv, k, red.as<double2>(), w.as<T>(), n, reinterpret_cast<double*>(part.p),
                               nrm.as<double>(), s);
            SB_CUDA(cudaMemcpyAsync(hbuf, red.p, sizeof(double2) * (k + 1), cudaMemcpyDeviceToHost, s));
            SB_CUDA(cudaMemcpyAsync(hbuf + m + 2, nrm.p, sizeof(double), cudaMemcpyDeviceToHost, s));
            SB_CUDA(cudaStreamSynchronize(s));
            const double wnb = std::sqrt(hbuf[k].x);
            double wn = std::sqrt(hbuf[m + 2].x);
            for (int i = 0; i < k; ++i) H[i * m + j] = cd(hbuf[i].x, hbuf[i].y);
            if (wn < 0.707 * wnb) {
                arnoldi_dots<T>(Vp, ldv, k, w.as<T>(), n, part.as<double2>(), red2.as<double2>(), s);
                arnoldi_project<T>(Vp, ldv, k, red2.as<double2>(), w.as<T>(), n,
                                   reinterpret_cast<double*>(part.p), nrm.as<double>(), s);
                SB_CUDA(cudaMemcpyAsync(hbuf, red2.p, sizeof(double2) * k, cudaMemcpyDeviceToHost, s));
                SB_CUDA(cudaMemcpyAsync(hbuf + m + 2, nrm.p, sizeof(double), cudaMemcpyDeviceToHost, s));
                SB_CUDA(cudaStreamSynchronize(s));
                for (int i = 0; i < k; ++i) H[i * m + j] += cd(hbuf[i].x, hbuf[i].y);
                wn = std::sqrt(hbuf[m + 2].x);
            }
            H[(j + 1) * m + j] = wn;
            bool inner_conv = false;
            if (wn < 1e-20) inner_conv = true;
            else scale_vec<T, T>(w.as<T>(), 1.0 / wn, Vj(j + 1), n, s);
            for (int64_t i = 0; i < j; ++i) {
                const cd t = std::conj(cs[i]) * H[i * m + j] + std::conj(sn[i]) * H[(i + 1) * m + j];
                H[(i + 1) * m + j] = cd(0, 0) - sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
                H[i * m + j] = t;
            }
            cd c, sg;
            givens(H[j * m + j], H[(j + 1) * m + j], c, sg);
            cs.push_back(c);
            sn.push_back(sg);
            H[j * m + j] = std::conj(c) * H[j * m + j] + std::conj(sg) * H[(j + 1) * m + j];
            H[(j + 1) * m + j] = 0.0;
            const cd t = std::conj(c) * g[j] + std::conj(sg) * g[j + 1];
            g[j + 1] = cd(0, 0) - sg * g[j] + c * g[j + 1];
            g[j] = t;
            const double absr = std::abs(g[j + 1]);
            const double relr = absr / pbnorm;
            const bool should_check = (j % std::max<int64_t>(check_interval, 1)) == 0 || j == m - 1 || inner_conv;
            const bool conv = relr < tol || (!inner_conv && absr < 1e-20);
            if (should_check && conv) {
                update_x(upper_solve(H, m, g, j + 1));
                const double tr = true_rel(bnorm);
                if (tr >= tol && tr >= 1e-20) {
                    ++R.restarts;
                    restart_now = true;
                    break;
                }
                R.converged = true;
                R.status = SB_SOLVER_CONVERGED;
                R.estimated = relr;
                R.residual = tr;
                return R;
            }
            if (inner_conv) {
                update_x(upper_solve(H, m, g, j + 1));
                const double ar = true_rel(bnorm);
                R.estimated = relr;
                R.residual = ar;
                R.converged = ar < tol;
                R.status = R.converged ? SB_SOLVER_CONVERGED : SB_SOLVER_BREAKDOWN;
                return R;
            }
        }
        if (restart_now) continue;
        update_x(upper_solve(H, m, g, m));
        const double tr = true_rel(bnorm);
        if (tr < tol) {
            R.converged = true;
            R.status = SB_SOLVER_CONVERGED;
            R.estimated = tr;
            R.residual = tr;
            return R;
        }
        ++R.restarts;
    }
    R.residual = true_rel(bnorm);
    R.estimated = R.residual;
    R.status = SB_SOLVER_MAX_ITERATIONS;
    return R;
}

// finalize_gmres_solution (gmres.rs:159-247): residual and backward error from one more product.
void finalize(const Operator& op, const double2* b, const double2* x, sb_gmres_stats& st,
              double tol) {
    const int64_t n = op.n;
    DevBuf ax, part, sums;
    ax.alloc(sizeof(double2) * n);
    part.alloc(sizeof(double2) * (n + 255) / 256 * 4 + 64);
    gemv_c128(op.A64.as<double2>(), n, x, ax.as<double2>(), Trans::N, op.stream,
              const_cast<Operator&>(op).scratch);
    ++st.matvecs;
    // |b - Ax|^2, |Ax|^2, |b|^2 on the host (n complex copies: cheap next to the solve).
    std::vector<double2> hb(n), hax(n), hx(n);
    SB_CUDA(cudaMemcpyAsync(hb.data(), b, sizeof(double2) * n, cudaMemcpyDeviceToHost, op.stream));
    SB_CUDA(cudaMemcpyAsync(hax.data(), ax.p, sizeof(double2) * n, cudaMemcpyDeviceToHost, op.stream));
    SB_CUDA(cudaMemcpyAsync(hx.data(), x, sizeof(double2) * n, cudaMemcpyDeviceToHost, op.stream));
    SB_CUDA(cudaStreamSynchronize(op.stream));
    double rs = 0, as = 0, bs = 0;
    bool finite = true;
    for (int64_t i = 0; i < n; ++i) {
        const double dr = hb[i].x - hax[i].x, di = hb[i].y - hax[i].y;
        rs += dr * dr + di * di;
        as += hax[i].x * hax[i].x + hax[i].y * hax[i].y;
        bs += hb[i].x * hb[i].x + hb[i].y * hb[i].y;
        if (!std::isfinite(hx[i].x) || !std::isfinite(hx[i].y) || !std::isfinite(hax[i].x) ||
            !std::isfinite(hax[i].y))
            finite = false;
    }
    if (!finite || !std::isfinite(rs)) {
        st.status = SB_SOLVER_NUMERICAL_ERROR;
        st.converged = 0;
        st.residual = INFINITY;
        st.backward_error = INFINITY;
        return;
    }
    const double rn = std::sqrt(rs), bn = std::sqrt(bs);
    st.residual = bn > 0 ? rn / bn : rn;
    st.backward_error = rn / std::max(std::sqrt(as) + bn, 2.2250738585072014e-308);
    (void)tol;
}

}  // namespace

void gmres_fp64(const Operator& op, const double2* b, double2* x, bool x0_given,
                const sb_gmres_config& cfg, int precond, sb_gmres_stats& st) {
    SB_CUDA(cudaSetDevice(op.device));
    const int64_t n = op.n;
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, op.stream));
    if (!x0_given) SB_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, op.stream));
    DevBuf part;
    part.alloc(sizeof(double) * gemv_partials(n));
    DevBuf nrm;
    nrm.alloc(sizeof(double));
    Operator& mop = const_cast<Operator&>(op);
    Problem<double2> P;
    P.n = n;
    P.stream = op.stream;
    P.jacobi = precond == SB_PRECOND_JACOBI ? op.diag.as<double2>() : nullptr;
    P.apply = [&](const double2* xi, double2* yo) {
        gemv_c128(op.A64.as<double2>(), n, xi, yo, Trans::N, op.stream, mop.scratch);
    };
    P.residual = [&](const double2* xi, const double2* bi, double2* ro) {
        gemv_residual_c128(op.A64.as<double2>(), n, xi, bi, ro, part.as<double>(), op.stream);
        sum_real(part.as<double>(), gemv_partials(n), nrm.as<double>(), op.stream);
        double h = 0;
        SB_CUDA(cudaMemcpyAsync(&h, nrm.p, sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        SB_CUDA(cudaStreamSynchronize(op.stream));
        return std::sqrt(h);
    };
    CoreResult R = gmres_core<double2>(P, b, x, cfg.max_iterations, cfg.restart, cfg.tolerance,
                                       cfg.convergence_check_interval);
    st = sb_gmres_stats{};
    st.iterations = R.iterations;
    st.restarts = R.restarts;
    st.matvecs = R.matvecs;
    st.estimated_residual = R.estimated;
    st.converged = R.converged ? 1 : 0;
    st.status = R.status;
    finalize(op, b, x, st, cfg.tolerance);
    SB_CUDA(cudaEventRecord(e1, op.stream));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    st.device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

void gmres_mixed_ir(const Operator& op, const double2* b, double2* x, bool x0_given,
                    const sb_ir_config& cfg, sb_gmres_stats& st) {
    SB_REQUIRE(op.precision == SB_PRECISION_FP64_FP32 && op.A32.p, SB_ERR_INVALID_ARGUMENT,
               "mixed solve: the operator has no complex64 copy (assemble with SB_PRECISION_FP64_FP32)");
    SB_CUDA(cudaSetDevice(op.device));
    const int64_t n = op.n;
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, op.stream));
    if (!x0_given) SB_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, op.stream));
    DevBuf r64, r32, d32, part, nrm, one;
    r64.alloc(sizeof(double2) * n);
    r32.alloc(sizeof(float2) * n);
    d32.alloc(sizeof(float2) * n);
    part.alloc(sizeof(double) * gemv_partials(n));
    nrm.alloc(sizeof(double));
    one.alloc(sizeof(double2));
    const double2 h_one = make_double2(1.0, 0.0);
    SB_CUDA(cudaMemcpy(one.p, &h_one, sizeof(double2), cudaMemcpyHostToDevice));
    auto residual64 = [&]() {
        gemv_residual_c128(op.A64.as<double2>(), n, x, b, r64.as<double2>(), part.as<double>(), op.stream);
        sum_real(part.as<double>(), gemv_partials(n), nrm.as<double>(), op.stream);
        double h = 0;
        SB_CUDA(cudaMemcpyAsync(&h, nrm.p, sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        SB_CUDA(cudaStreamSynchronize(op.stream));
        return std::sqrt(h);
    };
    Problem<float2> P;
    P.n = n;
    P.stream = op.stream;
    P.apply = [&](const float2* xi, float2* yo) {
        gemv_c64(op.A32.as<float2>(), n, op.lda32, xi, yo, nullptr, nullptr, op.stream);
    };
    P.residual = [&](const float2* xi, const float2* bi, float2* ro) {
        gemv_c64(op.A32.as<float2>(), n, op.lda32, xi, ro, bi, part.as<double>(), op.stream);
        sum_real(part.as<double>(), gemv_partials(n), nrm.as<double>(), op.stream);
        double h = 0;
        SB_CUDA(cudaMemcpyAsync(&h, nrm.p, sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        SB_CUDA(cudaStreamSynchronize(op.stream));
        return std::sqrt(h);
    };
    st = sb_gmres_stats{};
    // ||b|| from the residual of x = 0 when no guess is given, else separately.
    double bnorm;
    {
        DevBuf zero;
        zero.alloc(sizeof(double2) * n);
        SB_CUDA(cudaMemsetAsync(zero.p, 0, sizeof(double2) * n, op.stream));
        gemv_residual_c128(op.A64.as<double2>(), n, zero.as<double2>(), b, r64.as<double2>(), part.as<double>(), op.stream);
        sum_real(part.as<double>(), gemv_partials(n), nrm.as<double>(), op.stream);
        double h = 0;
        SB_CUDA(cudaMemcpyAsync(&h, nrm.p, sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        SB_CUDA(cudaStreamSynchronize(op.stream));
        bnorm = std::sqrt(h);
        ++st.matvecs;
    }
    const double bref = bnorm < 1e-15 ? 1.0 : bnorm;
    int status = SB_SOLVER_MAX_ITERATIONS;
    bool converged = false;
    double rel = 1.0;
    for (int64_t it = 0; it <= cfg.max_refinements; ++it) {
        const double rn = residual64();
        ++st.matvecs;
        rel = rn / bref;
        if (rel < cfg.tolerance) {
            converged = true;
            status = SB_SOLVER_CONVERGED;
            break;
        }
        if (!std::isfinite(rn)) {
            status = SB_SOLVER_NUMERICAL_ERROR;
            break;
        }
        if (it == cfg.max_refinements) break;
        // Inner correction: A32 d = r / ||r|| in FP32, then x += ||r|| d in FP64.
        scale_vec<double2, float2>(r64.as<double2>(), 1.0 / rn, r32.as<float2>(), n, op.stream);
        SB_CUDA(cudaMemsetAsync(d32.p, 0, sizeof(float2) * n, op.stream));
        CoreResult R = gmres_core<float2>(P, r32.as<float2>(), d32.as<float2>(), cfg.inner_max_iterations,
                                          cfg.inner_restart, cfg.inner_tolerance, 1);
        st.iterations += R.iterations;
        st.restarts += R.restarts;
        st.matvecs += R.matvecs;
        st.matvecs_fp32 += R.matvecs;
        basis_update<float2, double2>(d32.as<float2>(), n, 1, one.as<double2>(), rn, x, n, op.stream);
        ++st.refinements;
        if (R.status == SB_SOLVER_BREAKDOWN && R.iterations == 0) {
            status = SB_SOLVER_BREAKDOWN;
            break;
        }
    }
    st.estimated_residual = rel;
    st.converged = converged ? 1 : 0;
    st.status = status;
    finalize(op, b, x, st, cfg.tolerance);
    SB_CUDA(cudaEventRecord(e1, op.stream));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    st.device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

}  // namespace sb
