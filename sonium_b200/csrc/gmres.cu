// Restarted GMRES and mixed-precision iterative refinement with device-resident Arnoldi cycles.
//
// Reference: gmres_core (crates/sonium-solvers/crates/sonium-solvers-iterative/src/gmres.rs:631-1047)
// with finalize_gmres_solution (gmres.rs:159-247), givens_rotation / solve_upper_triangular
// (gmres_common.rs:91-127) and the CGS + DGKS (0.707) orthogonalisation of cgs_orth.rs:180-300.
//
// One restart cycle is a fixed sequence of kernels per Arnoldi step: matvec, Gram-Schmidt dots
// and projection, a single-thread FP64 kernel that fills the Hessenberg column, applies the
// Givens rotations and tests convergence, the optional DGKS second pass, and the normalisation of
// the next basis vector. Every kernel of the cycle is gated by the instance's `active` flag, so
// the whole cycle is captured once as a CUDA graph and replayed: after convergence the rest of
// the cycle costs only empty launches, and the host synchronises twice per cycle (initial
// residual, then true residual after the update) instead of once per step. The arithmetic and the
// decisions (DGKS threshold, convergence tests, restart / breakdown logic) are the reference's.

#include <complex>
#include <functional>
#include <mutex>

#include "sb_blas.cuh"
#include "sb_device.cuh"
#include "sb_internal.cuh"
#include "sb_krylov.cuh"
#include "sb_profile.cuh"

namespace sb {

using cd = std::complex<double>;

namespace {

__global__ void k_cycle_init(KState* __restrict__ st, double2* __restrict__ H, double2* __restrict__ g,
                             int m, int interval, double beta, double pbnorm, double tol) {
    cycle_init_dev(st, H, g, m, interval, beta, pbnorm, tol, blockIdx.x * (int64_t)blockDim.x + threadIdx.x,
                   (int64_t)gridDim.x * blockDim.x, true);
}

__global__ void k_after_first(KState* __restrict__ st, const double2* __restrict__ red,
                              const double* __restrict__ nrm, double2* __restrict__ H, int j) {
    after_first_dev(st, red, nrm, H, j);
}

__global__ void k_givens(KState* __restrict__ st, const double2* __restrict__ red2,
                         const double* __restrict__ nrm2, double2* __restrict__ H,
                         double2* __restrict__ cs, double2* __restrict__ sn, double2* __restrict__ g,
                         int j) {
    givens_step_dev(st, red2, nrm2, H, cs, sn, g, j);
}

__global__ void k_upper_solve(const KState* __restrict__ st, const double2* __restrict__ H,
                              const double2* __restrict__ g, double2* __restrict__ y) {
    upper_solve_dev(st, H, g, y);
}

// Final statistics of a solve: per-CTA sums of |b - A x|^2, |A x|^2, |b|^2 and the count of
// non-finite x or A x entries (from A x itself, or from a residual r as A x = b - r), then one warp
// adds the CTAs' sums in CTA order.
constexpr int kFinThreads = 256, kFinBlocks = 296;
__global__ void __launch_bounds__(kFinThreads) k_final_sums(const double2* __restrict__ b,
                                                            const double2* __restrict__ axr, bool is_r,
                                                            const double2* __restrict__ x, int64_t n,
                                                            double* __restrict__ part) {
    __shared__ double red[kFinThreads / 32][4];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)kFinThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kFinThreads) {
        const double2 bb = b[i];
        double2 ax = axr[i];
        if (is_r) ax = make_double2(bb.x - ax.x, bb.y - ax.y);
        const double dr = bb.x - ax.x, di = bb.y - ax.y;
        v[0] += dr * dr + di * di;
        v[1] += ax.x * ax.x + ax.y * ax.y;
        v[2] += bb.x * bb.x + bb.y * bb.y;
        const double2 xx = x[i];
        if (!isfinite(xx.x) || !isfinite(xx.y) || !isfinite(ax.x) || !isfinite(ax.y)) v[3] += 1.0;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 4; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0)
        for (int c = 0; c < 4; ++c) red[warp][c] = v[c];
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < kFinThreads / 32; ++w) t += red[w][threadIdx.x];
        part[4 * blockIdx.x + threadIdx.x] = t;
    }
}

__global__ void k_final_reduce(const double* __restrict__ part, int nb, double* __restrict__ out) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = threadIdx.x; c < nb; c += 32)
        for (int t = 0; t < 4; ++t) v[t] += part[4 * c + t];
    for (int t = 0; t < 4; ++t) v[t] = warp_sum(v[t]);
    if (threadIdx.x == 0)
        for (int t = 0; t < 4; ++t) out[t] = v[t];
}

struct PinnedBuf {
    void* p = nullptr;
    void alloc(size_t bytes) {
        if (p) return;
        SB_CUDA(cudaMallocHost(&p, bytes));
    }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

// Persistent per-operator workspace of one vector type.
template <class T>
struct KrylovWork {
    int64_t n = 0, m = 0, ldv = 0;
    DevBuf V, w, opb, r, part, red, red2, nrm, ydev, H, cs, sn, g, st;
    DevBuf cnt;  // last-CTA reduction counters of the Arnoldi kernels (zero between launches)
    PinnedBuf host;  // KState + two doubles, then two KState slots of the chunk checks
    // The cycle is captured as chunks of kCycleChunk Arnoldi steps (one graph each), launched
    // while the cycle is still active, so a converged cycle stops paying for gated launches.
    std::vector<cudaGraph_t> graphs;
    std::vector<cudaGraphExec_t> execs;
    std::vector<int64_t> chunk_kernels;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const void* key_A = nullptr;
    const void* key_jac = nullptr;  // the Jacobi diagonal the cycle reads, if any
    const void* key_pre = nullptr;  // the block-Jacobi inverses the cycle reads, if any
    int key_pre_bs = 0;
    int key_jacobi = -1;
    unsigned key_prof = 0;
    std::vector<ProfPair> prof_pairs;

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
    ~KrylovWork() {
        reset_graph();
        for (cudaEvent_t& e : ev)
            if (e) cudaEventDestroy(e);
    }

    void ensure(int64_t n_, int64_t m_) {
        if (n_ == n && m_ == m) return;
        reset_graph();
        n = n_;
        m = m_;
        ldv = (n + 1) / 2 * 2;  // even: every basis vector 16-byte aligned for vector loads
        V.alloc(sizeof(T) * (m + 1) * ldv);
        w.alloc(sizeof(T) * ldv);
        opb.alloc(sizeof(T) * ldv);
        r.alloc(sizeof(T) * ldv);
        const int64_t dchunks = arnoldi_dot_chunks(n);
        part.alloc(sizeof(double2) * std::max<int64_t>(dchunks * (m + 2), (n + 255) / 256 + gemv_partials(n)));
        red.alloc(sizeof(double2) * (m + 2));
        red2.alloc(sizeof(double2) * (m + 2));
        nrm.alloc(sizeof(double) * 4);
        ydev.alloc(sizeof(double2) * (m + 1));
        H.alloc(sizeof(double2) * (m + 1) * m);
        cs.alloc(sizeof(double2) * m);
        sn.alloc(sizeof(double2) * m);
        g.alloc(sizeof(double2) * (m + 1));
        st.alloc(sizeof(KState));
        if (!cnt.p) {
            cnt.alloc(sizeof(unsigned) * 2 * kArnoldiCounters);
            memset_sync(cnt.p, 0, sizeof(unsigned) * 2 * kArnoldiCounters);
        }
        host.alloc(3 * sizeof(KState) + 64);
        for (cudaEvent_t& e : ev)
            if (!e) SB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    KState* hstate() { return static_cast<KState*>(host.p); }
    KState* hslot(int i) {
        return reinterpret_cast<KState*>(static_cast<char*>(host.p) + sizeof(KState) + 64) + i;
    }
    double* hscalar() { return reinterpret_cast<double*>(static_cast<char*>(host.p) + sizeof(KState)); }
};

struct SolveWork {
    KrylovWork<double2> k64;
    KrylovWork<float2> k32;
    DevBuf r64, r32, d32, t32, partg, nrmg, one, ax;
    DevBuf t64, z64;  // the FP64 solver's block-Jacobi vectors (allocated on first use)
    PinnedBuf pin;
    DevBuf npart, nred;  // scratch of the ||b|| reduction
    DevBuf fin;          // partial sums of the final statistics (k_final_sums) and their totals
    int64_t n = 0;
    double2* k64_part(int64_t) { return npart.as<double2>(); }
    double2* k64_red() { return nred.as<double2>(); }
    void ensure(int64_t n_) {
        if (n_ == n) return;
        n = n_;
        pin.alloc(64);
        npart.alloc(sizeof(double2) * arnoldi_dot_chunks(n));
        nred.alloc(sizeof(double2) * 2);
        fin.alloc(sizeof(double) * 4 * (kFinBlocks + 1));
        r64.alloc(sizeof(double2) * n);
        r32.alloc(sizeof(float2) * n);
        d32.alloc(sizeof(float2) * n);
        t32.alloc(sizeof(float2) * n);
        partg.alloc(sizeof(double) * gemv_partials(n));
        nrmg.alloc(sizeof(double) * 2);
        one.alloc(sizeof(double2));
        const double2 h_one = make_double2(1.0, 0.0);
        SB_CUDA(cudaMemcpy(one.p, &h_one, sizeof(double2), cudaMemcpyHostToDevice)); SB_CUDA(cudaStreamSynchronize(0));
        ax.alloc(sizeof(double2) * n);
        t64.release();
        z64.release();
    }
    void ensure_bj64(int64_t n_) {
        if (t64.bytes == sizeof(double2) * n_) return;
        t64.release();
        z64.release();
        t64.alloc(sizeof(double2) * n_);
        z64.alloc(sizeof(double2) * n_);
    }
};

// Workspaces of destroyed operators are kept (a few per process) for the next operator of the
// same size and device: its buffers, pinned host memory and captured cycle graphs are reused (a
// graph is replayed only when every pointer it bakes in matches; see run_cycle).
namespace {
std::mutex g_ws_mu;
std::vector<std::pair<int, SolveWork*>> g_ws_pool;
constexpr size_t kWsPool = 4;
}  // namespace

void destroy_solve_work(Operator& op) {
    if (!op.work) return;
    cudaSetDevice(op.device);
    SolveWork* w = static_cast<SolveWork*>(op.work);
    op.work = nullptr;
    std::lock_guard<std::mutex> lock(g_ws_mu);
    if (g_ws_pool.size() < kWsPool) {
        g_ws_pool.push_back({op.device, w});
    } else {
        delete w;
    }
}

void solve_work_pool_trim(int device) {
    std::lock_guard<std::mutex> lock(g_ws_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto it = g_ws_pool.begin(); it != g_ws_pool.end();) {
        if (device >= 0 && it->first != device) {
            ++it;
            continue;
        }
        cudaSetDevice(it->first);
        delete it->second;
        it = g_ws_pool.erase(it);
    }
    cudaSetDevice(cur);
}

static SolveWork& solve_work(const Operator& op) {
    Operator& o = const_cast<Operator&>(op);
    if (!o.work) {
        std::lock_guard<std::mutex> lock(g_ws_mu);
        for (auto it = g_ws_pool.begin(); it != g_ws_pool.end(); ++it)
            if (it->first == op.device && it->second->n == op.n) {
                o.work = it->second;
                g_ws_pool.erase(it);
                break;
            }
        if (!o.work) o.work = new SolveWork();
    }
    SolveWork& w = *static_cast<SolveWork*>(o.work);
    w.ensure(op.n);
    return w;
}

// y = A x with FP64 vectors: the complex128 matrix when present, else the complex64 one with
// FP64 accumulation.
void op_gemv64(const Operator& op, const double2* x, double2* y, Gate g) {
    if (op.A64.p)
        gemv_c128(op.A64.as<double2>(), op.n, x, y, Trans::N, op.stream, const_cast<Operator&>(op).scratch, g);
    else
        gemv_c64_x64(op.A32.as<float2>(), op.n, op.lda32, x, y, nullptr, nullptr, op.stream, g);
}

int64_t op_residual64_partials(const Operator& op) {
    return op.A64.p ? gemv_partials(op.n) : gemv_x64_partials(op.n);
}

// r = b - A x with FP64 vectors and per-CTA partial norms (op_residual64_partials entries).
void op_residual64(const Operator& op, const double2* x, const double2* b, double2* r, double* part) {
    if (op.A64.p)
        gemv_residual_c128(op.A64.as<double2>(), op.n, x, b, r, part, op.stream);
    else
        gemv_c64_x64(op.A32.as<float2>(), op.n, op.lda32, x, r, b, part, op.stream);
}

namespace {

// Device operator callbacks of one GMRES problem.
template <class T>
struct Problem {
    int64_t n = 0;
    const void* key_A = nullptr;                                // identifies the captured graph
    std::function<void(const T*, T*, Gate)> apply;              // y = A x (gated)
    std::function<void(const T*, const T*, T*, double*)> residual;  // r = b - A x, partials
    int64_t partials = 0;                                       // partial norms residual writes
    const void* key_pre = nullptr;                              // right preconditioner's data
    int key_pre_bs = 0;
    const double2* jacobi = nullptr;                            // diagonal for Jacobi, or null
    cudaStream_t stream = nullptr;
};

struct CoreResult {
    int64_t iterations = 0, restarts = 0, matvecs = 0;
    double residual = 1.0, estimated = 1.0;
    bool converged = false;
    int status = SB_SOLVER_MAX_ITERATIONS;
    const void* r_last = nullptr;  // device b - A x for the returned x, when one was formed
};

// Arnoldi steps [j0, j1) of one cycle, every launch gated by st->active.
template <class T>
void launch_cycle(KrylovWork<T>& W, const Problem<T>& P, int64_t j0, int64_t j1) {
    const int64_t n = P.n;
    const cudaStream_t s = P.stream;
    KState* st = W.st.template as<KState>();
    const Gate ga{&st->active, nullptr};
    const Gate gb{&st->active, &st->reorth};
    T* Vp = W.V.template as<T>();
    T* w = W.w.template as<T>();
    double* nrm = W.nrm.template as<double>();
    for (int64_t j = j0; j < j1; ++j) {
        capture_step(static_cast<int>(j));
        const int k = static_cast<int>(j + 1);
        if (P.jacobi) {
            P.apply(Vp + j * W.ldv, W.opb.template as<T>(), ga);
            jacobi_apply<T>(P.jacobi, W.opb.template as<T>(), w, n, s, ga);
        } else {
            P.apply(Vp + j * W.ldv, w, ga);
        }
        unsigned* cd = W.cnt.template as<unsigned>();           // dots counters
        unsigned* cp = cd + kArnoldiCounters;                    // projection counter
        arnoldi_dots<T>(Vp, W.ldv, k, w, n, W.part.template as<double2>(), W.red.template as<double2>(), s, ga, cd);
        arnoldi_project<T>(Vp, W.ldv, k, W.red.template as<double2>(), w, n, W.part.template as<double>(), nrm, s, ga,
                           cp);
        k_after_first<<<1, 1, 0, s>>>(st, W.red.template as<double2>(), nrm, W.H.template as<double2>(), static_cast<int>(j));
        count_launch();
        arnoldi_dots<T>(Vp, W.ldv, k, w, n, W.part.template as<double2>(), W.red2.template as<double2>(), s, gb, cd);
        arnoldi_project<T>(Vp, W.ldv, k, W.red2.template as<double2>(), w, n, W.part.template as<double>(), nrm + 1,
                           s, gb, cp);
        k_givens<<<1, 1, 0, s>>>(st, W.red2.template as<double2>(), nrm + 1, W.H.template as<double2>(),
                                 W.cs.template as<double2>(), W.sn.template as<double2>(), W.g.template as<double2>(),
                                 static_cast<int>(j));
        count_launch();
        scale_vec<T, T>(w, 0.0, &st->inv_wn, Vp + (j + 1) * W.ldv, n, s, ga);
    }
    SB_CUDA(cudaGetLastError());
}

// Steps per captured chunk of a restart cycle: smaller chunks leave fewer gated launches after
// convergence (N = 20480 mixed solve: 4 steps 13.43 ms, 6 steps 13.49 ms, 8 steps 13.64 ms, 12
// steps 13.64 ms).
constexpr int64_t kCycleChunk = 4;

// Replays the captured cycle (capturing it first when buffers, matrix or profiling changed):
// chunk c + 1 is queued before the host reads chunk c's state, so the device never waits for the
// host; launching stops once a chunk leaves the cycle inactive (the queued one returns at once).
template <class T>
void run_cycle(KrylovWork<T>& W, const Problem<T>& P, int64_t m) {
    const int jac = P.jacobi ? 1 : 0;
    const int64_t nch = (m + kCycleChunk - 1) / kCycleChunk;
    if (W.execs.empty() || W.key_A != P.key_A || W.key_jacobi != jac || W.key_jac != P.jacobi ||
        W.key_prof != prof_key() || W.key_pre != P.key_pre || W.key_pre_bs != P.key_pre_bs) {
        W.reset_graph();
        capture_begin(&W.prof_pairs);
        for (int64_t c = 0; c < nch; ++c) {
            const int64_t before = kernel_count();
            cudaGraph_t g = nullptr;
            SB_CUDA(cudaStreamBeginCapture(P.stream, cudaStreamCaptureModeThreadLocal));
            try {
                launch_cycle<T>(W, P, c * kCycleChunk, std::min(m, (c + 1) * kCycleChunk));
            } catch (...) {
                cudaStreamEndCapture(P.stream, &g);
                if (g) cudaGraphDestroy(g);
                capture_end();
                W.reset_graph();
                throw;
            }
            SB_CUDA(cudaStreamEndCapture(P.stream, &g));
            W.graphs.push_back(g);
            cudaGraphExec_t e = nullptr;
            SB_CUDA(cudaGraphInstantiate(&e, g, 0));
            W.execs.push_back(e);
            W.chunk_kernels.push_back(kernel_count() - before);
            add_kernel_count(-(kernel_count() - before));
        }
        capture_end();
        W.key_A = P.key_A;
        W.key_jac = P.jacobi;
        W.key_jacobi = jac;
        W.key_prof = prof_key();
        W.key_pre = P.key_pre;
        W.key_pre_bs = P.key_pre_bs;
    }
    auto launch = [&](int64_t c) {
        SB_CUDA(cudaGraphLaunch(W.execs[c], P.stream));
        add_kernel_count(W.chunk_kernels[c]);
        SB_CUDA(cudaMemcpyAsync(W.hslot(static_cast<int>(c & 1)), W.st.p, sizeof(KState), cudaMemcpyDeviceToHost,
                                P.stream));
        SB_CUDA(cudaEventRecord(W.ev[c & 1], P.stream));
    };
    launch(0);
    if (nch > 1) launch(1);
    for (int64_t c = 0; c + 1 < nch; ++c) {
        SB_CUDA(cudaEventSynchronize(W.ev[c & 1]));
        if (!W.hslot(static_cast<int>(c & 1))->active) break;
        if (c + 2 < nch) launch(c + 2);
    }
}

// gmres_core (gmres.rs:631-1047) with an identity or Jacobi left preconditioner.
// x_zero: x enters as zero, so the first residual is b itself (no product needed).
// trust_estimate: an inner solve of iterative refinement, whose caller forms the FP64 residual
// itself: an estimated convergence ends the solve without the exact residual product.
template <class T>
CoreResult gmres_core(KrylovWork<T>& W, const Problem<T>& P, const T* b, T* x, int64_t max_it,
                      int64_t m, double tol, int64_t check_interval, bool x_zero = false,
                      bool trust_estimate = false) {
    const int64_t n = P.n;
    const cudaStream_t s = P.stream;
    W.ensure(n, m);
    CoreResult R;
    KState* hst = W.hstate();
    double* hsc = W.hscalar();
    double* nrm = W.nrm.template as<double>();
    double* partd = W.part.template as<double>();
    auto norm_of = [&](const T* v) -> double {
        arnoldi_dots<T>(v, n, 0, v, n, W.part.template as<double2>(), W.red2.template as<double2>(), s);
        SB_CUDA(cudaMemcpyAsync(hsc, W.red2.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        return std::sqrt(hsc[0]);
    };
    auto residual = [&](T* out, bool with_state) -> double {
        P.residual(x, b, out, partd);
        sum_real(partd, P.partials, nrm + 2, s);
        SB_CUDA(cudaMemcpyAsync(hsc, nrm + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
        if (with_state) SB_CUDA(cudaMemcpyAsync(hst, W.st.p, sizeof(KState), cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        ++R.matvecs;
        return std::sqrt(hsc[0]);
    };
    const double raw_bn = norm_of(b);
    const bool rhs_zero = raw_bn < 1e-15;
    const double bnorm = rhs_zero ? 1.0 : raw_bn;
    double pbnorm = bnorm;
    if (P.jacobi) {
        jacobi_apply<T>(P.jacobi, b, W.w.template as<T>(), n, s);
        const double raw_pb = norm_of(W.w.template as<T>());
        if (!rhs_zero && raw_pb < 1e-15) {
            R.status = SB_SOLVER_BREAKDOWN;
            return R;
        }
        pbnorm = rhs_zero ? 1.0 : raw_pb;
    }
    for (int64_t outer = 0; outer < max_it; ++outer) {
        double rn;
        if (outer == 0 && x_zero) {
            SB_CUDA(cudaMemcpyAsync(W.opb.p, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
            rn = raw_bn;
        } else {
            rn = residual(W.opb.template as<T>(), false);
        }
        R.r_last = W.opb.p;
        const double trel = rn / bnorm;
        double beta = rn;
        const T* src = W.opb.template as<T>();
        if (P.jacobi) {
            jacobi_apply<T>(P.jacobi, W.opb.template as<T>(), W.w.template as<T>(), n, s);
            beta = norm_of(W.w.template as<T>());
            src = W.w.template as<T>();
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
        scale_vec<T, T>(src, 1.0 / beta, nullptr, W.V.template as<T>(), n, s);
        k_cycle_init<<<8, 256, 0, s>>>(W.st.template as<KState>(), W.H.template as<double2>(),
                                       W.g.template as<double2>(), static_cast<int>(m),
                                       static_cast<int>(check_interval), beta, pbnorm, tol);
        count_launch();
        SB_CUDA(cudaGetLastError());
        run_cycle<T>(W, P, m);
        k_upper_solve<<<1, 1, 0, s>>>(W.st.template as<KState>(), W.H.template as<double2>(),
                                      W.g.template as<double2>(), W.ydev.template as<double2>());
        count_launch();
        SB_CUDA(cudaGetLastError());
        basis_update<T, T>(W.V.template as<T>(), W.ldv, 0, &W.st.template as<KState>()->jdone,
                           W.ydev.template as<double2>(), 1.0, x, n, s);
        R.r_last = nullptr;
        if (trust_estimate) {
            SB_CUDA(cudaMemcpyAsync(hst, W.st.p, sizeof(KState), cudaMemcpyDeviceToHost, s));
            SB_CUDA(cudaStreamSynchronize(s));
            profile_account(W.prof_pairs, hst->jdone);
            R.iterations += hst->jdone;
            R.matvecs += hst->jdone;
            if (hst->reason != 0) {
                R.estimated = R.residual = hst->relres;
                R.converged = hst->relres < tol;
                R.status = R.converged ? SB_SOLVER_CONVERGED : SB_SOLVER_BREAKDOWN;
                return R;
            }
            ++R.restarts;
            continue;
        }
        const double tr = residual(W.r.template as<T>(), true) / bnorm;
        R.r_last = W.r.p;
        profile_account(W.prof_pairs, hst->jdone);
        R.iterations += hst->jdone;
        R.matvecs += hst->jdone;
        if (hst->reason == 1) {
            if (tr >= tol && tr >= 1e-20) {
                ++R.restarts;
                continue;
            }
            R.converged = true;
            R.status = SB_SOLVER_CONVERGED;
            R.estimated = hst->relres;
            R.residual = tr;
            return R;
        }
        if (hst->reason == 2) {
            R.estimated = hst->relres;
            R.residual = tr;
            R.converged = tr < tol;
            R.status = R.converged ? SB_SOLVER_CONVERGED : SB_SOLVER_BREAKDOWN;
            return R;
        }
        if (tr < tol) {
            R.converged = true;
            R.status = SB_SOLVER_CONVERGED;
            R.estimated = tr;
            R.residual = tr;
            return R;
        }
        ++R.restarts;
    }
    R.residual = residual(W.r.template as<T>(), false) / bnorm;
    R.r_last = W.r.p;
    R.estimated = R.residual;
    R.status = SB_SOLVER_MAX_ITERATIONS;
    return R;
}

// finalize_gmres_solution (gmres.rs:159-247): residual and backward error of the returned x.
// `r`, when given, is b - A x already formed for this x (A x = b - r then needs no product).
void finalize(const Operator& op, SolveWork& sw, const double2* b, const double2* x, sb_gmres_stats& st,
              const double2* r = nullptr) {
    const int64_t n = op.n;
    const double2* axr = r;
    if (!r) {
        op_gemv64(op, x, sw.ax.as<double2>(), Gate{});
        ++st.matvecs;
        axr = sw.ax.as<double2>();
    }
    k_final_sums<<<kFinBlocks, kFinThreads, 0, op.stream>>>(b, axr, r != nullptr, x, n, sw.fin.as<double>());
    count_launch();
    k_final_reduce<<<1, 32, 0, op.stream>>>(sw.fin.as<double>(), kFinBlocks, sw.fin.as<double>() + 4 * kFinBlocks);
    count_launch();
    SB_CUDA(cudaGetLastError());
    double* h = static_cast<double*>(sw.pin.p) + 2;
    SB_CUDA(cudaMemcpyAsync(h, sw.fin.as<double>() + 4 * kFinBlocks, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                            op.stream));
    SB_CUDA(cudaStreamSynchronize(op.stream));
    const double rs = h[0], as = h[1], bs = h[2];
    const bool finite = h[3] == 0.0;
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
}

struct DeviceTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit DeviceTimer(cudaStream_t s_) : s(s_) {
        SB_CUDA(cudaEventCreate(&a));
        SB_CUDA(cudaEventCreate(&b));
        SB_CUDA(cudaEventRecord(a, s));
    }
    double stop() {
        SB_CUDA(cudaEventRecord(b, s));
        SB_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        SB_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
    ~DeviceTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

Problem<double2> problem64(const Operator& op) {
    Problem<double2> P;
    P.n = op.n;
    P.stream = op.stream;
    P.key_A = op.A64.p ? op.A64.p : op.A32.p;
    P.partials = op_residual64_partials(op);
    P.apply = [&op](const double2* xi, double2* yo, Gate g) { op_gemv64(op, xi, yo, g); };
    P.residual = [&op](const double2* xi, const double2* bi, double2* ro, double* part) {
        op_residual64(op, xi, bi, ro, part);
    };
    return P;
}

Problem<float2> problem32(const Operator& op) {
    Problem<float2> P;
    P.n = op.n;
    P.stream = op.stream;
    P.key_A = op.A32.p;
    P.partials = gemv_partials(op.n);
    P.apply = [&op](const float2* xi, float2* yo, Gate g) {
        gemv_c64(op.A32.as<float2>(), op.n, op.lda32, xi, yo, nullptr, nullptr, op.stream, g);
    };
    P.residual = [&op](const float2* xi, const float2* bi, float2* ro, double* part) {
        gemv_c64(op.A32.as<float2>(), op.n, op.lda32, xi, ro, bi, part, op.stream);
    };
    return P;
}

// The inner problem on the complex-half copy (SB_INNER_FP16).
Problem<float2> problem16(const Operator& op) {
    Problem<float2> P;
    P.n = op.n;
    P.stream = op.stream;
    P.key_A = op.A16.p;
    P.partials = gemv16_partials(op.n);
    const float* inv = op.half_scale.as<float>() + op.n;  // per-row inverse scales
    P.apply = [&op, inv](const float2* xi, float2* yo, Gate g) {
        gemv_c16(op.A16.as<uint32_t>(), op.n, op.lda16, inv, xi, yo, nullptr, nullptr, op.stream, g);
    };
    P.residual = [&op, inv](const float2* xi, const float2* bi, float2* ro, double* part) {
        gemv_c16(op.A16.as<uint32_t>(), op.n, op.lda16, inv, xi, ro, bi, part, op.stream);
    };
    return P;
}

}  // namespace

namespace {

// Right block-Jacobi preconditioning of the FP64 solver: GMRES on (A M^-1) z = b - A x0 from z = 0,
// then x = x0 + M^-1 z. The restart and convergence tests of gmres_core see b - A M^-1 z, which is
// b - A x for that x, so the tolerance keeps its meaning (relative to ||b||: the inner tolerance
// is scaled by ||b|| / ||b - A x0|| when an initial guess is given).
void gmres_fp64_block_jacobi(const Operator& op, SolveWork& sw, Problem<double2>& P, const double2* b, double2* x,
                             bool x0_given, const sb_gmres_config& cfg, sb_gmres_stats& st) {
    const int64_t n = op.n;
    bj64_prepare(const_cast<Operator&>(op));
    sw.ensure_bj64(n);
    double2* t = sw.t64.as<double2>();
    double2* z = sw.z64.as<double2>();
    auto a_apply = P.apply;
    auto a_res = P.residual;
    P.apply = [&op, t, a_apply](const double2* xi, double2* yo, Gate g) {
        bj64_apply(op, xi, t, g);
        a_apply(t, yo, g);
    };
    P.residual = [&op, t, a_res](const double2* xi, const double2* bi, double2* ro, double* part) {
        bj64_apply(op, xi, t, Gate{});
        a_res(t, bi, ro, part);
    };
    P.key_pre = op.bj64_inv.p;
    P.key_pre_bs = op.bj_size;
    st = sb_gmres_stats{};
    const double2* rhs = b;
    double tol = cfg.tolerance;
    if (x0_given) {
        // r0 = b - A x0 (one product), and the tolerance relative to ||b||
        double* hsc = static_cast<double*>(sw.pin.p);
        arnoldi_dots<double2>(b, n, 0, b, n, sw.k64_part(n), sw.k64_red(), op.stream);
        SB_CUDA(cudaMemcpyAsync(hsc, sw.k64_red(), sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        op_residual64(op, x, b, sw.r64.as<double2>(), sw.partg.as<double>());
        sum_real(sw.partg.as<double>(), op_residual64_partials(op), sw.nrmg.as<double>(), op.stream);
        SB_CUDA(cudaMemcpyAsync(hsc + 1, sw.nrmg.p, sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        SB_CUDA(cudaStreamSynchronize(op.stream));
        ++st.matvecs;
        const double bn = std::sqrt(hsc[0]), rn = std::sqrt(hsc[1]);
        if (bn >= 1e-15 && rn > 0.0) tol = cfg.tolerance * bn / rn;
        rhs = sw.r64.as<double2>();
    }
    // gmres_core accumulates its updates into z and takes it to be zero on entry
    SB_CUDA(cudaMemsetAsync(z, 0, sizeof(double2) * n, op.stream));
    CoreResult R = gmres_core<double2>(sw.k64, P, rhs, z, cfg.max_iterations, cfg.restart, tol,
                                       cfg.convergence_check_interval, /*x_zero=*/true, false);
    // x = x0 + M^-1 z (x = M^-1 z without an initial guess)
    bj64_apply(op, z, t, Gate{});
    if (x0_given) {
        basis_update<double2, double2>(t, n, 1, nullptr, sw.one.as<double2>(), 1.0, x, n, op.stream);
    } else {
        SB_CUDA(cudaMemcpyAsync(x, t, sizeof(double2) * n, cudaMemcpyDeviceToDevice, op.stream));
    }
    st.iterations = R.iterations;
    st.restarts = R.restarts;
    st.matvecs += R.matvecs;
    st.estimated_residual = R.estimated;
    st.converged = R.converged ? 1 : 0;
    st.status = R.status;
    // Without an initial guess the last residual gmres_core formed is b - A x for this very x
    // (the same M^-1 z, by the same kernel); otherwise finalize forms it.
    finalize(op, sw, b, x, st, x0_given ? nullptr : static_cast<const double2*>(R.r_last));
}

}  // namespace

void gmres_fp64(const Operator& op, const double2* b, double2* x, bool x0_given,
                const sb_gmres_config& cfg, int precond, sb_gmres_stats& st) {
    SB_CUDA(cudaSetDevice(op.device));
    SB_REQUIRE(cfg.restart <= kMaxKrylov, SB_ERR_INVALID_ARGUMENT, "restart exceeds the supported Krylov dimension");
    SolveWork& sw = solve_work(op);
    DeviceTimer timer(op.stream);
    if (!x0_given) SB_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * op.n, op.stream));
    Problem<double2> P = problem64(op);
    P.jacobi = precond == SB_PRECOND_JACOBI ? op.diag.as<double2>() : nullptr;
    if (precond == SB_PRECOND_BLOCK_JACOBI) {
        gmres_fp64_block_jacobi(op, sw, P, b, x, x0_given, cfg, st);
        st.device_ms = timer.stop();
        return;
    }
    CoreResult R = gmres_core<double2>(sw.k64, P, b, x, cfg.max_iterations, cfg.restart, cfg.tolerance,
                                       cfg.convergence_check_interval, !x0_given, false);
    st = sb_gmres_stats{};
    st.iterations = R.iterations;
    st.restarts = R.restarts;
    st.matvecs = R.matvecs;
    st.estimated_residual = R.estimated;
    st.converged = R.converged ? 1 : 0;
    st.status = R.status;
    finalize(op, sw, b, x, st, static_cast<const double2*>(R.r_last));
    st.device_ms = timer.stop();
}

void gmres_mixed_ir(const Operator& op, const double2* b, double2* x, bool x0_given,
                    const sb_ir_config& cfg, sb_gmres_stats& st) {
    SB_REQUIRE(op.A32.p, SB_ERR_INVALID_ARGUMENT,
               "mixed solve: the operator has no complex64 matrix (assemble with SB_PRECISION_FP64_FP32 or "
               "SB_PRECISION_FP32)");
    SB_REQUIRE(cfg.inner_restart <= kMaxKrylov, SB_ERR_INVALID_ARGUMENT,
               "inner_restart exceeds the supported Krylov dimension");
    SB_CUDA(cudaSetDevice(op.device));
    const int64_t n = op.n;
    SolveWork& sw = solve_work(op);
    DeviceTimer timer(op.stream);
    if (!x0_given) SB_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, op.stream));
    double* hsc = static_cast<double*>(sw.pin.p);
    auto residual64 = [&](const double2* xv) {
        op_residual64(op, xv, b, sw.r64.as<double2>(), sw.partg.as<double>());
        sum_real(sw.partg.as<double>(), op_residual64_partials(op), sw.nrmg.as<double>(), op.stream);
        SB_CUDA(cudaMemcpyAsync(hsc, sw.nrmg.p, sizeof(double), cudaMemcpyDeviceToHost, op.stream));
        SB_CUDA(cudaStreamSynchronize(op.stream));
        return std::sqrt(hsc[0]);
    };
    const bool half = op.inner == SB_INNER_FP16;
    if (half) half_prepare(const_cast<Operator&>(op));
    Problem<float2> P = half ? problem16(op) : problem32(op);
    // Right block-Jacobi preconditioning of the inner solve: (A M^-1) y = r, d = M^-1 y.
    const bool bj = op.inner_precond == SB_INNER_PRECOND_BLOCK_JACOBI;
    if (bj) {
        bj_prepare(const_cast<Operator&>(op));
        float2* t = sw.t32.as<float2>();
        auto inner_apply = P.apply;
        auto inner_res = P.residual;
        P.apply = [&op, t, inner_apply](const float2* xi, float2* yo, Gate g) {
            bj_apply(op, xi, t, g);
            inner_apply(t, yo, g);
        };
        P.residual = [&op, t, inner_res](const float2* xi, const float2* bi, float2* ro, double* part) {
            bj_apply(op, xi, t, Gate{});
            inner_res(t, bi, ro, part);
        };
        P.key_pre = op.bj_inv.p;
        P.key_pre_bs = op.bj_size;
    }
    st = sb_gmres_stats{};
    // ||b|| by a norm kernel; with a zero initial guess the first residual is b itself.
    arnoldi_dots<double2>(b, n, 0, b, n, sw.k64_part(n), sw.k64_red(), op.stream);
    SB_CUDA(cudaMemcpyAsync(hsc, sw.k64_red(), sizeof(double), cudaMemcpyDeviceToHost, op.stream));
    SB_CUDA(cudaStreamSynchronize(op.stream));
    const double bnorm = std::sqrt(hsc[0]);
    const double bref = bnorm < 1e-15 ? 1.0 : bnorm;
    int status = SB_SOLVER_MAX_ITERATIONS;
    bool converged = false;
    double rel = 1.0;
    bool r_valid = false;  // r64 holds b - A x for the current x
    for (int64_t it = 0; it <= cfg.max_refinements; ++it) {
        double rn;
        if (it == 0 && !x0_given) {
            SB_CUDA(cudaMemcpyAsync(sw.r64.p, b, sizeof(double2) * n, cudaMemcpyDeviceToDevice, op.stream));
            rn = bnorm;
        } else {
            rn = residual64(x);
            ++st.matvecs;
        }
        r_valid = true;
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
        scale_vec<double2, float2>(sw.r64.as<double2>(), 1.0 / rn, nullptr, sw.r32.as<float2>(), n, op.stream);
        SB_CUDA(cudaMemsetAsync(sw.d32.p, 0, sizeof(float2) * n, op.stream));
        // The inner solve need not reduce the residual further than the outer target asks:
        // relax its tolerance (never below inner_tolerance) on the last refinements.
        const double inner_tol = std::max(cfg.inner_tolerance, 0.5 * cfg.tolerance / rel);
        CoreResult R = gmres_core<float2>(sw.k32, P, sw.r32.as<float2>(), sw.d32.as<float2>(),
                                          cfg.inner_max_iterations, cfg.inner_restart, inner_tol, 1,
                                          /*x_zero=*/true, /*trust_estimate=*/true);
        st.iterations += R.iterations;
        st.restarts += R.restarts;
        st.matvecs += R.matvecs;
        st.matvecs_fp32 += R.matvecs;
        const float2* dcorr = sw.d32.as<float2>();
        if (bj) {
            bj_apply(op, sw.d32.as<float2>(), sw.t32.as<float2>(), Gate{});
            dcorr = sw.t32.as<float2>();
        }
        basis_update<float2, double2>(dcorr, n, 1, nullptr, sw.one.as<double2>(), rn, x, n, op.stream);
        r_valid = false;
        ++st.refinements;
        if (R.status == SB_SOLVER_BREAKDOWN && R.iterations == 0) {
            status = SB_SOLVER_BREAKDOWN;
            break;
        }
    }
    st.estimated_residual = rel;
    st.converged = converged ? 1 : 0;
    st.status = status;
    finalize(op, sw, b, x, st, r_valid ? sw.r64.as<double2>() : nullptr);
    st.device_ms = timer.stop();
}

}  // namespace sb
