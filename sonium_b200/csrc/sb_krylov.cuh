// Device-side Arnoldi cycle state and the FP64 Hessenberg / Givens step shared by the
// single-instance and the batched GMRES drivers (internal).
//
// Reference: gmres_core (crates/sonium-solvers/crates/sonium-solvers-iterative/src/gmres.rs:
// 790-900), givens_rotation / solve_upper_triangular (gmres_common.rs:91-127).
#pragma once

#include <cuda_runtime.h>

namespace sb {

// Device state of one Arnoldi cycle.
struct KState {
    int active;     // the cycle is still running
    int reorth;     // the current step needs the DGKS second pass
    int jdone;      // Arnoldi steps taken in this cycle
    int reason;     // 0 = m steps completed, 1 = estimated convergence, 2 = inner breakdown
    int m, interval;
    double pbnorm, tol;
    double wnb, wn, inv_wn;
    double absres, relres;
};

__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double2 cconj_mul(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cmul_(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 csub_(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cadd_(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// Cycle start: H = 0, g = (beta, 0, ...), state reset (all threads of the launch cooperate on H).
__device__ __forceinline__ void cycle_init_dev(KState* st, double2* H, double2* g, int m, int interval, double beta,
                                               double pbnorm, double tol, int64_t tid, int64_t nthreads, bool active) {
    const int64_t tot = (int64_t)(m + 1) * m;
    for (int64_t t = tid; t < tot; t += nthreads) H[t] = make_double2(0.0, 0.0);
    for (int64_t t = tid; t <= m; t += nthreads) g[t] = make_double2(t == 0 ? beta : 0.0, 0.0);
    if (tid == 0) {
        st->active = active ? 1 : 0;
        st->reorth = 0;
        st->jdone = 0;
        st->reason = 0;
        st->m = m;
        st->interval = interval < 1 ? 1 : interval;
        st->pbnorm = pbnorm;
        st->tol = tol;
        st->wn = st->wnb = st->inv_wn = 0.0;
        st->absres = st->relres = 0.0;
    }
}

// After the first Gram-Schmidt pass: Hessenberg column j and the DGKS (0.707) decision.
__device__ __forceinline__ void after_first_dev(KState* st, const double2* red, const double* nrm, double2* H,
                                                int j) {
    if (!st->active) return;
    const int m = st->m;
    for (int i = 0; i <= j; ++i) H[i * m + j] = red[i];
    const double wnb = sqrt(red[j + 1].x);
    const double wn = sqrt(*nrm);
    st->wnb = wnb;
    st->wn = wn;
    st->reorth = wn < 0.707 * wnb ? 1 : 0;
}

// givens_rotation (gmres_common.rs:91-106).
__device__ __forceinline__ void givens_dev(double2 a, double2 b, double2& c, double2& s) {
    const double tol = 1e-30;
    if (cabs_(b) < tol) {
        c = make_double2(1.0, 0.0);
        s = make_double2(0.0, 0.0);
        return;
    }
    if (cabs_(a) < tol) {
        c = make_double2(0.0, 0.0);
        s = make_double2(1.0, 0.0);
        return;
    }
    const double r = sqrt((a.x * a.x + a.y * a.y) + (b.x * b.x + b.y * b.y));
    const double ir = 1.0 / r;
    c = make_double2(a.x * ir, a.y * ir);
    s = make_double2(b.x * ir, b.y * ir);
}

// Second-pass update, Hessenberg subdiagonal, rotations and the convergence test of step j.
__device__ __forceinline__ void givens_step_dev(KState* st, const double2* red2, const double* nrm2, double2* H,
                                                double2* cs, double2* sn, double2* g, int j) {
    if (!st->active) return;
    const int m = st->m;
    if (st->reorth) {
        for (int i = 0; i <= j; ++i) H[i * m + j] = cadd_(H[i * m + j], red2[i]);
        st->wn = sqrt(*nrm2);
    }
    const double wn = st->wn;
    H[(j + 1) * m + j] = make_double2(wn, 0.0);
    const bool inner = wn < 1e-20;
    st->inv_wn = inner ? 0.0 : 1.0 / wn;
    for (int i = 0; i < j; ++i) {
        const double2 hij = H[i * m + j], hi1 = H[(i + 1) * m + j];
        const double2 t = cadd_(cconj_mul(cs[i], hij), cconj_mul(sn[i], hi1));
        H[(i + 1) * m + j] = csub_(cmul_(cs[i], hi1), cmul_(sn[i], hij));
        H[i * m + j] = t;
    }
    double2 c, s;
    givens_dev(H[j * m + j], H[(j + 1) * m + j], c, s);
    cs[j] = c;
    sn[j] = s;
    H[j * m + j] = cadd_(cconj_mul(c, H[j * m + j]), cconj_mul(s, H[(j + 1) * m + j]));
    H[(j + 1) * m + j] = make_double2(0.0, 0.0);
    const double2 t = cadd_(cconj_mul(c, g[j]), cconj_mul(s, g[j + 1]));
    g[j + 1] = csub_(cmul_(c, g[j + 1]), cmul_(s, g[j]));
    g[j] = t;
    const double absr = cabs_(g[j + 1]);
    const double relr = absr / st->pbnorm;
    const bool should_check = (j % st->interval) == 0 || j == m - 1 || inner;
    const bool conv = relr < st->tol || (!inner && absr < 1e-20);
    st->jdone = j + 1;
    st->absres = absr;
    st->relres = relr;
    if (should_check && conv) {
        st->active = 0;
        st->reason = 1;
    } else if (inner) {
        st->active = 0;
        st->reason = 2;
    } else if (j == m - 1) {
        st->active = 0;
        st->reason = 0;
    }
}

// solve_upper_triangular for the jdone x jdone leading block.
__device__ __forceinline__ void upper_solve_dev(const KState* st, const double2* H, const double2* g, double2* y) {
    const int m = st->m, k = st->jdone;
    for (int i = k - 1; i >= 0; --i) {
        double2 s = g[i];
        for (int j = i + 1; j < k; ++j) s = csub_(s, cmul_(H[i * m + j], y[j]));
        const double2 h = H[i * m + i];
        if (cabs_(h) > 1e-30) {
            const double d = h.x * h.x + h.y * h.y;
            const double2 inv = make_double2(h.x / d, -h.y / d);
            y[i] = cmul_(s, inv);
        } else {
            y[i] = make_double2(0.0, 0.0);
        }
    }
}

}  // namespace sb
