// Per-kernel-class device timing with CUDA events on the launching stream (off by default).

#include <atomic>
#include <mutex>

#include "sb_profile.cuh"

namespace sb {

bool g_prof_on = false;
static std::atomic<int64_t> g_kernels{0};

void count_launch() { g_kernels.fetch_add(1, std::memory_order_relaxed); }
static std::mutex g_prof_mu;
struct Pending {
    int kind;
    cudaEvent_t a, b;
};
static std::vector<Pending> g_pending;
static double g_ms[SB_PROF_KINDS] = {};
static int64_t g_launches[SB_PROF_KINDS] = {};

ProfScope::ProfScope(int kind, cudaStream_t s) : kind_(kind), s_(s) {
    if (!g_prof_on) return;
    if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
        cudaGetLastError();
        a_ = b_ = nullptr;
        return;
    }
    cudaEventRecord(a_, s_);
    active_ = true;
}

ProfScope::~ProfScope() {
    if (!active_) return;
    cudaEventRecord(b_, s_);
    std::lock_guard<std::mutex> lock(g_prof_mu);
    g_pending.push_back({kind_, a_, b_});
}

void profile_flush() {
    std::lock_guard<std::mutex> lock(g_prof_mu);
    for (auto& p : g_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            g_ms[p.kind] += ms;
            g_launches[p.kind] += 1;
        } else {
            cudaGetLastError();
        }
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    g_pending.clear();
}

void profile_read(sb_profile* out, bool reset) {
    profile_flush();
    std::lock_guard<std::mutex> lock(g_prof_mu);
    out->kernels = reset ? g_kernels.exchange(0) : g_kernels.load();
    for (int k = 0; k < SB_PROF_KINDS; ++k) {
        out->ms[k] = g_ms[k];
        out->launches[k] = g_launches[k];
        if (reset) {
            g_ms[k] = 0.0;
            g_launches[k] = 0;
        }
    }
}

}  // namespace sb
