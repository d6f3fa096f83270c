// Per-kernel-class device timing with CUDA events on the launching stream (off by default).

#include <atomic>
#include <mutex>

#include "sb_profile.cuh"

namespace sb {

bool g_prof_on = false;
unsigned g_prof_mask = ~0u;
static std::atomic<int64_t> g_kernels{0};
static std::mutex g_prof_mu;
static std::vector<ProfPair> g_pending;
static double g_ms[SB_PROF_KINDS] = {};
static int64_t g_launches[SB_PROF_KINDS] = {};
static thread_local std::vector<ProfPair>* t_capture = nullptr;
static thread_local int t_step = 0;

void count_launch() { g_kernels.fetch_add(1, std::memory_order_relaxed); }
int64_t kernel_count() { return g_kernels.load(); }
void add_kernel_count(int64_t d) { g_kernels.fetch_add(d); }

void capture_begin(std::vector<ProfPair>* pairs) {
    t_capture = pairs;
    t_step = 0;
}
void capture_step(int step) { t_step = step; }
void capture_end() { t_capture = nullptr; }

ProfScope::ProfScope(int kind, cudaStream_t s) : kind_(kind), s_(s) {
    if (!g_prof_on || !(g_prof_mask & (1u << kind_))) return;
    if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
        cudaGetLastError();
        a_ = b_ = nullptr;
        return;
    }
    // Inside a capture a plain record only expresses a dependency; an external record becomes an
    // event-record node that every replay executes, so the pair can time the captured launches.
    if (t_capture) cudaEventRecordWithFlags(a_, s_, cudaEventRecordExternal);
    else cudaEventRecord(a_, s_);
    active_ = true;
}

ProfScope::~ProfScope() {
    if (!active_) return;
    if (t_capture) cudaEventRecordWithFlags(b_, s_, cudaEventRecordExternal);
    else cudaEventRecord(b_, s_);
    if (t_capture) {
        t_capture->push_back({kind_, t_step, a_, b_});
        return;
    }
    std::lock_guard<std::mutex> lock(g_prof_mu);
    g_pending.push_back({kind_, 0, a_, b_});
}

static void flush_locked() {
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

void profile_account(const std::vector<ProfPair>& pairs, int steps_done) {
    if (pairs.empty()) return;
    std::lock_guard<std::mutex> lock(g_prof_mu);
    for (const auto& p : pairs) {
        if (p.step >= steps_done) continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            g_ms[p.kind] += ms;
            g_launches[p.kind] += 1;
        } else {
            cudaGetLastError();
        }
    }
}

void profile_release(std::vector<ProfPair>& pairs) {
    for (auto& p : pairs) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    pairs.clear();
}

void profile_read(sb_profile* out, bool reset) {
    std::lock_guard<std::mutex> lock(g_prof_mu);
    flush_locked();
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
