// Kernel-class timing scopes (internal). A ProfScope records a CUDA event pair around the
// launches it encloses on their stream when profiling is on; sb_profile_read() collects them.
// Inside a stream capture the pair becomes part of the graph instead: its events are re-recorded
// by every replay and accounted with profile_account() after the replay completes.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "sb_internal.cuh"

namespace sb {

extern bool g_prof_on;
extern unsigned g_prof_mask;  // kernel classes timed while profiling is on (bit = SB_PROF_*)
// Identifies the profiling configuration a captured graph was recorded under.
inline unsigned prof_key() { return g_prof_on ? g_prof_mask : 0u; }

struct ProfPair {
    int kind;
    int step;  // Arnoldi step of the captured cycle the launch belongs to
    cudaEvent_t a, b;
};

class ProfScope {
   public:
    ProfScope(int kind, cudaStream_t s);
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

   private:
    int kind_;
    cudaStream_t s_;
    cudaEvent_t a_ = nullptr, b_ = nullptr;
    bool active_ = false;
};

void profile_read(sb_profile* out, bool reset);
// Stream-capture support: scopes created between capture_begin and capture_end append their
// event pairs to `pairs` (tagged with the step set by capture_step).
void capture_begin(std::vector<ProfPair>* pairs);
void capture_step(int step);
void capture_end();
// Adds the elapsed times of the pairs of steps < steps_done (call after the replay finished).
void profile_account(const std::vector<ProfPair>& pairs, int steps_done);
void profile_release(std::vector<ProfPair>& pairs);
int64_t kernel_count();
void add_kernel_count(int64_t delta);

}  // namespace sb
