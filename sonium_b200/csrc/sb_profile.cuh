// Kernel-class timing scopes (internal). A ProfScope records a CUDA event pair around the
// launches it encloses on their stream when profiling is on; sb_profile_read() collects them.
#pragma once

#include <cuda_runtime.h>

#include "sb_internal.cuh"

namespace sb {

extern bool g_prof_on;

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

}  // namespace sb
