// FP32 fused multiply-add rate of the device (sb_measure_fp32_rate): the denominator of the FP32
// far-field kernel's roofline, measured on the part the kernel runs on instead of taken from a
// data sheet. No reference counterpart (instrumentation).
//
// Every thread runs 8 independent dependency chains of FMAs (enough to cover the pipe latency at
// full occupancy), scalar or as sm_100's packed f32x2 FMA; the grid is 8 CTAs of 256 threads per
// SM. The result of every chain is stored so that no FMA can be removed.

#include "sb_internal.cuh"
#include "sb_profile.cuh"

namespace sb {
namespace {

constexpr int kChains = 8;
constexpr int kRateThreads = 256;

template <bool kPacked>
__global__ void __launch_bounds__(kRateThreads) k_fma_rate(float* __restrict__ out, int iters, float a, float b) {
    const float seed = 1e-3f * static_cast<float>(threadIdx.x & 31);
    if constexpr (kPacked) {
        float2 acc[kChains];
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc[c] = make_float2(seed + c, seed - c);
        const float2 A = make_float2(a, a), B = make_float2(b, b);
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) acc[c] = __ffma2_rn(acc[c], A, B);
        }
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < kChains; ++c) s += acc[c].x + acc[c].y;
        out[blockIdx.x * (int64_t)kRateThreads + threadIdx.x] = s;
    } else {
        float acc[kChains];
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc[c] = seed + c;
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) acc[c] = fmaf(acc[c], a, b);
        }
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < kChains; ++c) s += acc[c];
        out[blockIdx.x * (int64_t)kRateThreads + threadIdx.x] = s;
    }
}

template <bool kPacked>
double rate_tflops(int sms, float* out, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    const int blocks = sms * 8;
    const int iters = 1 << 14;
    k_fma_rate<kPacked><<<blocks, kRateThreads, 0, s>>>(out, iters, 0.9999999f, 1e-7f);  // warm-up
    count_launch();
    SB_CUDA(cudaGetLastError());
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        SB_CUDA(cudaEventRecord(e0, s));
        k_fma_rate<kPacked><<<blocks, kRateThreads, 0, s>>>(out, iters, 0.9999999f, 1e-7f);
        count_launch();
        SB_CUDA(cudaEventRecord(e1, s));
        SB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = ms < best ? ms : best;
    }
    const double flop = 2.0 * (kPacked ? 2.0 : 1.0) * kChains * static_cast<double>(iters) * blocks * kRateThreads;
    return flop / (best * 1e-3) / 1e12;
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" SB_API int sb_measure_fp32_rate(int device, double* scalar_tflops, double* packed_tflops) {
    return abi_guard([&] {
        SB_REQUIRE(scalar_tflops && packed_tflops, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_CUDA(cudaSetDevice(device));
        const int sms = device_sm_count(device);
        DevBuf out;
        out.alloc(sizeof(float) * static_cast<size_t>(sms) * 8 * kRateThreads);
        cudaStream_t s = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        SB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            SB_CUDA(cudaEventCreate(&e0));
            SB_CUDA(cudaEventCreate(&e1));
            *scalar_tflops = rate_tflops<false>(sms, out.as<float>(), s, e0, e1);
            *packed_tflops = rate_tflops<true>(sms, out.as<float>(), s, e0, e1);
        } catch (...) {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        SB_CUDA(cudaStreamSynchronize(s));
        SB_CUDA(cudaStreamDestroy(s));
    });
}
