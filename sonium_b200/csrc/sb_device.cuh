// Device-side math shared by the assembly kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sb {

constexpr double kPiD = 3.141592653589793116;     // RN(pi)
constexpr double kInv4Pi = 0x1.45f306dc9c883p-4;  // RN(1/(4 pi))

// ---------------------------------------------------------------------------------------------
// sincos in FP64, written from the published Cody-Waite method: q = rint(x * 2/pi), the
// argument is reduced with a three-double split of pi/2 applied by fused multiply-adds, and
// sin / cos of the reduced argument |r| <= pi/4 (+ rounding) come from their Taylor series
// (coefficients (-1)^k / n!, rounded to double) up to r^19 / r^20, where the truncation error
// is below 1e-19. The quadrant picks the signs. For |x| > 2^20 the reduction loses accuracy,
// so that (never used by the assembly, where |x| = k r) case calls CUDA's sincos.
// Constants: c1 = RN(pi/2), c2 = RN(pi/2 - c1), c3 = RN(pi/2 - c1 - c2); 2/pi rounded.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void sb_sincos(double x, double* s_out, double* c_out) {
    if (!(fabs(x) <= 1048576.0)) {
        sincos(x, s_out, c_out);
        return;
    }
    const double q = rint(x * 0x1.45f306dc9c883p-1);
    double r = fma(-q, 0x1.921fb54442d18p+0, x);
    r = fma(-q, 0x1.1a62633145c07p-54, r);
    r = fma(-q, -0x1.f1976b7ed8fbcp-110, r);
    const double r2 = r * r;
    // sin(r) = r + r^3 * P(r^2)
    double ps = 0x1.952c77030ad4ap-49;
    ps = fma(ps, r2, -0x1.ae7f3e733b81fp-41);
    ps = fma(ps, r2, 0x1.6124613a86d09p-33);
    ps = fma(ps, r2, -0x1.ae64567f544e4p-26);
    ps = fma(ps, r2, 0x1.71de3a556c734p-19);
    ps = fma(ps, r2, -0x1.a01a01a01a01ap-13);
    ps = fma(ps, r2, 0x1.1111111111111p-7);
    ps = fma(ps, r2, -0x1.5555555555555p-3);
    const double sn = fma(ps * r2, r, r);
    // cos(r) = 1 + r^2 * Q(r^2)
    double pc = -0x1.6827863b97d97p-53;
    pc = fma(pc, r2, 0x1.ae7f3e733b81fp-45);
    pc = fma(pc, r2, -0x1.93974a8c07c9dp-37);
    pc = fma(pc, r2, 0x1.1eed8eff8d898p-29);
    pc = fma(pc, r2, -0x1.27e4fb7789f5cp-22);
    pc = fma(pc, r2, 0x1.a01a01a01a01ap-16);
    pc = fma(pc, r2, -0x1.6c16c16c16c17p-10);
    pc = fma(pc, r2, 0x1.5555555555555p-5);
    pc = fma(pc, r2, -0.5);
    const double cs = fma(pc, r2, 1.0);
    const int quad = static_cast<int>(static_cast<long long>(q) & 3);
    double s = sn, c = cs;
    if (quad & 1) {
        s = cs;
        c = -sn;
    }
    if (quad & 2) {
        s = -s;
        c = -c;
    }
    *s_out = s;
    *c_out = c;
}

// 1/sqrt(a) for normal a > 0: FP32 hardware estimate refined by Newton-Raphson
// y <- y (3 - a y^2) / 2 in FP64 (three steps take the ~2^-22 estimate to full precision).
__device__ __forceinline__ double sb_rsqrt(double a) {
    double y = static_cast<double>(rsqrtf(static_cast<float>(a)));
    double h = 0.5 * a;
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    return y;
}

// One Newton step from the hardware's FP64 reciprocal square-root estimate (about 2^-22 relative,
// from the special-function unit without FP32 conversions): relative error below 1e-13, enough
// for the FP64 phase k r of the FP32 far field, whose entries carry FP32 rounding.
__device__ __forceinline__ double sb_rsqrt1(double a) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    return y * fma(-0.5 * a * y, y, 1.5);
}

// The same with two Newton steps: relative error below 2e-14, enough for the phase k r and the
// 1e-10 parity bar of the assembled entries.
__device__ __forceinline__ double sb_rsqrt2(double a) {
    double y = static_cast<double>(rsqrtf(static_cast<float>(a)));
    double h = 0.5 * a;
    y = y * fma(-h * y, y, 1.5);
    y = y * fma(-h * y, y, 1.5);
    return y;
}

// Reduce over the 32 lanes of a warp.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Complex helpers on double2 (x = re, y = im).
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // a*b + c
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) {
    return make_double2(a.x * s, a.y * s);
}

}  // namespace sb
