// Host launchers of the dense kernels in blas.cu (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sb_internal.cuh"

namespace sb {

constexpr int kMaxKrylov = 127;  // largest Krylov dimension (restart) the kernels accept

// A launch gate: the kernel does nothing unless *a != 0 (when a is set) and *b != 0 (when b is
// set). Captured Krylov cycles use it to stop work of converged instances without a host round
// trip.
struct Gate {
    const int* a = nullptr;
    const int* b = nullptr;
};

// y = op(A) x for the complex128 matrix (row-major, leading dimension n). T / C use `scratch`.
void gemv_c128(const double2* A, int64_t n, const double2* x, double2* y, Trans t,
               cudaStream_t s, DevBuf& scratch, Gate gate = {});
// r = b - A x with per-CTA partial ||r||^2 in part[gemv_partials(n)].
void gemv_residual_c128(const double2* A, int64_t n, const double2* x, const double2* b,
                        double2* r, double* part, cudaStream_t s, Gate gate = {});
int64_t gemv_partials(int64_t n);
// Complex64 matrix with even leading dimension lda: FP32 vectors / FP32 accumulation, or FP64
// vectors / FP64 accumulation. With b != null the result is b - A x and part gets ||.||^2.
void gemv_c64(const float2* A, int64_t n, int64_t lda, const float2* x, float2* y,
              const float2* b, double* part, cudaStream_t s, Gate gate = {});
void gemv_c64_x64(const float2* A, int64_t n, int64_t lda, const double2* x, double2* y,
                  const double2* b, double* part, cudaStream_t s, Gate gate = {});
int64_t gemv_x64_partials(int64_t n);  // partial norms gemv_c64_x64 writes with b
// Complex-half matrix (uint32 = FP16 re | FP16 im << 16; lda a multiple of 4), FP32 vectors and
// accumulation: y_i = (A x)_i * inv_scale[i], or b_i - (A x)_i * inv_scale[i] with part = ||.||^2.
void gemv_c16(const uint32_t* A, int64_t n, int64_t lda, const float* inv_scale, const float2* x, float2* y,
              const float2* b, double* part, cudaStream_t s, Gate gate = {});
int64_t gemv16_partials(int64_t n);

// out[i] = V_i^H w (i < k), out[k].x = |w|^2; part holds arnoldi_dot_chunks(n) * (k + 1).
// With cnt (kArnoldiCounters zeroed unsigned, owned by one stream's work) the reduction runs in
// the same launch (the last CTA reduces).
constexpr int kArnoldiCounters = 16;
template <class T>
void arnoldi_dots(const T* V, int64_t ldv, int k, const T* w, int64_t n, double2* part,
                  double2* out, cudaStream_t s, Gate gate = {}, unsigned* cnt = nullptr);
int64_t arnoldi_dot_chunks(int64_t n);
// w -= sum_i coeff[i] V_i; *out_norm2 = |w|^2 (part holds ceil(n / 256) doubles); cnt as above.
template <class T>
void arnoldi_project(const T* V, int64_t ldv, int k, const double2* coeff, T* w, int64_t n,
                     double* part, double* out_norm2, cudaStream_t s, Gate gate = {}, unsigned* cnt = nullptr);
void sum_real(const double* part, int64_t m, double* out, cudaStream_t s, Gate gate = {});
// y = alpha x (alpha_dev, when given, overrides alpha).
template <class TI, class TO>
void scale_vec(const TI* x, double alpha, const double* alpha_dev, TO* y, int64_t n,
               cudaStream_t s, Gate gate = {});
// x += alpha * sum_{i < k} y_i V_i, with k read from k_dev when given.
template <class T, class TX>
void basis_update(const T* V, int64_t ldv, int k, const int* k_dev, const double2* y,
                  double alpha, TX* x, int64_t n, cudaStream_t s);
template <class T>
void jacobi_apply(const double2* d, const T* x, T* y, int64_t n, cudaStream_t s, Gate gate = {});

}  // namespace sb
