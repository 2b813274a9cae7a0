// Shared helpers for the MaoMi B200 kernels: complex arithmetic on float2,
// status codes, the thread-local error message and launch checking.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>

#include "../../include/maomi_b200.h"

namespace mm {

// ----------------------------------------------------------------- errors --
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

#define MM_CHECK_ARG(cond, ...)                     \
  do {                                              \
    if (!(cond)) {                                  \
      ::mm::set_error(__VA_ARGS__);                 \
      return MM_ERR_ARGUMENT;                       \
    }                                               \
  } while (0)

#define MM_CHECK_CUDA(call, what)                                 \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return ::mm::cuda_status(e_, what);    \
  } while (0)

#define MM_CHECK_LAUNCH(what) MM_CHECK_CUDA(cudaGetLastError(), what)

// ---------------------------------------------------------------- complex --
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float cnorm2(float2 a) { return a.x * a.x + a.y * a.y; }

// a * (SIGN * i): SIGN = -1 is the forward-DFT quarter turn, +1 the inverse one.
template <int SIGN>
__device__ __forceinline__ float2 quarter(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// |E|^(2*order) as the reference resample kernel forms it: p = x^2+y^2, then
// p^order by repeated multiplication (optical_kernels.cu:29-32).
__device__ __forceinline__ float photon_power(float2 e, int order) {
  float p = cnorm2(e);
  return order == 1 ? p : (order == 2 ? p * p : p * p * p);
}

// Acquire load of a counter written by other CTAs (GPU scope).
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

}  // namespace mm
