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
void count_launch();
// Sites in flight that mm_propagate_sites actually uses for `slots` asked:
// at most the site count, and for the persistent schedule balanced so the
// last wave is (nearly) full.  Defined in propagate.cu.
int propagation_slots(int nsites, int slots, int schedule);

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

#define MM_CHECK_LAUNCH(what)  \
  do {                          \
    ::mm::count_launch();       \
    MM_CHECK_CUDA(cudaGetLastError(), what); \
  } while (0)

// ---------------------------------------------------------------- complex --
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float cnorm2(float2 a) { return a.x * a.x + a.y * a.y; }

__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cmul(double2 a, float2 b) { return cmul(a, make_double2(b.x, b.y)); }
__host__ __device__ __forceinline__ double cnorm2(double2 a) { return a.x * a.x + a.y * a.y; }

// FP32 complex arithmetic whose multiplications by the DFT rotation
// constants take each constant as an unevaluated pair hi + lo of floats; with
// TW the twiddle tables are carried the same way (entries {hi, lo}).  The
// rounding of a constant is the same in every transform, so its error adds up
// coherently over hundreds of line transforms; carrying the constant to
// ~2^-48 leaves only the data-dependent (incoherent) roundings of FP32
// butterflies.  The rotations dominate that coherent error, the twiddle
// tables add a smaller share.
template <bool TW>
struct __align__(8) cfx_t {
  float x, y;
};
using cfx = cfx_t<true>;  // rotations and twiddle tables compensated
template <class C> struct IsCompensated { static constexpr bool value = false; };
template <bool TW> struct IsCompensated<cfx_t<TW>> { static constexpr bool value = true; };

template <bool TW>
__host__ __device__ __forceinline__ cfx_t<TW> cadd(cfx_t<TW> a, cfx_t<TW> b) { return {a.x + b.x, a.y + b.y}; }
template <bool TW>
__host__ __device__ __forceinline__ cfx_t<TW> csub(cfx_t<TW> a, cfx_t<TW> b) { return {a.x - b.x, a.y - b.y}; }
// a * b for a data value or a plain FP32 twiddle b: ordinary FP32 product.
template <bool TW>
__host__ __device__ __forceinline__ cfx_t<TW> cmul(cfx_t<TW> a, float2 b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * w for a constant w = (hi.x + lo.x) + i (hi.y + lo.y), packed {hi.x, hi.y, lo.x, lo.y}.
__device__ __forceinline__ cfx cmul(cfx a, float4 w) {
  const float cx = fmaf(a.x, w.z, -a.y * w.w);
  const float cy = fmaf(a.x, w.w, a.y * w.z);
  return cfx{fmaf(a.x, w.x, fmaf(-a.y, w.y, cx)), fmaf(a.x, w.y, fmaf(a.y, w.x, cy))};
}

// Conversions between the storage type (float2) and a register type.
template <class C> __device__ __forceinline__ C from_f2(float2 a);
template <> __device__ __forceinline__ float2 from_f2<float2>(float2 a) { return a; }
template <> __device__ __forceinline__ double2 from_f2<double2>(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ float2 to_f2(float2 a) { return a; }
__device__ __forceinline__ float2 to_f2(double2 a) { return make_float2(float(a.x), float(a.y)); }
template <class C> __device__ __forceinline__ C promote(float2 a) { return from_f2<C>(a); }
template <class C> __device__ __forceinline__ C promote(double2 a);
template <> __device__ __forceinline__ double2 promote<double2>(double2 a) { return a; }
template <class C> __device__ __forceinline__ C make_c(double re, double im);
template <> __device__ __forceinline__ float2 make_c<float2>(double re, double im) { return make_float2(float(re), float(im)); }
template <> __device__ __forceinline__ double2 make_c<double2>(double re, double im) { return make_double2(re, im); }
template <> __device__ __forceinline__ cfx from_f2<cfx>(float2 a) { return cfx{a.x, a.y}; }
template <bool TW> __device__ __forceinline__ float2 to_f2(cfx_t<TW> a) { return make_float2(a.x, a.y); }
template <class C, bool TW> __device__ __forceinline__ C promote(cfx_t<TW> a) { return a; }
// Twiddle-table entries of a register type: cfx keeps {hi, lo} pairs.
template <class C> struct TwiddleOf { using T = C; };
template <> struct TwiddleOf<cfx> { using T = float4; };
template <class T> __device__ __forceinline__ T make_tw(double re, double im) { return make_c<T>(re, im); }
template <> __device__ __forceinline__ float4 make_tw<float4>(double re, double im) {
  const float hx = float(re), hy = float(im);
  return make_float4(hx, hy, float(re - double(hx)), float(im - double(hy)));
}

// a * (SIGN * i): SIGN = -1 is the forward-DFT quarter turn, +1 the inverse one.
template <int SIGN>
__device__ __forceinline__ float2 quarter(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
template <int SIGN, bool TW>
__device__ __forceinline__ cfx_t<TW> quarter(cfx_t<TW> a) {
  return SIGN < 0 ? cfx_t<TW>{a.y, -a.x} : cfx_t<TW>{-a.y, a.x};
}
template <int SIGN>
__device__ __forceinline__ double2 quarter(double2 a) {
  return SIGN < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

// |E|^(2*order) as the reference resample kernel forms it: p = x^2+y^2, then
// p^order by repeated multiplication (optical_kernels.cu:29-32).
__device__ __forceinline__ float photon_power(float2 e, int order) {
  float p = cnorm2(e);
  return order == 1 ? p : (order == 2 ? p * p : p * p * p);
}
__device__ __forceinline__ float photon_power(double2 e, int order) {
  const double p = cnorm2(e);
  return float(order == 1 ? p : (order == 2 ? p * p : p * p * p));
}

// Asynchronous 8-byte global -> shared copy (L1-allocating), its commit and
// the wait for all of this thread's outstanding copies.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
// The same copy with zero fill: `valid` false writes 8 zero bytes to smem and
// reads nothing (gmem must still be a valid address).
__device__ __forceinline__ void cp_async8_zfill(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const unsigned n = valid ? 8u : 0u;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Acquire load of a counter written by other CTAs (GPU scope).
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

}  // namespace mm
