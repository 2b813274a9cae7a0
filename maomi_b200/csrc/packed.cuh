// Complex FP32 arithmetic on the packed instructions of sm_100 (add / mul /
// fma .f32x2: two IEEE single-precision operations per instruction, each
// lane rounded exactly as its scalar form).
//
// A cpk is an ordinary (re, im) pair of floats.  A complex sum is one packed
// add; a product by w = (c, s) is one packed multiply and one packed fma on
// the pair and its swapped halves:
//
//     (re, im) * w = (re, im) * (c, c) + (im, re) * (-s, s)
//
// Swapped halves, a negated half and broadcast or immediate factors are
// operand forms of the packed instructions, so none of them costs an extra
// instruction.  Rotation constants are carried as hi + lo float pairs, as in
// the scalar compensated type (cfx_t).
#pragma once

#include "common.cuh"

namespace mm {

struct __align__(8) cpk {
  float x, y;
};

__device__ __forceinline__ float2 f2(cpk a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cpk pk(float2 a) { return cpk{a.x, a.y}; }
__device__ __forceinline__ float2 bc(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 swapped(cpk a) { return make_float2(a.y, a.x); }

__device__ __forceinline__ cpk cadd(cpk a, cpk b) { return pk(__fadd2_rn(f2(a), f2(b))); }
__device__ __forceinline__ cpk csub(cpk a, cpk b) { return pk(__fadd2_rn(f2(a), make_float2(-b.x, -b.y))); }
__device__ __forceinline__ cpk cneg(cpk a) { return cpk{-a.x, -a.y}; }
// a * (SIGN * i), left to the consumer as swapped, half-negated operands
template <int SIGN>
__device__ __forceinline__ cpk quarter(cpk a) {
  return SIGN < 0 ? cpk{a.y, -a.x} : cpk{-a.y, a.x};
}
// a * w for an FP32 factor w (twiddle-table entry, filter tap, screen sample)
__device__ __forceinline__ cpk cmul(cpk a, float2 w) {
  return pk(__ffma2_rn(f2(a), bc(w.x), __fmul2_rn(swapped(a), make_float2(-w.y, w.y))));
}
// a * conj(w)
__device__ __forceinline__ cpk cmul_conj(cpk a, float2 w) {
  return pk(__ffma2_rn(f2(a), bc(w.x), __fmul2_rn(swapped(a), make_float2(w.y, -w.y))));
}
// a * (hi + lo) for a rotation constant (c, s) given as hi + lo float pairs
__device__ __forceinline__ cpk cmul_hl(cpk a, float ch, float sh, float cl, float sl) {
  const float2 lo = __ffma2_rn(f2(a), bc(cl), __fmul2_rn(swapped(a), make_float2(-sl, sl)));
  return pk(__ffma2_rn(f2(a), bc(ch), __ffma2_rn(swapped(a), make_float2(-sh, sh), lo)));
}
// a * g * (ex + i ey) for |ex| = |ey| = 1 and g = gh + gl: the signed sum
// (ex re - ey im, ey re + ex im) once rounded, then scaled by g
__device__ __forceinline__ cpk cmul_diag(cpk a, float ex, float ey, float gh, float gl) {
  const float2 u = __fadd2_rn(make_float2(ex * a.x, ex * a.y), make_float2(-ey * a.y, ey * a.x));
  return pk(__ffma2_rn(u, bc(gh), __fmul2_rn(u, bc(gl))));
}

template <> __device__ __forceinline__ cpk from_f2<cpk>(float2 a) { return cpk{a.x, a.y}; }
__device__ __forceinline__ float2 to_f2(cpk a) { return make_float2(a.x, a.y); }
template <class C> __device__ __forceinline__ C promote(cpk a) { return a; }
template <> struct TwiddleOf<cpk> { using T = float2; };

}  // namespace mm
