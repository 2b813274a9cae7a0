// Register-resident small DFTs (sizes 2..32) and the line propagator built on
// them.
//
// A line of N = R1 * R2 complex samples is held by R2 threads, thread t owning
// samples t + R2*m (m < R1).  One "propagate" applies x -> IDFT(Q * DFT(x))
// (the 1-D angular-spectrum step along that axis) as a four-step transform:
//
//   forward : DFT_R1 in registers, twiddle W_N^(t*k1), exchange through
//             shared memory, DFT_R2 in registers -> X[k1 + R1*k2]
//   filter  : multiply by Q in FFT order (Q carries the 1/N of the inverse)
//   inverse : IDFT_R2 in registers, twiddle W_N^(-n_a*k1), exchange,
//             IDFT_R1 in registers -> x[n_a + R2*n_b], back in the input layout.
//
// The spectrum never needs reordering: the filter is applied in the order the
// forward transform produces, and the inverse consumes that order.
#pragma once

#include "common.cuh"

namespace mm {

// cos / sin of pi*k/16, k = 0..16 (exact values rounded once to float).
__device__ constexpr float kCos16[17] = {
    1.0f, 0.98078528040323043058f, 0.92387953251128673848f, 0.83146961230254523567f,
    0.70710678118654752440f, 0.55557023301960222474f, 0.38268343236508977173f, 0.19509032201612826785f,
    0.0f, -0.19509032201612826785f, -0.38268343236508977173f, -0.55557023301960222474f,
    -0.70710678118654752440f, -0.83146961230254523567f, -0.92387953251128673848f, -0.98078528040323043058f,
    -1.0f};
__device__ constexpr float kSin16[17] = {
    0.0f, 0.19509032201612826785f, 0.38268343236508977173f, 0.55557023301960222474f,
    0.70710678118654752440f, 0.83146961230254523567f, 0.92387953251128673848f, 0.98078528040323043058f,
    1.0f, 0.98078528040323043058f, 0.92387953251128673848f, 0.83146961230254523567f,
    0.70710678118654752440f, 0.55557023301960222474f, 0.38268343236508977173f, 0.19509032201612826785f,
    0.0f};

// a * W_32^k with W = exp(SIGN * 2*pi*i/32), k = 0..15 (angle pi*k/16).
template <int SIGN, int K>
__device__ __forceinline__ float2 rot32(float2 a) {
  if constexpr (K == 0) {
    return a;
  } else if constexpr (K == 8) {
    return quarter<SIGN>(a);
  } else {
    const float c = kCos16[K], s = SIGN * kSin16[K];
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

template <int SIGN>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

// 4-point DFT on v[0], v[S], v[2S], v[3S] (natural order in and out).
template <int SIGN, int S = 1>
__device__ __forceinline__ void dft4s(float2* v) {
  float2 t0 = cadd(v[0], v[2 * S]);
  float2 t1 = csub(v[0], v[2 * S]);
  float2 t2 = cadd(v[S], v[3 * S]);
  float2 t3 = quarter<SIGN>(csub(v[S], v[3 * S]));
  v[0] = cadd(t0, t2);
  v[2 * S] = csub(t0, t2);
  v[S] = cadd(t1, t3);
  v[3 * S] = csub(t1, t3);
}

template <int SIGN>
__device__ __forceinline__ void dft4(float2* v) { dft4s<SIGN, 1>(v); }

// 8-point DFT: two interleaved 4-point DFTs and a radix-2 combine.
template <int SIGN>
__device__ __forceinline__ void dft8(float2* v) {
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  dft4<SIGN>(e);
  dft4<SIGN>(o);
  o[1] = rot32<SIGN, 4>(o[1]);
  o[2] = rot32<SIGN, 8>(o[2]);
  o[3] = rot32<SIGN, 12>(o[3]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

// 16-point DFT: radix-4 decimation in time (4 x 4 with W_16 twiddles).
template <int SIGN>
__device__ __forceinline__ void dft16(float2* v) {
  // F_r = DFT4(v[r], v[r+4], v[r+8], v[r+12]) computed in place (stride 4).
#pragma unroll
  for (int r = 0; r < 4; ++r) dft4s<SIGN, 4>(v + r);
  // v[r + 4*k1] now holds F_r[k1]; twiddle by W_16^(r*k1) = W_32^(2*r*k1).
  v[1 + 4 * 1] = rot32<SIGN, 2>(v[1 + 4 * 1]);
  v[1 + 4 * 2] = rot32<SIGN, 4>(v[1 + 4 * 2]);
  v[1 + 4 * 3] = rot32<SIGN, 6>(v[1 + 4 * 3]);
  v[2 + 4 * 1] = rot32<SIGN, 4>(v[2 + 4 * 1]);
  v[2 + 4 * 2] = rot32<SIGN, 8>(v[2 + 4 * 2]);
  v[2 + 4 * 3] = rot32<SIGN, 12>(v[2 + 4 * 3]);
  v[3 + 4 * 1] = rot32<SIGN, 6>(v[3 + 4 * 1]);
  v[3 + 4 * 2] = rot32<SIGN, 12>(v[3 + 4 * 2]);
  {  // W_16^9 = -W_16^1
    float2 a = rot32<SIGN, 2>(v[3 + 4 * 3]);
    v[3 + 4 * 3] = make_float2(-a.x, -a.y);
  }
  // X[k1 + 4*k2] = DFT4 over r of the twiddled F_r[k1]: rows of 4.
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4s<SIGN, 1>(v + 4 * k1);
  // v[4*k1 + k2] holds X[k1 + 4*k2]: transpose the 4x4 index in registers.
  float2 t[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// 32-point DFT: radix-2 decimation in time over two 16-point DFTs.
template <int SIGN>
__device__ __forceinline__ void dft32(float2* v) {
  float2 e[16], o[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  dft16<SIGN>(e);
  dft16<SIGN>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    float2 w;
    switch (k) {  // resolved at compile time after unrolling
      case 0: w = o[k]; break;
      case 1: w = rot32<SIGN, 1>(o[k]); break;
      case 2: w = rot32<SIGN, 2>(o[k]); break;
      case 3: w = rot32<SIGN, 3>(o[k]); break;
      case 4: w = rot32<SIGN, 4>(o[k]); break;
      case 5: w = rot32<SIGN, 5>(o[k]); break;
      case 6: w = rot32<SIGN, 6>(o[k]); break;
      case 7: w = rot32<SIGN, 7>(o[k]); break;
      case 8: w = rot32<SIGN, 8>(o[k]); break;
      case 9: w = rot32<SIGN, 9>(o[k]); break;
      case 10: w = rot32<SIGN, 10>(o[k]); break;
      case 11: w = rot32<SIGN, 11>(o[k]); break;
      case 12: w = rot32<SIGN, 12>(o[k]); break;
      case 13: w = rot32<SIGN, 13>(o[k]); break;
      case 14: w = rot32<SIGN, 14>(o[k]); break;
      default: w = rot32<SIGN, 15>(o[k]); break;
    }
    v[k] = cadd(e[k], w);
    v[k + 16] = csub(e[k], w);
  }
}

template <int R, int SIGN>
__device__ __forceinline__ void dft(float2* v) {
  static_assert(R == 2 || R == 4 || R == 8 || R == 16 || R == 32, "unsupported radix");
  if constexpr (R == 2) dft2<SIGN>(v);
  else if constexpr (R == 4) dft4<SIGN>(v);
  else if constexpr (R == 8) dft8<SIGN>(v);
  else if constexpr (R == 16) dft16<SIGN>(v);
  else dft32<SIGN>(v);
}

// --------------------------------------------------------------------------
// One line of length N = R1*R2 on R2 threads.  Shared memory per line and per
// exchange buffer: R1 rows of (R2 + 1) float2 (the +1 keeps the transposed
// reads bank-conflict free).  Two buffers alternate so one barrier per
// exchange suffices.
template <int R1_, int R2_>
struct FftLine {
  static constexpr int R1 = R1_;
  static constexpr int R2 = R2_;
  static constexpr int N = R1 * R2;
  static constexpr int J = R1 / R2;  // columns of the second pass per thread
  static constexpr int PITCH = R2 + 1;
  static constexpr int XBUF = R1 * PITCH;  // float2 per line per buffer
  static_assert(R1 % R2 == 0, "R2 must divide R1");

  // twf[k1*R2 + t] = W_N^(t*k1); twi[n*R1 + k1] = W_N^(-n*k1)   (shared memory)
  __device__ static void propagate(float2 (&v)[R1], int t, const float2* __restrict__ q,
                                   float2* xa, float2* xb, const float2* twf, const float2* twi) {
    // ---- forward pass 1: DFT over m of x[t + R2*m], twiddle, exchange
    dft<R1, -1>(v);
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) v[k1] = cmul(v[k1], twf[k1 * R2 + t]);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) xa[k1 * PITCH + t] = v[k1];
    __syncthreads();
    // ---- forward pass 2: thread t owns k1 = t + R2*j
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) v[j * R2 + n2] = xa[(t + R2 * j) * PITCH + n2];
#pragma unroll
    for (int j = 0; j < J; ++j) dft<R2, -1>(v + j * R2);
    // v[j*R2 + k2] = X[k1 + R1*k2];  filter in FFT order
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[j * R2 + k2] = cmul(v[j * R2 + k2], __ldg(q + t + R2 * j + R1 * k2));
    // ---- inverse pass 1: IDFT over k2 -> n_a, twiddle W_N^(-n_a*k1), exchange
#pragma unroll
    for (int j = 0; j < J; ++j) dft<R2, +1>(v + j * R2);
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
      for (int na = 0; na < R2; ++na) {
        const int k1 = t + R2 * j;
        float2 z = v[j * R2 + na];
        if (na) z = cmul(z, twi[na * R1 + k1]);
        xb[k1 * PITCH + na] = z;
      }
    __syncthreads();
    // ---- inverse pass 2: thread t = n_a gathers every k1
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) v[k1] = xb[k1 * PITCH + t];
    dft<R1, +1>(v);
  }
};

}  // namespace mm
