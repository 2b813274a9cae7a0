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

#include <type_traits>

#include "common.cuh"
#include "packed.cuh"

namespace mm {

// cos / sin of pi*k/16, k = 0..16 (exact values; rounded once to the
// register precision where used).
__device__ constexpr double kCos16[17] = {
    1.0, 0.98078528040323043058, 0.92387953251128673848, 0.83146961230254523567,
    0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173, 0.19509032201612826785,
    0.0, -0.19509032201612826785, -0.38268343236508977173, -0.55557023301960222474,
    -0.70710678118654752440, -0.83146961230254523567, -0.92387953251128673848, -0.98078528040323043058,
    -1.0};
__device__ constexpr double kSin16[17] = {
    0.0, 0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
    0.70710678118654752440, 0.83146961230254523567, 0.92387953251128673848, 0.98078528040323043058,
    1.0, 0.98078528040323043058, 0.92387953251128673848, 0.83146961230254523567,
    0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173, 0.19509032201612826785,
    0.0};

template <class C> struct Real;
template <> struct Real<float2> { using T = float; };
template <> struct Real<double2> { using T = double; };
template <bool TW> struct Real<cfx_t<TW>> { using T = float; };
template <> struct Real<cpk> { using T = float; };

__device__ __forceinline__ float2 cneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
template <bool TW>
__device__ __forceinline__ cfx_t<TW> cneg(cfx_t<TW> a) { return cfx_t<TW>{-a.x, -a.y}; }

// a * W_32^k with W = exp(SIGN * 2*pi*i/32), k = 0..15 (angle pi*k/16).
template <int SIGN, int K, class C>
__device__ __forceinline__ C rot32(C a) {
  using T = typename Real<C>::T;
  if constexpr (K == 0) {
    return a;
  } else if constexpr (K == 8) {
    return quarter<SIGN>(a);
  } else if constexpr (std::is_same_v<C, cpk>) {
    // packed (re, im), constants as hi + lo float pairs (see cmul_hl)
    constexpr double c = kCos16[K], s = SIGN * kSin16[K];
    constexpr float ch = float(c), sh = float(s);
    constexpr float cl = float(c - double(ch)), sl = float(s - double(sh));
    if constexpr (K == 4 || K == 12) {
      constexpr float g = c > 0 ? ch : -ch, gl = c > 0 ? cl : -cl;
      return cmul_diag(a, c > 0 ? 1.f : -1.f, s > 0 ? 1.f : -1.f, g, gl);
    } else {
      return cmul_hl(a, ch, sh, cl, sl);
    }
  } else if constexpr (IsCompensated<C>::value) {
    // constants as hi + lo float pairs (see cfx)
    constexpr double c = kCos16[K], s = SIGN * kSin16[K];
    constexpr float ch = float(c), sh = float(s);
    constexpr float cl = float(c - double(ch)), sl = float(s - double(sh));
    if constexpr (K == 4 || K == 12) {
      // |c| = |s| = sqrt(1/2): one rounded sum, then the scaled product
      constexpr float g = c > 0 ? ch : -ch, gl = c > 0 ? cl : -cl;  // +sqrt(1/2) as hi + lo
      constexpr float ex = c > 0 ? 1.f : -1.f, ey = s > 0 ? 1.f : -1.f;
      const float u = ex * a.x - ey * a.y, w = ey * a.x + ex * a.y;
      return C{fmaf(u, g, u * gl), fmaf(w, g, w * gl)};
    } else {
      const float rx = fmaf(a.x, cl, -a.y * sl), ry = fmaf(a.x, sl, a.y * cl);
      return C{fmaf(a.x, ch, fmaf(-a.y, sh, rx)), fmaf(a.x, sh, fmaf(a.y, ch, ry))};
    }
  } else {
    const T c = T(kCos16[K]), s = T(SIGN * kSin16[K]);
    C r;
    r.x = a.x * c - a.y * s;
    r.y = a.x * s + a.y * c;
    return r;
  }
}

template <int SIGN, class C>
__device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

// 4-point DFT on v[0], v[S], v[2S], v[3S] (natural order in and out).
template <int SIGN, int S = 1, class C>
__device__ __forceinline__ void dft4s(C* v) {
  C t0 = cadd(v[0], v[2 * S]);
  C t1 = csub(v[0], v[2 * S]);
  C t2 = cadd(v[S], v[3 * S]);
  C t3 = quarter<SIGN>(csub(v[S], v[3 * S]));
  v[0] = cadd(t0, t2);
  v[2 * S] = csub(t0, t2);
  v[S] = cadd(t1, t3);
  v[3 * S] = csub(t1, t3);
}

template <int SIGN, class C>
__device__ __forceinline__ void dft4(C* v) { dft4s<SIGN, 1>(v); }

// 8-point DFT: two interleaved 4-point DFTs and a radix-2 combine.
template <int SIGN, class C>
__device__ __forceinline__ void dft8(C* v) {
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
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
template <int SIGN, class C>
__device__ __forceinline__ void dft16(C* v) {
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
    v[3 + 4 * 3] = cneg(rot32<SIGN, 2>(v[3 + 4 * 3]));
  }
  // X[k1 + 4*k2] = DFT4 over r of the twiddled F_r[k1]: rows of 4.
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4s<SIGN, 1>(v + 4 * k1);
  // v[4*k1 + k2] holds X[k1 + 4*k2]: transpose the 4x4 index in registers.
  C t[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// 32-point DFT: radix-2 decimation in time over two 16-point DFTs.
template <int SIGN, class C>
__device__ __forceinline__ void dft32(C* v) {
  C e[16], o[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  dft16<SIGN>(e);
  dft16<SIGN>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    C w;
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

template <int R, int SIGN, class C>
__device__ __forceinline__ void dft(C* v) {
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
//
// CF / CI are the register arithmetic types of the forward and the inverse
// half: float2 (FP32), cpk (FP32 on the packed .f32x2 instructions, rotation
// constants as hi + lo pairs, FP32 twiddle tables), cfx (scalar FP32,
// rotations and twiddle tables as hi + lo pairs) or double2 (FP64
// butterflies, twiddles and filter).
// The line enters and leaves as complex64 and the exchanges are complex64.
// The inverse half carries most of the rounding that reaches the saved
// intensities, so <float2, double2> ("mixed") recovers most of the FP64
// accuracy for half of its cost.
template <int R1_, int R2_, class CF_ = float2, class CI_ = CF_>
struct FftLine {
  using CF = CF_;
  using CI = CI_;
  using TF = typename TwiddleOf<CF>::T;  // twiddle-table entries of each half
  using TI = typename TwiddleOf<CI>::T;
  static constexpr int R1 = R1_;
  static constexpr int R2 = R2_;
  static constexpr int N = R1 * R2;
  static constexpr int J = R1 / R2;  // columns of the second pass per thread
  static constexpr int PITCH = R2 + 1;
  // float2 per line per buffer.  In the column layout a warp holds 8-16
  // lines at the same in-line offset, in the row layout 2-4 lines at
  // consecutive offsets; the line stride (mod 16 eight-byte bank pairs) is
  // chosen so both layouts reach the fewest shared-memory wavefronts for the
  // CTA shapes of the propagation kernels (128 threads: 8 lines for R2 = 16,
  // 16 for R2 = 8, 32 for R2 = 4).
  static constexpr int kStrideResidue = R2 == 16 ? 2 : (R1 == 8 ? (R2 == 8 ? 10 : 9) : 3);
  static constexpr int XBUF = R1 * PITCH + ((kStrideResidue - (R1 * PITCH) % 16) + 16) % 16;
  static constexpr bool kFft = true;
  using XT = float2;
  // Packed halves (cpk) keep one twiddle table: the inverse twiddles are the
  // conjugates of the forward ones (the same rounded values); the shared
  // memory saved stays with L1.  For R1 == R2 the table W^(t*k) is
  // symmetric, so it is stored thread-major — row t holds every twiddle
  // thread t applies in either direction — and read 16 bytes at a time
  // (rows of R2 + 2 entries: 16-byte aligned, conflict-free).
  static constexpr bool kConjTw = std::is_same_v<CF, cpk> && std::is_same_v<CI, cpk>;
  static constexpr bool kRowTw = kConjTw && R1 == R2;
  static constexpr int TWP = kRowTw ? R2 + 2 : (kConjTw ? R2 + 1 : R2);  // pitch of the forward table's rows
  static constexpr size_t kTwiddleBytes =
      kConjTw ? (size_t)R1 * TWP * sizeof(TF) : (size_t)N * (sizeof(TF) + sizeof(TI));
  // CTAs of 128 threads resident per SM the kernels are compiled for: the
  // FP32 forms fit in 80 registers (6 CTAs); FP64 halves need the 4-CTA budget.
  static constexpr int kMinBlocks =
      R1 > 16 ? 2 : ((std::is_same_v<CF, double2> || std::is_same_v<CI, double2>) ? 4 : 6);
  static_assert(R1 % R2 == 0, "R2 must divide R1");

  // twf[k1*TWP + t] = W_N^(t*k1) (CF);  twi[n*R1 + k1] = W_N^(-n*k1) (CI),
  // each formed in FP64 and rounded once.
  __device__ static void fill_twiddles(TF* twf, TI* twi) {
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      double s, c;
      const int k1 = i / R2, t = i % R2;
      sincospi(-2.0 * double((t * k1) % N) / N, &s, &c);
      twf[k1 * TWP + t] = make_tw<TF>(c, s);  // row k1 = thread-major row t (symmetric) when kRowTw
      if constexpr (!kConjTw) {
        const int nn = i / R1, kk = i % R1;
        sincospi(2.0 * double((nn * kk) % N) / N, &s, &c);
        twi[i] = make_tw<TI>(c, s);
      }
    }
  }

  // SINGLE: xa and xb are the same buffer; two more barriers keep the
  // exchanges apart (and the next call's first exchange after this one's last).
  // With R1 == R2 they are not needed: thread t reads back exactly the row it
  // writes next (row t: forward pass 2, then inverse pass 1) and the column
  // it writes next (column t: inverse pass 2, then the next forward pass 1),
  // so no thread overwrites a word another thread has still to read.
  // warp_local: the line's R2 threads share one warp (row layout), so a warp
  // barrier orders the exchanges; otherwise the whole CTA synchronises.
  template <bool SINGLE = false>
  __device__ static void propagate(float2 (&x)[R1], int t, const float2* __restrict__ q, int /*n*/,
                                   float2* xa, float2* xb, const TF* twf, const TI* twi, bool warp_local = false) {
    auto sync = [warp_local]() {
      if (warp_local) __syncwarp();
      else __syncthreads();
    };
    CF v[R1];
#pragma unroll
    for (int m = 0; m < R1; ++m) v[m] = from_f2<CF>(x[m]);
    // ---- forward pass 1: DFT over m of x[t + R2*m], twiddle, exchange
    dft<R1, -1>(v);
    if constexpr (kRowTw) {
      const float4* row = reinterpret_cast<const float4*>(twf + t * TWP);
#pragma unroll
      for (int k = 0; k < R1; k += 2) {
        const float4 w2 = row[k / 2];
        if (k) v[k] = cmul(v[k], make_float2(w2.x, w2.y));
        v[k + 1] = cmul(v[k + 1], make_float2(w2.z, w2.w));
      }
    } else {
#pragma unroll
      for (int k1 = 1; k1 < R1; ++k1) v[k1] = cmul(v[k1], twf[k1 * TWP + t]);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) xa[k1 * PITCH + t] = to_f2(v[k1]);
    sync();
    // ---- forward pass 2: thread t owns k1 = t + R2*j
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) v[j * R2 + n2] = from_f2<CF>(xa[(t + R2 * j) * PITCH + n2]);
#pragma unroll
    for (int j = 0; j < J; ++j) dft<R2, -1>(v + j * R2);
    // v[j*R2 + k2] = X[k1 + R1*k2];  filter in FFT order (inverse precision)
    CI w[R1];
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2)
        w[j * R2 + k2] = cmul(promote<CI>(v[j * R2 + k2]), __ldg(q + t + R2 * j + R1 * k2));
    // ---- inverse pass 1: IDFT over k2 -> n_a, twiddle W_N^(-n_a*k1), exchange
#pragma unroll
    for (int j = 0; j < J; ++j) dft<R2, +1>(w + j * R2);
    if constexpr (SINGLE && J > 1) sync();  // forward reads of the shared buffer done
    if constexpr (kRowTw) {  // J == 1, k1 = t: row t, conjugated
      const float4* row = reinterpret_cast<const float4*>(twf + t * TWP);
#pragma unroll
      for (int na = 0; na < R2; na += 2) {
        const float4 w2 = row[na / 2];
        CI z0 = w[na], z1 = w[na + 1];
        if (na) z0 = cmul_conj(z0, make_float2(w2.x, w2.y));
        z1 = cmul_conj(z1, make_float2(w2.z, w2.w));
        xb[t * PITCH + na] = to_f2(z0);
        xb[t * PITCH + na + 1] = to_f2(z1);
      }
    } else {
#pragma unroll
      for (int j = 0; j < J; ++j)
#pragma unroll
        for (int na = 0; na < R2; ++na) {
          const int k1 = t + R2 * j;
          CI z = w[j * R2 + na];
          if constexpr (kConjTw) {
            if (na) z = cmul_conj(z, twf[k1 * TWP + na]);
          } else {
            if (na) z = cmul(z, twi[na * R1 + k1]);
          }
          xb[k1 * PITCH + na] = to_f2(z);
        }
    }
    sync();
    // ---- inverse pass 2: thread t = n_a gathers every k1
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) w[k1] = from_f2<CI>(xb[k1 * PITCH + t]);
    dft<R1, +1>(w);
#pragma unroll
    for (int m = 0; m < R1; ++m) x[m] = to_f2(w[m]);
    if constexpr (SINGLE && J > 1) sync();  // inverse reads done before the buffer is reused
  }
};

// --------------------------------------------------------------------------
// Any line length n <= 16*RMAX: the step along the line is the circular
// convolution with p = IDFT(Q) (one n-tap complex kernel per step, formed in
// FP64 on the host), accumulated in FP64.  Used for window sizes without a
// radix-2 factorisation (e.g. the 112 / 72 windows of supersampled configs).
template <int RMAX>
struct DenseLine {
  using CF = float2;
  using CI = float2;
  using TF = float2;
  using TI = float2;
  static constexpr size_t kTwiddleBytes = 0;
  static constexpr int R1 = RMAX;
  static constexpr int R2 = 16;
  static constexpr int N = RMAX * 16;  // capacity
  static constexpr int XBUF = N + 1;  // odd stride: lines start on different banks
  static constexpr bool kFft = false;
  static constexpr bool kConjTw = false;
  using XT = float2;
  static constexpr int kMinBlocks = RMAX > 16 ? 2 : 4;
  __device__ static void fill_twiddles(TF*, TI*) {}

  template <bool SINGLE = false>
  __device__ static void propagate(float2 (&v)[R1], int t, const float2* __restrict__ ker, int n, float2* xa,
                                   float2* /*xb*/, const TF* /*twf*/, const TI* /*twi*/, bool /*warp_local*/ = false) {
#pragma unroll
    for (int j = 0; j < R1; ++j) {
      const int e = t + R2 * j;
      if (e < n) xa[e] = v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < R1; ++j) {
      const int e = t + R2 * j;
      if (e < n) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k < n; ++k) {
          int m = e - k;
          m += m < 0 ? n : 0;
          const float2 a = __ldg(ker + m), b = xa[k];
          re += double(a.x) * b.x - double(a.y) * b.y;
          im += double(a.x) * b.y + double(a.y) * b.x;
        }
        v[j] = make_float2(float(re), float(im));
      }
    }
    __syncthreads();
  }
};

}  // namespace mm
