// Static and per-frame scan operators (maomi/scanning.py:8-53 zstack;
// maomi/movie.py:14-102 conv2_same, psf_fft, single_scan, blurred_background):
// 2-D linear convolutions of real planes with real kernel planes, coupled
// along Z by a per-bin rule.
//
// Design.  Every operator is  out[x, y, o] = sum_(z,l in rule(o)) (src_z * k_l)(x + cx, y + cy)
// with * the 2-D linear convolution.  Planes are zero padded to fx x fy
// (powers of two, >= the extent that keeps the kept window alias free) and
// transformed in pairs: two real planes a, b as one complex plane a + i b.
//
//   rows_fwd   one CTA per (input row, 2*LPC planes): the row tile of every
//              plane is read once (coalesced along whichever of y / z is
//              contiguous; grouping, masks and periodic wrap applied in the
//              read), packed into pairs and DFT'd along y in registers;
//   cols       one CTA per (column block, pair): DFT along x of the nonzero
//              rows (forward), or inverse DFT keeping only the crop rows;
//   combine    one thread per conjugate bin pair (k, -k): unpack the source
//              spectra of every plane (Hermitian split), apply the Z rule
//              against the kernel half spectra, repack the output pairs;
//   rows_inv   one CTA per kept output row: inverse DFT along y, unpack the
//              pair into two planes, crop, scale, store or accumulate.
//
// The line DFT of N = R1 * R2 samples runs on R2 threads (thread t holds
// samples t + R2*m): a radix-R1 DFT in registers, twiddles W_N^(t*k1), one
// shared-memory exchange, radix-R2 DFTs; the result is in natural order in
// the same thread layout.  The 1/(fx*fy) of the inverse is folded into the
// combine.  HBM-bound: each transform pass reads and writes every plane once.
#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "dft.cuh"

namespace mm {
namespace scan {

template <class T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

template <int N> struct Split;
template <> struct Split<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Split<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct Split<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Split<512> { static constexpr int R1 = 32, R2 = 16; };
template <> struct Split<384> { static constexpr int R1 = 48, R2 = 8; };   // FP32 planes only
template <> struct Split<768> { static constexpr int R1 = 48, R2 = 16; };  // FP32 planes only
template <> struct Split<1024> { static constexpr int R1 = 32, R2 = 32; };

constexpr int kThreads = 256;
constexpr int kCombineThreads = 128;

// W_N^-n (forward direction) for n < N, formed in FP64 and rounded once.
template <class C>
__device__ void fill_twiddles(C* tw, int N) {
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    double s, c;
    sincospi(-2.0 * double(n) / double(N), &s, &c);
    tw[n] = make_c<C>(c, s);
  }
}

// After line_dft, X[t + R2*m] sits in v[slot(m)].
template <int R1, int R2>
__host__ __device__ constexpr int slot(int m) {
  return (m % (R1 / R2)) * R2 + m / (R1 / R2);
}

// 48-point DFT in registers, natural order in and out: n = 3 m + r, k = k1 +
// 16 k2; three 16-point DFTs over m, twiddles W_48^(r k1) (entry stride * r *
// k1 of the line's table of W_N^n, conjugated for SIGN > 0), then radix-3
// butterflies over r: X[k1 + 16 k2] = sum_r W_3^(r k2) W_48^(r k1) F_r[k1].
template <int SIGN, class C>
__device__ __forceinline__ void dft48(C (&v)[48], const C* tw, int stride) {
  using R = decltype(v[0].x);
  C f[3][16];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int m = 0; m < 16; ++m) f[r][m] = v[3 * m + r];
    dft<16, SIGN>(f[r]);
  }
#pragma unroll
  for (int r = 1; r < 3; ++r)
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) {
      C w = tw[stride * r * k1];
      if constexpr (SIGN > 0) w.y = -w.y;
      f[r][k1] = cmul(f[r][k1], w);
    }
  const R h = R(0.5), q = R(SIGN) * R(0.86602540378443864676);  // SIGN * sqrt(3) / 2
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) {
    const C a = f[0][k1], t1 = cadd(f[1][k1], f[2][k1]), t2 = csub(f[1][k1], f[2][k1]);
    C m1 = a, m2 = t2;
    m1.x = a.x - h * t1.x;
    m1.y = a.y - h * t1.y;
    m2.x = -q * t2.y;  // i * SIGN * sqrt(3)/2 * (b - c)
    m2.y = q * t2.x;
    v[k1] = cadd(a, t1);
    v[k1 + 16] = cadd(m1, m2);
    v[k1 + 32] = csub(m1, m2);
  }
}

// In-place DFT of one line (SIGN -1 forward, +1 inverse, unnormalised).
// Thread t holds x[t + R2*m] in v[m]; on return it holds X[t + R2*m] in
// v[slot(m)].  xb: R1 * (R2 + 1) complex of this line.  Every thread of the
// CTA calls it (two CTA barriers).
template <int R1, int R2, int SIGN, class C>
__device__ __forceinline__ void line_dft(C (&v)[R1], int t, C* xb, const C* tw) {
  constexpr int J = R1 / R2, P = R2 + 1;
  if constexpr (R1 == 48)
    dft48<SIGN>(v, tw, R2);  // W_48^j = W_N^(j * N / 48), N / 48 = R2
  else
    dft<R1, SIGN>(v);
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) {
    C w = tw[t * k1];
    if constexpr (SIGN > 0) w.y = -w.y;
    v[k1] = cmul(v[k1], w);
  }
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) xb[k1 * P + t] = v[k1];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < J; ++j)
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) v[j * R2 + n2] = xb[(t + R2 * j) * P + n2];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < J; ++j) dft<R2, SIGN>(v + j * R2);
}

// ------------------------------------------------------------------ params
struct Planes {
  const void* data;
  long long s0, s1, s2;
  int nx, ny, nz, group, planes;  // planes = ceil(nz / group)
  const void* m0;
  const void* m1;
  const void* data2;  // optional second volume (same strides), added element-wise
  int wrap, wx0, wy0, ext_x, ext_y;
};

// Transform-input value at row i, column j of transform plane p (grouped,
// masked, wrapped).  i < ext_x, j < ext_y, p < planes.
template <class T>
__device__ __forceinline__ T plane_value(const Planes& P, int i, int j, int p) {
  int x = i, y = j;
  if (P.wrap) {
    x = (i + P.wx0) % P.nx;
    y = (j + P.wy0) % P.ny;
  }
  const T* d = static_cast<const T*>(P.data);
  const long long base = (long long)x * P.s0 + (long long)y * P.s1;
  const int z0 = p * P.group;
  const int z1 = min(z0 + P.group, P.nz);
  T s = T(0);
  if (P.data2) {
    const T* d2 = static_cast<const T*>(P.data2);
    for (int z = z0; z < z1; ++z) s += d[base + (long long)z * P.s2] + d2[base + (long long)z * P.s2];
  } else {
    for (int z = z0; z < z1; ++z) s += d[base + (long long)z * P.s2];
  }
  if (P.m0) s *= static_cast<const T*>(P.m0)[(long long)x * P.ny + y];
  if (P.m1) s *= static_cast<const T*>(P.m1)[(long long)x * P.ny + y];
  return s;
}

template <class T, int N>
struct RowShape {
  using C = typename Cplx<T>::type;
  static constexpr int R1 = Split<N>::R1, R2 = Split<N>::R2, LPC = kThreads / R2, TP = 2 * LPC + 1;
  static constexpr size_t kTile = (size_t)N * TP * sizeof(T);
  static constexpr size_t kXb = (size_t)LPC * R1 * (R2 + 1) * sizeof(C);
  static constexpr size_t kSmem = N * sizeof(C) + (kTile > kXb ? kTile : kXb);
};

// Forward row pass.  grid (ext_x, ceil(pairs / LPC)); S: (pairs, fx, N).
template <class T, int N>
__global__ void __launch_bounds__(kThreads, Split<N>::R1 == 48 ? 2 : 1) rows_fwd_kernel(Planes P, int fx, typename Cplx<T>::type* __restrict__ S,
                                                            int pairs) {
  using Sh = RowShape<T, N>;
  using C = typename Sh::C;
  constexpr int R1 = Sh::R1, R2 = Sh::R2, LPC = Sh::LPC, TP = Sh::TP;
  extern __shared__ __align__(16) unsigned char smem[];
  C* tw = reinterpret_cast<C*>(smem);
  unsigned char* body = smem + N * sizeof(C);
  T* tile = reinterpret_cast<T*>(body);  // (N, TP): the row of every plane of this CTA
  C* xb = reinterpret_cast<C*>(body);    // exchange buffers, after the tile is consumed
  fill_twiddles(tw, N);
  const int i = blockIdx.x;
  const int p0 = blockIdx.y * 2 * LPC;
  const int np = min(2 * LPC, P.planes - p0);
  const int ey = P.ext_y;
  const bool pfast = P.s2 < P.s1 && !P.wrap;  // planes contiguous: read planes fastest
  const int total = ey * np;
  for (int e = threadIdx.x; e < total; e += kThreads) {
    int j, q;
    if (pfast) { j = e / np; q = e - j * np; }
    else { q = e / ey; j = e - q * ey; }
    tile[j * TP + q] = plane_value<T>(P, i, j, p0 + q);
  }
  __syncthreads();
  const int line = threadIdx.x / R2, t = threadIdx.x % R2;
  C v[R1];
#pragma unroll
  for (int m = 0; m < R1; ++m) {
    const int j = t + R2 * m;
    T a = T(0), b = T(0);
    if (j < ey) {
      if (2 * line < np) a = tile[j * TP + 2 * line];
      if (2 * line + 1 < np) b = tile[j * TP + 2 * line + 1];
    }
    v[m].x = a;
    v[m].y = b;
  }
  __syncthreads();  // the tile is consumed; xb overwrites it
  line_dft<R1, R2, -1>(v, t, xb + line * R1 * (R2 + 1), tw);
  const int pair = blockIdx.y * LPC + line;
  if (pair < pairs) {
    C* dst = S + ((long long)pair * fx + i) * N;
#pragma unroll
    for (int m = 0; m < R1; ++m) dst[t + R2 * m] = v[slot<R1, R2>(m)];
  }
}

// Column pass along x.  grid (fy / CB, pairs).  Forward (SIGN -1): rows
// [0, rows_in) are read (the others are zero), every row written.  Inverse
// (SIGN +1): every row read, rows [row0, row0 + rows_out) written to rows
// [0, rows_out) of the same plane (in place: a CTA owns its columns).
template <class T, int N>
struct ColShape {
  using C = typename Cplx<T>::type;
  static constexpr int R1 = Split<N>::R1, R2 = Split<N>::R2, CB = kThreads / R2;
  static constexpr size_t kSmem = N * sizeof(C) + (size_t)CB * R1 * (R2 + 1) * sizeof(C);
};

template <class T, int N, int SIGN>
__global__ void __launch_bounds__(kThreads, Split<N>::R1 == 48 ? 2 : 1) cols_kernel(typename Cplx<T>::type* __restrict__ S, int fy, int rows_in,
                                                        int row0, int rows_out) {
  using Sh = ColShape<T, N>;
  using C = typename Sh::C;
  constexpr int R1 = Sh::R1, R2 = Sh::R2, CB = Sh::CB;
  extern __shared__ __align__(16) unsigned char smem[];
  C* tw = reinterpret_cast<C*>(smem);
  C* xb = tw + N;
  fill_twiddles(tw, N);
  __syncthreads();
  const int c = threadIdx.x % CB, t = threadIdx.x / CB;
  const int col = blockIdx.x * CB + c;
  C* plane = S + (long long)blockIdx.y * N * fy;
  C v[R1];
#pragma unroll
  for (int m = 0; m < R1; ++m) {
    const int r = t + R2 * m;
    v[m] = (r < rows_in) ? plane[(long long)r * fy + col] : make_c<C>(0.0, 0.0);
  }
  line_dft<R1, R2, SIGN>(v, t, xb + c * R1 * (R2 + 1), tw);
#pragma unroll
  for (int m = 0; m < R1; ++m) {
    const int r = t + R2 * m - row0;
    if (r >= 0 && r < rows_out) plane[(long long)r * fy + col] = v[slot<R1, R2>(m)];
  }
}

// ----------------------------------------------------------------- combine
struct Rule {
  int zrule, zoff;
  int nin;    // source transform planes
  int nk;     // kernel planes
  int nout;   // output planes
};

template <class C>
__device__ __forceinline__ void hsplit(C w, C wm, C& a, C& b) {
  // w = A(k) + i B(k), wm = A(-k) + i B(-k) for real planes A, B
  a.x = (w.x + wm.x) * 0.5f;
  a.y = (w.y - wm.y) * 0.5f;
  b.x = (w.y + wm.y) * 0.5f;
  b.y = (wm.x - w.x) * 0.5f;
}

// CONV / CORR rule for one chunk of kOutChunk outputs with register windows
// (FP32): 16 taps at a time, the 31 source bins they reach read once from
// shared memory and the 16 kernel bins once from global memory; terms outside
// the source or kernel range are exact zeros, so every output sums its taps
// in increasing l exactly as the one-tap loop does.
constexpr int kOutChunk = 16;

template <bool CONV, class C>
__device__ __forceinline__ void zrule_window(C (&y)[kOutChunk], const C* sv, int nt, int tid, const C* kk,
                                             long long kplane, int o0, int zoff, int lo, int hi, int nin) {
  constexpr int TB = 16;
  const C zero = make_c<C>(0.0, 0.0);
  for (int l0 = lo; l0 <= hi; l0 += TB) {
    C kb[TB];
#pragma unroll
    for (int ll = 0; ll < TB; ++ll) kb[ll] = (l0 + ll <= hi) ? kk[(long long)(l0 + ll) * kplane] : zero;
    // CONV: z = o0 + j + zoff - l0 - ll = zb + (TB - 1) + j - ll;  CORR: z = zb + j + ll
    const int zb = CONV ? o0 + zoff - l0 - (TB - 1) : o0 - zoff + l0;
    C w[2 * TB - 1];
#pragma unroll
    for (int i = 0; i < 2 * TB - 1; ++i) {
      const int z = zb + i;
      w[i] = (z >= 0 && z < nin) ? sv[z * nt + tid] : zero;
    }
#pragma unroll
    for (int ll = 0; ll < TB; ++ll)
#pragma unroll
      for (int j = 0; j < kOutChunk; ++j) y[j] = cadd(y[j], cmul(w[CONV ? j - ll + TB - 1 : j + ll], kb[ll]));
  }
}

// Bin pair representative: ky in [0, fy/2]; on the self-paired columns
// (ky = 0, fy/2) only kx in [0, fx/2].  One thread per representative.
// Source spectra Sin (pairs_in, fx, fy) -> output spectra S (pairs_out, fx,
// fy), stored or (accumulate) added.  S may be Sin: a thread reads its two
// bins of every source plane before it writes any output bin.  Kernel half
// spectra K (nk, fx, fy/2 + 1).
template <class T>
__global__ void __launch_bounds__(kCombineThreads) combine_kernel(const typename Cplx<T>::type* Sin,
                                                                  typename Cplx<T>::type* S,
                                                                  const typename Cplx<T>::type* __restrict__ K,
                                                                  int fx, int fy, Rule R, T scale, int accumulate) {
  using C = typename Cplx<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  C* sv = reinterpret_cast<C*>(smem);  // (nin, blockDim) source bins of this thread
  const int hy = fy / 2 + 1;
  const long long nb = (long long)fx * hy;
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;  // no barriers below
  const int kx = int(b / hy), ky = int(b - (long long)kx * hy);
  if ((ky == 0 || ky == fy / 2) && kx > fx / 2) return;  // its partner handles the pair
  const int mx = kx == 0 ? 0 : fx - kx, my = ky == 0 ? 0 : fy - ky;  // conjugate bin
  const bool self = (mx == kx) && (my == ky);
  const long long plane = (long long)fx * fy;
  const long long ik = (long long)kx * fy + ky, im = (long long)mx * fy + my;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int pin = (R.nin + 1) / 2;
  for (int p = 0; p < pin; ++p) {
    C a, bb;
    hsplit(Sin[p * plane + ik], Sin[p * plane + im], a, bb);
    sv[(2 * p) * nt + tid] = a;
    if (2 * p + 1 < R.nin) sv[(2 * p + 1) * nt + tid] = bb;
  }
  const C* kk = K + (long long)kx * hy + ky;
  const long long kplane = (long long)fx * hy;
  const int pout = (R.nout + 1) / 2;
  const C zero = make_c<C>(0.0, 0.0);
  // packed output: W(k) = Y0(k) + i Y1(k);  W(-k) = conj(Y0(k)) + i conj(Y1(k))
  auto store = [&](int q, C y0, C y1) {
    C wk, wm;
    wk.x = y0.x - y1.y;
    wk.y = y0.y + y1.x;
    wm.x = y0.x + y1.y;
    wm.y = y1.x - y0.y;
    if (accumulate) {
      wk = cadd(S[q * plane + ik], wk);
      if (!self) wm = cadd(S[q * plane + im], wm);
    }
    S[q * plane + ik] = wk;
    if (!self) S[q * plane + im] = wm;
  };
  auto scaled = [&](C a) { return make_c<C>(a.x * scale, a.y * scale); };
  if (R.zrule == MM_SCAN_SUM_Z || R.zrule == MM_SCAN_EACH_Z) {
    for (int q = 0; q < pout; ++q) {
      C y[2] = {zero, zero};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int o = 2 * q + h;
        if (o >= R.nout) break;
        C acc = zero;
        if (R.zrule == MM_SCAN_SUM_Z) {
          for (int z = 0; z < R.nin; ++z) acc = cadd(acc, cmul(sv[z * nt + tid], kk[z * kplane]));
        } else {
          acc = cmul(sv[o * nt + tid], kk[o * kplane]);
        }
        y[h] = scaled(acc);
      }
      store(q, y[0], y[1]);
    }
    return;
  }
  // CONV: z = o + zoff - l;  CORR: z = o - zoff + l.  Outputs in register
  // chunks of kOutChunk: each kernel bin is read once per chunk, every
  // output still sums its taps in increasing l.
  const bool conv = R.zrule == MM_SCAN_CONV_Z;
  for (int o0 = 0; o0 < R.nout; o0 += kOutChunk) {
    C y[kOutChunk];
#pragma unroll
    for (int j = 0; j < kOutChunk; ++j) y[j] = zero;
    const int oe = min(o0 + kOutChunk, R.nout) - 1;
    const int lo = conv ? max(0, o0 + R.zoff - (R.nin - 1)) : max(0, R.zoff - oe);
    const int hi = conv ? min(R.nk - 1, oe + R.zoff) : min(R.nk - 1, R.nin - 1 - o0 + R.zoff);
    if constexpr (std::is_same_v<T, float>) {
      if (conv) zrule_window<true>(y, sv, nt, tid, kk, kplane, o0, R.zoff, lo, hi, R.nin);
      else zrule_window<false>(y, sv, nt, tid, kk, kplane, o0, R.zoff, lo, hi, R.nin);
    } else {
    for (int l = lo; l <= hi; ++l) {
      const C kl = kk[l * kplane];
      const int z0 = conv ? o0 + R.zoff - l : o0 - R.zoff + l;  // source plane of output o0
      if (z0 >= 0 && z0 + kOutChunk <= R.nin && o0 + kOutChunk - 1 <= oe) {
        // interior: every output of the chunk reads a source plane
        const C* vp = sv + (long long)z0 * nt + tid;
#pragma unroll
        for (int j = 0; j < kOutChunk; ++j) y[j] = cadd(y[j], cmul(vp[j * nt], kl));
      } else {
#pragma unroll
        for (int j = 0; j < kOutChunk; ++j) {
          const int z = z0 + j;
          if (o0 + j <= oe && z >= 0 && z < R.nin) y[j] = cadd(y[j], cmul(sv[z * nt + tid], kl));
        }
      }
    }
    }
#pragma unroll
    for (int j = 0; j < kOutChunk; j += 2) {
      if (o0 + j > oe) break;
      store((o0 + j) / 2, scaled(y[j]), o0 + j + 1 <= oe ? scaled(y[j + 1]) : zero);
    }
  }
}

// Kernel half spectra from the packed kernel spectra: K_(2p)(k), K_(2p+1)(k)
// for ky in [0, fy/2].
template <class T>
__global__ void unpack_kernel(const typename Cplx<T>::type* __restrict__ S, typename Cplx<T>::type* __restrict__ K,
                              int fx, int fy, int nk) {
  using C = typename Cplx<T>::type;
  const int hy = fy / 2 + 1;
  const long long nb = (long long)fx * hy;
  const long long plane = (long long)fx * fy;
  const int pairs = (nk + 1) / 2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nb * pairs;
       e += (long long)gridDim.x * blockDim.x) {
    const int p = int(e / nb);
    const long long b = e - (long long)p * nb;
    const int kx = int(b / hy), ky = int(b - (long long)kx * hy);
    const int mx = kx == 0 ? 0 : fx - kx, my = ky == 0 ? 0 : fy - ky;  // conjugate bin
    C a, bb;
    hsplit(S[p * plane + (long long)kx * fy + ky], S[p * plane + (long long)mx * fy + my], a, bb);
    K[(2 * p) * nb + b] = a;
    if (2 * p + 1 < nk) K[(2 * p + 1) * nb + b] = bb;
  }
}

// Inverse row pass.  grid (out_x, ceil(pairs_out / LPC)): kept row r (spectra
// row r after the column pass), inverse DFT along y, columns
// [crop_y, crop_y + out_y) of both planes of each pair, times alpha, into out.
struct Out {
  void* data;
  long long o0, o1, o2;
  int out_x, out_y, planes, crop_y, accumulate;
  double alpha;
  const void* weight;  // (out_x, out_y) row-major weights of the kept window, or NULL
};

template <class T, int N>
__global__ void __launch_bounds__(kThreads, Split<N>::R1 == 48 ? 2 : 1) rows_inv_kernel(const typename Cplx<T>::type* __restrict__ S, int fx,
                                                            Out O) {
  using Sh = RowShape<T, N>;
  using C = typename Sh::C;
  constexpr int R1 = Sh::R1, R2 = Sh::R2, LPC = Sh::LPC, TP = Sh::TP;
  extern __shared__ __align__(16) unsigned char smem[];
  C* tw = reinterpret_cast<C*>(smem);
  unsigned char* body = smem + N * sizeof(C);
  T* tile = reinterpret_cast<T*>(body);
  C* xb = reinterpret_cast<C*>(body);
  fill_twiddles(tw, N);
  __syncthreads();
  const int r = blockIdx.x;
  const int line = threadIdx.x / R2, t = threadIdx.x % R2;
  const int pairs = (O.planes + 1) / 2;
  const int pair = blockIdx.y * LPC + line;
  C v[R1];
  const C* src = S + ((long long)min(pair, pairs - 1) * fx + r) * N;
#pragma unroll
  for (int m = 0; m < R1; ++m) v[m] = src[t + R2 * m];
  line_dft<R1, R2, +1>(v, t, xb + line * R1 * (R2 + 1), tw);
  // xb is free again (line_dft ends with a barrier): stage the kept columns
#pragma unroll
  for (int m = 0; m < R1; ++m) {
    const int j = t + R2 * m - O.crop_y;
    if (j >= 0 && j < O.out_y) {
      const C w = v[slot<R1, R2>(m)];
      tile[j * TP + 2 * line] = w.x;
      tile[j * TP + 2 * line + 1] = w.y;
    }
  }
  __syncthreads();
  const int p0 = blockIdx.y * 2 * LPC;
  const int np = min(2 * LPC, O.planes - p0);
  const bool pfast = O.o2 < O.o1;
  T* out = static_cast<T*>(O.data);
  const T alpha = T(O.alpha);
  const T* wrow = O.weight ? static_cast<const T*>(O.weight) + (long long)r * O.out_y : nullptr;
  const int total = O.out_y * np;
  for (int e = threadIdx.x; e < total; e += kThreads) {
    int j, q;
    if (pfast) { j = e / np; q = e - j * np; }
    else { q = e / O.out_y; j = e - q * O.out_y; }
    const long long a = (long long)r * O.o0 + (long long)j * O.o1 + (long long)(p0 + q) * O.o2;
    T val = alpha * tile[j * TP + q];
    if (wrow) val *= wrow[j];
    out[a] = O.accumulate ? out[a] + val : val;
  }
}

// Background source plane (movie.py:86-95).
template <class T>
struct BgVols {
  const T* v[4];
};

template <class T>
__global__ void background_kernel(BgVols<T> V, int nvol, long long s0, long long s1, long long s2, int nx, int ny,
                                  int nz, const int32_t* __restrict__ idx, const double* __restrict__ scale, int n,
                                  double power, const T* __restrict__ mask, T* __restrict__ out) {
  const long long np = (long long)nx * ny;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < np; e += (long long)gridDim.x * blockDim.x) {
    const int x = int(e / ny), y = int(e - (long long)x * ny);
    const long long base = (long long)x * s0 + (long long)y * s1;
    double acc = 0.0;
    for (int v = 0; v < nvol; ++v) {
      double s = 0.0;
      for (int i = 0; i < n; ++i) {
        const int z = idx[i];
        if (z >= 0 && z < nz) s += double(V.v[v][base + (long long)z * s2]) * scale[i];  // host-checked; never read out of range
      }
      acc += s / n;
    }
    acc *= power;
    if (mask) acc *= double(mask[e]);
    out[e] = T(acc);
  }
}

// ------------------------------------------------------------------- host
// Transform sizes of one axis: powers of two 64..1024, and 384 = 48 x 8 and
// 768 = 48 x 16 for FP32 planes.
bool supported_size(int n, int fp64) {
  return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024 || ((n == 384 || n == 768) && !fp64);
}

template <class T>
int set_smem(const void* fn, size_t bytes, const char* what) {
  MM_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), what);
  return MM_OK;
}

template <class T, int N>
int rows_fwd(const Planes& P, int fx, void* S, int pairs, cudaStream_t st) {
  using Sh = RowShape<T, N>;
  auto fn = rows_fwd_kernel<T, N>;
  int rc = set_smem<T>((const void*)fn, Sh::kSmem, "cudaFuncSetAttribute(scan rows)");
  if (rc) return rc;
  dim3 grid(P.ext_x, (pairs + Sh::LPC - 1) / Sh::LPC);
  fn<<<grid, kThreads, Sh::kSmem, st>>>(P, fx, static_cast<typename Cplx<T>::type*>(S), pairs);
  MM_CHECK_LAUNCH("scan rows (forward)");
  return MM_OK;
}

template <class T, int N, int SIGN>
int cols(void* S, int fy, int pairs, int rows_in, int row0, int rows_out, cudaStream_t st) {
  using Sh = ColShape<T, N>;
  auto fn = cols_kernel<T, N, SIGN>;
  int rc = set_smem<T>((const void*)fn, Sh::kSmem, "cudaFuncSetAttribute(scan columns)");
  if (rc) return rc;
  dim3 grid(fy / Sh::CB, pairs);
  fn<<<grid, kThreads, Sh::kSmem, st>>>(static_cast<typename Cplx<T>::type*>(S), fy, rows_in, row0, rows_out);
  MM_CHECK_LAUNCH("scan columns");
  return MM_OK;
}

template <class T, int N>
int rows_inv(const void* S, int fx, const Out& O, cudaStream_t st) {
  using Sh = RowShape<T, N>;
  auto fn = rows_inv_kernel<T, N>;
  int rc = set_smem<T>((const void*)fn, Sh::kSmem, "cudaFuncSetAttribute(scan rows inverse)");
  if (rc) return rc;
  const int pairs = (O.planes + 1) / 2;
  dim3 grid(O.out_x, (pairs + Sh::LPC - 1) / Sh::LPC);
  fn<<<grid, kThreads, Sh::kSmem, st>>>(static_cast<const typename Cplx<T>::type*>(S), fx, O);
  MM_CHECK_LAUNCH("scan rows (inverse)");
  return MM_OK;
}

// Dispatch on the transform size of one axis.
template <class T, class F>
int by_size(int n, F&& f) {
  switch (n) {
    case 64: return f(std::integral_constant<int, 64>{});
    case 128: return f(std::integral_constant<int, 128>{});
    case 256: return f(std::integral_constant<int, 256>{});
    case 384:
      if constexpr (std::is_same_v<T, float>) return f(std::integral_constant<int, 384>{});
      set_error("scan transform size 384 is for FP32 planes only");
      return MM_ERR_UNSUPPORTED;
    case 512: return f(std::integral_constant<int, 512>{});
    case 768:
      if constexpr (std::is_same_v<T, float>) return f(std::integral_constant<int, 768>{});
      set_error("scan transform size 768 is for FP32 planes only");
      return MM_ERR_UNSUPPORTED;
    case 1024: return f(std::integral_constant<int, 1024>{});
    default:
      set_error("scan transform size %d is not one of 64, 128, 256, 384 (FP32), 512, 768 (FP32), 1024", n);
      return MM_ERR_UNSUPPORTED;
  }
}

int check_desc(const mm_scan_desc* d) {
  MM_CHECK_ARG(d != nullptr, "scan: null descriptor");
  MM_CHECK_ARG(d->fp64 == 0 || d->fp64 == 1, "scan: fp64 must be 0 or 1");
  if (!supported_size(d->fx, d->fp64) || !supported_size(d->fy, d->fp64)) {
    set_error("scan transform sizes %d x %d: each must be 64, 128, 256, 512, 1024 or (FP32) 384, 768", d->fx,
              d->fy);
    return MM_ERR_UNSUPPORTED;
  }
  MM_CHECK_ARG(d->kx >= 1 && d->ky >= 1 && d->kplanes >= 1, "scan: kernel extents must be positive");
  return MM_OK;
}

int check_planes(const mm_scan_planes* p, int fx, int fy, int ext_x, int ext_y) {
  MM_CHECK_ARG(p != nullptr && p->data != nullptr, "scan: null planes");
  MM_CHECK_ARG(p->nx >= 1 && p->ny >= 1 && p->nz >= 1 && p->group >= 1, "scan: plane extents must be positive");
  MM_CHECK_ARG(ext_x >= 1 && ext_y >= 1 && ext_x <= fx && ext_y <= fy,
               "scan: transform input %d x %d exceeds the transform %d x %d", ext_x, ext_y, fx, fy);
  return MM_OK;
}

Planes make_planes(const mm_scan_planes* p, int wrap, int wx0, int wy0, int ext_x, int ext_y) {
  Planes P;
  P.data = p->data;
  P.s0 = p->s0;
  P.s1 = p->s1;
  P.s2 = p->s2;
  P.nx = p->nx;
  P.ny = p->ny;
  P.nz = p->nz;
  P.group = p->group;
  P.planes = (p->nz + p->group - 1) / p->group;
  P.m0 = p->mask0;
  P.m1 = p->mask1;
  P.data2 = p->data2;
  P.wrap = wrap;
  P.wx0 = wx0;
  P.wy0 = wy0;
  P.ext_x = ext_x;
  P.ext_y = ext_y;
  return P;
}

size_t complex_bytes(int fp64) { return fp64 ? sizeof(double2) : sizeof(float2); }

// forward transform of P's planes into S (pairs, fx, fy)
template <class T>
int forward(const Planes& P, int fx, int fy, void* S, cudaStream_t st) {
  const int pairs = (P.planes + 1) / 2;
  int rc = by_size<T>(fy, [&](auto n) { return rows_fwd<T, decltype(n)::value>(P, fx, S, pairs, st); });
  if (rc) return rc;
  return by_size<T>(fx, [&](auto n) { return cols<T, decltype(n)::value, -1>(S, fy, pairs, P.ext_x, 0, fx, st); });
}

template <class T>
int kernel_spectrum(const mm_scan_desc* d, const mm_scan_planes* k, void* spectrum, void* work, size_t wbytes,
                    cudaStream_t st) {
  Planes P = make_planes(k, 0, 0, 0, k->nx, k->ny);
  MM_CHECK_ARG(P.planes == d->kplanes, "scan: kernel has %d transform planes, descriptor says %d", P.planes,
               d->kplanes);
  MM_CHECK_ARG(k->nx == d->kx && k->ny == d->ky, "scan: kernel extents %d x %d differ from the descriptor's %d x %d",
               k->nx, k->ny, d->kx, d->ky);
  const size_t need = mm_scan_workspace_size(d, P.planes);
  MM_CHECK_ARG(work != nullptr && wbytes >= need, "scan: workspace of %zu bytes needed", need);
  MM_CHECK_ARG(spectrum != nullptr, "scan: null spectrum");
  int rc = forward<T>(P, d->fx, d->fy, work, st);
  if (rc) return rc;
  const long long n = (long long)d->fx * (d->fy / 2 + 1) * ((P.planes + 1) / 2);
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  unpack_kernel<T><<<blocks, 256, 0, st>>>(static_cast<const typename Cplx<T>::type*>(work),
                                          static_cast<typename Cplx<T>::type*>(spectrum), d->fx, d->fy, P.planes);
  MM_CHECK_LAUNCH("scan kernel unpack");
  return MM_OK;
}

// Inverse passes of packed spectra S (overwritten): columns keeping the crop
// rows, rows keeping the crop columns, unpacked, weighted, scaled, stored.
template <class T>
int inverse(const mm_scan_desc* d, const mm_scan_conv* c, int planes, void* S, cudaStream_t st) {
  MM_CHECK_ARG(c->out != nullptr, "scan: null output");
  MM_CHECK_ARG(c->out_x >= 1 && c->out_y >= 1 && c->crop_x >= 0 && c->crop_y >= 0 &&
                   c->crop_x + c->out_x <= d->fx && c->crop_y + c->out_y <= d->fy,
               "scan: kept window [%d, %d) x [%d, %d) outside the transform %d x %d", c->crop_x, c->crop_x + c->out_x,
               c->crop_y, c->crop_y + c->out_y, d->fx, d->fy);
  const int pairs = (planes + 1) / 2;
  int rc = by_size<T>(d->fx, [&](auto n) {
    return cols<T, decltype(n)::value, +1>(S, d->fy, pairs, d->fx, c->crop_x, c->out_x, st);
  });
  if (rc) return rc;
  Out O;
  O.data = c->out;
  O.o0 = c->o0;
  O.o1 = c->o1;
  O.o2 = c->o2;
  O.out_x = c->out_x;
  O.out_y = c->out_y;
  O.planes = planes;
  O.crop_y = c->crop_y;
  O.accumulate = c->accumulate;
  O.alpha = c->alpha;
  O.weight = c->out_weight;
  return by_size<T>(d->fy, [&](auto n) { return rows_inv<T, decltype(n)::value>(S, d->fx, O, st); });
}

template <class T>
int convolve(const mm_scan_desc* d, const mm_scan_conv* c, const void* spectrum, void* work, size_t wbytes,
             cudaStream_t st) {
  using C = typename Cplx<T>::type;
  int rc = check_planes(&c->src, d->fx, d->fy, c->ext_x, c->ext_y);
  if (rc) return rc;
  MM_CHECK_ARG(spectrum != nullptr && (c->out != nullptr || c->out_spectra != nullptr),
               "scan: null spectrum or output");
  Planes P = make_planes(&c->src, c->wrap, c->wrap_x0, c->wrap_y0, c->ext_x, c->ext_y);
  MM_CHECK_ARG(!c->wrap || (c->wrap_x0 >= 0 && c->wrap_y0 >= 0), "scan: wrap offsets must be nonnegative");
  Rule R;
  R.zrule = c->zrule;
  R.zoff = c->zoff;
  R.nin = P.planes;
  R.nk = d->kplanes;
  R.nout = c->out_planes;
  switch (c->zrule) {
    case MM_SCAN_CONV_Z:
    case MM_SCAN_CORR_Z:
      MM_CHECK_ARG(c->out_planes >= 1, "scan: output planes must be positive");
      MM_CHECK_ARG(c->zoff >= 0 && c->zoff < R.nk, "scan: Z offset %d outside the %d kernel planes", c->zoff, R.nk);
      break;
    case MM_SCAN_SUM_Z:
      MM_CHECK_ARG(R.nk == R.nin && c->out_planes == 1, "scan: SUM_Z needs as many kernel as source planes (%d, %d) "
                   "and one output plane", R.nk, R.nin);
      break;
    case MM_SCAN_EACH_Z:
      MM_CHECK_ARG(R.nk == R.nin && c->out_planes == R.nin, "scan: EACH_Z needs equal source, kernel and output "
                   "planes (%d, %d, %d)", R.nin, R.nk, c->out_planes);
      break;
    default:
      MM_CHECK_ARG(false, "scan: unknown Z rule %d", c->zrule);
  }
  // alias-free: the linear convolution's support ends at ext + k - 1
  MM_CHECK_ARG(c->ext_x + d->kx - 1 <= d->fx + c->crop_x && c->ext_y + d->ky - 1 <= d->fy + c->crop_y,
               "scan: transform %d x %d too small for inputs %d x %d and kernels %d x %d at crop (%d, %d)", d->fx,
               d->fy, c->ext_x, c->ext_y, d->kx, d->ky, c->crop_x, c->crop_y);
  const int pairs_out = (R.nout + 1) / 2;
  // workspace: the source spectra (unless given) and the output spectra
  // (unless stored elsewhere)
  const int wplanes = c->src_spectra ? (c->out_spectra ? 0 : R.nout) : std::max(R.nin, R.nout);
  const size_t need = wplanes ? mm_scan_workspace_size(d, wplanes) : 0;
  MM_CHECK_ARG(!need || (work != nullptr && wbytes >= need), "scan: workspace of %zu bytes needed", need);
  // combine: per-thread source bins in shared memory
  int threads = kCombineThreads;
  while (threads > 32 && (size_t)R.nin * threads * sizeof(C) > 200 * 1024) threads /= 2;
  const size_t csmem = (size_t)R.nin * threads * sizeof(C);
  MM_CHECK_ARG(csmem <= 200 * 1024, "scan: %d source planes exceed the combine kernel's shared memory", R.nin);
  const C* sin = static_cast<const C*>(c->src_spectra);
  if (!sin) {
    rc = forward<T>(P, d->fx, d->fy, work, st);
    if (rc) return rc;
    sin = static_cast<const C*>(work);
  }
  C* sout = c->out_spectra ? static_cast<C*>(c->out_spectra) : static_cast<C*>(work);
  MM_CHECK_CUDA(cudaFuncSetAttribute(combine_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem),
                "cudaFuncSetAttribute(scan combine)");
  const long long bins = (long long)d->fx * (d->fy / 2 + 1);
  const T scale = T(1.0 / (double(d->fx) * double(d->fy)));
  combine_kernel<T><<<(unsigned)((bins + threads - 1) / threads), threads, csmem, st>>>(
      sin, sout, static_cast<const C*>(spectrum), d->fx, d->fy, R, scale, c->out_spectra ? c->accumulate : 0);
  MM_CHECK_LAUNCH("scan combine");
  if (c->out_spectra) return MM_OK;
  return inverse<T>(d, c, R.nout, sout, st);
  (void)pairs_out;
}

}  // namespace scan
}  // namespace mm

using namespace mm;

extern "C" size_t mm_scan_spectrum_bytes(const mm_scan_desc* d) {
  if (scan::check_desc(d)) return 0;
  return (size_t)d->kplanes * d->fx * (d->fy / 2 + 1) * scan::complex_bytes(d->fp64);
}

extern "C" size_t mm_scan_workspace_size(const mm_scan_desc* d, int planes) {
  if (scan::check_desc(d) || planes < 1) return 0;
  return (size_t)((planes + 1) / 2) * d->fx * d->fy * scan::complex_bytes(d->fp64);
}

extern "C" int mm_scan_kernel_spectrum(const mm_scan_desc* d, const mm_scan_planes* k, void* spectrum, void* work,
                                       size_t wbytes, void* stream) {
  int rc = scan::check_desc(d);
  if (rc) return rc;
  rc = scan::check_planes(k, d->fx, d->fy, k ? k->nx : 0, k ? k->ny : 0);
  if (rc) return rc;
  auto st = static_cast<cudaStream_t>(stream);
  return d->fp64 ? scan::kernel_spectrum<double>(d, k, spectrum, work, wbytes, st)
                 : scan::kernel_spectrum<float>(d, k, spectrum, work, wbytes, st);
}

extern "C" int mm_scan_convolve(const mm_scan_desc* d, const mm_scan_conv* c, const void* spectrum, void* work,
                                size_t wbytes, void* stream) {
  int rc = scan::check_desc(d);
  if (rc) return rc;
  MM_CHECK_ARG(c != nullptr, "scan: null convolution");
  auto st = static_cast<cudaStream_t>(stream);
  return d->fp64 ? scan::convolve<double>(d, c, spectrum, work, wbytes, st)
                 : scan::convolve<float>(d, c, spectrum, work, wbytes, st);
}

extern "C" int mm_scan_forward(const mm_scan_desc* d, const mm_scan_conv* c, void* spectra, void* stream) {
  int rc = scan::check_desc(d);
  if (rc) return rc;
  MM_CHECK_ARG(c != nullptr && spectra != nullptr, "scan: null convolution or spectra");
  rc = scan::check_planes(&c->src, d->fx, d->fy, c->ext_x, c->ext_y);
  if (rc) return rc;
  MM_CHECK_ARG(!c->wrap || (c->wrap_x0 >= 0 && c->wrap_y0 >= 0), "scan: wrap offsets must be nonnegative");
  scan::Planes P = scan::make_planes(&c->src, c->wrap, c->wrap_x0, c->wrap_y0, c->ext_x, c->ext_y);
  auto st = static_cast<cudaStream_t>(stream);
  return d->fp64 ? scan::forward<double>(P, d->fx, d->fy, spectra, st) : scan::forward<float>(P, d->fx, d->fy, spectra, st);
}

extern "C" int mm_scan_inverse(const mm_scan_desc* d, const mm_scan_conv* c, void* spectra, void* stream) {
  int rc = scan::check_desc(d);
  if (rc) return rc;
  MM_CHECK_ARG(c != nullptr && spectra != nullptr && c->out_planes >= 1, "scan: bad inverse arguments");
  auto st = static_cast<cudaStream_t>(stream);
  return d->fp64 ? scan::inverse<double>(d, c, c->out_planes, spectra, st)
                 : scan::inverse<float>(d, c, c->out_planes, spectra, st);
}

extern "C" int mm_scan_background(int fp64, const void* const* volumes, int nvol, long long s0, long long s1,
                                  long long s2, int nx, int ny, int nz, const int32_t* idx, const double* scale, int n,
                                  double power, const void* mask, void* out, void* stream) {
  MM_CHECK_ARG(volumes != nullptr && nvol >= 1 && nvol <= 4, "scan background: 1..4 volumes");
  MM_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1 && n >= 1 && idx && scale && out, "scan background: bad arguments");
  auto st = static_cast<cudaStream_t>(stream);
  const long long np = (long long)nx * ny;
  const int blocks = (int)std::min<long long>((np + 255) / 256, 148LL * 8);
  if (fp64) {
    scan::BgVols<double> V{};
    for (int v = 0; v < nvol; ++v) V.v[v] = static_cast<const double*>(volumes[v]);
    scan::background_kernel<double><<<blocks, 256, 0, st>>>(V, nvol, s0, s1, s2, nx, ny, nz, idx, scale, n, power,
                                                            static_cast<const double*>(mask),
                                                            static_cast<double*>(out));
  } else {
    scan::BgVols<float> V{};
    for (int v = 0; v < nvol; ++v) V.v[v] = static_cast<const float*>(volumes[v]);
    scan::background_kernel<float><<<blocks, 256, 0, st>>>(V, nvol, s0, s1, s2, nx, ny, nz, idx, scale, n, power,
                                                           static_cast<const float*>(mask), static_cast<float*>(out));
  }
  MM_CHECK_LAUNCH("scan background");
  return MM_OK;
}
