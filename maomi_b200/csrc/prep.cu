// Per-run preparation kernels: phase screens, the screen gather of the
// reference backend, the FP64 pupil and the pupil -> tissue base field.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "dft.cuh"

namespace mm {
namespace {

// -------------------------------------------------------------- screens --
// out[z, i, j] = exp(1j * scale * raw[i, j, z]) without resizing (ss = 1).
__global__ void screens_direct_kernel(const float* __restrict__ raw, int H, int W, int Z, float scale,
                                      float2* __restrict__ out) {
  const long long total = (long long)Z * H * W;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const int j = int(o % W);
    const int i = int((o / W) % H);
    const int z = int(o / ((long long)W * H));
    const float ph = __ldg(raw + ((size_t)i * W + j) * Z + z) * scale;
    float s, c;
    sincosf(ph, &s, &c);
    out[o] = make_float2(c, s);
  }
}

// Resize along axis 0: tmp[i, w, z] = sum_a wx[i,a] * raw[ix[i,a], w, z].
__global__ void resize_rows_kernel(const float* __restrict__ raw, int W, int Z, const int* __restrict__ ix,
                                   const float* __restrict__ wx, int Ho, int KX, float* __restrict__ tmp) {
  const long long total = (long long)Ho * W * Z;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const int z = int(o % Z);
    const int w = int((o / Z) % W);
    const int i = int(o / ((long long)Z * W));
    float acc = 0.f;
    for (int a = 0; a < KX; ++a) acc += __ldg(raw + ((size_t)__ldg(ix + i * KX + a) * W + w) * Z + z) * __ldg(wx + i * KX + a);
    tmp[o] = acc;
  }
}

// Resize along axis 1 and form the screen: out[z, i, j] = exp(1j*scale*sum_b wy[j,b] tmp[i, iy[j,b], z]).
__global__ void resize_cols_screens_kernel(const float* __restrict__ tmp, int Ho, int W, int Z, const int* __restrict__ iy,
                                           const float* __restrict__ wy, int Wo, int KY, float scale,
                                           float2* __restrict__ out) {
  const long long total = (long long)Z * Ho * Wo;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const int j = int(o % Wo);
    const int i = int((o / Wo) % Ho);
    const int z = int(o / ((long long)Wo * Ho));
    float acc = 0.f;
    for (int b = 0; b < KY; ++b) acc += __ldg(tmp + ((size_t)i * W + __ldg(iy + j * KY + b)) * Z + z) * __ldg(wy + j * KY + b);
    float s, c;
    sincosf(acc * scale, &s, &c);
    out[o] = make_float2(c, s);
  }
}

__global__ void gather_kernel(const float2* __restrict__ src, const float* __restrict__ edge, const int* __restrict__ off,
                              float2* __restrict__ dst, int B, int Z, int H, int W, int N) {
  const long long total = (long long)B * Z * N * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int y = int(t % N), x = int((t / N) % N), z = int((t / ((long long)N * N)) % Z);
    const int b = int(t / ((long long)N * N * Z));
    const float2 a = __ldg(src + ((size_t)z * H + __ldg(off + 2 * b) + x) * W + __ldg(off + 2 * b + 1) + y);
    const float e = __ldg(edge + x * N + y);
    dst[t] = make_float2(a.x * e, a.y * e);
  }
}

int grid_for(long long total, int block = 256) {
  long long g = (total + block - 1) / block;
  return int(std::min<long long>(std::max<long long>(g, 1), 148LL * 64));
}

// ---------------------------------------------------------------- pupil --
struct PupilDev {
  int n;
  double pitch, rad, aper, k, fl;
  int nmodes;
  double mode_coef[32];
  int mode_m[32], mode_cos[32], mode_t0[32], mode_nt[32];
  double term_coef[128];
  int term_pow[128];
  const float* custom;
  int ch, cw;
  double crad, cscale;
};

// Zernike phase of one pixel accumulated like the reference: a float32 buffer
// receiving float64 terms one mode at a time (_optical_math.py:190-195).
__device__ float zernike_phase32(const PupilDev& d, double x, double y) {
  const double xs = x / d.aper, ys = y / d.aper;
  const double r = sqrt(xs * xs + ys * ys);
  const double th = atan2(ys, xs);
  float ph = 0.f;
  for (int m = 0; m < d.nmodes; ++m) {
    double rad = 0.0;
    for (int t = 0; t < d.mode_nt[m]; ++t) {
      const int i = d.mode_t0[m] + t;
      double pw = 1.0;
      for (int e = 0; e < d.term_pow[i]; ++e) pw *= r;
      rad += d.term_coef[i] * pw;
    }
    double ang = 1.0;
    if (d.mode_m[m] > 0) ang = d.mode_cos[m] ? cos(d.mode_m[m] * th) : sin(d.mode_m[m] * th);
    ph = float(double(ph) + d.mode_coef[m] * rad * ang);
  }
  return ph;
}

__global__ void pupil_phase_kernel(PupilDev d, float* __restrict__ phase, double* __restrict__ partial) {
  __shared__ double red[32];
  const int total = d.n * d.n;
  double acc = 0.0;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
    const int i = o / d.n, j = o % d.n;
    const double X = (j - d.n / 2.0) * d.pitch, Y = (i - d.n / 2.0) * d.pitch;
    const float ph = d.nmodes ? zernike_phase32(d, X, Y) : 0.f;
    phase[o] = ph;
    acc += ph;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void pupil_field_kernel(PupilDev d, const float* __restrict__ phase, const double* __restrict__ partial,
                                   int nparts, float2* __restrict__ out) {
  __shared__ float s_mean;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += partial[b];
    s_mean = float(s / (double(d.n) * d.n));
  }
  __syncthreads();
  const float mean = s_mean;
  const int total = d.n * d.n;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
    const int i = o / d.n, j = o % d.n;
    const double X = (j - d.n / 2.0) * d.pitch, Y = (i - d.n / 2.0) * d.pitch;
    const double rho2 = X * X + Y * Y;
    double amp = exp(-(X * X + Y * Y) / (d.rad * d.rad));
    if (!(rho2 < d.aper * d.aper)) amp = 0.0;
    double s, c;
    sincos(-d.k / (2.0 * d.fl) * rho2, &s, &c);
    double re = amp * c, im = amp * s;
    if (d.nmodes) {
      // exp(1j * k * (phase - mean)) formed in complex64 by the reference.
      const float arg = float(d.k) * (phase[o] - mean);
      double zs, zc;
      sincos(double(arg), &zs, &zc);
      const double zr = double(float(zc)), zi = double(float(zs));
      const double r2 = re * zr - im * zi, i2 = re * zi + im * zr;
      re = r2;
      im = i2;
    }
    if (d.custom) {
      // nearest sample, align_corners=True, zero outside (optics.py:109-117)
      const double gx = X / d.crad, gy = Y / d.crad;
      const double fx = rint((gx + 1.0) / 2.0 * (d.cw - 1)), fy = rint((gy + 1.0) / 2.0 * (d.ch - 1));
      double ph = 0.0;
      if (fx >= 0 && fx <= d.cw - 1 && fy >= 0 && fy <= d.ch - 1) ph = __ldg(d.custom + int(fy) * d.cw + int(fx));
      double cs, cc;
      sincos(ph * d.cscale, &cs, &cc);
      const double r2 = re * cc - im * cs, i2 = re * cs + im * cc;
      re = r2;
      im = i2;
    }
    out[o] = make_float2(float(re), float(im));
  }
}

// ------------------------------------------------------------ base field --
// v = u * exp(1j*pre(r)) * edge / sc, pre = k ((x d1)^2 + (y d1)^2) (1-sc)/(2 dz)  (FP64 phase)
__global__ void base_pre_kernel(const float2* __restrict__ u, const float* __restrict__ edge, int n, double d1,
                                double k, double sc, double dz, float2* __restrict__ v) {
  const int total = n * n;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
    const int i = o / n, j = o % n;
    const double x = (i - n / 2.0) * d1, y = (j - n / 2.0) * d1;
    double s, c;
    sincos(k * (x * x + y * y) * (1.0 - sc) / (2.0 * dz), &s, &c);
    const double e = double(__ldg(edge + i)) * double(__ldg(edge + j)) / sc;
    const float2 a = __ldg(u + o);
    v[o] = make_float2(float((a.x * c - a.y * s) * e), float((a.x * s + a.y * c) * e));
  }
}

// out = v * edge * exp(1j*post(r)), post = k/2 (sc-1)/(sc dz) ((x d2)^2 + (y d2)^2); norm^2 accumulated.
__global__ void base_post_kernel(const float2* __restrict__ v, const float* __restrict__ edge, int n, double d2,
                                 double k, double sc, double dz, double* __restrict__ parts, float2* __restrict__ out) {
  __shared__ double red[32];
  const int total = n * n;
  double acc = 0.0;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
    const int i = o / n, j = o % n;
    const double x = (i - n / 2.0) * d2, y = (j - n / 2.0) * d2;
    double s, c;
    sincos(k / 2.0 * (sc - 1.0) / (sc * dz) * (x * x + y * y), &s, &c);
    const double e = double(__ldg(edge + i)) * double(__ldg(edge + j));
    const float2 a = v[o];
    const double re = (a.x * c - a.y * s) * e, im = (a.x * s + a.y * c) * e;
    acc += re * re + im * im;
    out[o] = make_float2(float(re), float(im));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
    parts[blockIdx.x] = s;
  }
}

__global__ void base_norm_kernel(float2* __restrict__ out, int total, const double* __restrict__ parts, int nparts) {
  __shared__ float s_inv;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += parts[b];
    s_inv = float(1.0 / sqrt(s));
  }
  __syncthreads();
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x)
    out[o] = cscale(out[o], s_inv);
}

// One 1-D propagate along rows (axis 0) or columns (axis 1) of an n x n field.
template <class L, int LINES>
__global__ void __launch_bounds__(LINES * L::R2) line_pass_kernel(float2* __restrict__ f, int n, int axis,
                                                                  const float2* __restrict__ q) {
  extern __shared__ float4 smem_raw[];
  using CF = typename L::TF;
  using CI = typename L::TI;
  float2* xa = reinterpret_cast<float2*>(smem_raw);
  float2* xb = xa + LINES * L::XBUF;
  CF* twf = reinterpret_cast<CF*>(xb + LINES * L::XBUF);
  CI* twi = reinterpret_cast<CI*>(twf + L::N);
  if constexpr (L::kFft) {
    for (int i = threadIdx.x; i < L::N; i += blockDim.x) {
      double s, c;
      const int k1 = i / L::R2, t = i % L::R2;
      sincospi(-2.0 * double((t * k1) % L::N) / L::N, &s, &c);
      twf[i] = make_tw<CF>(c, s);
      const int nn = i / L::R1, k2 = i % L::R1;
      sincospi(2.0 * double((nn * k2) % L::N) / L::N, &s, &c);
      twi[i] = make_tw<CI>(c, s);
    }
  }
  __syncthreads();
  const int tid = threadIdx.x;
  const int line_local = axis == 0 ? tid / L::R2 : tid % LINES;
  const int t = axis == 0 ? tid % L::R2 : tid / LINES;
  const int line = blockIdx.x * LINES + line_local;
  float2 v[L::R1];
#pragma unroll
  for (int j = 0; j < L::R1; ++j) {
    const int e = t + L::R2 * j;
    v[j] = make_float2(0.f, 0.f);
    if (line < n && e < n) v[j] = axis == 0 ? f[(size_t)line * n + e] : f[(size_t)e * n + line];
  }
  L::propagate(v, t, q, n, xa + line_local * L::XBUF, xb + line_local * L::XBUF, twf, twi);
#pragma unroll
  for (int j = 0; j < L::R1; ++j) {
    const int e = t + L::R2 * j;
    if (line >= n || e >= n) continue;
    if (axis == 0) f[(size_t)line * n + e] = v[j];
    else f[(size_t)e * n + line] = v[j];
  }
}

template <class L, int LINES>
int line_pass(int n, float2* f, int axis, const float2* q, cudaStream_t s) {
  const size_t smem = 2 * (size_t)LINES * L::XBUF * sizeof(float2) + L::kTwiddleBytes;
  MM_CHECK_CUDA(cudaFuncSetAttribute(line_pass_kernel<L, LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(line_pass)");
  line_pass_kernel<L, LINES><<<(n + LINES - 1) / LINES, LINES * L::R2, smem, s>>>(f, n, axis, q);
  MM_CHECK_LAUNCH("line pass");
  return MM_OK;
}

bool fft_size(int n) { return n == 64 || n == 128 || n == 256 || n == 512; }

int line_pass_any(int n, float2* f, int axis, const float2* q, cudaStream_t s) {
  switch (n) {
    case 64: return line_pass<FftLine<8, 8, double2>, 32>(n, f, axis, q, s);
    case 128: return line_pass<FftLine<16, 8, double2>, 32>(n, f, axis, q, s);
    case 256: return line_pass<FftLine<16, 16, double2>, 16>(n, f, axis, q, s);
    case 512: return line_pass<FftLine<32, 16, double2>, 8>(n, f, axis, q, s);
    default:
      if (n <= 128) return line_pass<DenseLine<8>, 16>(n, f, axis, q, s);
      return line_pass<DenseLine<32>, 16>(n, f, axis, q, s);
  }
}

// Circulant kernel of the scaled step for dense lines: p[m] = IDFT(Q)[m] (FP64).
__global__ void base_p_kernel(float2* p, int n, double lam, double dz, double dx, double sc) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double re = 0.0, im = 0.0;
  for (int k = 0; k < n; ++k) {
    const int ks = k < n / 2 ? k : k - n;
    const double f = ks / (n * dx);
    double s, c;
    sincos(-M_PI * lam * dz * f * f / sc, &s, &c);
    double ws, wc;
    sincospi(2.0 * double((long long)k * m % n) / n, &ws, &wc);
    re += c * wc - s * ws;
    im += c * ws + s * wc;
  }
  p[m] = make_float2(float(re / n), float(im / n));
}

// Transfer function of the scaled step along one axis, FFT order, 1/n folded.
__global__ void base_q_kernel(float2* q, int n, double lam, double dz, double dx, double sc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int ks = k < n / 2 ? k : k - n;
  const double f = ks / (n * dx);
  double s, c;
  sincos(-M_PI * lam * dz * f * f / sc, &s, &c);
  q[k] = make_float2(float(c / n), float(s / n));
}

}  // namespace
}  // namespace mm

using namespace mm;

extern "C" int mm_gather_screens(const void* src, const float* edge, const int32_t* offsets, void* dst, int B, int Z,
                                 int H, int W, int N, void* stream) {
  MM_CHECK_ARG(src && edge && offsets && dst, "NULL pointer");
  MM_CHECK_ARG(B >= 0 && Z >= 1 && N >= 1 && H >= N && W >= N, "bad gather sizes B=%d Z=%d H=%d W=%d N=%d", B, Z, H, W, N);
  if (B == 0) return MM_OK;
  const long long total = (long long)B * Z * N * N;
  gather_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(src), edge, offsets, static_cast<float2*>(dst), B, Z, H, W, N);
  MM_CHECK_LAUNCH("gather_screens");
  return MM_OK;
}

extern "C" int mm_phase_prepare(const float* raw, int H, int W, int Z, const int32_t* ix, const float* wx, int Ho, int KX,
                                const int32_t* iy, const float* wy, int Wo, int KY, float scale, void* screens,
                                float* scratch, void* stream) {
  MM_CHECK_ARG(raw && screens, "NULL pointer");
  MM_CHECK_ARG(H >= 1 && W >= 1 && Z >= 1, "bad raw shape (%d,%d,%d)", H, W, Z);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* out = static_cast<float2*>(screens);
  if (!ix && !iy) {
    MM_CHECK_ARG(Ho == H && Wo == W, "without resize tables the output must match the input");
    const long long total = (long long)Z * H * W;
    screens_direct_kernel<<<grid_for(total), 256, 0, s>>>(raw, H, W, Z, scale, out);
    MM_CHECK_LAUNCH("phase screens");
    return MM_OK;
  }
  MM_CHECK_ARG(ix && wx && iy && wy && scratch && KX >= 1 && KY >= 1 && Ho >= 1 && Wo >= 1, "incomplete resize tables");
  resize_rows_kernel<<<grid_for((long long)Ho * W * Z), 256, 0, s>>>(raw, W, Z, ix, wx, Ho, KX, scratch);
  MM_CHECK_LAUNCH("resize rows");
  resize_cols_screens_kernel<<<grid_for((long long)Z * Ho * Wo), 256, 0, s>>>(scratch, Ho, W, Z, iy, wy, Wo, KY, scale, out);
  MM_CHECK_LAUNCH("resize columns + screens");
  return MM_OK;
}

extern "C" int mm_pupil(const mm_pupil_desc* desc, void* out, double* scratch, void* stream) {
  MM_CHECK_ARG(desc && out && scratch, "NULL pointer");
  MM_CHECK_ARG(desc->n >= 2 && desc->n <= 8192, "pupil grid %d out of range", desc->n);
  MM_CHECK_ARG(desc->nmodes >= 0 && desc->nmodes <= 32, "at most 32 Zernike modes (got %d)", desc->nmodes);
  PupilDev d{};
  d.n = desc->n;
  d.pitch = desc->pitch;
  d.rad = desc->beam_radius;
  d.aper = desc->aperture;
  d.k = desc->k;
  d.fl = desc->focal_length;
  d.nmodes = desc->nmodes;
  int t0 = 0;
  for (int m = 0; m < desc->nmodes; ++m) {
    d.mode_coef[m] = desc->mode_coef[m];
    d.mode_m[m] = desc->mode_m[m];
    d.mode_cos[m] = desc->mode_cos[m];
    d.mode_t0[m] = t0;
    d.mode_nt[m] = desc->mode_nterms[m];
    MM_CHECK_ARG(t0 + d.mode_nt[m] <= 128, "too many radial terms");
    for (int t = 0; t < d.mode_nt[m]; ++t) {
      d.term_coef[t0 + t] = desc->term_coef[t0 + t];
      d.term_pow[t0 + t] = desc->term_pow[t0 + t];
    }
    t0 += d.mode_nt[m];
  }
  d.custom = desc->custom_phase;
  d.ch = desc->custom_h;
  d.cw = desc->custom_w;
  d.crad = desc->custom_radius;
  d.cscale = desc->custom_scale;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int total = d.n * d.n;
  const int blocks = std::min(1024, (total + 255) / 256);
  float* phase = reinterpret_cast<float*>(scratch);
  double* parts = scratch + ((size_t)total + 1) / 2 + 1;
  pupil_phase_kernel<<<blocks, 256, 0, s>>>(d, phase, parts);
  MM_CHECK_LAUNCH("pupil phase");
  pupil_field_kernel<<<blocks, 256, 0, s>>>(d, phase, parts, blocks, static_cast<float2*>(out));
  MM_CHECK_LAUNCH("pupil field");
  return MM_OK;
}

extern "C" int mm_base_field(const mm_base_desc* desc, const void* pupil, void* out, void* work, double* scratch,
                             void* stream) {
  MM_CHECK_ARG(desc && pupil && out && work && scratch && desc->edge1d, "NULL pointer");
  const int n = desc->n;
  MM_CHECK_ARG(n >= 2 && n <= 512 && n % 2 == 0, "base field needs an even n <= 512 (got %d)", n);
  MM_CHECK_ARG(desc->dz > 0 && desc->d1 > 0 && desc->d2 > 0, "bad base-field geometry");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double lam = desc->lambda_medium;
  const double k = 2.0 * M_PI / lam;
  const double sc = desc->d2 / desc->d1;
  float2* v = static_cast<float2*>(work);
  float2* o = static_cast<float2*>(out);
  // q for the step lives after the norm partials in scratch (n complex64 = n/2... doubles)
  float2* q = reinterpret_cast<float2*>(scratch + 256);
  MM_CHECK_ARG(n <= 1536, "scratch too small");
  const int blocks = std::min(256, (n * n + 255) / 256);
  if (fft_size(n)) base_q_kernel<<<(n + 127) / 128, 128, 0, s>>>(q, n, lam, desc->dz, desc->d1, sc);
  else base_p_kernel<<<(n + 127) / 128, 128, 0, s>>>(q, n, lam, desc->dz, desc->d1, sc);
  MM_CHECK_LAUNCH("base transfer function");
  base_pre_kernel<<<blocks, 256, 0, s>>>(static_cast<const float2*>(pupil), desc->edge1d, n, desc->d1, k, sc, desc->dz, v);
  MM_CHECK_LAUNCH("base pre-chirp");
  if (int rc = line_pass_any(n, v, 0, q, s)) return rc;
  if (int rc = line_pass_any(n, v, 1, q, s)) return rc;
  base_post_kernel<<<blocks, 256, 0, s>>>(v, desc->edge1d, n, desc->d2, k, sc, desc->dz, scratch, o);
  MM_CHECK_LAUNCH("base post-chirp");
  base_norm_kernel<<<blocks, 256, 0, s>>>(o, n * n, scratch, blocks);
  MM_CHECK_LAUNCH("base normalise");
  return MM_OK;
}
