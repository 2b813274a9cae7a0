// MATLAB "v4" biharmonic-spline mask assembly in FP64: the Green system
// matrix and the evaluation of r^2 (0.5 log r^2 - 1) against the solved
// coefficients for every query (pixel centre).
#include <algorithm>

#include "common.cuh"

namespace mm {
namespace {

constexpr int kTile = 256;   // points staged per shared-memory tile
constexpr int kMaxCoef = 4;  // value columns evaluated per pass

__device__ __forceinline__ double green_r2(double r2) { return r2 > 0.0 ? r2 * (0.5 * log(r2) - 1.0) : 0.0; }

__global__ void green_matrix_kernel(const double* __restrict__ p, int n, double* __restrict__ G) {
  const long long total = (long long)n * n;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const int i = int(o / n), j = int(o % n);
    const double dx = p[2 * i] - p[2 * j], dy = p[2 * i + 1] - p[2 * j + 1];
    const double d = sqrt(dx * dx + dy * dy);
    G[o] = d == 0.0 ? 0.0 : d * d * (log(d) - 1.0);
  }
}

// Queries either explicit (q != NULL, (m,2)) or the grid (i+0.5, j+0.5), i<X, j<Y.
template <int C>
__global__ void __launch_bounds__(256) green_eval_kernel(const double* __restrict__ p, const double* __restrict__ coef,
                                                         int ncoef, int c0, int n, const double* __restrict__ q,
                                                         int m, int Y, double* __restrict__ out) {
  __shared__ double sp[kTile][2 + C];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double qx = 0.0, qy = 0.0;
  if (t < m) {
    if (q) {
      qx = q[2 * t];
      qy = q[2 * t + 1];
    } else {
      qx = (t / Y) + 0.5;
      qy = (t % Y) + 0.5;
    }
  }
  double acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0.0;
  for (int base = 0; base < n; base += kTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
      const int g = base + i;
      if (g < n) {
        sp[i][0] = p[2 * g];
        sp[i][1] = p[2 * g + 1];
#pragma unroll
        for (int c = 0; c < C; ++c) sp[i][2 + c] = coef[(size_t)g * ncoef + c0 + c];
      } else {
        sp[i][0] = 0.0;
        sp[i][1] = 0.0;
#pragma unroll
        for (int c = 0; c < C; ++c) sp[i][2 + c] = 0.0;
      }
    }
    __syncthreads();
    const int cnt = min(kTile, n - base);
    for (int i = 0; i < cnt; ++i) {
      const double dx = qx - sp[i][0], dy = qy - sp[i][1];
      const double g = green_r2(dx * dx + dy * dy);
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = fma(g, sp[i][2 + c], acc[c]);
    }
  }
  if (t < m) {
#pragma unroll
    for (int c = 0; c < C; ++c) out[(size_t)t * ncoef + c0 + c] = acc[c];
  }
}

int eval_all(const double* p, const double* coef, int n, const double* q, int m, int Y, int ncoef, double* out,
             cudaStream_t s) {
  const int blocks = (m + 255) / 256;
  for (int c0 = 0; c0 < ncoef; c0 += kMaxCoef) {
    const int c = std::min(kMaxCoef, ncoef - c0);
    switch (c) {
      case 1: green_eval_kernel<1><<<blocks, 256, 0, s>>>(p, coef, ncoef, c0, n, q, m, Y, out); break;
      case 2: green_eval_kernel<2><<<blocks, 256, 0, s>>>(p, coef, ncoef, c0, n, q, m, Y, out); break;
      case 3: green_eval_kernel<3><<<blocks, 256, 0, s>>>(p, coef, ncoef, c0, n, q, m, Y, out); break;
      default: green_eval_kernel<4><<<blocks, 256, 0, s>>>(p, coef, ncoef, c0, n, q, m, Y, out); break;
    }
    MM_CHECK_LAUNCH("green evaluation");
  }
  return MM_OK;
}

}  // namespace
}  // namespace mm

using namespace mm;

extern "C" int mm_green_matrix(const double* points, double* G, int n, void* stream) {
  MM_CHECK_ARG(points && G, "NULL pointer");
  MM_CHECK_ARG(n >= 1, "need at least one point");
  const long long total = (long long)n * n;
  const int blocks = int(std::min<long long>((total + 255) / 256, 148LL * 32));
  green_matrix_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(points, n, G);
  MM_CHECK_LAUNCH("green matrix");
  return MM_OK;
}

extern "C" int mm_green_apply(const double* points, const double* coef, const double* queries, double* out, int n,
                              int m, int ncoef, void* stream) {
  MM_CHECK_ARG(points && coef && queries && out, "NULL pointer");
  MM_CHECK_ARG(n >= 1 && m >= 0 && ncoef >= 1, "bad v4 sizes n=%d m=%d ncoef=%d", n, m, ncoef);
  if (m == 0) return MM_OK;
  return eval_all(points, coef, n, queries, m, 1, ncoef, out, static_cast<cudaStream_t>(stream));
}

extern "C" int mm_green_apply_grid(const double* points, const double* coef, double* out, int n, int X, int Y,
                                   int ncoef, void* stream) {
  MM_CHECK_ARG(points && coef && out, "NULL pointer");
  MM_CHECK_ARG(n >= 1 && X >= 1 && Y >= 1 && ncoef >= 1, "bad v4 grid sizes");
  return eval_all(points, coef, n, nullptr, X * Y, Y, ncoef, out, static_cast<cudaStream_t>(stream));
}
