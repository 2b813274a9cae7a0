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

// ---------------------------------------------------------------------------
// Points on a full nx x ny lattice whose coordinates are symmetric under
// x -> reflection and y -> reflection: G commutes with both reflections, so in
// the basis of even / odd reflection pairs it splits into four independent
// blocks (parities (sx, sy) in {+,-}^2).  Lattice index (i, j) -> point
// idx[i*ny + j]; orbit O(i) = {i, nx-1-i}; even blocks use representatives
// i < (nx+1)/2, odd blocks i < nx/2.  Block b = 2*(sx<0) + (sy<0), padded to
// m x m with the identity.
__host__ __device__ __forceinline__ int reps(int n, int sign) { return sign > 0 ? (n + 1) / 2 : n / 2; }

__device__ __forceinline__ double green_d(const double* p, int k, int l) {
  const double dx = p[2 * k] - p[2 * l], dy = p[2 * k + 1] - p[2 * l + 1];
  const double d = sqrt(dx * dx + dy * dy);
  return d == 0.0 ? 0.0 : d * d * (log(d) - 1.0);
}

__global__ void green_blocks_kernel(const double* __restrict__ p, const int* __restrict__ idx, int nx, int ny, int m,
                                    double* __restrict__ blocks) {
  const long long total = 4LL * m * m;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const int b = int(o / ((long long)m * m));
    const int r = int((o / m) % m), c = int(o % m);
    const int sx = (b & 2) ? -1 : 1, sy = (b & 1) ? -1 : 1;
    const int hx = reps(nx, sx), hy = reps(ny, sy);
    if (r >= hx * hy || c >= hx * hy) {
      blocks[o] = r == c ? 1.0 : 0.0;
      continue;
    }
    const int i = r / hy, j = r % hy, i2 = c / hy, j2 = c % hy;
    const int k = idx[i * ny + j];
    const int ox = (i == nx - 1 - i) ? 1 : 2, oy = (j == ny - 1 - j) ? 1 : 2;
    const int ox2 = (i2 == nx - 1 - i2) ? 1 : 2, oy2 = (j2 == ny - 1 - j2) ? 1 : 2;
    double acc = 0.0;
    for (int u = 0; u < ox2; ++u)
      for (int v = 0; v < oy2; ++v) {
        const int a = u ? nx - 1 - i2 : i2, bb = v ? ny - 1 - j2 : j2;
        const double sgn = (u ? sx : 1) * (v ? sy : 1);
        acc += sgn * green_d(p, k, idx[a * ny + bb]);
      }
    blocks[o] = acc * sqrt(double(ox * oy) / double(ox2 * oy2));
  }
}

// Forward (dir 0): values (n, C) -> parity components W (4, m, C) (padding 0).
// Inverse (dir 1): components D (4, m, C) -> coefficients (n, C).
__global__ void parity_transform_kernel(const int* __restrict__ idx, int nx, int ny, int m, int C, int dir,
                                        const double* __restrict__ in, double* __restrict__ out) {
  const long long total = dir == 0 ? 4LL * m * C : (long long)nx * ny * C;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    if (dir == 0) {
      const int b = int(o / ((long long)m * C)), r = int((o / C) % m), c = int(o % C);
      const int sx = (b & 2) ? -1 : 1, sy = (b & 1) ? -1 : 1;
      const int hx = reps(nx, sx), hy = reps(ny, sy);
      double acc = 0.0;
      if (r < hx * hy) {
        const int i = r / hy, j = r % hy;
        const int ox = (i == nx - 1 - i) ? 1 : 2, oy = (j == ny - 1 - j) ? 1 : 2;
        for (int u = 0; u < ox; ++u)
          for (int v = 0; v < oy; ++v) {
            const int a = u ? nx - 1 - i : i, bb = v ? ny - 1 - j : j;
            acc += (u ? sx : 1) * (v ? sy : 1) * in[(size_t)idx[a * ny + bb] * C + c];
          }
        acc /= sqrt(double(ox * oy));
      }
      out[o] = acc;
    } else {
      const int pt = int(o / C), c = int(o % C);
      const int a = pt / ny, bb = pt % ny;
      const int i = min(a, nx - 1 - a), j = min(bb, ny - 1 - bb);
      const int ox = (i == nx - 1 - i) ? 1 : 2, oy = (j == ny - 1 - j) ? 1 : 2;
      double acc = 0.0;
      for (int b = 0; b < 4; ++b) {
        const int sx = (b & 2) ? -1 : 1, sy = (b & 1) ? -1 : 1;
        if ((sx < 0 && ox == 1) || (sy < 0 && oy == 1)) continue;  // the centre has no odd component
        const int hy = reps(ny, sy);
        const double sgn = (a != i ? sx : 1) * (bb != j ? sy : 1);
        acc += sgn * in[((size_t)b * m + i * hy + j) * C + c];
      }
      out[(size_t)idx[pt] * C + c] = acc / sqrt(double(ox * oy));
    }
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

// Integer point coordinates and pixel-centre queries: every query-point
// offset is (dx + 0.5, dy + 0.5) with integer dx, dy, so the Green function
// takes one of TW x TH tabulated values; table[(dx - dx0) * TH + (dy - dy0)].
__global__ void green_table_kernel(int dx0, int dy0, int TW, int TH, double* __restrict__ table) {
  const long long total = (long long)TW * TH;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const double dx = double(dx0 + int(o / TH)) + 0.5, dy = double(dy0 + int(o % TH)) + 0.5;
    table[o] = green_r2(dx * dx + dy * dy);
  }
}

// Same sums as green_eval_kernel on the grid (same point order, same FMA
// chain), with the Green function read from the table.  A CTA covers a
// 16 x 16 query tile, so for each point it reads one 16 x 16 table window.
template <int C>
__global__ void __launch_bounds__(256) green_eval_table_kernel(const double* __restrict__ p,
                                                               const double* __restrict__ coef, int ncoef, int c0, int n,
                                                               int X, int Y, const double* __restrict__ table, int dx0,
                                                               int dy0, int TH, double* __restrict__ out) {
  __shared__ int sp[kTile][2];
  __shared__ double sc[kTile][C];
  const int qx = blockIdx.x * 16 + threadIdx.x / 16, qy = blockIdx.y * 16 + threadIdx.x % 16;
  double acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0.0;
  const bool live = qx < X && qy < Y;
  for (int base = 0; base < n; base += kTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
      const int g = base + i;
      sp[i][0] = g < n ? int(p[2 * g]) : 0;
      sp[i][1] = g < n ? int(p[2 * g + 1]) : 0;
#pragma unroll
      for (int c = 0; c < C; ++c) sc[i][c] = g < n ? coef[(size_t)g * ncoef + c0 + c] : 0.0;
    }
    __syncthreads();
    if (live) {
      const int cnt = min(kTile, n - base);
      for (int i = 0; i < cnt; ++i) {
        const double g = __ldg(table + (size_t)(qx - sp[i][0] - dx0) * TH + (qy - sp[i][1] - dy0));
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] = fma(g, sc[i][c], acc[c]);
      }
    }
  }
  if (live) {
#pragma unroll
    for (int c = 0; c < C; ++c) out[((size_t)qx * Y + qy) * ncoef + c0 + c] = acc[c];
  }
}

// Solve LU x = P b in place for one m x m factorisation per CTA, LU stored
// column-major (element (i, k) at k*m + i, as getrf leaves it: unit-lower L
// below the diagonal, U on and above it; 1-based LAPACK row interchanges),
// C right-hand sides held in shared memory.  Blocked by 32 columns: warp 0
// solves the diagonal block, then every thread updates its rows with the
// block's 32 columns (consecutive threads read consecutive rows: coalesced).
constexpr int kSolveBlock = 32;
// One CTA per (system b, right-hand side blockIdx.y): the columns are
// independent, so each runs its own substitution chain (the same operations
// in the same order as a CTA that carries all columns together).
__global__ void __launch_bounds__(512) lu_solve_kernel(const double* __restrict__ lu, const int* __restrict__ piv,
                                                        int m, int ldx, double* __restrict__ x) {
  constexpr int C = 1;
  extern __shared__ double xs[];  // m values of this column, then m pivots
  int* sp = reinterpret_cast<int*>(xs + (size_t)m * C);
  const int b = blockIdx.x, col = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* A = lu + (size_t)b * m * m;
  double* xb = x + (size_t)b * m * ldx + col;
  for (int e = tid; e < m; e += blockDim.x) xs[e] = xb[(size_t)e * ldx];
  for (int e = tid; e < m; e += blockDim.x) sp[e] = piv[(size_t)b * m + e];
  __syncthreads();
  if (tid == 0) {
    for (int i = 0; i < m; ++i) {
      const int r = sp[i] - 1;
      if (r != i && r >= 0 && r < m)
        for (int c = 0; c < C; ++c) {
          const double t = xs[i * C + c];
          xs[i * C + c] = xs[r * C + c];
          xs[r * C + c] = t;
        }
    }
  }
  __syncthreads();
  // forward substitution with unit-lower L
  for (int kb = 0; kb < m; kb += kSolveBlock) {
    const int ke = min(kb + kSolveBlock, m);
    if (warp == 0) {
      // the block's 32 x 32 L tile in registers (lane = row), x rows in registers
      const int i = kb + lane;
      double lr[kSolveBlock], xr[C];
#pragma unroll
      for (int kk = 0; kk < kSolveBlock; ++kk) lr[kk] = (i < ke && kb + kk < ke) ? A[(size_t)(kb + kk) * m + i] : 0.0;
#pragma unroll
      for (int c = 0; c < C; ++c) xr[c] = (c < C && i < ke) ? xs[i * C + c] : 0.0;
#pragma unroll
      for (int kk = 0; kk < kSolveBlock; ++kk) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const double xk = __shfl_sync(0xffffffffu, xr[c], kk);
          if (lane > kk) xr[c] -= lr[kk] * xk;
        }
      }
      if (i < ke)
        for (int c = 0; c < C; ++c) xs[i * C + c] = xr[c];
    }
    __syncthreads();
    for (int i = ke + tid; i < m; i += blockDim.x) {
      double a[kSolveBlock];
#pragma unroll
      for (int kk = 0; kk < kSolveBlock; ++kk) a[kk] = kb + kk < ke ? A[(size_t)(kb + kk) * m + i] : 0.0;
      for (int c = 0; c < C; ++c) {
        double acc = xs[i * C + c];
#pragma unroll
        for (int kk = 0; kk < kSolveBlock; ++kk) acc -= a[kk] * (kb + kk < ke ? xs[(kb + kk) * C + c] : 0.0);
        xs[i * C + c] = acc;
      }
    }
    __syncthreads();
  }
  // back substitution with U
  for (int ke = m; ke > 0; ke -= kSolveBlock) {
    const int kb = max(ke - kSolveBlock, 0);
    if (warp == 0) {
      const int i = kb + lane;
      double ur[kSolveBlock], xr[C];
#pragma unroll
      for (int kk = 0; kk < kSolveBlock; ++kk) ur[kk] = (i < ke && kb + kk < ke) ? A[(size_t)(kb + kk) * m + i] : 1.0;
#pragma unroll
      for (int c = 0; c < C; ++c) xr[c] = (c < C && i < ke) ? xs[i * C + c] : 0.0;
#pragma unroll
      for (int kk = kSolveBlock - 1; kk >= 0; --kk) {
        if (kb + kk >= ke) continue;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          if (lane == kk) xr[c] /= ur[kk];
          const double xk = __shfl_sync(0xffffffffu, xr[c], kk);
          if (lane < kk) xr[c] -= ur[kk] * xk;
        }
      }
      if (i < ke)
        for (int c = 0; c < C; ++c) xs[i * C + c] = xr[c];
    }
    __syncthreads();
    for (int i = tid; i < kb; i += blockDim.x) {
      double a[kSolveBlock];
#pragma unroll
      for (int kk = 0; kk < kSolveBlock; ++kk) a[kk] = kb + kk < ke ? A[(size_t)(kb + kk) * m + i] : 0.0;
      for (int c = 0; c < C; ++c) {
        double acc = xs[i * C + c];
#pragma unroll
        for (int kk = 0; kk < kSolveBlock; ++kk) acc -= a[kk] * (kb + kk < ke ? xs[(kb + kk) * C + c] : 0.0);
        xs[i * C + c] = acc;
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < m; e += blockDim.x) xb[(size_t)e * ldx] = xs[e];
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

extern "C" int mm_green_blocks(const double* points, const int* lattice, int nx, int ny, int m, double* blocks,
                               void* stream) {
  MM_CHECK_ARG(points && lattice && blocks, "NULL pointer");
  MM_CHECK_ARG(nx >= 1 && ny >= 1 && m >= reps(nx, 1) * reps(ny, 1), "block size %d too small for a %d x %d lattice", m,
               nx, ny);
  const long long total = 4LL * m * m;
  const int nblk = int(std::min<long long>((total + 255) / 256, 148LL * 32));
  green_blocks_kernel<<<nblk, 256, 0, static_cast<cudaStream_t>(stream)>>>(points, lattice, nx, ny, m, blocks);
  MM_CHECK_LAUNCH("green parity blocks");
  return MM_OK;
}

extern "C" int mm_v4_parity(const int* lattice, int nx, int ny, int m, int ncoef, int inverse, const double* in,
                            double* out, void* stream) {
  MM_CHECK_ARG(lattice && in && out, "NULL pointer");
  MM_CHECK_ARG(nx >= 1 && ny >= 1 && ncoef >= 1 && m >= reps(nx, 1) * reps(ny, 1), "bad parity transform sizes");
  const long long total = inverse ? (long long)nx * ny * ncoef : 4LL * m * ncoef;
  const int nblk = int(std::min<long long>((total + 255) / 256, 148LL * 8));
  parity_transform_kernel<<<nblk, 256, 0, static_cast<cudaStream_t>(stream)>>>(lattice, nx, ny, m, ncoef, inverse ? 1 : 0,
                                                                              in, out);
  MM_CHECK_LAUNCH("v4 parity transform");
  return MM_OK;
}

extern "C" int mm_green_apply_grid_table(const double* points, const double* coef, double* out, int n, int X, int Y,
                                         int ncoef, int px_min, int px_max, int py_min, int py_max, double* table,
                                         size_t table_bytes, void* stream) {
  MM_CHECK_ARG(points && coef && out && table, "NULL pointer");
  MM_CHECK_ARG(n >= 1 && X >= 1 && Y >= 1 && ncoef >= 1 && px_max >= px_min && py_max >= py_min,
               "bad v4 grid sizes");
  // integer offsets dx = qx - px range over [-px_max, X - 1 - px_min]
  const int dx0 = -px_max, dy0 = -py_max;
  const int TW = X - 1 - px_min - dx0 + 1, TH = Y - 1 - py_min - dy0 + 1;
  MM_CHECK_ARG(table_bytes >= sizeof(double) * (size_t)TW * TH, "v4 table needs %zu bytes, %zu given",
               sizeof(double) * (size_t)TW * TH, table_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long total = (long long)TW * TH;
  green_table_kernel<<<int(std::min<long long>((total + 255) / 256, 148LL * 16)), 256, 0, s>>>(dx0, dy0, TW, TH, table);
  MM_CHECK_LAUNCH("green table");
  const dim3 grid((X + 15) / 16, (Y + 15) / 16);
  for (int c0 = 0; c0 < ncoef; c0 += kMaxCoef) {
    const int c = std::min(kMaxCoef, ncoef - c0);
    switch (c) {
      case 1: green_eval_table_kernel<1><<<grid, 256, 0, s>>>(points, coef, ncoef, c0, n, X, Y, table, dx0, dy0, TH, out); break;
      case 2: green_eval_table_kernel<2><<<grid, 256, 0, s>>>(points, coef, ncoef, c0, n, X, Y, table, dx0, dy0, TH, out); break;
      case 3: green_eval_table_kernel<3><<<grid, 256, 0, s>>>(points, coef, ncoef, c0, n, X, Y, table, dx0, dy0, TH, out); break;
      default: green_eval_table_kernel<4><<<grid, 256, 0, s>>>(points, coef, ncoef, c0, n, X, Y, table, dx0, dy0, TH, out); break;
    }
    MM_CHECK_LAUNCH("green table evaluation");
  }
  return MM_OK;
}

extern "C" int mm_lu_solve_batched(const double* lu, const int* pivots, int batch, int m, int nrhs, double* x,
                                   void* stream) {
  MM_CHECK_ARG(lu && pivots && x, "NULL pointer");
  MM_CHECK_ARG(batch >= 1 && m >= 1 && nrhs >= 1 && nrhs <= 4, "bad LU solve sizes (1..4 right-hand sides)");
  const size_t smem = sizeof(double) * (size_t)m + sizeof(int) * (size_t)m;
  MM_CHECK_ARG(smem <= 200 * 1024, "LU solve: systems of %d unknowns exceed shared memory", m);
  if (smem > 48 * 1024)
    MM_CHECK_CUDA(cudaFuncSetAttribute(lu_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "cudaFuncSetAttribute(lu solve)");
  lu_solve_kernel<<<dim3(batch, nrhs), 512, smem, static_cast<cudaStream_t>(stream)>>>(lu, pivots, m, nrhs, x);
  MM_CHECK_LAUNCH("LU solve");
  return MM_OK;
}
