// Spatially varying local-PSF render (the RANA compact-support operator), FP64.
//
// The reference evaluates, for every field-node pair (i, j), an FFT
// convolution of the source tile around the node's support and overlap-adds
// the weighted piece (maomi/rana/_fft.py:74-95).  Because every tile is zero
// padded to a linear-convolution length, that equals the direct sum
//
//   excitation (correlate): out[r] += wz(r_z) sum_ij w_ij(r) sum_u src[r + u - K/2]   k_ij[u]
//   native (convolve)     : out[r] += wz(r_z) sum_ij w_ij(r) sum_u src[r - u + K/2]   k_ij[u]
//   detection (convolve)  : out[r] +=         sum_ij sum_u w_ij(s) wz(s_z) src[s] k_ij[u],  s = r - u + K/2
//
// with zero source outside the volume (K/2 = floor per axis; plane mode sums
// the 2-D operator over z with kernel plane z acting on source plane z).  This
// kernel computes that sum directly in FP64: one CTA per output tile of
// 16 x 16 pixels x 4 planes, looping over the node pairs active on the tile;
// per kernel plane the four source planes (with halo) and the kernel plane are
// staged in shared memory, and each thread slides an 8-wide register window
// along y so every staged value feeds 8 FMAs.  Convolutions are turned into
// correlations by staging the kernel flipped.
#include <algorithm>

#include "common.cuh"

namespace mm {
namespace {

constexpr int TX = 16, TY = 16, TZ = 4;  // output tile
constexpr int QY = 8;                    // y outputs per thread (register window)
constexpr int THREADS = TX * (TY / QY) * TZ;  // 128

struct LocalP {
  int sx, sy, sz, kx, ky, kz, nx, ny;
  int kyp;         // ky padded to a multiple of QY
  int hx, hy;      // staged halo extents: TX + kx - 1, TY + kyp - 1 (+QY slack)
  const double* kern;
  const double* wx;
  const double* wy;
  const double* wz;  // nullable
  int detection, flip, plane;
  int cx, cy, cz;  // correlation offsets of the staged (possibly flipped) kernel
  double* out;
  const double* src;
};

__device__ __forceinline__ double wz_at(const LocalP& p, int z) { return p.wz ? p.wz[z] : 1.0; }

constexpr int kMaxNodes = 64;  // field nodes per axis

// Support [lo, hi] (first / last nonzero sample) of every node's weight row.
__device__ void node_support(const double* w, int nodes, int n, int* lo, int* hi) {
  for (int i = threadIdx.x; i < nodes; i += blockDim.x) {
    lo[i] = n;
    hi[i] = -1;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nodes * n; e += blockDim.x)
    if (w[e] != 0.0) {
      atomicMin(lo + e / n, e % n);
      atomicMax(hi + e / n, e % n);
    }
  __syncthreads();
}

// Node with support [lo, hi] touches [a, b)?
__device__ __forceinline__ bool touches(int lo, int hi, int a, int b) { return lo <= hi && lo < b && hi >= a; }

__global__ void __launch_bounds__(THREADS) local_render_kernel(LocalP p) {
  extern __shared__ double smem[];
  const int tiles_y = (p.sy + TY - 1) / TY;
  const int x0 = (blockIdx.x / tiles_y) * TX;
  const int y0 = (blockIdx.x % tiles_y) * TY;
  const int z0 = p.plane ? 0 : blockIdx.y * TZ;
  const int nzo = p.plane ? 1 : TZ;   // output planes of this tile
  const int tid = threadIdx.x;
  const int tx = tid % TX, tq = (tid / TX) % (TY / QY), tzi = tid / (TX * (TY / QY));
  __shared__ int lox[kMaxNodes], hix[kMaxNodes], loy[kMaxNodes], hiy[kMaxNodes];
  node_support(p.wx, p.nx, p.sx, lox, hix);
  node_support(p.wy, p.ny, p.sy, loy, hiy);
  const int hplane = p.hx * p.hy;
  double* halo = smem;                       // [TZ][hx][hy]
  double* ks = smem + (size_t)TZ * hplane;   // [kx][kyp]
  // Source reach of the tile along x / y (for the node-activity test in detection mode).
  const int sx_lo = x0 - p.cx, sx_hi = x0 + TX - 1 - p.cx + p.kx;
  const int sy_lo = y0 - p.cy, sy_hi = y0 + TY - 1 - p.cy + p.kyp;
  double acc_total[QY];
#pragma unroll
  for (int q = 0; q < QY; ++q) acc_total[q] = 0.0;
  for (int i = 0; i < p.nx; ++i) {
    const bool ai = p.detection ? touches(lox[i], hix[i], sx_lo, sx_hi) : touches(lox[i], hix[i], x0, x0 + TX);
    if (!ai) continue;
    for (int j = 0; j < p.ny; ++j) {
      const bool aj = p.detection ? touches(loy[j], hiy[j], sy_lo, sy_hi) : touches(loy[j], hiy[j], y0, y0 + TY);
      if (!aj) continue;
      const double* kij = p.kern + ((size_t)i * p.ny + j) * p.kx * p.ky * p.kz;
      double acc[QY];
#pragma unroll
      for (int q = 0; q < QY; ++q) acc[q] = 0.0;
      const int nplanes = p.kz;  // kernel planes (3-D: z taps; plane mode: summed source planes)
      for (int dz = 0; dz < nplanes; ++dz) {
        __syncthreads();
        // ---- stage the source planes this dz needs (one per output plane)
        for (int e = tid; e < nzo * hplane; e += THREADS) {
          const int zi = e / hplane, rem = e % hplane, hxi = rem / p.hy, hyi = rem % p.hy;
          const int gx = x0 - p.cx + hxi, gy = y0 - p.cy + hyi;
          const int gz = p.plane ? dz : z0 + zi + dz - p.cz;
          double v = 0.0;
          if (gx >= 0 && gx < p.sx && gy >= 0 && gy < p.sy && gz >= 0 && gz < p.sz && z0 + zi < p.sz) {
            v = p.src[((size_t)gx * p.sy + gy) * p.sz + gz];
            if (p.detection) v *= p.wx[(size_t)i * p.sx + gx] * p.wy[(size_t)j * p.sy + gy] * wz_at(p, gz);
          }
          halo[e] = v;
        }
        // ---- stage kernel plane dz (flipped for convolutions), zero padded to kyp
        for (int e = tid; e < p.kx * p.kyp; e += THREADS) {
          const int ux = e / p.kyp, uy = e % p.kyp;
          double v = 0.0;
          if (uy < p.ky) {
            const int fx = p.flip ? p.kx - 1 - ux : ux, fy = p.flip ? p.ky - 1 - uy : uy;
            const int fz = (p.flip && !p.plane) ? p.kz - 1 - dz : dz;
            v = kij[((size_t)fx * p.ky + fy) * p.kz + fz];
          }
          ks[e] = v;
        }
        __syncthreads();
        if (tzi < nzo) {
          const double* hrow0 = halo + (size_t)tzi * hplane + (size_t)tx * p.hy + tq * QY;
          for (int ux = 0; ux < p.kx; ++ux) {
            const double* hrow = hrow0 + (size_t)ux * p.hy;
            const double* krow = ks + (size_t)ux * p.kyp;
            double w[2 * QY];
#pragma unroll
            for (int q = 0; q < QY; ++q) w[q] = hrow[q];
            for (int uy0 = 0; uy0 < p.kyp; uy0 += QY) {
#pragma unroll
              for (int q = 0; q < QY; ++q) w[QY + q] = hrow[uy0 + QY + q];
#pragma unroll
              for (int ph = 0; ph < QY; ++ph) {
                const double kv = krow[uy0 + ph];
#pragma unroll
                for (int q = 0; q < QY; ++q) acc[q] = fma(w[q + ph], kv, acc[q]);
              }
#pragma unroll
              for (int q = 0; q < QY; ++q) w[q] = w[QY + q];
            }
          }
        }
      }
      // ---- weight the pair's contribution at the output pixel (excitation / native)
      const int ox = x0 + tx;
#pragma unroll
      for (int q = 0; q < QY; ++q) {
        const int oy = y0 + tq * QY + q;
        double wgt = 1.0;
        if (!p.detection) wgt = (ox < p.sx && oy < p.sy) ? p.wx[(size_t)i * p.sx + ox] * p.wy[(size_t)j * p.sy + oy] : 0.0;
        acc_total[q] = fma(wgt, acc[q], acc_total[q]);
      }
    }
  }
  if (tzi >= nzo) return;
  const int ox = x0 + tx, oz = z0 + tzi;
  if (ox >= p.sx || (!p.plane && oz >= p.sz)) return;
  const double zw = (!p.detection && !p.plane) ? wz_at(p, oz) : 1.0;
#pragma unroll
  for (int q = 0; q < QY; ++q) {
    const int oy = y0 + tq * QY + q;
    if (oy >= p.sy) continue;
    double* dst = p.plane ? p.out + (size_t)ox * p.sy + oy : p.out + ((size_t)ox * p.sy + oy) * p.sz + oz;
    *dst += zw * acc_total[q];
  }
}

}  // namespace
}  // namespace mm

extern "C" size_t mm_local_render_workspace_size(const mm_local_desc* desc) {
  (void)desc;
  return 0;  // the render needs no workspace
}

extern "C" int mm_local_render(const mm_local_desc* d, const double* source, const double* zweight, double* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  using namespace mm;
  (void)workspace;
  (void)workspace_bytes;
  MM_CHECK_ARG(d && source && out && d->kernels && d->wx && d->wy, "NULL pointer");
  MM_CHECK_ARG(d->sx >= 1 && d->sy >= 1 && d->sz >= 1 && d->kx >= 1 && d->ky >= 1 && d->kz >= 1 && d->nodes_x >= 1 &&
                   d->nodes_y >= 1,
               "bad local-render sizes");
  MM_CHECK_ARG(!d->plane || d->kz == d->sz, "plane mode needs kernel depth == source depth (%d vs %d)", d->kz, d->sz);
  MM_CHECK_ARG(d->nodes_x <= kMaxNodes && d->nodes_y <= kMaxNodes, "at most %d field nodes per axis", kMaxNodes);
  LocalP p{};
  p.sx = d->sx; p.sy = d->sy; p.sz = d->sz;
  p.kx = d->kx; p.ky = d->ky; p.kz = d->kz;
  p.nx = d->nodes_x; p.ny = d->nodes_y;
  p.kyp = (d->ky + QY - 1) / QY * QY;
  p.hx = TX + p.kx - 1;
  p.hy = TY + p.kyp - 1 + QY;  // the window reads QY past the last tap
  p.kern = d->kernels; p.wx = d->wx; p.wy = d->wy; p.wz = zweight;
  p.detection = d->detection;
  p.flip = !d->correlate;  // convolutions become correlations with the flipped kernel
  p.plane = d->plane;
  // correlation offset of the staged kernel: K/2 (correlate) or K-1-K/2 (flipped)
  p.cx = d->correlate ? d->kx / 2 : d->kx - 1 - d->kx / 2;
  p.cy = d->correlate ? d->ky / 2 : d->ky - 1 - d->ky / 2;
  p.cz = d->correlate ? d->kz / 2 : d->kz - 1 - d->kz / 2;
  p.out = out;
  p.src = source;
  const size_t smem = ((size_t)TZ * p.hx * p.hy + (size_t)p.kx * p.kyp) * sizeof(double);
  MM_CHECK_ARG(smem <= 227 * 1024, "kernel %dx%d too large for the shared-memory tile (%zu bytes)", d->kx, d->ky, smem);
  MM_CHECK_CUDA(cudaFuncSetAttribute(local_render_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(local render)");
  const int tiles = ((d->sx + TX - 1) / TX) * ((d->sy + TY - 1) / TY);
  const int zblocks = d->plane ? 1 : (d->sz + TZ - 1) / TZ;
  local_render_kernel<<<dim3(tiles, zblocks), THREADS, smem, static_cast<cudaStream_t>(stream)>>>(p);
  MM_CHECK_LAUNCH("local render");
  return MM_OK;
}
