// Spatially varying local-PSF render (the RANA compact-support operator), FP64.
//
// The reference evaluates, for every field-node pair (i, j), an FFT
// convolution of the source tile around the node's support and overlap-adds
// the weighted piece (maomi/rana/_fft.py:74-95).  Every tile is zero padded to
// a linear-convolution length, so that equals the direct sum
//
//   excitation (correlate): out[r] += wz(r_z) sum_ij w_ij(r) sum_u src[r + u - K/2]   k_ij[u]
//   native (convolve)     : out[r] += wz(r_z) sum_ij w_ij(r) sum_u src[r - u + K/2]   k_ij[u]
//   detection (convolve)  : out[r] +=         sum_ij sum_u w_ij(s) wz(s_z) src[s] k_ij[u],  s = r - u + K/2
//
// with w_ij(r) = wx[i, r_x] wy[j, r_y], zero source outside the volume
// (K/2 = floor per axis) and, in plane mode, the 2-D operator summed over z
// with kernel plane z acting on source plane z.  Convolutions become
// correlations with the kernel staged flipped.
//
// Two kernels evaluate that sum in FP64:
//
// * cell_kernel (excitation, native): the output is cut along x and along y
//   into tiles over which the set of nodes with nonzero weight is constant
//   (mm_local_tiles; the smoothstep weights give two nodes per axis, so a tile
//   of one node interval needs exactly its 2 x 2 node pairs, where a fixed
//   16 x 16 grid straddling the intervals touched about nine).  One CTA owns a
//   tile (<= 18 x 18 pixels) x 2 planes and loops over the depth fields whose
//   weight is nonzero on its planes, so a whole depth bank is one launch.
//   Per kernel plane it stages the source halo plane(s) and the four pairs'
//   kernel planes in shared memory; each thread slides a register window of
//   2 x 6 source values along y for 6 outputs and keeps one 6-wide
//   accumulator per pair (24 FMAs per staged kernel value quartet), and folds
//   the pairs with their pixel weights at the end.
// * generic_kernel (detection, where the weights sit on the source side):
//   16 x 16 x 4 output tiles, node pairs whose weighted source reaches the
//   tile, source halo staged pre-weighted per pair.
//
// Both read the source transposed to (z, x, y) (a workspace filled by
// transpose_kernel) so every staged halo row is a contiguous run of y.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace mm {
namespace {

constexpr int kMaxNodes = 64;  // field nodes per axis
constexpr int kTileInts = 8;   // mm_local_tiles record: start, len, nact, node[4], 0
constexpr int kMaxActive = 4;  // nodes with nonzero weight inside one tile, per axis

// ------------------------------------------------------------ common pieces
__global__ void transpose_kernel(const double* __restrict__ src, int sx, int sy, int sz, double* __restrict__ dst) {
  // src (x, y, z) -> dst (z, x, y); one CTA per (x, 32-row block of y)
  __shared__ double t[32][17];
  const int x = blockIdx.x;
  const int y0 = blockIdx.y * 32;
  for (int z0 = 0; z0 < sz; z0 += 16) {
    for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
      const int yy = e / 16, zz = e % 16;
      const int y = y0 + yy, z = z0 + zz;
      t[yy][zz] = (y < sy && z < sz) ? src[((size_t)x * sy + y) * sz + z] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
      const int zz = e / 32, yy = e % 32;
      const int y = y0 + yy, z = z0 + zz;
      if (y < sy && z < sz) dst[((size_t)z * sx + x) * sy + y] = t[yy][zz];
    }
    __syncthreads();
  }
}

struct Common {
  int sx, sy, sz, kx, ky, kz, nx, ny, nf;
  const double* kern;   // (nf, nx, ny, kx, ky, kz)
  const double* wx;     // (nx, sx)
  const double* wy;     // (ny, sy)
  const double* wz;     // (nf, sz) or null
  const double* srcT;   // (sz, sx, sy)
  double* out;
  int flip, plane;
  int cx, cy, cz;       // correlation offsets of the staged (possibly flipped) kernel
};

__device__ __forceinline__ double wz_at(const Common& c, int f, int z) { return c.wz ? c.wz[(size_t)f * c.sz + z] : 1.0; }


// Kernels re-laid for staging: (nf, nx, ny, kz, kx, ky), already flipped for
// convolutions (x and y always, z only in 3-D mode), so one kernel plane of
// one node pair is a contiguous run of kx*ky values.
__global__ void kernel_prep_kernel(const double* __restrict__ k, int n_pairs, int kx, int ky, int kz, int flip,
                                   int plane, double* __restrict__ kt) {
  const size_t per = (size_t)kx * ky * kz;
  const size_t total = per * n_pairs;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t pair = e / per;
    const int r = int(e % per);
    const int kp = r / (kx * ky), uv = r % (kx * ky), ux = uv / ky, uy = uv % ky;
    const int fx = flip ? kx - 1 - ux : ux, fy = flip ? ky - 1 - uy : uy;
    const int fz = (flip && !plane) ? kz - 1 - kp : kp;
    kt[e] = k[pair * per + ((size_t)fx * ky + fy) * kz + fz];
  }
}

// ---------------------------------------------------- cell kernel (gather)
constexpr int QY = 6;              // y outputs per thread
constexpr int TMAX = 18;           // tile extent per axis
constexpr int CH = TMAX / QY;      // y chunks per tile row
constexpr int GROUP = 64;          // threads per output plane (>= TMAX * CH)
constexpr int TZC = 2;             // output planes per CTA
constexpr int CELL_THREADS = GROUP * TZC;
constexpr int PG = 4;              // node pairs per register pass
static_assert(TMAX * CH <= GROUP, "one unit per thread");

struct CellP {
  Common c;
  const double* kt;  // kernel_prep_kernel layout
  const int* tx;     // x tiles (kTileInts each)
  const int* ty;
  int ntx, nty;
  int hx, hy;        // halo plane extents (hy padded against bank conflicts)
  int kplanes;       // kernel-plane slots in shared memory (1, or TZC in plane mode)
};

// One halo row of taps for NP node pairs: acc[p][q] += sum_uy h[q + uy] k_p[uy].
// The window w slides along y in chunks of QY taps; the chunk loop has no
// data-dependent branches (the remainder of ky is a separate tail).
template <int NP>
__device__ __forceinline__ void taps_row(const double* __restrict__ hrow, const double* __restrict__ krow, int kplane,
                                         int ky, double (&acc)[PG][QY]) {
  double w[2 * QY];
#pragma unroll
  for (int q = 0; q < QY; ++q) w[q] = hrow[q];
  const int nfull = ky / QY;
#pragma unroll 1
  for (int cidx = 0; cidx < nfull; ++cidx) {
    const int uy0 = cidx * QY;
#pragma unroll
    for (int q = 0; q < QY; ++q) w[QY + q] = hrow[uy0 + QY + q];
#pragma unroll
    for (int ph = 0; ph < QY; ++ph)
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const double kv = krow[p * kplane + uy0 + ph];
#pragma unroll
        for (int q = 0; q < QY; ++q) acc[p][q] = fma(w[q + ph], kv, acc[p][q]);
      }
#pragma unroll
    for (int q = 0; q < QY; ++q) w[q] = w[QY + q];
  }
  const int rem = ky - nfull * QY;
  if (rem > 0) {
    const int uy0 = nfull * QY;
#pragma unroll
    for (int q = 0; q < QY; ++q) w[QY + q] = hrow[uy0 + QY + q];
#pragma unroll
    for (int ph = 0; ph < QY; ++ph)
      if (ph < rem)
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const double kv = krow[p * kplane + uy0 + ph];
#pragma unroll
          for (int q = 0; q < QY; ++q) acc[p][q] = fma(w[q + ph], kv, acc[p][q]);
        }
  }
}

template <int NP>
__device__ __forceinline__ void taps_plane(const double* hbase, const double* kbase, int hy, int kx, int ky,
                                           double (&acc)[PG][QY]) {
  const int kplane = kx * ky;
#pragma unroll 1
  for (int ux = 0; ux < kx; ++ux) taps_row<NP>(hbase + (size_t)ux * hy, kbase + (size_t)ux * ky, kplane, ky, acc);
}

__global__ void __launch_bounds__(CELL_THREADS, 2) cell_kernel(CellP P) {
  extern __shared__ double smem[];
  const Common& c = P.c;
  const int* tx = P.tx + (size_t)(blockIdx.x / P.nty) * kTileInts;
  const int* ty = P.ty + (size_t)(blockIdx.x % P.nty) * kTileInts;
  const int x0 = tx[0], lx = tx[1], ax = tx[2];
  const int y0 = ty[0], ly = ty[1], ay = ty[2];
  // a malformed tile record renders nothing rather than reading out of bounds
  bool ok = lx >= 1 && lx <= TMAX && ly >= 1 && ly <= TMAX && ax >= 1 && ax <= kMaxActive && ay >= 1 &&
            ay <= kMaxActive && x0 >= 0 && x0 + lx <= c.sx && y0 >= 0 && y0 + ly <= c.sy;
  for (int m = 0; m < kMaxActive; ++m) {
    ok = ok && (m >= ax || (tx[3 + m] >= 0 && tx[3 + m] < c.nx));
    ok = ok && (m >= ay || (ty[3 + m] >= 0 && ty[3 + m] < c.ny));
  }
  if (!ok) return;  // uniform per CTA
  const int tid = threadIdx.x;
  const int warp = tid / 32, lane = tid % 32;
  const int g = tid / GROUP;                 // plane group
  const int u = tid % GROUP;
  const int ch = u / TMAX, row = u % TMAX;   // rows fastest: conflict-free halo reads
  const bool unit = u < TMAX * CH && row < lx && ch * QY < ly;
  const int z0 = c.plane ? 0 : blockIdx.y * TZC;
  const int oz = z0 + g;                     // 3-D: this group's output plane
  const int hplane = P.hx * P.hy;
  const int kplane = c.kx * c.ky;
  double* halo = smem;                                         // [TZC][hx][hy]
  double* ks = smem + (size_t)TZC * hplane;                    // [kplanes][PG][kx*ky]
  const int npairs = ax * ay;
  const int iters = c.plane ? (c.kz + TZC - 1) / TZC : c.kz;
  const size_t pair_stride = (size_t)c.kz * kplane;

  double fin[QY];
#pragma unroll
  for (int q = 0; q < QY; ++q) fin[q] = 0.0;

  for (int f = 0; f < c.nf; ++f) {
    // skip fields with zero weight on this CTA's planes (uniform per CTA)
    if (!c.plane && c.wz) {
      bool any = false;
      for (int zz = z0; zz < min(z0 + TZC, c.sz); ++zz) any |= (c.wz[(size_t)f * c.sz + zz] != 0.0);
      if (!any) continue;
    }
    const double wzo = (!c.plane && oz < c.sz) ? wz_at(c, f, oz) : 1.0;
    const bool live = unit && (c.plane || (oz < c.sz && wzo != 0.0));
    const double* kf = P.kt + (size_t)f * c.nx * c.ny * pair_stride;
    for (int p0 = 0; p0 < npairs; p0 += PG) {
      const int np = min(PG, npairs - p0);
      double acc[PG][QY];
#pragma unroll
      for (int p = 0; p < PG; ++p)
#pragma unroll
        for (int q = 0; q < QY; ++q) acc[p][q] = 0.0;
      for (int it = 0; it < iters; ++it) {
        __syncthreads();  // the previous iteration's readers are done
        // ---- source halo planes, rows per warp, y across lanes (zero fill
        // outside the volume); all copies of the iteration in flight at once
        for (int gg = 0; gg < TZC; ++gg) {
          const int gz = c.plane ? it * TZC + gg : z0 + gg + it - c.cz;
          const bool zin = gz >= 0 && gz < c.sz;
          const double* splane = c.srcT + (size_t)(zin ? gz : 0) * c.sx * c.sy;
          for (int hxi = warp; hxi < P.hx; hxi += CELL_THREADS / 32) {
            const int gx = x0 - c.cx + hxi;
            const bool xin = zin && gx >= 0 && gx < c.sx;
            const double* srow = splane + (size_t)(xin ? gx : 0) * c.sy;
            double* drow = halo + (size_t)gg * hplane + (size_t)hxi * P.hy;
            for (int hyi = lane; hyi < P.hy; hyi += 32) {
              const int gy = y0 - c.cy + hyi;
              const bool in = xin && gy >= 0 && gy < c.sy;
              cp_async8_zfill(drow + hyi, srow + (in ? gy : 0), in);
            }
          }
        }
        // ---- this pass's kernel planes: contiguous runs of kx*ky values
        for (int slot = 0; slot < P.kplanes; ++slot) {
          const int kp = c.plane ? it * TZC + slot : it;
          for (int p = 0; p < np; ++p) {
            const int pair = p0 + p, i = tx[3 + pair / ay], j = ty[3 + pair % ay];
            const bool kin = kp < c.kz;
            const double* src = kf + ((size_t)i * c.ny + j) * pair_stride + (size_t)(kin ? kp : 0) * kplane;
            double* dst = ks + ((size_t)slot * PG + p) * kplane;
            for (int e = tid; e < kplane; e += CELL_THREADS) cp_async8_zfill(dst + e, src + e, kin);
          }
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        if (!live) continue;
        if (c.plane && it * TZC + g >= c.kz) continue;
        const double* hbase = halo + (size_t)g * hplane + (size_t)row * P.hy + ch * QY;
        const double* kbase = ks + (size_t)(c.plane ? g : 0) * PG * kplane;
        switch (np) {
          case 4: taps_plane<4>(hbase, kbase, P.hy, c.kx, c.ky, acc); break;
          case 3: taps_plane<3>(hbase, kbase, P.hy, c.kx, c.ky, acc); break;
          case 2: taps_plane<2>(hbase, kbase, P.hy, c.kx, c.ky, acc); break;
          default: taps_plane<1>(hbase, kbase, P.hy, c.kx, c.ky, acc); break;
        }
      }
      // ---- fold the pairs with their pixel weights
      if (live) {
        const int ox = x0 + row;
#pragma unroll
        for (int p = 0; p < PG; ++p) {
          if (p < np) {
            const int pair = p0 + p, i = tx[3 + pair / ay], j = ty[3 + pair % ay];
            const double wxi = c.wx[(size_t)i * c.sx + ox] * wzo;
#pragma unroll
            for (int q = 0; q < QY; ++q) {
              const int oy = y0 + ch * QY + q;
              const double wyj = oy < c.sy ? c.wy[(size_t)j * c.sy + oy] : 0.0;
              fin[q] = fma(wxi * wyj, acc[p][q], fin[q]);
            }
          }
        }
      }
    }
  }
  // ---- write: 3-D, one writer per voxel; plane mode, the groups' partial
  // sums over kernel planes are reduced through shared memory first
  if (c.plane) {
    __syncthreads();
    double* red = smem;
    if (g > 0 && unit)
#pragma unroll
      for (int q = 0; q < QY; ++q) red[((size_t)(g - 1) * GROUP + u) * QY + q] = fin[q];
    __syncthreads();
    if (g != 0 || !unit) return;
    for (int gg = 1; gg < TZC; ++gg)
#pragma unroll
      for (int q = 0; q < QY; ++q) fin[q] += red[((size_t)(gg - 1) * GROUP + u) * QY + q];
  }
  if (!unit || (!c.plane && oz >= c.sz)) return;
  const int ox = x0 + row;
#pragma unroll
  for (int q = 0; q < QY; ++q) {
    const int yq = ch * QY + q;
    if (yq >= ly) continue;
    const int oy = y0 + yq;
    double* dst = c.plane ? c.out + (size_t)ox * c.sy + oy : c.out + ((size_t)ox * c.sy + oy) * c.sz + oz;
    *dst += fin[q];
  }
}

// ------------------------------------------------- generic kernel (detection)
constexpr int TX = 16, TY = 16, TZ = 4;  // output tile
constexpr int GQY = 8;                   // y outputs per thread (register window)
constexpr int GEN_THREADS = TX * (TY / GQY) * TZ;  // 128

struct GenP {
  Common c;
  const double* kt;  // kernel_prep_kernel layout
  int kyp;         // ky padded to a multiple of GQY
  int hx, hy;
  int detection;
};

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

__device__ __forceinline__ bool touches(int lo, int hi, int a, int b) { return lo <= hi && lo < b && hi >= a; }

__global__ void __launch_bounds__(GEN_THREADS) generic_kernel(GenP P) {
  extern __shared__ double smem[];
  const Common& c = P.c;
  const int tiles_y = (c.sy + TY - 1) / TY;
  const int x0 = (blockIdx.x / tiles_y) * TX;
  const int y0 = (blockIdx.x % tiles_y) * TY;
  const int z0 = c.plane ? 0 : blockIdx.y * TZ;
  const int nzo = c.plane ? 1 : TZ;
  const int tid = threadIdx.x;
  const int tx = tid % TX, tq = (tid / TX) % (TY / GQY), tzi = tid / (TX * (TY / GQY));
  __shared__ int lox[kMaxNodes], hix[kMaxNodes], loy[kMaxNodes], hiy[kMaxNodes];
  node_support(c.wx, c.nx, c.sx, lox, hix);
  node_support(c.wy, c.ny, c.sy, loy, hiy);
  const int hplane = P.hx * P.hy;
  double* halo = smem;                       // [TZ][hx][hy]
  double* ks = smem + (size_t)TZ * hplane;   // [kx][kyp]
  const int sx_lo = x0 - c.cx, sx_hi = x0 + TX - 1 - c.cx + c.kx;
  const int sy_lo = y0 - c.cy, sy_hi = y0 + TY - 1 - c.cy + P.kyp;
  // source planes this tile reaches (detection weights sit on the source)
  const int szlo = c.plane ? 0 : max(0, z0 - c.cz), szhi = c.plane ? c.sz - 1 : min(c.sz - 1, z0 + TZ - 1 + c.kz - 1 - c.cz);
  double acc_total[GQY];
#pragma unroll
  for (int q = 0; q < GQY; ++q) acc_total[q] = 0.0;
  for (int f = 0; f < c.nf; ++f) {
    if (c.wz) {
      bool any = false;
      if (P.detection) {
        for (int zz = szlo; zz <= szhi; ++zz) any |= wz_at(c, f, zz) != 0.0;
      } else {
        for (int zz = z0; zz < min(z0 + nzo, c.sz); ++zz) any |= wz_at(c, f, zz) != 0.0;
      }
      if (!any) continue;
    }
    const double* kf = P.kt + (size_t)f * c.nx * c.ny * c.kx * c.ky * c.kz;
    for (int i = 0; i < c.nx; ++i) {
      const bool ai = P.detection ? touches(lox[i], hix[i], sx_lo, sx_hi) : touches(lox[i], hix[i], x0, x0 + TX);
      if (!ai) continue;
      for (int j = 0; j < c.ny; ++j) {
        const bool aj = P.detection ? touches(loy[j], hiy[j], sy_lo, sy_hi) : touches(loy[j], hiy[j], y0, y0 + TY);
        if (!aj) continue;
        const double* kij = kf + ((size_t)i * c.ny + j) * c.kx * c.ky * c.kz;
        double acc[GQY];
#pragma unroll
        for (int q = 0; q < GQY; ++q) acc[q] = 0.0;
        for (int dz = 0; dz < c.kz; ++dz) {
          __syncthreads();
          for (int e = tid; e < nzo * hplane; e += GEN_THREADS) {
            const int zi = e / hplane, rem = e % hplane, hxi = rem / P.hy, hyi = rem % P.hy;
            const int gx = x0 - c.cx + hxi, gy = y0 - c.cy + hyi;
            const int gz = c.plane ? dz : z0 + zi + dz - c.cz;
            double v = 0.0;
            if (gx >= 0 && gx < c.sx && gy >= 0 && gy < c.sy && gz >= 0 && gz < c.sz && z0 + zi < c.sz) {
              v = c.srcT[((size_t)gz * c.sx + gx) * c.sy + gy];
              if (P.detection) v *= c.wx[(size_t)i * c.sx + gx] * c.wy[(size_t)j * c.sy + gy] * wz_at(c, f, gz);
            }
            halo[e] = v;
          }
          const double* kpl = kij + (size_t)dz * c.kx * c.ky;  // prepped: flips applied
          for (int e = tid; e < c.kx * P.kyp; e += GEN_THREADS) {
            const int ux = e / P.kyp, uy = e % P.kyp;
            ks[e] = uy < c.ky ? kpl[(size_t)ux * c.ky + uy] : 0.0;
          }
          __syncthreads();
          if (tzi < nzo) {
            const double* hrow0 = halo + (size_t)tzi * hplane + (size_t)tx * P.hy + tq * GQY;
            for (int ux = 0; ux < c.kx; ++ux) {
              const double* hrow = hrow0 + (size_t)ux * P.hy;
              const double* krow = ks + (size_t)ux * P.kyp;
              double w[2 * GQY];
#pragma unroll
              for (int q = 0; q < GQY; ++q) w[q] = hrow[q];
              for (int uy0 = 0; uy0 < P.kyp; uy0 += GQY) {
#pragma unroll
                for (int q = 0; q < GQY; ++q) w[GQY + q] = hrow[uy0 + GQY + q];
#pragma unroll
                for (int ph = 0; ph < GQY; ++ph) {
                  const double kv = krow[uy0 + ph];
#pragma unroll
                  for (int q = 0; q < GQY; ++q) acc[q] = fma(w[q + ph], kv, acc[q]);
                }
#pragma unroll
                for (int q = 0; q < GQY; ++q) w[q] = w[GQY + q];
              }
            }
          }
        }
        const int ox = x0 + tx;
#pragma unroll
        for (int q = 0; q < GQY; ++q) {
          const int oy = y0 + tq * GQY + q;
          double wgt = 1.0;
          if (!P.detection)
            wgt = (ox < c.sx && oy < c.sy) ? c.wx[(size_t)i * c.sx + ox] * c.wy[(size_t)j * c.sy + oy] : 0.0;
          if (!P.detection && !c.plane) wgt *= (z0 + tzi < c.sz) ? wz_at(c, f, z0 + tzi) : 0.0;
          acc_total[q] = fma(wgt, acc[q], acc_total[q]);
        }
      }
    }
  }
  if (tzi >= nzo) return;
  const int ox = x0 + tx, oz = z0 + tzi;
  if (ox >= c.sx || (!c.plane && oz >= c.sz)) return;
#pragma unroll
  for (int q = 0; q < GQY; ++q) {
    const int oy = y0 + tq * GQY + q;
    if (oy >= c.sy) continue;
    double* dst = c.plane ? c.out + (size_t)ox * c.sy + oy : c.out + ((size_t)ox * c.sy + oy) * c.sz + oz;
    *dst += acc_total[q];
  }
}

// Row pitch of the cell kernel's halo planes: at least `need`, chosen so the
// 16 lanes of each half-warp (rows fastest, QY-wide chunks) read from
// distinct 8-byte bank pairs.
int cell_halo_pitch(int need) {
  int best = need, best_ways = 1 << 30;
  for (int hy = need; hy < need + 16; ++hy) {
    int worst = 0;
    for (int half = 0; half < GROUP / 16; ++half) {
      int count[16] = {0};
      for (int u = half * 16; u < half * 16 + 16 && u < TMAX * CH; ++u) {
        const int chk = u / TMAX, row = u % TMAX;
        worst = std::max(worst, ++count[(row * hy + chk * QY) % 16]);
      }
    }
    if (worst < best_ways) {
      best_ways = worst;
      best = hy;
    }
  }
  return best;
}

Common common_params(const mm_local_desc* d, const double* srcT, const double* zweight, double* out) {
  Common c{};
  c.sx = d->sx; c.sy = d->sy; c.sz = d->sz;
  c.kx = d->kx; c.ky = d->ky; c.kz = d->kz;
  c.nx = d->nodes_x; c.ny = d->nodes_y; c.nf = d->nfields;
  c.kern = d->kernels; c.wx = d->wx; c.wy = d->wy; c.wz = zweight;
  c.srcT = srcT;
  c.out = out;
  c.flip = !d->correlate;  // convolutions become correlations with the flipped kernel
  c.plane = d->plane;
  // correlation offset of the staged kernel: K/2 (correlate) or K-1-K/2 (flipped)
  c.cx = d->correlate ? d->kx / 2 : d->kx - 1 - d->kx / 2;
  c.cy = d->correlate ? d->ky / 2 : d->ky - 1 - d->ky / 2;
  c.cz = d->correlate ? d->kz / 2 : d->kz - 1 - d->kz / 2;
  return c;
}

}  // namespace
}  // namespace mm

extern "C" int mm_local_tiles(const double* w, int nodes, int n, int max_len, int* table, int capacity) {
  using namespace mm;
  MM_CHECK_ARG(w && nodes >= 1 && n >= 1, "bad weight table");
  if (max_len <= 0 || max_len > TMAX) max_len = TMAX;
  // active node set per pixel
  std::vector<int> sets((size_t)n * kMaxActive, -1);
  std::vector<int> counts(n, 0);
  for (int x = 0; x < n; ++x)
    for (int i = 0; i < nodes; ++i)
      if (w[(size_t)i * n + x] != 0.0) {
        if (counts[x] == kMaxActive) {
          set_error("pixel %d has more than %d nodes with nonzero weight", x, kMaxActive);
          return MM_ERR_UNSUPPORTED;
        }
        sets[(size_t)x * kMaxActive + counts[x]++] = i;
      }
  int ntiles = 0;
  for (int a = 0; a < n;) {
    int b = a + 1;
    while (b < n && counts[b] == counts[a] &&
           std::equal(&sets[(size_t)b * kMaxActive], &sets[(size_t)b * kMaxActive] + kMaxActive,
                      &sets[(size_t)a * kMaxActive]))
      ++b;
    // [a, b) shares one node set; split it evenly into pieces of <= max_len
    const int len = b - a, pieces = (len + max_len - 1) / max_len;
    for (int k = 0; k < pieces; ++k) {
      const int s = a + (int)((long long)len * k / pieces), e = a + (int)((long long)len * (k + 1) / pieces);
      if (counts[a] > 0) {  // pixels with no active node get no tile (their sum is zero)
        if (table && ntiles < capacity) {
          int* t = table + (size_t)ntiles * kTileInts;
          t[0] = s;
          t[1] = e - s;
          t[2] = counts[a];
          for (int m = 0; m < kMaxActive; ++m) t[3 + m] = sets[(size_t)a * kMaxActive + m];
          t[7] = 0;
        }
        ++ntiles;
      }
    }
    a = b;
  }
  return ntiles;
}

namespace mm {
namespace {
size_t round256(size_t b) { return (b + 255) / 256 * 256; }
size_t source_bytes(const mm_local_desc* d) { return round256((size_t)d->sx * d->sy * d->sz * sizeof(double)); }
size_t kernel_bytes(const mm_local_desc* d) {
  return round256((size_t)d->nfields * d->nodes_x * d->nodes_y * d->kx * d->ky * d->kz * sizeof(double));
}
}  // namespace
}  // namespace mm

extern "C" size_t mm_local_render_workspace_size(const mm_local_desc* d) {
  if (!d || d->sx < 1 || d->sy < 1 || d->sz < 1 || d->kx < 1 || d->ky < 1 || d->kz < 1 || d->nodes_x < 1 ||
      d->nodes_y < 1 || d->nfields < 1)
    return 0;
  return mm::source_bytes(d) + mm::kernel_bytes(d);
}

extern "C" int mm_local_render(const mm_local_desc* d, const double* source, const double* zweight, double* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  using namespace mm;
  MM_CHECK_ARG(d && source && out && d->kernels && d->wx && d->wy, "NULL pointer");
  MM_CHECK_ARG(d->sx >= 1 && d->sy >= 1 && d->sz >= 1 && d->kx >= 1 && d->ky >= 1 && d->kz >= 1 && d->nodes_x >= 1 &&
                   d->nodes_y >= 1 && d->nfields >= 1,
               "bad local-render sizes");
  MM_CHECK_ARG(!d->plane || d->kz == d->sz, "plane mode needs kernel depth == source depth (%d vs %d)", d->kz, d->sz);
  MM_CHECK_ARG(!d->plane || (d->nfields == 1 && !zweight), "plane mode renders one field with pre-weighted source");
  MM_CHECK_ARG(zweight || d->nfields == 1, "several fields need their depth weights");
  MM_CHECK_ARG(d->nodes_x <= kMaxNodes && d->nodes_y <= kMaxNodes, "at most %d field nodes per axis", kMaxNodes);
  const size_t need = mm_local_render_workspace_size(d);
  MM_CHECK_ARG(workspace && workspace_bytes >= need, "workspace too small: %zu bytes given, %zu needed",
               workspace_bytes, need);
  MM_CHECK_ARG(reinterpret_cast<uintptr_t>(workspace) % 256 == 0, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* srcT = static_cast<double*>(workspace);
  double* kt = reinterpret_cast<double*>(static_cast<char*>(workspace) + source_bytes(d));
  transpose_kernel<<<dim3(d->sx, (d->sy + 31) / 32), 256, 0, s>>>(source, d->sx, d->sy, d->sz, srcT);
  MM_CHECK_LAUNCH("local render transpose");
  const Common c = common_params(d, srcT, zweight, out);
  kernel_prep_kernel<<<1184, 256, 0, s>>>(d->kernels, d->nfields * d->nodes_x * d->nodes_y, d->kx, d->ky, d->kz,
                                          c.flip, c.plane, kt);
  MM_CHECK_LAUNCH("local render kernel layout");
  if (!d->detection) {
    MM_CHECK_ARG(d->tiles_x && d->tiles_y && d->ntiles_x >= 0 && d->ntiles_y >= 0,
                 "excitation/native render needs the mm_local_tiles tables");
    if (d->ntiles_x == 0 || d->ntiles_y == 0) return MM_OK;  // no active node anywhere
    CellP P{};
    P.c = c;
    P.kt = kt;
    P.tx = d->tiles_x;
    P.ty = d->tiles_y;
    P.ntx = d->ntiles_x;
    P.nty = d->ntiles_y;
    P.hx = TMAX + d->kx - 1;
    P.hy = cell_halo_pitch((CH + (d->ky + QY - 1) / QY) * QY);
    P.kplanes = d->plane ? TZC : 1;
    const size_t smem = ((size_t)TZC * P.hx * P.hy + (size_t)P.kplanes * PG * d->kx * d->ky) * sizeof(double);
    const size_t red = (size_t)(TZC - 1) * GROUP * QY * sizeof(double);
    const size_t bytes = std::max(smem, red);
    MM_CHECK_ARG(bytes <= 227 * 1024, "kernel %dx%d too large for the shared-memory tile (%zu bytes)", d->kx, d->ky,
                 bytes);
    MM_CHECK_CUDA(cudaFuncSetAttribute(cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                  "cudaFuncSetAttribute(local cell render)");
    const long long tiles = (long long)d->ntiles_x * d->ntiles_y;
    MM_CHECK_ARG(tiles < (1ll << 31), "too many tiles");
    const int zblocks = d->plane ? 1 : (d->sz + TZC - 1) / TZC;
    cell_kernel<<<dim3((unsigned)tiles, zblocks), CELL_THREADS, bytes, s>>>(P);
    MM_CHECK_LAUNCH("local cell render");
    return MM_OK;
  }
  GenP P{};
  P.c = c;
  P.kt = kt;
  P.detection = d->detection;
  P.kyp = (d->ky + GQY - 1) / GQY * GQY;
  P.hx = TX + d->kx - 1;
  P.hy = TY + P.kyp - 1 + GQY;  // the window reads GQY past the last tap
  const size_t smem = ((size_t)TZ * P.hx * P.hy + (size_t)d->kx * P.kyp) * sizeof(double);
  MM_CHECK_ARG(smem <= 227 * 1024, "kernel %dx%d too large for the shared-memory tile (%zu bytes)", d->kx, d->ky, smem);
  MM_CHECK_CUDA(cudaFuncSetAttribute(generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(local render)");
  const int tiles = ((d->sx + TX - 1) / TX) * ((d->sy + TY - 1) / TY);
  const int zblocks = d->plane ? 1 : (d->sz + TZ - 1) / TZ;
  generic_kernel<<<dim3(tiles, zblocks), GEN_THREADS, smem, s>>>(P);
  MM_CHECK_LAUNCH("local render");
  return MM_OK;
}
