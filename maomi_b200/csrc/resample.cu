// Intensity resampling and the site reductions of the optical stage.
#include <algorithm>

#include "common.cuh"

namespace mm {
namespace {

int grid_for(long long total, int block = 256) {
  long long g = (total + block - 1) / block;
  return int(std::min<long long>(std::max<long long>(g, 1), 148LL * 64));
}

// out[b,x,y,z] = scale*axial[z]*sum_i wx[x,i] sum_j wy[y,j] |field[b,z,ix,iy]|^(2*order)
__global__ void resample_power_kernel(const float2* __restrict__ field, const int* __restrict__ ix,
                                      const float* __restrict__ wx, const int* __restrict__ iy,
                                      const float* __restrict__ wy, const float* __restrict__ axial,
                                      float* __restrict__ out, int B, int Z, int H, int W, int X, int Y, int KX,
                                      int KY, int order, float scale) {
  const long long total = (long long)B * X * Y * Z;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int z = int(t % Z), y = int((t / Z) % Y), x = int((t / ((long long)Z * Y)) % X);
    const long long b = t / ((long long)Z * Y * X);
    const float2* plane = field + ((size_t)b * Z + z) * H * W;
    float value = 0.f;
    for (int i = 0; i < KX; ++i) {
      const float a = __ldg(wx + x * KX + i);
      if (a == 0.f) continue;
      const int sx = __ldg(ix + x * KX + i);
      float row = 0.f;
      for (int j = 0; j < KY; ++j) {
        const float w = __ldg(wy + y * KY + j);
        if (w == 0.f) continue;
        row += w * photon_power(__ldg(plane + (size_t)sx * W + __ldg(iy + y * KY + j)), order);
      }
      value += a * row;
    }
    out[t] = scale * value * __ldg(axial + z);
  }
}

// One CTA per (site, output row x): psf[p,x,:,:] (Y*Z values, z fastest).
// Inputs are read plane by plane with y fastest (coalesced rows of the focal
// crops), staged in shared memory and written out with z fastest.
__global__ void focal_finalize_kernel(const float* __restrict__ focal, const int* __restrict__ ix,
                                      const float* __restrict__ wx, int KX, const int* __restrict__ iy,
                                      const float* __restrict__ wy, int KY, const float* __restrict__ axial,
                                      float scale, int Z, int H, int W, int X, int Y, float* __restrict__ psf,
                                      double* __restrict__ energies) {
  extern __shared__ float tile[];  // Y x (Z + 1)
  __shared__ double red[32];
  const int p = blockIdx.y, x = blockIdx.x;
  const float* src = focal + (size_t)p * Z * H * W;
  double acc = 0.0;
  for (int o = threadIdx.x; o < Y * Z; o += blockDim.x) {
    const int z = o / Y, y = o % Y;
    const float* plane = src + (size_t)z * H * W;
    float value = 0.f;
    for (int i = 0; i < KX; ++i) {
      const float a = __ldg(wx + x * KX + i);
      if (a == 0.f) continue;
      const int sx = __ldg(ix + x * KX + i);
      float row = 0.f;
      for (int j = 0; j < KY; ++j) {
        const float w = __ldg(wy + y * KY + j);
        if (w == 0.f) continue;
        row += w * __ldg(plane + (size_t)sx * W + __ldg(iy + y * KY + j));
      }
      value += a * row;
    }
    const float v = scale * value * __ldg(axial + z);
    tile[y * (Z + 1) + z] = v;
    acc += v;
  }
  __syncthreads();
  if (psf) {
    float* dst = psf + ((size_t)p * X + x) * Y * Z;
    for (int o = threadIdx.x; o < Y * Z; o += blockDim.x) dst[o] = tile[(o / Z) * (Z + 1) + o % Z];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
    atomicAdd(energies + p, s);
  }
}

// Identity resample (ss = 1: X = H, Y = W): a tiled transpose of the focal
// crops (P, Z, X, Y) -> psf (P, X, Y, Z) with the scale and axial weights.
// grid (ceil(X / kFocalRows), P); both the reads (rows of a plane, y fastest)
// and the writes (z fastest) are contiguous runs.  Same value expression as
// focal_finalize_kernel (scale * v * axial[z]).
constexpr int kFocalRows = 8;

__global__ void focal_transpose_kernel(const float* __restrict__ focal, const float* __restrict__ axial, float scale,
                                       int Z, int X, int Y, float* __restrict__ psf, double* __restrict__ energies) {
  extern __shared__ __align__(16) float tile[];  // (rows * Y) x Z: the block's output run, in order
  __shared__ double red[32];
  const int p = blockIdx.y, x0 = blockIdx.x * kFocalRows;
  const int rows = min(kFocalRows, X - x0);
  const int ry = rows * Y;
  const float* src = focal + (size_t)p * Z * X * Y + (size_t)x0 * Y;
  const int tid = threadIdx.x, nt = blockDim.x;
  double acc = 0.0;
  // planes outer, kFocalBatch of them in flight per thread: every load of a
  // batch is issued before any is used, and no index needs a division
  constexpr int kFocalBatch = 16;
  for (int o = tid; o < ry; o += nt) {
    for (int z0 = 0; z0 < Z; z0 += kFocalBatch) {
      float v[kFocalBatch];
#pragma unroll
      for (int u = 0; u < kFocalBatch; ++u)
        v[u] = z0 + u < Z ? __ldg(src + (size_t)(z0 + u) * X * Y + o) : 0.f;
#pragma unroll
      for (int u = 0; u < kFocalBatch; ++u) {
        if (z0 + u >= Z) break;
        const float w = scale * v[u] * __ldg(axial + z0 + u);
        tile[o * Z + z0 + u] = w;
        acc += w;
      }
    }
  }
  __syncthreads();
  if (psf) {
    // the tile is the block's whole output run (pixels x planes, z fastest):
    // a linear copy, 16 bytes per thread and step when aligned
    float* dst = psf + ((size_t)p * X + x0) * Y * Z;
    const int total = ry * Z;
    if ((total & 3) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
      const float4* t4 = reinterpret_cast<const float4*>(tile);
      float4* d4 = reinterpret_cast<float4*>(dst);
      for (int i = tid; i < (total >> 2); i += nt) d4[i] = t4[i];
    } else {
      for (int i = tid; i < total; i += nt) dst[i] = tile[i];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < int(nt >> 5); ++w) s += red[w];
    atomicAdd(energies + p, s);
  }
}

// Partial site sums of psf and |psf|: grid (ceil(E/256), chunks).
__global__ void site_sums_kernel(const float* __restrict__ psf, long long E, int P, int chunk,
                                 double* __restrict__ sum, double* __restrict__ abs_sum) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= E) return;
  const int p0 = blockIdx.y * chunk, p1 = min(P, p0 + chunk);
  double s = 0.0, a = 0.0;
  int p = p0;
  for (; p + 8 <= p1; p += 8) {  // eight independent loads in flight
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = __ldg(psf + (size_t)(p + u) * E + e);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      s += (double)v[u];
      a += fabs((double)v[u]);
    }
  }
  for (; p < p1; ++p) {
    const double v = __ldg(psf + (size_t)p * E + e);
    s += v;
    a += fabs(v);
  }
  atomicAdd(sum + e, s);
  atomicAdd(abs_sum + e, a);
}

// sum over images (float) into a float64 plane
__global__ void image_sum_kernel(const float* __restrict__ img, int S, int HW, double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < HW; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < S; ++i) s += __ldg(img + (size_t)i * HW + e);
    out[e] = s;
  }
}

// out[x,y] = scale * sum_h sum_w rx[x,h] ry[y,w] in[h,w]  (dense, float64)
__global__ void resample_plane_kernel(const double* __restrict__ in, int H, int W, const float* __restrict__ rx,
                                      const float* __restrict__ ry, int X, int Y, double scale, double* __restrict__ out) {
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < X * Y; o += gridDim.x * blockDim.x) {
    const int x = o / Y, y = o % Y;
    double acc = 0.0;
    for (int h = 0; h < H; ++h) {
      const double a = __ldg(rx + (size_t)x * H + h);
      if (a == 0.0) continue;
      double row = 0.0;
      for (int w = 0; w < W; ++w) {
        const double b = __ldg(ry + (size_t)y * W + w);
        if (b != 0.0) row += b * in[(size_t)h * W + w];
      }
      acc += a * row;
    }
    out[o] = scale * acc;
  }
}

// per-image sparse resample (float): out[s,x,y] = scale * sum wx*wy*in[s,ix,iy]
__global__ void resample_images_kernel(const float* __restrict__ in, int S, int H, int W, const int* __restrict__ ix,
                                       const float* __restrict__ wx, int KX, const int* __restrict__ iy,
                                       const float* __restrict__ wy, int KY, int X, int Y, float scale,
                                       float* __restrict__ out) {
  const long long total = (long long)S * X * Y;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int y = int(t % Y), x = int((t / Y) % X);
    const long long s = t / ((long long)X * Y);
    const float* plane = in + (size_t)s * H * W;
    float value = 0.f;
    for (int i = 0; i < KX; ++i) {
      const float a = __ldg(wx + x * KX + i);
      if (a == 0.f) continue;
      const int sx = __ldg(ix + x * KX + i);
      float row = 0.f;
      for (int j = 0; j < KY; ++j) {
        const float w = __ldg(wy + y * KY + j);
        if (w == 0.f) continue;
        row += w * __ldg(plane + (size_t)sx * W + __ldg(iy + y * KY + j));
      }
      value += a * row;
    }
    out[t] = scale * value;
  }
}

}  // namespace
}  // namespace mm

using namespace mm;

extern "C" int mm_resample_power(const void* field, const int32_t* ix, const float* wx, const int32_t* iy,
                                 const float* wy, const float* axial, float* out, int B, int Z, int H, int W, int X,
                                 int Y, int KX, int KY, int order, float scale, void* stream) {
  MM_CHECK_ARG(field && ix && wx && iy && wy && axial && out, "NULL pointer");
  MM_CHECK_ARG(order >= 1 && order <= 3, "Photon order must be 1, 2 or 3");
  MM_CHECK_ARG(B >= 0 && Z >= 1 && H >= 1 && W >= 1 && X >= 1 && Y >= 1 && KX >= 1 && KY >= 1, "bad resample sizes");
  if (B == 0) return MM_OK;
  const long long total = (long long)B * X * Y * Z;
  resample_power_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(field), ix, wx, iy, wy, axial, out, B, Z, H, W, X, Y, KX, KY, order, scale);
  MM_CHECK_LAUNCH("resample_power");
  return MM_OK;
}

extern "C" int mm_focal_finalize(const float* focal, const int32_t* ix, const float* wx, int KX, const int32_t* iy,
                                 const float* wy, int KY, const float* axial, float scale, int P, int Z, int H, int W,
                                 int X, int Y, float* psf, double* energies, double* psf_sum, double* psf_abs_sum,
                                 void* stream) {
  const bool identity = !ix && !wx && !iy && !wy;
  MM_CHECK_ARG(focal && axial && energies && (identity || (ix && wx && iy && wy)), "NULL pointer");
  MM_CHECK_ARG(P >= 1 && Z >= 1 && H >= 1 && W >= 1 && X >= 1 && Y >= 1 && P <= 65535, "bad focal sizes");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  MM_CHECK_CUDA(cudaMemsetAsync(energies, 0, sizeof(double) * P, s), "zero energies");
  if (identity) {
    MM_CHECK_ARG(X == H && Y == W, "identity focal resample needs X == H and Y == W (got %d x %d from %d x %d)", X, Y,
                 H, W);
    const size_t tt = sizeof(float) * (size_t)kFocalRows * Y * Z;
    MM_CHECK_ARG(tt <= 200 * 1024, "focal crop %d x %d planes too large for one tile", Y, Z);
    if (tt > 48 * 1024)
      MM_CHECK_CUDA(cudaFuncSetAttribute(focal_transpose_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tt),
                    "cudaFuncSetAttribute(focal transpose)");
    const int threads = std::min(512, (std::min(kFocalRows, X) * Y + 31) / 32 * 32);  // one output run each
    focal_transpose_kernel<<<dim3((X + kFocalRows - 1) / kFocalRows, P), threads, tt, s>>>(focal, axial, scale, Z, X,
                                                                                              Y, psf, energies);
    MM_CHECK_LAUNCH("focal transpose");
  }
  const size_t tile = sizeof(float) * (size_t)Y * (Z + 1);
  MM_CHECK_ARG(tile <= 200 * 1024, "focal crop %d x %d planes too large for one tile", Y, Z);
  if (!identity) {
    if (tile > 48 * 1024)
      MM_CHECK_CUDA(cudaFuncSetAttribute(focal_finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile),
                    "cudaFuncSetAttribute(focal finalize)");
    focal_finalize_kernel<<<dim3(X, P), 256, tile, s>>>(focal, ix, wx, KX, iy, wy, KY, axial, scale, Z, H, W, X, Y,
                                                        psf, energies);
    MM_CHECK_LAUNCH("focal finalize");
  }
  if (psf_sum && psf_abs_sum && psf) {
    const long long E = (long long)X * Y * Z;
    MM_CHECK_CUDA(cudaMemsetAsync(psf_sum, 0, sizeof(double) * E, s), "zero psf sum");
    MM_CHECK_CUDA(cudaMemsetAsync(psf_abs_sum, 0, sizeof(double) * E, s), "zero psf abs sum");
    const int chunk = 128;
    dim3 grid((unsigned)((E + 255) / 256), (unsigned)((P + chunk - 1) / chunk));
    site_sums_kernel<<<grid, 256, 0, s>>>(psf, E, P, chunk, psf_sum, psf_abs_sum);
    MM_CHECK_LAUNCH("site sums");
  }
  return MM_OK;
}

extern "C" int mm_tail_finalize(const float* images, int S, int H, int W, const float* rx, const float* ry, int X, int Y,
                                double scale, double* out, double* scratch, void* stream) {
  MM_CHECK_ARG(images && rx && ry && out && scratch, "NULL pointer");
  MM_CHECK_ARG(S >= 1 && H >= 1 && W >= 1 && X >= 1 && Y >= 1, "bad tail sizes");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  image_sum_kernel<<<grid_for((long long)H * W), 256, 0, s>>>(images, S, H * W, scratch);
  MM_CHECK_LAUNCH("tail image sum");
  resample_plane_kernel<<<grid_for((long long)X * Y), 256, 0, s>>>(scratch, H, W, rx, ry, X, Y, scale, out);
  MM_CHECK_LAUNCH("tail resample");
  return MM_OK;
}

extern "C" int mm_resample_images(const float* in, int S, int H, int W, const int32_t* ix, const float* wx, int KX,
                                  const int32_t* iy, const float* wy, int KY, int X, int Y, float scale, float* out,
                                  void* stream) {
  MM_CHECK_ARG(in && ix && wx && iy && wy && out, "NULL pointer");
  MM_CHECK_ARG(S >= 0 && H >= 1 && W >= 1 && X >= 1 && Y >= 1 && KX >= 1 && KY >= 1, "bad image resample sizes");
  if (S == 0) return MM_OK;
  resample_images_kernel<<<grid_for((long long)S * X * Y), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      in, S, H, W, ix, wx, KX, iy, wy, KY, X, Y, scale, out);
  MM_CHECK_LAUNCH("resample images");
  return MM_OK;
}
