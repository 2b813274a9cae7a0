// Scattering-field generation on the device: the Gaussian-process draw of
// maomi/_optical_math.py:20-67 (masked_3DGP_test) and the occupancy
// combination of maomi/optics.py:174-196 (prepare_fields with vessels).
// All three take device arrays except the vessel slab bounds (host, nz + 1).
//
//   mm_gp_spectrum  the shaped, shifted spectrum: spec = ifftshift(noise * S)
//                   with S = sqrt(sum_i prod(l_i) (kx ky kz)^2 w_i^2), the
//                   separable squared-exponential factors evaluated in
//                   float32 in the reference's order of operations;
//   (inverse 3-D DFT of spec, normalised by 1/N, between the two kernels)
//   mm_gp_finish    out = scale * Re(ifftshift(y)), the first / last z slab
//                   times its optical-thickness factor;
//   mm_vessel_combine  out = occ + raw * (1 - occ / denom) with occ the sum of
//                   the vessel volume over each field slab's z range.
#include "common.cuh"

namespace mm {
namespace {

// One thread per voxel (used when the per-plane tables below do not fit).
__global__ void gp_spectrum_kernel(int nx, int ny, int nz, const float* __restrict__ g2x, const float* __restrict__ g2y,
                                   const float* __restrict__ g2z, int K, const float* __restrict__ l2,
                                   const float* __restrict__ prod_l, const float* __restrict__ w2,
                                   const float* __restrict__ re, const float* __restrict__ im, float2* __restrict__ spec) {
  const long long total = (long long)nx * ny * nz;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int z = int(o % nz);
    const long long xy = o / nz;
    const int y = int(xy % ny), x = int(xy / ny);
    // ifftshift: output i takes input (i + n/2) mod n along every axis
    const int sx = (x + nx / 2) % nx, sy = (y + ny / 2) % ny, sz = (z + nz / 2) % nz;
    const float gx = __ldg(g2x + sx), gy = __ldg(g2y + sy), gz = __ldg(g2z + sz);
    float acc = 0.f;
    for (int k = 0; k < K; ++k) {
      const float kx = expf(-gx * __ldg(l2 + 3 * k)), ky = expf(-gy * __ldg(l2 + 3 * k + 1)),
                  kz = expf(-gz * __ldg(l2 + 3 * k + 2));
      const float k3 = kx * ky * kz;
      acc += __ldg(prod_l + k) * (k3 * k3) * __ldg(w2 + k);
    }
    const float s = sqrtf(acc);
    const long long j = ((long long)sx * ny + sy) * nz + sz;
    spec[o] = make_float2(__ldg(re + j) * s, __ldg(im + j) * s);
  }
}

// One block per x plane (ifftshifted source sx): the separable factors are
// tabulated once per block in shared memory (ky, kz for every scale; kx per
// scale), then every voxel of the plane combines them in the same order as
// gp_spectrum_kernel, so both give the same floats.
__global__ void gp_spectrum_plane_kernel(int nx, int ny, int nz, const float* __restrict__ g2x,
                                         const float* __restrict__ g2y, const float* __restrict__ g2z, int K,
                                         const float* __restrict__ l2, const float* __restrict__ prod_l,
                                         const float* __restrict__ w2, const float* __restrict__ re,
                                         const float* __restrict__ im, float2* __restrict__ spec) {
  extern __shared__ float tab[];  // kx[K], ky[K][ny], kz[K][nz]
  float* kx = tab;
  float* ky = tab + K;
  float* kz = ky + (size_t)K * ny;
  const int x = blockIdx.x, sx = (x + nx / 2) % nx;
  const float gx = __ldg(g2x + sx);
  for (int i = threadIdx.x; i < K; i += blockDim.x) kx[i] = expf(-gx * __ldg(l2 + 3 * i));
  for (int i = threadIdx.x; i < K * ny; i += blockDim.x) {
    const int k = i / ny, y = i % ny;
    ky[i] = expf(-__ldg(g2y + (y + ny / 2) % ny) * __ldg(l2 + 3 * k + 1));
  }
  for (int i = threadIdx.x; i < K * nz; i += blockDim.x) {
    const int k = i / nz, z = i % nz;
    kz[i] = expf(-__ldg(g2z + (z + nz / 2) % nz) * __ldg(l2 + 3 * k + 2));
  }
  __syncthreads();
  const int plane = ny * nz;
  float2* out = spec + (size_t)x * plane;
  const float* rs = re + (size_t)sx * plane;
  const float* is = im + (size_t)sx * plane;
  // (y, z) of o = threadIdx.x + i * blockDim.x, stepped without divisions
  const int dy = blockDim.x / nz, dz = blockDim.x % nz;
  int y = threadIdx.x / nz, z = threadIdx.x % nz;
  for (int o = threadIdx.x; o < plane; o += blockDim.x) {
    float acc = 0.f;
    for (int k = 0; k < K; ++k) {
      const float k3 = kx[k] * ky[k * ny + y] * kz[k * nz + z];
      acc += __ldg(prod_l + k) * (k3 * k3) * __ldg(w2 + k);
    }
    const float s = sqrtf(acc);
    int sy = y + ny / 2, sz = z + nz / 2;
    sy -= sy >= ny ? ny : 0;
    sz -= sz >= nz ? nz : 0;
    const int j = sy * nz + sz;
    out[o] = make_float2(__ldg(rs + j) * s, __ldg(is + j) * s);
    z += dz;
    y += dy;
    if (z >= nz) {
      z -= nz;
      ++y;
    }
  }
}

// Plane-per-block form of gp_finish_kernel (same values).
__global__ void gp_finish_plane_kernel(const float2* __restrict__ yv, int nx, int ny, int nz, float scale, float first,
                                       float last, float* __restrict__ out) {
  const int x = blockIdx.x, sx = (x + nx / 2) % nx;
  const int plane = ny * nz;
  const float2* src = yv + (size_t)sx * plane;
  float* dst = out + (size_t)x * plane;
  const int dy = blockDim.x / nz, dz = blockDim.x % nz;
  int y = threadIdx.x / nz, z = threadIdx.x % nz;
  for (int o = threadIdx.x; o < plane; o += blockDim.x) {
    int sy = y + ny / 2, sz = z + nz / 2;
    sy -= sy >= ny ? ny : 0;
    sz -= sz >= nz ? nz : 0;
    float v = scale * src[sy * nz + sz].x;
    if (z == 0) v *= first;
    if (z == nz - 1) v *= last;
    dst[o] = v;
    z += dz;
    y += dy;
    if (z >= nz) {
      z -= nz;
      ++y;
    }
  }
}

__global__ void gp_finish_kernel(const float2* __restrict__ y, int nx, int ny, int nz, float scale, float first,
                                 float last, float* __restrict__ out) {
  const long long total = (long long)nx * ny * nz;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int z = int(o % nz);
    const long long xy = o / nz;
    const int yy = int(xy % ny), x = int(xy / ny);
    const long long j = ((long long)((x + nx / 2) % nx) * ny + (yy + ny / 2) % ny) * nz + (z + nz / 2) % nz;
    float v = scale * y[j].x;
    if (z == 0) v *= first;
    if (z == nz - 1) v *= last;
    out[o] = v;
  }
}

constexpr int kMaxSlabs = 512;
struct ZBounds {
  int z[kMaxSlabs + 1];  // slab c covers vessel planes z[c] .. z[c+1]-1
};

__global__ void vessel_combine_kernel(const float* __restrict__ ves, int vy, int vz, int x0, int y0, ZBounds zb,
                                      float denom, float* __restrict__ raw, int nx, int ny, int nz) {
  const long long total = (long long)nx * ny * nz;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int c = int(o % nz);
    const long long xy = o / nz;
    const int y = int(xy % ny), x = int(xy / ny);
    const float* col = ves + ((long long)(x0 + x) * vy + (y0 + y)) * vz;
    float occ = 0.f;
    for (int z = zb.z[c]; z < zb.z[c + 1]; ++z) occ += __ldg(col + z);
    raw[o] = occ + raw[o] * (1.f - occ / denom);
  }
}

unsigned grid_of(long long total) {
  const long long b = (total + 255) / 256;
  return (unsigned)(b < 148 * 64 ? (b > 0 ? b : 1) : 148 * 64);
}

}  // namespace
}  // namespace mm

extern "C" int mm_gp_spectrum(int nx, int ny, int nz, const float* g2x, const float* g2y, const float* g2z,
                              int nscales, const float* l2, const float* prod_l, const float* w2, const float* noise_re,
                              const float* noise_im, void* spec, void* stream) {
  MM_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1 && nscales >= 1, "bad GP grid %d x %d x %d (%d scales)", nx, ny, nz,
               nscales);
  MM_CHECK_ARG(g2x && g2y && g2z && l2 && prod_l && w2 && noise_re && noise_im && spec, "NULL pointer");
  const long long total = (long long)nx * ny * nz;
  const size_t tab = sizeof(float) * (size_t)nscales * (1 + (size_t)ny + nz);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (tab <= 48 * 1024 && (long long)ny * nz < (1ll << 31)) {
    mm::gp_spectrum_plane_kernel<<<nx, 256, tab, s>>>(nx, ny, nz, g2x, g2y, g2z, nscales, l2, prod_l, w2, noise_re,
                                                      noise_im, static_cast<float2*>(spec));
  } else {
    mm::gp_spectrum_kernel<<<mm::grid_of(total), 256, 0, s>>>(nx, ny, nz, g2x, g2y, g2z, nscales, l2, prod_l, w2,
                                                              noise_re, noise_im, static_cast<float2*>(spec));
  }
  MM_CHECK_LAUNCH("GP spectrum");
  return MM_OK;
}

extern "C" int mm_gp_finish(const void* y, int nx, int ny, int nz, float scale, float first, float last, float* out,
                            void* stream) {
  MM_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1, "bad GP grid %d x %d x %d", nx, ny, nz);
  MM_CHECK_ARG(y && out, "NULL pointer");
  const long long total = (long long)nx * ny * nz;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if ((long long)ny * nz < (1ll << 31))
    mm::gp_finish_plane_kernel<<<nx, 256, 0, s>>>(static_cast<const float2*>(y), nx, ny, nz, scale, first, last, out);
  else
    mm::gp_finish_kernel<<<mm::grid_of(total), 256, 0, s>>>(static_cast<const float2*>(y), nx, ny, nz, scale, first,
                                                            last, out);
  MM_CHECK_LAUNCH("GP finish");
  return MM_OK;
}

extern "C" int mm_vessel_combine(const float* vessels, int vx, int vy, int vz, int x0, int y0, const int* zbounds,
                                 float denom, float* raw, int nx, int ny, int nz, void* stream) {
  MM_CHECK_ARG(vessels && zbounds && raw, "NULL pointer");
  MM_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1 && x0 >= 0 && y0 >= 0 && x0 + nx <= vx && y0 + ny <= vy,
               "field %d x %d at (%d, %d) outside the %d x %d vessel volume", nx, ny, x0, y0, vx, vy);
  MM_CHECK_ARG(denom > 0.f, "bad occupancy denominator");
  MM_CHECK_ARG(nz <= mm::kMaxSlabs, "at most %d slabs (got %d)", mm::kMaxSlabs, nz);
  mm::ZBounds zb{};
  for (int c = 0; c <= nz; ++c) {
    MM_CHECK_ARG(zbounds[c] >= 0 && zbounds[c] <= vz && (c == 0 || zbounds[c] >= zbounds[c - 1]),
                 "slab bounds must rise within 0..%d (entry %d is %d)", vz, c, zbounds[c]);
    zb.z[c] = zbounds[c];
  }
  const long long total = (long long)nx * ny * nz;
  mm::vessel_combine_kernel<<<mm::grid_of(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      vessels, vy, vz, x0, y0, zb, denom, raw, nx, ny, nz);
  MM_CHECK_LAUNCH("vessel occupancy");
  return MM_OK;
}
