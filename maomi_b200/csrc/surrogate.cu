// Learned surrogate of the scattered focal PSF: a Fourier-neural-operator
// (4 spectral layers of width 32, 12 x 12 retained modes, pointwise 1x1
// branch) trained and evaluated with BF16 tcgen05 GEMMs that accumulate in
// FP32.  This file holds the GEMM launchers, the CUDA-core kernels between
// them (spectral mixing, activations, loss, optimiser) and the C ABI.
#include <algorithm>

#include <cuda_bf16.h>

#include "common.cuh"
#include "gemm.cuh"
#include "tmap.cuh"

namespace mm {
namespace {

// ------------------------------------------------------------ launching --
// One persistent CTA per SM over the grid.x * grid.y tiles of `t`.
template <int NT, int NB, class Epi>
int launch_gemm(const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap& a2, const CUtensorMap& b2,
                gemm::Tiles t, dim3 grid, const Epi& epi, cudaStream_t s) {
  auto kernel = gemm::gemm_kernel<NT, NB, Epi>;
  const size_t smem = gemm::Smem<NT, NB>::bytes;
  MM_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(gemm)");
  int per_sm = 0, device = 0, sms = 0;
  MM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, gemm::kThreads, smem),
                "occupancy(gemm)");
  constexpr int cols = 2 * (int)gemm::tmem_cols<(NT > 8 * NB ? NT : 8 * NB)>();
  if (per_sm < 1 || per_sm * cols > 512) {
    set_error("GEMM tile %dx%d: %d CTAs per SM would not fit tensor memory", 128, NT, per_sm);
    return MM_ERR_UNSUPPORTED;
  }
  if (grid.x == 0 || grid.y == 0) return MM_OK;
  MM_CHECK_CUDA(cudaGetDevice(&device), "cudaGetDevice");
  MM_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  const long long ntiles = (long long)grid.x * grid.y;
  MM_CHECK_ARG(ntiles < (1ll << 31), "GEMM: %lld tiles exceed the tile index range", ntiles);
  t.grid_x = (int)grid.x;
  t.ntiles = (int)ntiles;
  const int ctas = (int)std::min<long long>(ntiles, (long long)sms * per_sm);
  kernel<<<ctas, gemm::kThreads, smem, s>>>(a, b, a2, b2, t, epi);
  MM_CHECK_LAUNCH("tcgen05 GEMM");
  return MM_OK;
}

// D[m x n] (FP32, row stride ld) for the plain TN product.
struct StoreF32 {
  float* d;
  int m, n, nt;
  long long ld;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int r = bx * gemm::kBM + row;
    if (r >= m) return;
    const int c0 = by * nt + c;
    float* dst = d + (size_t)r * ld + c0;
#pragma unroll
    for (int k = 0; k < 32; ++k)
      if (c + k < nt && c0 + k < n) dst[k] = v[k];
  }
};

template <int NT>
int gemm_tn(const void* a, const void* b, float* d, int m, int n, int k, int* err, cudaStream_t s) {
  CUtensorMap ma, mb;
  if (int rc = bf16_map(&ma, a, m, k, gemm::kBM)) return rc;
  if (int rc = bf16_map(&mb, b, n, k, NT)) return rc;
  gemm::Tiles t{};
  t.nk = (k + gemm::kBK - 1) / gemm::kBK;
  t.a_row_step = gemm::kBM;
  t.b_row_step = NT;
  t.ncols = (NT + 31) / 32 * 32;
  t.err = err;
  const dim3 grid((m + gemm::kBM - 1) / gemm::kBM, (n + NT - 1) / NT);
  return launch_gemm<NT, 32>(ma, mb, ma, mb, t, grid, StoreF32{d, m, n, NT, n}, s);
}


// ================================================================ surrogate
// Per-site grid 64 x 64 (4,096 pixels, p = 64 x + y), width 32 channels,
// 288 retained modes = 576 real rows (re, im of mode q at rows 2q, 2q+1).
constexpr int kGrid = 64, kPix = 4096, kWidth = 32, kModes = 12, kNModes = 288, kRows = 576;
constexpr int kPlanes = 9, kOut = 16, kLayers = 4, kCin = 18, kGroup = 8;  // sites per wide tile

// tanh-form GELU on the hardware tanh approximation (PTX tanh.approx.f32,
// relative error about 2^-11, below the BF16 rounding of the layer outputs).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float z) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * z, z * z, z);
  const float hz = 0.5f * z;
  return fmaf(hz, tanh_hw(u), hz);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * z, z * z, z);
  const float t = tanh_hw(u);
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * 0.7978845608028654f * (1.f + 3.f * 0.044715f * z * z);
}

// Mode q -> (kx, ky): kx in {0..11, 52..63}, ky in 0..11, q = ikx * 12 + ky.
__host__ __device__ __forceinline__ void mode_of(int q, int& kx, int& ky) {
  const int ikx = q / kModes;
  ky = q % kModes;
  kx = ikx < kModes ? ikx : kGrid - 2 * kModes + ikx;
}

// F (576 x 4096), G (4096 x 576), FT = F^T, GT = G^T in BF16.
__global__ void spectral_constants_kernel(__nv_bfloat16* F, __nv_bfloat16* G, __nv_bfloat16* FT, __nv_bfloat16* GT) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kNModes * kPix) return;
  const int q = idx / kPix, p = idx % kPix;
  int kx, ky;
  mode_of(q, kx, ky);
  const int x = p / kGrid, y = p % kGrid;
  double s, c;
  sincospi(2.0 * double((kx * x + ky * y) % kGrid) / kGrid, &s, &c);
  const double w = (ky == 0 ? 1.0 : 2.0) / kPix;
  const __nv_bfloat16 fr = __float2bfloat16_rn(float(c)), fi = __float2bfloat16_rn(float(-s));
  const __nv_bfloat16 gr = __float2bfloat16_rn(float(w * c)), gi = __float2bfloat16_rn(float(-w * s));
  F[(size_t)(2 * q) * kPix + p] = fr;
  F[(size_t)(2 * q + 1) * kPix + p] = fi;
  FT[(size_t)p * kRows + 2 * q] = fr;
  FT[(size_t)p * kRows + 2 * q + 1] = fi;
  G[(size_t)p * kRows + 2 * q] = gr;
  G[(size_t)p * kRows + 2 * q + 1] = gi;
  GT[(size_t)(2 * q) * kPix + p] = gr;
  GT[(size_t)(2 * q + 1) * kPix + p] = gi;
}

// ---------------------------------------------------------------- epilogues
// V / dVo: rows of the spectral GEMM (mode rows) x (8 sites x 32 channels),
// FP32 (S, 576, 32) into `out` and / or BF16 mode-major (288, S, 64) into
// `vb` (row (q, s) = the re row then the im row of mode q); either may be NULL.
struct EpiSpectral {
  float* out;
  __nv_bfloat16* vb;
  int sites;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int r = bx * gemm::kBM + row, s = by * kGroup + c / kWidth;
    if (r >= kRows || s >= sites) return;
    if (out) {
      float4* dst = reinterpret_cast<float4*>(out + ((size_t)s * kRows + r) * kWidth);
#pragma unroll
      for (int k = 0; k < 8; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    }
    if (vb) {
      uint4* dst = reinterpret_cast<uint4*>(vb + (((size_t)(r >> 1) * sites + s) * 2 + (r & 1)) * kWidth);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        __nv_bfloat162 a = __floats2bfloat162_rn(v[8 * k], v[8 * k + 1]), b = __floats2bfloat162_rn(v[8 * k + 2], v[8 * k + 3]);
        __nv_bfloat162 e = __floats2bfloat162_rn(v[8 * k + 4], v[8 * k + 5]), f = __floats2bfloat162_rn(v[8 * k + 6], v[8 * k + 7]);
        uint4 u;
        u.x = *reinterpret_cast<uint32_t*>(&a);
        u.y = *reinterpret_cast<uint32_t*>(&b);
        u.z = *reinterpret_cast<uint32_t*>(&e);
        u.w = *reinterpret_cast<uint32_t*>(&f);
        dst[k] = u;
      }
    }
  }
};

// Store one pixel's 32 channels of site s in both layouts (BF16); hc may be NULL.
__device__ __forceinline__ void store_both(__nv_bfloat16* hp, __nv_bfloat16* hc, int s, int pix, const float (&h)[32]) {
  uint4* dp = reinterpret_cast<uint4*>(hp + ((size_t)s * kPix + pix) * kWidth);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    __nv_bfloat162 a = __floats2bfloat162_rn(h[8 * k], h[8 * k + 1]), b = __floats2bfloat162_rn(h[8 * k + 2], h[8 * k + 3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(h[8 * k + 4], h[8 * k + 5]), d = __floats2bfloat162_rn(h[8 * k + 6], h[8 * k + 7]);
    uint4 u;
    u.x = *reinterpret_cast<uint32_t*>(&a);
    u.y = *reinterpret_cast<uint32_t*>(&b);
    u.z = *reinterpret_cast<uint32_t*>(&c);
    u.w = *reinterpret_cast<uint32_t*>(&d);
    dp[k] = u;
  }
  if (!hc) return;
  __nv_bfloat16* dc = hc + (size_t)s * kWidth * kPix + pix;
#pragma unroll
  for (int o = 0; o < kWidth; ++o) dc[(size_t)o * kPix] = __float2bfloat16_rn(h[o]);
}

// The same two stores from a whole warp whose lanes hold 32 consecutive
// pixels of site s (lane l: pixel pix0 + l).  The pixel-major rows go out
// through the warp's 1 KB shared scratch, 16 rows at a time, as 512-byte
// contiguous runs (four full-line requests per store instruction instead of
// sixteen half-filled ones); 16-byte pieces are XOR-swizzled by row pair so
// both the row writes and the linear reads are free of bank conflicts.
__device__ __forceinline__ void store_both_warp(__nv_bfloat16* hp, __nv_bfloat16* hc, int s, int pix,
                                                const float (&h)[32], unsigned char* scratch) {
  const int lane = threadIdx.x & 31, pix0 = pix - lane;
  uint4 u[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    __nv_bfloat162 a = __floats2bfloat162_rn(h[8 * k], h[8 * k + 1]), b = __floats2bfloat162_rn(h[8 * k + 2], h[8 * k + 3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(h[8 * k + 4], h[8 * k + 5]), d = __floats2bfloat162_rn(h[8 * k + 6], h[8 * k + 7]);
    u[k].x = *reinterpret_cast<uint32_t*>(&a);
    u[k].y = *reinterpret_cast<uint32_t*>(&b);
    u[k].z = *reinterpret_cast<uint32_t*>(&c);
    u[k].w = *reinterpret_cast<uint32_t*>(&d);
  }
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    if ((lane >> 4) == half) {
      const int r = lane & 15, g = (r >> 1) & 3;
#pragma unroll
      for (int k = 0; k < 4; ++k) *reinterpret_cast<uint4*>(scratch + r * 64 + ((k ^ g) << 4)) = u[k];
    }
    __syncwarp();
    uint4* dst = reinterpret_cast<uint4*>(hp + ((size_t)s * kPix + pix0 + 16 * half) * kWidth);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int m = lane + 32 * i, r = m >> 2, g = (r >> 1) & 3;
      dst[m] = *reinterpret_cast<const uint4*>(scratch + r * 64 + (((m & 3) ^ g) << 4));
    }
    __syncwarp();
  }
  if (!hc) return;
  __nv_bfloat16* dc = hc + (size_t)s * kWidth * kPix + pix;
#pragma unroll
  for (int o = 0; o < kWidth; ++o) dc[(size_t)o * kPix] = __float2bfloat16_rn(h[o]);
}

// Layer output: z = acc + bias; h = gelu(z) (or z); z kept (FP32) for the backward pass.
struct EpiLayer {
  const float* bias;
  float* z;  // (S, 4096, 32) or NULL
  __nv_bfloat16 *hp, *hc;  // hc NULL: pixel-major copy only
  int sites, act;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int pix = bx * gemm::kBM + row, s = by * kGroup + c / kWidth;
    if (s >= sites) return;
    float h[32];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float4 b = __ldg(reinterpret_cast<const float4*>(bias) + k);
      h[4 * k] = v[4 * k] + b.x;
      h[4 * k + 1] = v[4 * k + 1] + b.y;
      h[4 * k + 2] = v[4 * k + 2] + b.z;
      h[4 * k + 3] = v[4 * k + 3] + b.w;
    }
    if (z) {
      float4* dz = reinterpret_cast<float4*>(z + ((size_t)s * kPix + pix) * kWidth);
#pragma unroll
      for (int k = 0; k < 8; ++k) dz[k] = make_float4(h[4 * k], h[4 * k + 1], h[4 * k + 2], h[4 * k + 3]);
    }
    if (act) {
#pragma unroll
      for (int o = 0; o < 32; ++o) h[o] = gelu(h[o]);
    }
    store_both_warp(hp, hc, s, pix, h, scratch);
  }
};

// Backward through a layer input: dz_prev = acc * gelu'(z_prev) (or acc).
struct EpiBack {
  const float* zprev;  // (S, 4096, 32) or NULL (no activation)
  __nv_bfloat16 *dp, *dc;
  int sites;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int pix = bx * gemm::kBM + row, s = by * kGroup + c / kWidth;
    if (s >= sites) return;
    float d[32];
    if (zprev) {
      const float4* zp = reinterpret_cast<const float4*>(zprev + ((size_t)s * kPix + pix) * kWidth);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float4 z = zp[k];
        d[4 * k] = v[4 * k] * gelu_grad(z.x);
        d[4 * k + 1] = v[4 * k + 1] * gelu_grad(z.y);
        d[4 * k + 2] = v[4 * k + 2] * gelu_grad(z.z);
        d[4 * k + 3] = v[4 * k + 3] * gelu_grad(z.w);
      }
    } else {
#pragma unroll
      for (int o = 0; o < 32; ++o) d[o] = v[o];
    }
    store_both_warp(dp, dc, s, pix, d, scratch);
  }
};

// Projection: y = acc + bias + base (16 output channels per site, 2 sites per 32 columns).
struct EpiProject {
  const float* bias;  // (16)
  const float* base;  // (4096, 16)
  float* y;           // (S, 4096, 16)
  int sites;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int pix = bx * gemm::kBM + row;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int s = by * kGroup + c / kOut + half;
      if (s >= sites) continue;
      float4* dst = reinterpret_cast<float4*>(y + ((size_t)s * kPix + pix) * kOut);
      const float4* b4 = reinterpret_cast<const float4*>(base + (size_t)pix * kOut);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 b = __ldg(b4 + k);
        const int o = 16 * half + 4 * k;
        dst[k] = make_float4(v[o] + bias[4 * k] + b.x, v[o + 1] + bias[4 * k + 1] + b.y, v[o + 2] + bias[4 * k + 2] + b.z,
                             v[o + 3] + bias[4 * k + 3] + b.w);
      }
    }
  }
};

// Inference projection straight to the PSF planes: out (S, 9, 4096) =
// max(acc + bias + base, 0) for the first 9 output channels, one coalesced
// word per plane and pixel (the 16-channel y is not written).
struct EpiPlanes {
  const float* bias;  // (16)
  const float* base;  // (4096, 16)
  float* out;         // (S, 9, 4096)
  int sites;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int pix = bx * gemm::kBM + row;
    const float4* b4 = reinterpret_cast<const float4*>(base + (size_t)pix * kOut);
    float b[12];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 u = __ldg(b4 + k);
      b[4 * k] = u.x + __ldg(bias + 4 * k);
      b[4 * k + 1] = u.y + __ldg(bias + 4 * k + 1);
      b[4 * k + 2] = u.z + __ldg(bias + 4 * k + 2);
      b[4 * k + 3] = u.w + __ldg(bias + 4 * k + 3);
    }
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int s = by * kGroup + c / kOut + half;
      if (s >= sites) continue;
      float* dst = out + (size_t)s * kPlanes * kPix + pix;
#pragma unroll
      for (int k = 0; k < kPlanes; ++k) dst[(size_t)k * kPix] = fmaxf(v[16 * half + k] + b[k], 0.f);
    }
  }
};

// Weight gradient: the tile's rows are (site, a) pairs (rb rows per site), its
// columns (site', b) pairs (32 per site); only site == site' blocks belong to
// the gradient dW[a][b] (FP32, accumulated over all tiles).
struct EpiWeightGrad {
  float* dw;  // (rb, 32)
  int rb, sites;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32], unsigned char* scratch) const {
    const int per_tile = gemm::kBM / rb;
    const int j = row / rb, a = row % rb;
    if (c / kWidth != j || bx * per_tile + j >= sites) return;
#pragma unroll
    for (int b = 0; b < 32; ++b) atomicAdd(dw + a * kWidth + b, v[b]);
  }
};

// ------------------------------------------------------- spectral mixing
// The forward mixing Vo_q = V_q R_q runs on the tensor cores (mix_tc_kernel
// below).  Backward of the mixing for one mode over all sites: dV (-> dVc
// BF16) and dR, from the FP32 coefficients the training forward keeps.
__global__ void __launch_bounds__(256) mix_backward_kernel(const float* __restrict__ V, const float* __restrict__ dVo,
                                                           const float* __restrict__ Rr, const float* __restrict__ Ri,
                                                           __nv_bfloat16* __restrict__ dVc, float* __restrict__ dRr,
                                                           float* __restrict__ dRi, int sites) {
  __shared__ float rr[32][33], ri[32][33], vr[8][32], vi[8][32], gr[8][32], gi[8][32];
  const int q = blockIdx.x, t = threadIdx.x;
  for (int e = t; e < 1024; e += 256) {
    rr[e / 32][e % 32] = Rr[(size_t)q * 1024 + e];
    ri[e / 32][e % 32] = Ri[(size_t)q * 1024 + e];
  }
  const int sl = t / 32, lane = t % 32;
  // dR entries of this thread: (i, o) = (t / 8 + 32 * 0 .. ) -> 4 pairs: i = t / 8, o = (t % 8) * 4 + k
  const int di = t / 8, do0 = (t % 8) * 4;
  float ar[4] = {0.f, 0.f, 0.f, 0.f}, ai[4] = {0.f, 0.f, 0.f, 0.f};
  for (int s0 = 0; s0 < sites; s0 += 8) {
    __syncthreads();
    {
      const int s = s0 + sl;
      const bool ok = s < sites;
      vr[sl][lane] = ok ? V[((size_t)s * kRows + 2 * q) * kWidth + lane] : 0.f;
      vi[sl][lane] = ok ? V[((size_t)s * kRows + 2 * q + 1) * kWidth + lane] : 0.f;
      gr[sl][lane] = ok ? dVo[((size_t)s * kRows + 2 * q) * kWidth + lane] : 0.f;
      gi[sl][lane] = ok ? dVo[((size_t)s * kRows + 2 * q + 1) * kWidth + lane] : 0.f;
    }
    __syncthreads();
    {  // dV for (site sl, channel i = lane)
      float re = 0.f, im = 0.f;
#pragma unroll 8
      for (int o = 0; o < 32; ++o) {
        re += gr[sl][o] * rr[lane][o] + gi[sl][o] * ri[lane][o];
        im += -gr[sl][o] * ri[lane][o] + gi[sl][o] * rr[lane][o];
      }
      const int s = s0 + sl;
      if (s < sites)
        *reinterpret_cast<__nv_bfloat162*>(dVc + ((size_t)s * kWidth + lane) * kRows + 2 * q) =
            __floats2bfloat162_rn(re, im);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float a = vr[j][di], b = vi[j][di];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        ar[k] += a * gr[j][do0 + k] + b * gi[j][do0 + k];
        ai[k] += -b * gr[j][do0 + k] + a * gi[j][do0 + k];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    dRr[(size_t)q * 1024 + di * 32 + do0 + k] += ar[k];
    dRi[(size_t)q * 1024 + di * 32 + do0 + k] += ai[k];
  }
}

// ------------------------------------------------------------- loss, biases
// Per site: rel = ||y - t||^2 / ||t||^2 over planes 0..8; dy = 2 (y - t) / (S ||t||^2).
__global__ void __launch_bounds__(256) loss_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                                   __nv_bfloat16* __restrict__ dyp, __nv_bfloat16* __restrict__ dyc,
                                                   float* __restrict__ dbp, double* __restrict__ loss, int sites,
                                                   int batch) {
  const int s = blockIdx.x;
  const float* ys = y + (size_t)s * kPix * kOut;
  const float* ts = t + (size_t)s * kPix * kOut;
  __shared__ float red[2][8];
  __shared__ float s_scale;
  float num = 0.f, den = 0.f;
  for (int e = threadIdx.x; e < kPix * kOut; e += blockDim.x) {
    if (e % kOut >= kPlanes) continue;
    const float d = ys[e] - ts[e];
    num += d * d;
    den += ts[e] * ts[e];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, o);
    den += __shfl_xor_sync(0xffffffffu, den, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = num;
    red[1][threadIdx.x >> 5] = den;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.f, b = 0.f;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    b = fmaxf(b, 1e-30f);
    atomicAdd(loss, double(a) / double(b) / batch);
    s_scale = 2.f / (float(batch) * b);
  }
  __syncthreads();
  const float sc = s_scale;
  float db[kPlanes];
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) db[k] = 0.f;
  for (int p = threadIdx.x; p < kPix; p += blockDim.x) {
    float g[kOut];
#pragma unroll
    for (int k = 0; k < kOut; ++k) {
      g[k] = k < kPlanes ? sc * (ys[(size_t)p * kOut + k] - ts[(size_t)p * kOut + k]) : 0.f;
      if (k < kPlanes) db[k] += g[k];
      dyp[((size_t)s * kPix + p) * kOut + k] = __float2bfloat16_rn(g[k]);
      dyc[((size_t)s * kOut + k) * kPix + p] = __float2bfloat16_rn(g[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) {
    float v = db[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dbp + k, v);
  }
}

// db[o] += sum over pixels of dc[(s*32 + o), :]  (one warp per row).
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ dc, float* __restrict__ db, int rows) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const __nv_bfloat162* r = reinterpret_cast<const __nv_bfloat162*>(dc + (size_t)warp * kPix);
  float acc = 0.f;
  for (int e = lane; e < kPix / 2; e += 32) {
    const float2 f = __bfloat1622float2(r[e]);
    acc += f.x + f.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) atomicAdd(db + warp % kWidth, acc);
}

// ------------------------------------------------------------------- Adam
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 copies of the pointwise weights: W (o,i) and W^T for every layer, the
// lifting (o,c) and the projection (k,i) with its transpose (i,k).
struct WeightPtrs {
  const float* w[kLayers];
  __nv_bfloat16* wb[kLayers];
  __nv_bfloat16* wtb[kLayers];
  const float* wl;
  __nv_bfloat16* wlb;
  const float* wp;
  __nv_bfloat16* wpb;
  __nv_bfloat16* wptb;
};
__global__ void weights_bf16_kernel(WeightPtrs w) {
  const int e = threadIdx.x + blockIdx.x * blockDim.x;  // 0..1023
  if (e >= 1024) return;
  const int a = e / 32, b = e % 32;
#pragma unroll
  for (int l = 0; l < kLayers; ++l) {
    w.wb[l][e] = __float2bfloat16_rn(w.w[l][e]);
    w.wtb[l][b * 32 + a] = __float2bfloat16_rn(w.w[l][e]);
  }
  w.wlb[e] = __float2bfloat16_rn(w.wl[e]);
  if (e < kOut * kWidth) {
    const int k = e / 32, i = e % 32;
    w.wpb[e] = __float2bfloat16_rn(w.wp[e]);
    w.wptb[i * kOut + k] = __float2bfloat16_rn(w.wp[e]);
  }
}

// Per-mode mixing operators as tensor-core B operands (K-major BF16): for
// mode q, output n = 2 o + c (c = 0 real, 1 imaginary) and input k = 32 c' + i
// (the re then the im row of V_q), B[64 q + n][k] is the coefficient of input
// k in output n of Vo_q = V_q R_q:
//   re_o = sum_i Re(V_i) Rr_io - Im(V_i) Ri_io,  im_o = sum_i Re(V_i) Ri_io + Im(V_i) Rr_io.
__global__ void mix_operators_kernel(const float* __restrict__ Rr, const float* __restrict__ Ri,
                                     __nv_bfloat16* __restrict__ B) {
  const int q = blockIdx.x;
  for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
    const int n = e >> 6, k = e & 63, o = n >> 1, c = n & 1, ci = k >> 5, i = k & 31;
    const float rr = Rr[(size_t)q * 1024 + i * 32 + o], ri = Ri[(size_t)q * 1024 + i * 32 + o];
    const float w = c == 0 ? (ci == 0 ? rr : -ri) : (ci == 0 ? ri : rr);
    B[(size_t)q * 4096 + e] = __float2bfloat16_rn(w);
  }
}

// ------------------------------------------------------------------ inputs
// pooled[g][X][Y] = scale/16 * sum over the group's screens and the 4x4 block.
struct PoolArgs {
  const float* raw[3];  // (H, W, Z_part) float32
  int zpart[3];
  int H, W;
  int g0[17];           // screen range [g0[g], g0[g+1]) of group g (global screen index)
  float scale;
  float* pooled;        // (16, H/4, W/4)
};
__global__ void pool_inputs_kernel(PoolArgs a) {
  const int Hp = a.H / 4, Wp = a.W / 4;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 16 * Hp * Wp) return;
  const int g = idx / (Hp * Wp), r = idx % (Hp * Wp), X = r / Wp, Y = r % Wp;
  float acc = 0.f;
  for (int z = a.g0[g]; z < a.g0[g + 1]; ++z) {
    int part = 0, zl = z;
    while (part < 2 && zl >= a.zpart[part]) zl -= a.zpart[part++];
    const float* src = a.raw[part];
    const int Z = a.zpart[part];
    for (int dx = 0; dx < 4; ++dx)
      for (int dy = 0; dy < 4; ++dy) acc += src[((size_t)(4 * X + dx) * a.W + (4 * Y + dy)) * Z + zl];
  }
  a.pooled[idx] = acc * (a.scale / 16.f);
}

// Site inputs: channels 0..15 pooled screens in the site's 64 x 64 window,
// 16..17 the pixel coordinates (x - 31.5) / 32, (y - 31.5) / 32, rest 0.
__global__ void gather_inputs_kernel(const float* __restrict__ pooled, int Hp, int Wp, const int* __restrict__ offsets,
                                     int sites, __nv_bfloat16* __restrict__ xp, __nv_bfloat16* __restrict__ xc,
                                     int* __restrict__ err) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)sites * kPix) return;
  const int s = int(idx / kPix), p = int(idx % kPix), x = p / kGrid, y = p % kGrid;
  int ox = offsets[2 * s], oy = offsets[2 * s + 1];
  if (ox % 4 || oy % 4 || ox < 0 || oy < 0 || ox / 4 + kGrid > Hp || oy / 4 + kGrid > Wp) {
    if (p == 0) atomicOr(err, 2);
    ox = oy = 0;
  }
  float h[32];
#pragma unroll
  for (int g = 0; g < 16; ++g) h[g] = pooled[((size_t)g * Hp + ox / 4 + x) * Wp + oy / 4 + y];
  h[16] = (x - 31.5f) / 32.f;
  h[17] = (y - 31.5f) / 32.f;
#pragma unroll
  for (int c = kCin; c < 32; ++c) h[c] = 0.f;
  store_both(xp, xc, s, p, h);
}

// Prediction (S, 4096, 16) -> PSF planes (S, 9, 64, 64), negative values clipped.
// y (S, 4096, 16) -> planes (S, 9, 4096), negatives clipped: one thread per
// pixel reads its 64-byte output row and writes one coalesced word per plane.
constexpr int kPlanePixels = 128;
__global__ void __launch_bounds__(kPlanePixels) psf_planes_kernel(const float* __restrict__ y, float* __restrict__ out) {
  const int s = blockIdx.y, pix = blockIdx.x * kPlanePixels + threadIdx.x;
  const float4* src = reinterpret_cast<const float4*>(y + ((size_t)s * kPix + pix) * kOut);
  float v[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float4 a = __ldg(src + k);
    v[4 * k] = a.x;
    v[4 * k + 1] = a.y;
    v[4 * k + 2] = a.z;
    v[4 * k + 3] = a.w;
  }
  float* dst = out + (size_t)s * kPlanes * kPix + pix;
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) dst[(size_t)k * kPix] = fmaxf(v[k], 0.f);
}


// ------------------------------------------- spectral mixing on tensor cores
// Vo_q = V_q R_q for 8 modes q0..q0+7 of 128 sites per CTA: per mode one
// 128 x 64 x 64 BF16 MMA, A = the sites' mode-major rows (vb rows q S + s,
// [re | im] of V_q), B = the mode's operator (mixb rows 64 q ..), into TMEM
// columns 64 (q - q0) + 2 o + c.  All 8 modes' operands land in shared memory
// at once (8 x 24 KB, one mbarrier); one thread issues the 32 MMAs, then the
// four warps read, per group of 4 channels, the 8 modes' (re, im) pairs and
// write each (site, channel) row's 16 values as one 32-byte segment of Voc.
// Waits are bounded (bit 4 of *err); a failed CTA stores nothing.
constexpr int kMixTcModes = 8;
constexpr int kMixTcATile = 128 * 64 * 2, kMixTcBTile = 64 * 64 * 2;
constexpr size_t kMixTcSmem = 1024 + (size_t)kMixTcModes * (kMixTcATile + kMixTcBTile) + 64;

__global__ void __launch_bounds__(128, 1)
    mix_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                  __nv_bfloat16* __restrict__ Voc, int sites, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* a_tiles = base;
  unsigned char* b_tiles = base + kMixTcModes * kMixTcATile;
  uint64_t* full = reinterpret_cast<uint64_t*>(b_tiles + kMixTcModes * kMixTcBTile);
  uint64_t* done = full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int s_fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s0 = blockIdx.x * 128, q0 = blockIdx.y * kMixTcModes;
  if (threadIdx.x == 0) {
    umma::mbar_init(full, 1);
    umma::mbar_init(done, 1);
    umma::fence_barrier_init();
    s_fail = 0;
    umma::prefetch_map(&mapA);
    umma::prefetch_map(&mapB);
  }
  if (warp == 0) umma::tmem_alloc(tmem_slot, 512);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  if (threadIdx.x == 0) {
    umma::mbar_arrive_expect_tx(full, kMixTcModes * (kMixTcATile + kMixTcBTile));
    for (int i = 0; i < kMixTcModes; ++i) {
      umma::tma_load_2d(a_tiles + i * kMixTcATile, &mapA, full, 0, (q0 + i) * sites + s0);
      umma::tma_load_2d(b_tiles + i * kMixTcBTile, &mapB, full, 0, (q0 + i) * 64);
    }
    if (umma::mbar_wait(full, 0, gemm::kWaitLimit)) {
      umma::fence_after_sync();
      for (int i = 0; i < kMixTcModes; ++i) {
        const uint64_t da = umma::sw128_desc(a_tiles + i * kMixTcATile), db = umma::sw128_desc(b_tiles + i * kMixTcBTile);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          umma::mma_bf16(tmem + i * 64, da + 2 * k, db + 2 * k, umma::idesc_bf16(128, 64), k > 0 ? 1u : 0u);
      }
    } else {
      atomicOr(err, 16);
      s_fail = 1;
    }
    umma::mma_commit(done);  // arrives once the MMAs above (if any) have run
  }
  __syncwarp();
  bool ok = umma::mbar_wait(done, 0, gemm::kWaitLimit);
  if (!ok) atomicOr(err, 16);
  __syncthreads();  // s_fail is final
  ok = __all_sync(0xffffffffu, ok && !s_fail);
  umma::fence_after_sync();
  if (ok) {
    const int row = warp * 32 + lane, s = s0 + row;
    const uint32_t lane_addr = tmem + (uint32_t(warp * 32) << 16);
    for (int ob = 0; ob < kWidth / 4; ++ob) {  // channels 4 ob .. 4 ob + 3
      float v[kMixTcModes][8];
#pragma unroll
      for (int i = 0; i < kMixTcModes; ++i) umma::tmem_ld8(lane_addr + i * 64 + ob * 8, v[i]);
      if (s < sites) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          uint32_t w[kMixTcModes];
#pragma unroll
          for (int i = 0; i < kMixTcModes; ++i) {
            __nv_bfloat162 h = __floats2bfloat162_rn(v[i][2 * j], v[i][2 * j + 1]);
            w[i] = *reinterpret_cast<uint32_t*>(&h);
          }
          uint4* dst = reinterpret_cast<uint4*>(Voc + ((size_t)s * kWidth + 4 * ob + j) * kRows + 2 * q0);
          dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
          dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, 512);
  }
}

int mix_tc(const void* vb, const void* mixb, __nv_bfloat16* Voc, int S, int* err, cudaStream_t s) {
  CUtensorMap ma, mb;
  if (int rc = bf16_map(&ma, vb, (long long)kNModes * S, 64, 128)) return rc;
  if (int rc = bf16_map(&mb, mixb, (long long)kNModes * 64, 64, 64)) return rc;
  MM_CHECK_ARG((long long)kNModes * S < (1ll << 31), "mixing: %d sites exceed the row index range", S);
  MM_CHECK_CUDA(cudaFuncSetAttribute(mix_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMixTcSmem),
                "cudaFuncSetAttribute(mix)");
  int per_sm = 0;
  MM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mix_tc_kernel, 128, kMixTcSmem),
                "occupancy(mix)");
  if (per_sm != 1) {  // two CTAs of 512 tensor-memory columns would not fit on one SM
    set_error("tensor-core mixing: %d CTAs per SM would not fit tensor memory", per_sm);
    return MM_ERR_UNSUPPORTED;
  }
  mix_tc_kernel<<<dim3((S + 127) / 128, kNModes / kMixTcModes), 128, kMixTcSmem, s>>>(ma, mb, Voc, S, err);
  MM_CHECK_LAUNCH("tensor-core spectral mixing");
  return MM_OK;
}

// ------------------------------------------------------------ host side --
// Flat FP32 parameter layout: Wl (32x32), bl (32), per layer W (32x32), b (32),
// Rr (288x32x32), Ri (288x32x32), then Wp (16x32), bp (16).
constexpr long long kLayerStride = 1024 + 32 + 2LL * kNModes * 1024;
constexpr long long off_wl() { return 0; }
constexpr long long off_bl() { return 1024; }
constexpr long long off_w(int l) { return 1056 + l * kLayerStride; }
constexpr long long off_b(int l) { return off_w(l) + 1024; }
constexpr long long off_rr(int l) { return off_b(l) + 32; }
constexpr long long off_ri(int l) { return off_rr(l) + (long long)kNModes * 1024; }
constexpr long long off_wp() { return 1056 + kLayers * kLayerStride; }
constexpr long long off_bp() { return off_wp() + kOut * kWidth; }
constexpr long long kParams = off_bp() + kOut;

struct Maps {
  CUtensorMap a, b, a2, b2;
};

// Wide spectral GEMM: out (S, 576, 32) = A (576 x 4096) * act_c (S*32 x 4096)^T per site.
int spectral(const void* A, const void* act_c, float* out, __nv_bfloat16* vb, int S, int* err, cudaStream_t s) {
  Maps m;
  if (int rc = bf16_map(&m.a, A, kRows, kPix, gemm::kBM)) return rc;
  if (int rc = bf16_map(&m.b, act_c, (long long)S * kWidth, kPix, 256)) return rc;
  gemm::Tiles t{};
  t.nk = kPix / gemm::kBK;
  t.a_row_step = gemm::kBM;
  t.b_row_step = 256;
  t.ncols = 256;
  t.err = err;
  const dim3 grid((kRows + gemm::kBM - 1) / gemm::kBM, (S + kGroup - 1) / kGroup);
  return launch_gemm<256, 32>(m.a, m.b, m.a, m.b, t, grid, EpiSpectral{out, vb, S}, s);
}

// Fused layer GEMM: acc[pix, (site, o)] = A (4096 x 576) * coef_c (S*32 x 576)^T
//                                        + act_p (S*4096 x 32) * W (32 x 32)^T per site.
template <class Epi>
int fused(const void* A, const void* coef_c, const void* act_p, const void* W, int S, int* err, const Epi& epi,
          cudaStream_t s) {
  Maps m;
  if (int rc = bf16_map(&m.a, A, kPix, kRows, gemm::kBM)) return rc;
  if (int rc = bf16_map(&m.b, coef_c, (long long)S * kWidth, kRows, 256)) return rc;
  if (int rc = bf16_map(&m.a2, act_p, (long long)S * kPix, kWidth, gemm::kBM)) return rc;
  if (int rc = bf16_map(&m.b2, W, kWidth, kWidth, kWidth)) return rc;
  gemm::Tiles t{};
  t.nk = (kRows + gemm::kBK - 1) / gemm::kBK;
  t.a_row_step = gemm::kBM;
  t.b_row_step = 256;
  t.nsub = kGroup;
  t.ksub = kWidth / 16;
  t.sub_site = kPix;
  t.ncols = 256;
  t.err = err;
  const dim3 grid(kPix / gemm::kBM, (S + kGroup - 1) / kGroup);
  return launch_gemm<256, 32>(m.a, m.b, m.a2, m.b2, t, grid, epi, s);
}

// Pointwise-only GEMM: acc[pix, (site, n)] = act_p (S*4096 x kin) * W (NB x kin)^T per site.
template <int NB, class Epi>
int pointwise(const void* act_p, int kin, const void* W, int S, int* err, const Epi& epi, cudaStream_t s) {
  Maps m;
  if (int rc = bf16_map(&m.a2, act_p, (long long)S * kPix, kin, gemm::kBM)) return rc;
  if (int rc = bf16_map(&m.b2, W, NB, kin, NB)) return rc;
  gemm::Tiles t{};
  t.nsub = kGroup;
  t.ksub = kin / 16;
  t.sub_site = kPix;
  t.ncols = kGroup * NB;
  t.err = err;
  const dim3 grid(kPix / gemm::kBM, (S + kGroup - 1) / kGroup);
  return launch_gemm<kGroup * NB, NB>(m.a2, m.b2, m.a2, m.b2, t, grid, epi, s);
}

// Weight gradient dW[a][b] += sum_(site,pix) g[(site, a), pix] * act[(site, b), pix]
// with g channel-major (rb rows per site) and act channel-major (32 rows per site).
template <int RB>
int weight_grad(const void* g_c, const void* act_c, float* dw, int S, int* err, cudaStream_t s) {
  constexpr int per_tile = gemm::kBM / RB, NT = per_tile * kWidth;
  Maps m;
  if (int rc = bf16_map(&m.a, g_c, (long long)S * RB, kPix, gemm::kBM)) return rc;
  if (int rc = bf16_map(&m.b, act_c, (long long)S * kWidth, kPix, NT)) return rc;
  gemm::Tiles t{};
  t.nk = kPix / gemm::kBK;
  t.a_row_step = gemm::kBM;
  t.b_row_xstep = NT;
  t.ncols = NT;
  t.err = err;
  const dim3 grid((S + per_tile - 1) / per_tile, 1);
  return launch_gemm<NT, 32>(m.a, m.b, m.a, m.b, t, grid, EpiWeightGrad{dw, RB, S}, s);
}

int refresh_weights(const mm_surrogate_desc* d, cudaStream_t s) {
  WeightPtrs w{};
  for (int l = 0; l < kLayers; ++l) {
    w.w[l] = d->params + off_w(l);
    w.wb[l] = static_cast<__nv_bfloat16*>(d->wb[l]);
    w.wtb[l] = static_cast<__nv_bfloat16*>(d->wtb[l]);
  }
  w.wl = d->params + off_wl();
  w.wlb = static_cast<__nv_bfloat16*>(d->wlb);
  w.wp = d->params + off_wp();
  w.wpb = static_cast<__nv_bfloat16*>(d->wpb);
  w.wptb = static_cast<__nv_bfloat16*>(d->wptb);
  weights_bf16_kernel<<<4, 256, 0, s>>>(w);
  MM_CHECK_LAUNCH("surrogate weight copies");
  for (int l = 0; l < kLayers; ++l) {
    mix_operators_kernel<<<kNModes, 256, 0, s>>>(d->params + off_rr(l), d->params + off_ri(l),
                                                  static_cast<__nv_bfloat16*>(d->mixb[l]));
    MM_CHECK_LAUNCH("surrogate mixing operators");
  }
  return MM_OK;
}

int check_desc(const mm_surrogate_desc* d, bool backward) {
  MM_CHECK_ARG(d != nullptr, "surrogate descriptor is NULL");
  MM_CHECK_ARG(d->sites >= 1 && d->sites <= (1 << 19), "sites %d outside 1..524288", d->sites);
  MM_CHECK_ARG(d->F && d->G && d->params && d->base && d->xp && d->xc && d->voc && d->y && d->err && d->wlb &&
                   d->wpb && d->wptb,
               "surrogate descriptor has NULL buffers");
  MM_CHECK_ARG(d->vb, "surrogate descriptor has no mode-major coefficient buffer");
  for (int l = 0; l < kLayers; ++l)
    MM_CHECK_ARG(d->wb[l] && d->wtb[l] && d->v[l] && d->mixb[l], "layer %d buffers missing", l);
  for (int l = 0; l <= kLayers; ++l) MM_CHECK_ARG(d->hp[l] && d->hc[l], "activation %d buffers missing", l);
  if (backward) {
    MM_CHECK_ARG(d->FT && d->GT && d->grads && d->dyp && d->dyc && d->dzp[0] && d->dzp[1] && d->dzc[0] && d->dzc[1] &&
                     d->dvo && d->dvc,
                 "surrogate backward buffers missing");
    for (int l = 0; l < kLayers - 1; ++l) MM_CHECK_ARG(d->z[l], "pre-activation %d missing", l);
  }
  return MM_OK;
}

int finish(int check, int* err, cudaStream_t s, const char* what) {
  if (!check) return MM_OK;
  MM_CHECK_CUDA(cudaStreamSynchronize(s), what);
  int e = 0;
  MM_CHECK_CUDA(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost), "read surrogate error flag");
  if (e & 2) {
    set_error("%s: a site window is not on the 4-pixel input grid or leaves the volume", what);
    return MM_ERR_ARGUMENT;
  }
  if (e) {
    set_error("%s: a tensor-core pipeline wait timed out", what);
    return MM_ERR_TIMEOUT;
  }
  return MM_OK;
}

}  // namespace
}  // namespace mm

extern "C" int mm_gemm_bf16_tn(const void* a, const void* b, float* d, int m, int n, int k, int* err, int check,
                               void* stream) {
  using namespace mm;
  MM_CHECK_ARG(a && b && d && err, "NULL operand");
  MM_CHECK_ARG(m >= 1 && n >= 16 && k >= 16 && n % 16 == 0 && k % 16 == 0,
               "GEMM %d x %d x %d: n and k must be multiples of 16", m, n, k);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if (n % 256 == 0) rc = gemm_tn<256>(a, b, d, m, n, k, err, s);
  else if (n % 128 == 0) rc = gemm_tn<128>(a, b, d, m, n, k, err, s);
  else if (n % 64 == 0) rc = gemm_tn<64>(a, b, d, m, n, k, err, s);
  else if (n % 32 == 0) rc = gemm_tn<32>(a, b, d, m, n, k, err, s);
  else rc = gemm_tn<16>(a, b, d, m, n, k, err, s);
  if (rc != MM_OK || !check) return rc;
  MM_CHECK_CUDA(cudaStreamSynchronize(s), "GEMM");
  int e = 0;
  MM_CHECK_CUDA(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost), "read GEMM error flag");
  if (e) {
    set_error("tcgen05 GEMM: a pipeline wait timed out");
    return MM_ERR_TIMEOUT;
  }
  return MM_OK;
}


extern "C" int mm_surrogate_layout(long long* offsets, int n) {
  using namespace mm;
  MM_CHECK_ARG(offsets != nullptr && n >= 4 * mm::kLayers + 5, "layout needs %d entries", 4 * mm::kLayers + 5);
  int i = 0;
  offsets[i++] = off_wl();
  offsets[i++] = off_bl();
  for (int l = 0; l < kLayers; ++l) {
    offsets[i++] = off_w(l);
    offsets[i++] = off_b(l);
    offsets[i++] = off_rr(l);
    offsets[i++] = off_ri(l);
  }
  offsets[i++] = off_wp();
  offsets[i++] = off_bp();
  offsets[i++] = kParams;
  return MM_OK;
}

extern "C" int mm_surrogate_constants(void* F, void* G, void* FT, void* GT, void* stream) {
  using namespace mm;
  MM_CHECK_ARG(F && G && FT && GT, "NULL spectral matrix");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  spectral_constants_kernel<<<(kNModes * kPix + 255) / 256, 256, 0, s>>>(
      static_cast<__nv_bfloat16*>(F), static_cast<__nv_bfloat16*>(G), static_cast<__nv_bfloat16*>(FT),
      static_cast<__nv_bfloat16*>(GT));
  MM_CHECK_LAUNCH("surrogate spectral constants");
  return MM_OK;
}

namespace mm {
namespace {
// The forward pass; with `planes` the projection writes the clipped PSF
// planes (S, 9, 4096) instead of the prediction d->y.
int forward_pass(const mm_surrogate_desc* d, float* planes, cudaStream_t s) {
  const int S = d->sites;
  if (int rc = refresh_weights(d, s)) return rc;
  auto bf = [](const void* p) { return static_cast<__nv_bfloat16*>(const_cast<void*>(p)); };
  // lifting (no activation)
  if (int rc = pointwise<32>(d->xp, kWidth, d->wlb, S, d->err,
                             EpiLayer{d->params + off_bl(), nullptr, bf(d->hp[0]), bf(d->hc[0]), S, 0}, s))
    return rc;
  // without pre-activation buffers (inference) the FP32 spectral
  // coefficients and the last layer's channel-major copy, read only by the
  // backward pass, are skipped
  const bool train = d->z[0] != nullptr;
  for (int l = 0; l < kLayers; ++l) {
    if (int rc = spectral(d->F, d->hc[l], train ? d->v[l] : nullptr, bf(d->vb), S, d->err, s)) return rc;
    if (int rc = mix_tc(d->vb, d->mixb[l], bf(d->voc), S, d->err, s)) return rc;
    const EpiLayer epi{d->params + off_b(l), train ? d->z[l] : nullptr, bf(d->hp[l + 1]),
                       (train || l < kLayers - 1) ? bf(d->hc[l + 1]) : nullptr, S, l < kLayers - 1};
    if (int rc = fused(d->G, d->voc, d->hp[l], d->wb[l], S, d->err, epi, s)) return rc;
  }
  if (planes) return pointwise<16>(d->hp[kLayers], kWidth, d->wpb, S, d->err,
                                  EpiPlanes{d->params + off_bp(), d->base, planes, S}, s);
  return pointwise<16>(d->hp[kLayers], kWidth, d->wpb, S, d->err, EpiProject{d->params + off_bp(), d->base, d->y, S},
                       s);
}
}  // namespace
}  // namespace mm

extern "C" int mm_surrogate_forward(const mm_surrogate_desc* d, int check, void* stream) {
  using namespace mm;
  if (int rc = check_desc(d, false)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = forward_pass(d, nullptr, s)) return rc;
  return finish(check, d->err, s, "surrogate forward");
}

extern "C" int mm_surrogate_predict(const mm_surrogate_desc* d, float* planes, int check, void* stream) {
  using namespace mm;
  if (int rc = check_desc(d, false)) return rc;
  MM_CHECK_ARG(planes != nullptr, "NULL PSF planes");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = forward_pass(d, planes, s)) return rc;
  return finish(check, d->err, s, "surrogate predict");
}

extern "C" int mm_surrogate_backward(const mm_surrogate_desc* d, const float* target, double* loss, int check,
                                     void* stream) {
  using namespace mm;
  if (int rc = check_desc(d, true)) return rc;
  MM_CHECK_ARG(target && loss, "NULL target or loss");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int S = d->sites;
  auto bf = [](const void* p) { return static_cast<__nv_bfloat16*>(const_cast<void*>(p)); };
  float* g = d->grads;
  MM_CHECK_CUDA(cudaMemsetAsync(g, 0, sizeof(float) * kParams, s), "zero gradients");
  MM_CHECK_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), s), "zero loss");
  loss_kernel<<<S, 256, 0, s>>>(d->y, target, bf(d->dyp), bf(d->dyc), g + off_bp(), loss, S, S);
  MM_CHECK_LAUNCH("surrogate loss");
  if (int rc = weight_grad<16>(d->dyc, d->hc[kLayers], g + off_wp(), S, d->err, s)) return rc;
  int cur = 0;
  if (int rc = pointwise<32>(d->dyp, kOut, d->wptb, S, d->err,
                             EpiBack{nullptr, bf(d->dzp[cur]), bf(d->dzc[cur]), S}, s))
    return rc;
  const int rows = S * kWidth;
  for (int l = kLayers - 1; l >= 0; --l) {
    bias_grad_kernel<<<(rows * 32 + 255) / 256, 256, 0, s>>>(bf(d->dzc[cur]), g + off_b(l), rows);
    MM_CHECK_LAUNCH("surrogate bias gradient");
    if (int rc = weight_grad<32>(d->dzc[cur], d->hc[l], g + off_w(l), S, d->err, s)) return rc;
    if (int rc = spectral(d->GT, d->dzc[cur], d->dvo, nullptr, S, d->err, s)) return rc;
    mix_backward_kernel<<<kNModes, 256, 0, s>>>(d->v[l], d->dvo, d->params + off_rr(l), d->params + off_ri(l),
                                               bf(d->dvc), g + off_rr(l), g + off_ri(l), S);
    MM_CHECK_LAUNCH("surrogate mixing backward");
    const EpiBack epi{l > 0 ? d->z[l - 1] : nullptr, bf(d->dzp[1 - cur]), bf(d->dzc[1 - cur]), S};
    if (int rc = fused(d->FT, d->dvc, d->dzp[cur], d->wtb[l], S, d->err, epi, s)) return rc;
    cur = 1 - cur;
  }
  bias_grad_kernel<<<(rows * 32 + 255) / 256, 256, 0, s>>>(bf(d->dzc[cur]), g + off_bl(), rows);
  MM_CHECK_LAUNCH("surrogate bias gradient");
  if (int rc = weight_grad<32>(d->dzc[cur], d->xc, g + off_wl(), S, d->err, s)) return rc;
  return finish(check, d->err, s, "surrogate backward");
}

extern "C" int mm_surrogate_adam(float* params, const float* grads, float* m, float* v, long long n, float lr,
                                 float beta1, float beta2, float eps, int step, void* stream) {
  using namespace mm;
  MM_CHECK_ARG(params && grads && m && v && n >= 1 && step >= 1, "bad Adam arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  adam_kernel<<<592, 256, 0, s>>>(params, grads, m, v, n, lr, beta1, beta2, eps, c1, c2);
  MM_CHECK_LAUNCH("surrogate Adam step");
  return MM_OK;
}

extern "C" int mm_surrogate_inputs(const float* const* raw, const int* zpart, int h, int w, const int* groups,
                                   float scale, float* pooled, const int* offsets, int sites, void* xp, void* xc,
                                   int* err, int check, void* stream) {
  using namespace mm;
  MM_CHECK_ARG(raw && zpart && groups && pooled && err, "NULL surrogate input buffer");
  MM_CHECK_ARG(sites == 0 || (offsets && xp && xc), "NULL site buffers for %d sites", sites);
  MM_CHECK_ARG(h % 4 == 0 && w % 4 == 0 && h >= 4 * kGrid && w >= 4 * kGrid, "volume %d x %d", h, w);
  PoolArgs a{};
  for (int i = 0; i < 3; ++i) {
    MM_CHECK_ARG(raw[i] && zpart[i] >= 1, "raw field %d", i);
    a.raw[i] = raw[i];
    a.zpart[i] = zpart[i];
  }
  const int total = zpart[0] + zpart[1] + zpart[2];
  for (int g = 0; g <= 16; ++g) {
    MM_CHECK_ARG(groups[g] >= 0 && groups[g] <= total && (g == 0 || groups[g] >= groups[g - 1]),
                 "screen groups must be increasing within 0..%d", total);
    a.g0[g] = groups[g];
  }
  a.H = h;
  a.W = w;
  a.scale = scale;
  a.pooled = pooled;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = 16 * (h / 4) * (w / 4);
  pool_inputs_kernel<<<(n + 255) / 256, 256, 0, s>>>(a);
  MM_CHECK_LAUNCH("surrogate input pooling");
  if (sites > 0) {
    const long long m = (long long)sites * kPix;
    gather_inputs_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(
        pooled, h / 4, w / 4, offsets, sites, static_cast<__nv_bfloat16*>(xp), static_cast<__nv_bfloat16*>(xc), err);
    MM_CHECK_LAUNCH("surrogate input gather");
  }
  return finish(check, err, s, "surrogate inputs");
}

extern "C" int mm_surrogate_planes(const float* y, float* out, int sites, void* stream) {
  using namespace mm;
  MM_CHECK_ARG(y && out && sites >= 1, "bad surrogate plane arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  MM_CHECK_ARG(sites <= 65535, "surrogate planes: %d sites exceed one launch (65,535)", sites);
  psf_planes_kernel<<<dim3(kPix / kPlanePixels, sites), kPlanePixels, 0, s>>>(y, out);
  MM_CHECK_LAUNCH("surrogate PSF planes");
  return MM_OK;
}
