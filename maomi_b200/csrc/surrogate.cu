// Learned surrogate of the scattered focal PSF: a Fourier-neural-operator
// (4 spectral layers of width 32, 12 x 12 retained modes, pointwise 1x1
// branch) trained and evaluated with BF16 tcgen05 GEMMs that accumulate in
// FP32.  This file holds the GEMM launchers, the CUDA-core kernels between
// them (spectral mixing, activations, loss, optimiser) and the C ABI.
#include <algorithm>

#include "common.cuh"
#include "gemm.cuh"
#include "tmap.cuh"

namespace mm {
namespace {

// ------------------------------------------------------------ launching --
template <int NT, int NB, class Epi>
int launch_gemm(const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap& a2, const CUtensorMap& b2,
                const gemm::Tiles& t, dim3 grid, const Epi& epi, cudaStream_t s) {
  auto kernel = gemm::gemm_kernel<NT, NB, Epi>;
  const size_t smem = gemm::Smem<NT, NB>::bytes;
  MM_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(gemm)");
  int per_sm = 0;
  MM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, smem), "occupancy(gemm)");
  constexpr int cols = (int)gemm::tmem_cols<(NT > 8 * NB ? NT : 8 * NB)>();
  if (per_sm < 1 || per_sm * cols > 512) {
    set_error("GEMM tile %dx%d: %d CTAs per SM would not fit tensor memory", 128, NT, per_sm);
    return MM_ERR_UNSUPPORTED;
  }
  if (grid.x == 0 || grid.y == 0) return MM_OK;
  kernel<<<grid, 128, smem, s>>>(a, b, a2, b2, t, epi);
  MM_CHECK_LAUNCH("tcgen05 GEMM");
  return MM_OK;
}

// D[m x n] (FP32, row stride ld) for the plain TN product.
struct StoreF32 {
  float* d;
  int m, n, nt;
  long long ld;
  __device__ void store(int bx, int by, int row, int c, const float (&v)[32]) const {
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
