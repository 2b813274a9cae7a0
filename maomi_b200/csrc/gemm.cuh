// One-tile-per-CTA BF16 tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM).
//
//   D[128 x NT] = A[128 x K] * B[NT x K]^T                       ("wide" part)
//              (+) sum_j A2_j[128 x K2] * B2[NB x K2]^T -> columns j*NB..   ("sub-blocks")
//
// The wide part is the spectral transform / mixing contraction of the
// surrogate (K up to 4096, NT up to 256 = 8 sites x 32 channels); the
// sub-blocks are per-site pointwise (1x1) layers that add into the same
// accumulator columns (K2 <= 64, B2 = the layer weight, shared by all sites).
//
// Warp roles inside a 128-thread CTA: warp 0 lane 0 issues the TMA loads into
// a STAGES-deep shared-memory ring, warp 1 lane 0 issues the MMAs (one thread,
// accumulator in tensor memory), and all four warps run the epilogue: warp w
// reads accumulator rows 32w..32w+31, 32 FP32 columns at a time, and hands them
// to Epi::store(row, column0, values).  Every wait is bounded; a wait that runs
// out sets bit 4 of *err and the CTA winds down (still releasing its tensor
// memory).
#pragma once

#include <cuda.h>

#include "umma.cuh"

namespace mm {
namespace gemm {

constexpr int kStages = 4;  // default ring depth (long-K spectral GEMMs)
constexpr int kBM = 128;               // rows per tile
constexpr int kBK = 64;                // K elements per stage (one 128-byte swizzle row)
constexpr int kATile = kBM * kBK * 2;  // bytes
constexpr long long kWaitLimit = 1ll << 22;

struct Tiles {
  int nk;                // wide K blocks of 64 (0: no wide part)
  int a_row_step;        // wide A row of tile (x, y) = x * a_row_step + y * a_row_ystep
  int a_row_ystep;
  int b_row_step;        // wide B row = y * b_row_step + x * b_row_xstep
  int b_row_xstep;
  int nsub;              // sub-blocks (0..8)
  int ksub;              // K16 slices of a sub-block (K2 / 16)
  long long sub_site;    // sub-block A2 row = (y * nsub + j) * sub_site + x * 128 + sub_x0
  int sub_x0;
  int ncols;             // accumulator columns the epilogue reads (multiple of 32)
  int* err;
};

template <int NT, int NB, int ST = kStages>
struct Smem {
  static constexpr int kBTile = NT * kBK * 2;
  static constexpr int kStage = kATile + kBTile;
  static constexpr size_t bytes = 1024 + (size_t)ST * kStage + 256;
};

template <int NT>
__host__ __device__ constexpr uint32_t tmem_cols() {
  return NT <= 32 ? 32u : (NT <= 64 ? 64u : (NT <= 128 ? 128u : 256u));
}

template <int NT, int NB, class Epi, int ST = kStages>
__global__ void __launch_bounds__(128, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                const __grid_constant__ CUtensorMap mapA2, const __grid_constant__ CUtensorMap mapB2, Tiles t,
                Epi epi) {
  static_assert(NT % 16 == 0 && NT >= 16 && NT <= 256, "wide N");
  static_assert(NB % 16 == 0 && NB >= 16 && NB <= 64, "sub-block N");
  using S = Smem<NT, NB, ST>;
  constexpr int kStages = ST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kStages * S::kStage);
  uint64_t* empty = full + kStages;
  uint64_t* done = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int s_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr uint32_t kCols = tmem_cols<(NT > 8 * NB ? NT : 8 * NB)>();
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      umma::mbar_init(full + s, 1);
      umma::mbar_init(empty + s, 1);
    }
    umma::mbar_init(done, 1);
    umma::fence_barrier_init();
    s_fail = 0;
    umma::prefetch_map(&mapA);
    umma::prefetch_map(&mapB);
    umma::prefetch_map(&mapA2);
    umma::prefetch_map(&mapB2);
  }
  if (warp == 0) umma::tmem_alloc(tmem_slot, kCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  const int items = t.nk + t.nsub;
  const int bx = blockIdx.x, by = blockIdx.y;
  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------- producer
    for (int i = 0; i < items; ++i) {
      const int s = i % kStages, use = i / kStages;
      if (use > 0 && !umma::mbar_wait(empty + s, (use - 1) & 1, kWaitLimit)) {
        atomicOr(t.err, 16);
        s_fail = 1;
        break;
      }
      unsigned char* a = base + s * S::kStage;
      unsigned char* b = a + kATile;
      if (i < t.nk) {
        umma::mbar_arrive_expect_tx(full + s, kATile + S::kBTile);
        umma::tma_load_2d(a, &mapA, full + s, i * kBK, bx * t.a_row_step + by * t.a_row_ystep);
        umma::tma_load_2d(b, &mapB, full + s, i * kBK, by * t.b_row_step + bx * t.b_row_xstep);
      } else {
        const int j = i - t.nk;
        const long long row = (long long)(by * t.nsub + j) * t.sub_site + (long long)bx * kBM + t.sub_x0;
        umma::mbar_arrive_expect_tx(full + s, kATile + NB * kBK * 2);
        umma::tma_load_2d(a, &mapA2, full + s, 0, (int)row);
        umma::tma_load_2d(b, &mapB2, full + s, 0, 0);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // -------------------------------------------------------- MMA issuer
    for (int i = 0; i < items; ++i) {
      const int s = i % kStages, use = i / kStages;
      if (!umma::mbar_wait(full + s, use & 1, kWaitLimit)) {
        atomicOr(t.err, 16);
        s_fail = 1;
        break;
      }
      umma::fence_after_sync();
      const unsigned char* a = base + s * S::kStage;
      const unsigned char* b = a + kATile;
      const uint64_t da = umma::sw128_desc(a), db = umma::sw128_desc(b);
      if (i < t.nk) {
#pragma unroll
        for (int k = 0; k < kBK / 16; ++k)
          umma::mma_bf16(tmem, da + 2 * k, db + 2 * k, umma::idesc_bf16(kBM, NT), (i > 0 || k > 0) ? 1u : 0u);
      } else {
        const int j = i - t.nk;
        for (int k = 0; k < t.ksub; ++k)
          umma::mma_bf16(tmem + j * NB, da + 2 * k, db + 2 * k, umma::idesc_bf16(kBM, NB),
                         (t.nk > 0 || k > 0) ? 1u : 0u);
      }
      umma::mma_commit(empty + s);  // the stage is free once these MMAs have read it
    }
    umma::mma_commit(done);
  }
  __syncwarp();
  __syncthreads();  // both roles have stopped issuing; s_fail is final
  // -------------------------------------------------------------- epilogue
  // Always wait for the MMAs that were issued (bounded) before touching or
  // releasing the accumulator; the decision is made warp-uniform because the
  // tensor-memory loads are warp-collective.
  bool ok = umma::mbar_wait(done, 0, kWaitLimit);
  if (!ok) atomicOr(t.err, 16);
  ok = __all_sync(0xffffffffu, ok && !s_fail);
  umma::fence_after_sync();
  if (ok) {
    const int row = warp * 32 + lane;
    for (int c = 0; c < t.ncols; c += 32) {
      float v[32];
      umma::tmem_ld32(tmem + (uint32_t(warp * 32) << 16) + c, v);
      epi.store(bx, by, row, c, v);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, kCols);
  }
}

}  // namespace gemm
}  // namespace mm
