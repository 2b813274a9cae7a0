// Persistent BF16 tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM).
//
// Per 128 x NT output tile (bx, by):
//   D[128 x NT] = A[128 x K] * B[NT x K]^T                       ("wide" part)
//              (+) sum_j A2_j[128 x K2] * B2[NB x K2]^T -> columns j*NB..   ("sub-blocks")
//
// The wide part is the spectral transform / mixing contraction of the
// surrogate (K up to 4096, NT up to 256 = 8 sites x 32 channels); the
// sub-blocks are per-site pointwise (1x1) layers that add into the same
// accumulator columns (K2 <= 64, B2 = the layer weight, shared by all sites).
//
// One CTA per SM walks the tiles tile = blockIdx.x + k * gridDim.x (bx
// fastest, so the CTAs in flight share the B tiles of a few `by` in L2).
// Warp roles: warp 0 lane 0 issues the TMA loads into a shared-memory ring
// (4 to 8 stages) that runs on across tiles, warp 1 lane 0 issues the MMAs
// into one of two tensor-memory accumulators (tile k uses accumulator k & 1),
// and EW epilogue warps drain the other accumulator meanwhile: epilogue warp w
// reads TMEM lanes 32 (w % 4) .. + 31 (the lane quarter its warp index
// allows), every (EW / 4)-th group of 32 FP32 columns, and hands them to
// Epi::store(bx, by, row, column0, values, scratch) with a 1 KB shared
// scratch of its own (the calls of a warp are warp-uniform).  The accumulator handshake is a
// pair of mbarriers per buffer: `acc_full` (one tcgen05.commit after the
// tile's last MMA) and `acc_empty` (one arrival per epilogue warp after its
// last tensor-memory load).  Every wait is bounded; a wait that runs out sets
// bit 4 of *err and the CTA winds down, still waiting (bounded) for its MMAs
// and releasing its tensor memory.
#pragma once

#include <cuda.h>

#include "umma.cuh"

namespace mm {
namespace gemm {

constexpr int kBM = 128;               // rows per tile
constexpr int kBK = 64;                // K elements per stage (one 128-byte swizzle row)
constexpr int kATile = kBM * kBK * 2;  // bytes
constexpr int kEpiWarps = 16;          // epilogue warps (four per tensor-memory lane quarter)
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr long long kWaitLimit = 1ll << 22;
constexpr int kRingBytes = 196 * 1024;  // shared-memory ring budget of the one CTA per SM

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
  int grid_x;            // tiles along x; tile t = (t % grid_x, t / grid_x)
  int ntiles;            // grid_x * tiles along y
  int* err;
};

template <int NT>
__host__ __device__ constexpr int ring_stages() {
  return (kRingBytes / (kATile + NT * kBK * 2)) < 8 ? kRingBytes / (kATile + NT * kBK * 2) : 8;
}

// Shared memory: the ring, then the sub-block weight B2 (loaded once per
// CTA: every sub-block of every tile multiplies by the same layer weight),
// then the mbarriers.  A sub-block item packs the A2 rows of kSites sites
// into one ring stage (one 16 KB box each), so a tile's fresh DRAM rows
// arrive in a few large steps instead of one stage per site.
template <int NT, int NB>
struct Smem {
  static constexpr int kStages = ring_stages<NT>();
  static constexpr int kBTile = NT * kBK * 2;
  static constexpr int kStage = kATile + kBTile;
  static constexpr int kSites = kStage / kATile;
  static constexpr int kB2 = 64 * kBK * 2;  // room for NB <= 64 rows
  static constexpr int kScratch = 1024;     // per epilogue warp
  static constexpr size_t bytes = 1024 + (size_t)kStages * kStage + kB2 + kEpiWarps * kScratch + 256;
  static_assert(kStages >= 2, "ring");
  static_assert((2 * kStages + 6) * 8 + 4 <= 256, "barrier area");
  static_assert(kStage % 1024 == 0, "stages keep the 1024-byte swizzle-atom alignment");
};

// tensor-memory columns of ONE accumulator (the kernel holds two)
template <int NT>
__host__ __device__ constexpr uint32_t tmem_cols() {
  return NT <= 32 ? 32u : (NT <= 64 ? 64u : (NT <= 128 ? 128u : 256u));
}

// Item order within a tile.  When the sub-blocks cover every accumulator
// column (nsub * NB >= NT) they come first: their fresh DRAM rows are then
// requested together, while the MMAs still run on the previous tile's wide
// blocks from L2, and each sub-block's first K slice starts its own columns.
// Otherwise the wide blocks come first (block 0 starts all NT columns).
__device__ __forceinline__ void item_of(const Tiles& t, int nsub_items, bool subs_first, int i, bool& wide,
                                        int& idx) {
  if (subs_first) {
    wide = i >= nsub_items;
    idx = wide ? i - nsub_items : i;
  } else {
    wide = i < t.nk;
    idx = wide ? i : i - t.nk;
  }
}
__device__ __forceinline__ long long sub_row(const Tiles& t, int bx, int by, int j) {
  return (long long)(by * t.nsub + j) * t.sub_site + (long long)bx * kBM + t.sub_x0;
}

template <int NT, int NB, class Epi>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                const __grid_constant__ CUtensorMap mapA2, const __grid_constant__ CUtensorMap mapB2, Tiles t,
                Epi epi) {
  static_assert(NT % 16 == 0 && NT >= 16 && NT <= 256, "wide N");
  static_assert(NB % 16 == 0 && NB >= 16 && NB <= 64, "sub-block N");
  static_assert(kEpiWarps % 4 == 0, "epilogue warps cover whole lane quarters");
  using S = Smem<NT, NB>;
  constexpr int kStages = S::kStages;
  constexpr uint32_t kCols = tmem_cols<(NT > 8 * NB ? NT : 8 * NB)>();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* b2_tile = base + kStages * S::kStage;
  unsigned char* scratch_all = b2_tile + S::kB2;
  uint64_t* full = reinterpret_cast<uint64_t*>(scratch_all + kEpiWarps * S::kScratch);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* done = acc_empty + 2;
  uint64_t* b2_full = done + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(b2_full + 1);
  __shared__ int s_fail;
  volatile int* fail = &s_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      umma::mbar_init(full + s, 1);
      umma::mbar_init(empty + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      umma::mbar_init(acc_full + b, 1);
      umma::mbar_init(acc_empty + b, kEpiWarps);
    }
    umma::mbar_init(done, 1);
    umma::mbar_init(b2_full, 1);
    umma::fence_barrier_init();
    s_fail = 0;
    umma::prefetch_map(&mapA);
    umma::prefetch_map(&mapB);
    umma::prefetch_map(&mapA2);
    umma::prefetch_map(&mapB2);
  }
  if (warp == 0) umma::tmem_alloc(tmem_slot, 2 * kCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  const int nsub_items = (t.nsub + S::kSites - 1) / S::kSites;
  const int items = t.nk + nsub_items;
  const bool subs_first = t.nsub * NB >= NT;
  if (warp == 0) {
    if (lane == 0) {
      // -------------------------------------------------------- producer
      if (t.nsub > 0) {
        umma::mbar_arrive_expect_tx(b2_full, NB * kBK * 2);
        umma::tma_load_2d(b2_tile, &mapB2, b2_full, 0, 0);
      }
      int g = 0;  // ring position, continued across tiles
      for (int tile = blockIdx.x; tile < t.ntiles && !*fail; tile += gridDim.x) {
        const int bx = tile % t.grid_x, by = tile / t.grid_x;
        for (int i = 0; i < items; ++i, ++g) {
          const int s = g % kStages, use = g / kStages;
          if (use > 0 && !umma::mbar_wait(empty + s, (use - 1) & 1, kWaitLimit)) {
            atomicOr(t.err, 16);
            *fail = 1;
            break;
          }
          unsigned char* a = base + s * S::kStage;
          unsigned char* b = a + kATile;
          bool wide;
          int idx;
          item_of(t, nsub_items, subs_first, i, wide, idx);
          if (wide) {
            umma::mbar_arrive_expect_tx(full + s, kATile + S::kBTile);
            umma::tma_load_2d(a, &mapA, full + s, idx * kBK, bx * t.a_row_step + by * t.a_row_ystep);
            umma::tma_load_2d(b, &mapB, full + s, idx * kBK, by * t.b_row_step + bx * t.b_row_xstep);
          } else {
            const int j0 = idx * S::kSites, n = min(S::kSites, t.nsub - j0);
            umma::mbar_arrive_expect_tx(full + s, n * kATile);
            for (int jj = 0; jj < n; ++jj)
              umma::tma_load_2d(a + jj * kATile, &mapA2, full + s, 0, (int)sub_row(t, bx, by, j0 + jj));
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------------ MMA issuer
      if (t.nsub > 0 && !umma::mbar_wait(b2_full, 0, kWaitLimit)) {
        atomicOr(t.err, 16);
        *fail = 1;
      }
      int g = 0, lt = 0;
      for (int tile = blockIdx.x; tile < t.ntiles && !*fail; tile += gridDim.x, ++lt) {
        const int buf = lt & 1, use_buf = lt >> 1;
        if (use_buf > 0 && !umma::mbar_wait(acc_empty + buf, (use_buf - 1) & 1, kWaitLimit)) {
          atomicOr(t.err, 16);
          *fail = 1;
          break;
        }
        umma::fence_after_sync();
        const uint32_t acc = tmem + buf * kCols;
        bool ok = true;
        for (int i = 0; i < items; ++i, ++g) {
          const int s = g % kStages, use = g / kStages;
          if (!umma::mbar_wait(full + s, use & 1, kWaitLimit)) {
            atomicOr(t.err, 16);
            *fail = 1;
            ok = false;
            break;
          }
          umma::fence_after_sync();
          const unsigned char* a = base + s * S::kStage;
          bool wide;
          int idx;
          item_of(t, nsub_items, subs_first, i, wide, idx);
          if (wide) {
            const uint64_t da = umma::sw128_desc(a), db = umma::sw128_desc(a + kATile);
#pragma unroll
            for (int k = 0; k < kBK / 16; ++k)
              umma::mma_bf16(acc, da + 2 * k, db + 2 * k, umma::idesc_bf16(kBM, NT),
                             (subs_first || idx > 0 || k > 0) ? 1u : 0u);
          } else {
            const int j0 = idx * S::kSites, n = min(S::kSites, t.nsub - j0);
            const uint64_t db = umma::sw128_desc(b2_tile);
            for (int jj = 0; jj < n; ++jj) {
              const uint64_t da = umma::sw128_desc(a + jj * kATile);
              for (int k = 0; k < t.ksub; ++k)
                umma::mma_bf16(acc + (j0 + jj) * NB, da + 2 * k, db + 2 * k, umma::idesc_bf16(kBM, NB),
                               ((t.nk > 0 && !subs_first) || k > 0) ? 1u : 0u);
            }
          }
          umma::mma_commit(empty + s);  // the stage is free once these MMAs have read it
        }
        if (!ok) break;
        umma::mma_commit(acc_full + buf);  // the accumulator is complete once every MMA above has run
      }
      umma::mma_commit(done);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int quarter = warp & 3, part = (warp - 2) >> 2;  // part 0 .. kEpiWarps / 4 - 1
    const int row = quarter * 32 + lane;
    unsigned char* scratch = scratch_all + (warp - 2) * S::kScratch;
    int lt = 0;
    for (int tile = blockIdx.x; tile < t.ntiles; tile += gridDim.x, ++lt) {
      const int buf = lt & 1, use_buf = lt >> 1;
      // the tensor-memory loads are warp-collective: decide warp-uniformly
      bool ok = umma::mbar_wait(acc_full + buf, use_buf & 1, kWaitLimit);
      ok = __all_sync(0xffffffffu, ok && !*fail);
      if (!ok) {
        if (lane == 0) {
          atomicOr(t.err, 16);
          *fail = 1;
        }
        break;
      }
      umma::fence_after_sync();
      const int bx = tile % t.grid_x, by = tile / t.grid_x;
      const uint32_t acc = tmem + buf * kCols + (uint32_t(quarter * 32) << 16);
      for (int c = 32 * part; c < t.ncols; c += 32 * (kEpiWarps / 4)) {
        float v[32];
        umma::tmem_ld32(acc + c, v);
        epi.store(bx, by, row, c, v, scratch);
      }
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(acc_empty + buf);
    }
  }
  __syncwarp();
  __syncthreads();  // every role has stopped issuing
  if (warp == 0) {
    // release the accumulators only after every MMA this CTA issued has run
    const bool ok = umma::mbar_wait(done, 0, kWaitLimit);
    if (!ok && lane == 0) atomicOr(t.err, 16);
    __syncwarp();
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, 2 * kCols);
  }
}

}  // namespace gemm
}  // namespace mm
