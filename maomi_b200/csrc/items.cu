// Independent propagation items of uneven size and depth in one persistent
// launch per window size (the mixed workload of many small/large sites).
//
// An item is a field of n x n samples propagated through `steps` phase
// screens, u <- IDFT2(Q * DFT2(u * exp(i*phase_k))), as maomi/numerics.py:156-210
// does for constant pitch.  Items of one window size share a queue: they run
// in waves of `slots` items (callers sort them by depth so waves are even);
// inside a wave, (segment level, slot, line block) work items are handed out
// in dependency order and wait (bounded) on per-slot counters, exactly like
// the fixed-lattice stage.  Screens are formed from the float32 phase stacks
// in the kernel (cp.async prefetch, sincosf), so only the phases are stored.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "dft.cuh"

namespace mm {
namespace {

constexpr long long kItemSpinLimit = 1ll << 24;

struct ItemP {
  int n, nitems, slots, waves, nblocks;
  const int* steps;
  const long long* phase_off;
  const float* phase;
  const float2* field_in;
  float2* field_out;
  const float2* kern;
  const float* edge;
  const long long* wave_items;
  const int* wave_levels;
  const int* slot_base;
  float2* buf;
  unsigned* counters;
  unsigned* head;
  int* error;
  long long total;
};

struct IItem {
  int item, slot, level, block, wave;
};

__device__ __forceinline__ bool idecode(const ItemP& p, long long q, IItem& it) {
  int lo = 0, hi = p.waves;  // last wave w with wave_items[w] <= q
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (p.wave_items[mid] <= q) lo = mid;
    else hi = mid;
  }
  it.wave = lo;
  const long long r = q - p.wave_items[lo];
  const long long per_level = (long long)p.slots * p.nblocks;
  it.level = int(r / per_level);
  const long long rem = r % per_level;
  it.slot = int(rem / p.nblocks);
  it.block = int(rem % p.nblocks);
  it.item = it.wave * p.slots + it.slot;
  return it.item < p.nitems && it.level <= p.steps[it.item];
}

template <class L, int LINES>
struct ISmem {
  static constexpr size_t xbuf = (size_t)LINES * L::XBUF;
  static constexpr size_t screen = (size_t)LINES * L::R2 * L::R1;  // floats
  static constexpr size_t bytes = (xbuf + xbuf % 2) * sizeof(float2) + L::kTwiddleBytes + screen * sizeof(float);
};

// 128-thread CTAs resident per SM the item kernels are compiled for: the
// 512 window's lines hold 32 samples per thread, which fit 168 registers
// without spilling at three CTAs per SM (the line default is two).
template <class L>
constexpr int items_min_blocks() {
  return L::N == 512 ? 3 : L::kMinBlocks;
}

template <class L, int LINES>
__global__ void __launch_bounds__(LINES * L::R2, items_min_blocks<L>() * 128 / (LINES * L::R2)) items_kernel(ItemP p) {
  constexpr int R1 = L::R1, R2 = L::R2, N = L::N;
  extern __shared__ float4 smem_raw[];
  float2* xa = reinterpret_cast<float2*>(smem_raw);
  auto* twf = reinterpret_cast<typename L::TF*>(xa + ISmem<L, LINES>::xbuf + ISmem<L, LINES>::xbuf % 2);
  auto* twi = reinterpret_cast<typename L::TI*>(reinterpret_cast<char*>(twf) + (L::kConjTw ? 0 : N * sizeof(typename L::TF)));
  float* ph_s = reinterpret_cast<float*>(reinterpret_cast<char*>(twf) + L::kTwiddleBytes);
  // Thread 0 claims, decodes and waits for each item once for the CTA; an
  // item costs two CTA barriers (as in the fixed-lattice stage kernel).
  __shared__ long long s_item;
  __shared__ IItem s_it;
  __shared__ int s_live;
  __shared__ int s_abort;
  L::fill_twiddles(twf, twi);
  auto needed = [&](IItem it) {
    return unsigned(p.slot_base[it.wave * p.slots + it.slot] + it.level * p.nblocks);
  };
  auto wait_for = [&](IItem it) {
    const unsigned need = needed(it);
    long long spins = 0;
    unsigned ns = 32;
    while (ld_acquire(p.counters + it.slot) < need) {
      if (++spins > kItemSpinLimit || (ld_acquire(reinterpret_cast<unsigned*>(p.error)) & 1u) != 0u) {
        atomicOr(p.error, 1);
        return 1;
      }
      __nanosleep(ns);
      ns = ns < 256 ? ns * 2 : 256;
    }
    return 0;
  };
  if (threadIdx.x == 0) {
    IItem it{};
    s_item = (long long)atomicAdd(p.head, 1u);
    s_live = s_item < p.total ? int(idecode(p, s_item, it)) : 0;
    s_abort = s_live ? wait_for(it) : 0;
    s_it = it;
  }
  __syncthreads();
  while (true) {
    const long long q = s_item;
    if (q >= p.total || s_abort) break;
    unsigned next = 0;
    if (threadIdx.x == 0) next = atomicAdd(p.head, 1u);
    const IItem it = s_it;
    const bool live = s_live != 0;
    if (live) {
      const int S = p.steps[it.item];
      const int axis = it.level & 1;
      const int tid = threadIdx.x;
      const int line_local = axis == 0 ? tid / R2 : tid % LINES;
      const int t = axis == 0 ? tid % R2 : tid / LINES;
      const int line = it.block * LINES + line_local;
      const int row0 = axis == 0 ? line : t, col0 = axis == 0 ? t : line;
      const int jstep = axis == 0 ? R2 : R2 * N;
      // ---- this thread's phase samples, copied while the field loads
      if (it.level < S) {
        const float* ph = p.phase + p.phase_off[it.item] + (size_t)it.level * N * N + (size_t)row0 * N + col0;
#pragma unroll
        for (int j = 0; j < R1; ++j) {
          const unsigned sp = static_cast<unsigned>(__cvta_generic_to_shared(ph_s + j * blockDim.x + tid));
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sp), "l"(ph + (size_t)j * jstep) : "memory");
        }
        cp_async_commit();
      }
      float2* xl = xa + line_local * L::XBUF;
      const bool warp_local = axis == 0 && 32 % R2 == 0;
      float2 v[R1];
      const float2* src = it.level == 0 ? p.field_in : p.buf + (size_t)it.slot * N * N;
      src += (size_t)row0 * N + col0;
#pragma unroll
      for (int j = 0; j < R1; ++j) v[j] = it.level == 0 ? __ldg(src + (size_t)j * jstep) : __ldcg(src + (size_t)j * jstep);
      // half 0: the second half of step level-1; half 1: the first half of
      // step level (one unrolled copy of the line propagator)
#pragma unroll 1
      for (int half = 0; half < 2; ++half) {
        if (half == 0 ? it.level > 0 : it.level < S)
          L::template propagate<true>(v, t, p.kern, N, xl, xl, twf, twi, warp_local);
        if (half == 1 || it.level >= S) break;
        cp_async_wait_all();
        const float eline = p.edge ? __ldg(p.edge + line) : 1.f;
#pragma unroll
        for (int j = 0; j < R1; ++j) {
          const int e = t + R2 * j;
          float sn, cs;
          sincosf(ph_s[j * blockDim.x + tid], &sn, &cs);
          if (p.edge) {
            const float w = axis == 0 ? eline * __ldg(p.edge + e) : __ldg(p.edge + e) * eline;
            cs *= w;
            sn *= w;
          }
          if constexpr (std::is_same_v<typename L::CF, cpk>) v[j] = to_f2(cmul(from_f2<cpk>(v[j]), make_float2(cs, sn)));
          else v[j] = cmul(v[j], make_float2(cs, sn));
        }
      }
      float2* dst = (it.level == S ? p.field_out + (size_t)it.item * N * N : p.buf + (size_t)it.slot * N * N) +
                    (size_t)row0 * N + col0;
#pragma unroll
      for (int j = 0; j < R1; ++j) __stcg(dst + (size_t)j * jstep, v[j]);
    }
    // thread 0 decodes the next item and looks once at its dependency while
    // the other warps finish
    IItem nit{};
    int nlive = 0, ready = 0;
    if (threadIdx.x == 0) {
      nlive = (long long)next < p.total ? int(idecode(p, next, nit)) : 0;
      ready = !nlive || ld_acquire(p.counters + nit.slot) >= needed(nit);
    }
    __syncthreads();  // the item's stores are issued and every thread has read s_*
    if (threadIdx.x == 0) {
      if (live) {
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        atomicAdd(p.counters + it.slot, 1u);
      }
      s_abort = ready ? 0 : wait_for(nit);
      s_item = (long long)next;
      s_it = nit;
      s_live = nlive;
    }
    __syncthreads();
  }
}

size_t ialign(size_t x) { return (x + 255) & ~size_t(255); }

size_t iworkspace(int n, int slots, char* base, ItemP* p) {
  size_t off = 0;
  auto take = [&](size_t b) {
    char* q = base ? base + off : nullptr;
    off += ialign(b);
    return q;
  };
  float2* buf = reinterpret_cast<float2*>(take((size_t)slots * n * n * sizeof(float2)));
  unsigned* counters = reinterpret_cast<unsigned*>(take((size_t)slots * sizeof(unsigned)));
  unsigned* head = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
  int* error = reinterpret_cast<int*>(take(sizeof(int)));
  if (p) {
    p->buf = buf;
    p->counters = counters;
    p->head = head;
    p->error = error;
  }
  return off;
}

template <class L, int LINES>
int ilaunch(ItemP& p, cudaStream_t s) {
  const size_t smem = ISmem<L, LINES>::bytes;
  MM_CHECK_CUDA(cudaFuncSetAttribute(items_kernel<L, LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(items)");
  int dev = 0, sms = 0, per_sm = 0;
  MM_CHECK_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  MM_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  MM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, items_kernel<L, LINES>, LINES * L::R2, smem),
                "occupancy");
  MM_CHECK_ARG(per_sm >= 1, "item kernel cannot be resident");
  p.nblocks = L::N / LINES;
  const long long grid = std::min<long long>((long long)sms * per_sm, p.total);
  items_kernel<L, LINES><<<(unsigned)std::max<long long>(grid, 1), LINES * L::R2, smem, s>>>(p);
  MM_CHECK_LAUNCH("item propagation kernel");
  return MM_OK;
}

// (window, shape variant) -> kernel; variant 1 uses wider radices per thread.
template <class CF, class CI>
int ilaunch_any(ItemP& p, int shape, cudaStream_t s) {
  switch (p.n) {
    case 64: return shape ? ilaunch<FftLine<16, 4, CF, CI>, 32>(p, s) : ilaunch<FftLine<8, 8, CF, CI>, 16>(p, s);
    case 128: return shape ? ilaunch<FftLine<32, 4, CF, CI>, 32>(p, s) : ilaunch<FftLine<16, 8, CF, CI>, 16>(p, s);
    case 256: return shape ? ilaunch<FftLine<32, 8, CF, CI>, 16>(p, s) : ilaunch<FftLine<16, 16, CF, CI>, 8>(p, s);
    case 512: return ilaunch<FftLine<32, 16, CF, CI>, 8>(p, s);
    default: set_error("item windows must be 64, 128, 256 or 512 (got %d)", p.n); return MM_ERR_UNSUPPORTED;
  }
}

int lines_of(int n, int shape) {
  switch (n) {
    case 64: return shape ? 32 : 16;
    case 128: return shape ? 32 : 16;
    case 256: return shape ? 16 : 8;
    default: return 8;
  }
}

}  // namespace
}  // namespace mm

using namespace mm;

extern "C" int mm_items_blocks(int n, int shape) { return n / lines_of(n, shape); }

extern "C" size_t mm_propagate_items_workspace_size(const mm_item_class* c) {
  if (!c || c->slots < 1 || c->n < 1) return 0;
  return iworkspace(c->n, c->slots, nullptr, nullptr);
}

extern "C" int mm_propagate_items(const mm_item_class* c, void* workspace, size_t workspace_bytes, int check,
                                  void* stream) {
  MM_CHECK_ARG(c != nullptr, "class is NULL");
  MM_CHECK_ARG(c->n == 64 || c->n == 128 || c->n == 256 || c->n == 512, "item window %d unsupported", c->n);
  MM_CHECK_ARG(c->nitems >= 0 && c->slots >= 1 && c->waves >= 0, "bad item counts");
  MM_CHECK_ARG(c->shape == 0 || c->shape == 1, "unknown shape %d", c->shape);
  MM_CHECK_ARG(c->precision == MM_PRECISION_FP32 || c->precision == MM_PRECISION_FP64 ||
                   c->precision == MM_PRECISION_MIXED || c->precision == MM_PRECISION_COMPENSATED ||
                   c->precision == MM_PRECISION_COMPENSATED_FULL,
               "unknown precision %d", c->precision);
  if (c->nitems == 0) return MM_OK;
  MM_CHECK_ARG(c->steps && c->phase_offset && c->phase && c->field_in && c->field_out && c->kernel &&
                   c->wave_items && c->wave_levels && c->slot_base,
               "NULL pointer in item class");
  const size_t need = iworkspace(c->n, c->slots, nullptr, nullptr);
  MM_CHECK_ARG(workspace && workspace_bytes >= need, "workspace too small: %zu given, %zu needed", workspace_bytes, need);
  MM_CHECK_ARG(reinterpret_cast<uintptr_t>(workspace) % 256 == 0, "workspace must be 256-byte aligned");
  ItemP p{};
  p.n = c->n;
  p.nitems = c->nitems;
  p.slots = c->slots;
  p.waves = c->waves;
  p.steps = c->steps;
  p.phase_off = reinterpret_cast<const long long*>(c->phase_offset);
  p.phase = c->phase;
  p.field_in = static_cast<const float2*>(c->field_in);
  p.field_out = static_cast<float2*>(c->field_out);
  p.kern = static_cast<const float2*>(c->kernel);
  p.edge = c->edge1d;
  p.wave_items = reinterpret_cast<const long long*>(c->wave_items);
  p.wave_levels = c->wave_levels;
  p.slot_base = c->slot_base;
  p.total = (long long)c->total_items;
  iworkspace(c->n, c->slots, static_cast<char*>(workspace), &p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  MM_CHECK_CUDA(cudaMemsetAsync(p.counters, 0, (char*)p.error + sizeof(int) - (char*)p.counters, s), "zero queue");
  int rc;
  if (c->precision == MM_PRECISION_FP64) rc = ilaunch_any<double2, double2>(p, c->shape, s);
  else if (c->precision == MM_PRECISION_MIXED) rc = ilaunch_any<float2, double2>(p, c->shape, s);
  else if (c->precision == MM_PRECISION_COMPENSATED) rc = ilaunch_any<cpk, cpk>(p, c->shape, s);
  else if (c->precision == MM_PRECISION_COMPENSATED_FULL) rc = ilaunch_any<cfx, cfx>(p, c->shape, s);
  else rc = ilaunch_any<float2, float2>(p, c->shape, s);
  if (rc != MM_OK || !check) return rc;
  MM_CHECK_CUDA(cudaStreamSynchronize(s), "item propagation");
  int err = 0;
  MM_CHECK_CUDA(cudaMemcpy(&err, p.error, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
  if (err) {
    set_error("item propagation: a dependency wait timed out");
    return MM_ERR_TIMEOUT;
  }
  return MM_OK;
}
