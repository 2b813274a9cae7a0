// Fused split-step propagation of many sites through the A/B/C screen stacks.
//
// Each propagation step u <- IDFT2(Q * DFT2(u * S)) has a separable transfer
// function Q = Qx (x) Qy, so it factors into one 1-D propagate along rows and
// one along columns.  A "segment" applies, along one axis, the second half of
// step k-1, the screen of step k, the plane save, and the first half of step
// k; consecutive segments alternate axes.  The field therefore crosses global
// memory once per step (read + write) and every line is transformed fully in
// registers and shared memory.  Saved planes are reduced in the same pass:
// focal |E|^(2*order) crops, the tail images (trapezoid * axial weighted sums)
// and the per-plane tail profiles.
//
// Two schedules share the segment code:
//  * persistent: one launch; CTAs pull (site, segment, line-block) items from
//    a device queue in dependency order and wait (bounded) on per-slot
//    counters; `slots` sites are in flight, so their fields stay L2-resident.
//  * batched: one launch per segment for a batch of sites (kernel boundaries
//    order the segments), the launch structure of the reference's batches.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "dft.cuh"

namespace mm {
namespace {

struct StageP {
  int size, steps, nseg, nblocks;
  const float2* screens;
  int vol_h, vol_w;
  const float* edge;
  const float2* kern;
  long long cum0;  // blocks of one site before this stage's first segment
  int seg0;        // global segment index of this stage's first segment
};

struct Params {
  StageP st[3];
  const float2* base;
  int n, n2, crop0, order, cut;
  int fx0, fy0, fh, fw;
  const float* tail_w[2];
  float* focal;
  float* tail_img[2];
  int tail_per_site;
  double* profile[2];
  int planes[2];
  const int* offsets;
  int nsites;
  float2* bufA;
  float2* bufB;
  int slots;
  unsigned* counters;
  unsigned* head;
  int* error;
  long long blocks_per_site;
  long long total_items;
  // batched schedule: the stage / segment and first site of this launch
  int b_stage, b_k, b_site0;
  int precision;  // MM_PRECISION_*: arithmetic of the radix-2 line transforms
  int reserve_sms;  // persistent CTAs starting on SM ids below this leave at once
  int hold_site;    // fault drill: site + 1 whose first item waits for ever (0 = off)
  long long spin_limit;  // bound of a dependency wait, in polls
};

constexpr long long kSpinLimit = 1ll << 24;  // ~ seconds with the backoff below

// Lines per CTA (128 threads each: four CTAs, 16 warps, per SM).
constexpr int kLines64 = 16, kLines128 = 16, kLines256 = 8, kLines512 = 8, kLinesDense = 8;

struct Item {
  int stage, k, slot, block, site, wave;
};

__device__ __forceinline__ bool decode(const Params& p, long long item, Item& it) {
  const long long per_wave = p.blocks_per_site * p.slots;
  it.wave = int(item / per_wave);
  long long r = item % per_wave;
  for (int s = 0; s < 3; ++s) {
    const long long span = (long long)p.st[s].nseg * p.st[s].nblocks * p.slots;
    if (r < span || s == 2) {
      const long long per_seg = (long long)p.st[s].nblocks * p.slots;
      it.stage = s;
      it.k = int(r / per_seg);
      const long long rem = r % per_seg;
      it.slot = int(rem / p.st[s].nblocks);
      it.block = int(rem % p.st[s].nblocks);
      break;
    }
    r -= span;
  }
  it.site = it.wave * p.slots + it.slot;
  return it.site < p.nsites;
}

// Which line of the item this thread works on, and its place in the line:
// rows (axis 0) keep a line's threads in one warp; columns (axis 1) put 32
// consecutive columns in a warp so every global access is a full segment.
template <class L, int LINES>
struct Lane {
  int axis, line_local, t, line;
  __device__ Lane(const Params& p, const Item& it) {
    const StageP& st = p.st[it.stage];
    axis = (st.seg0 + it.k) & 1;
    const int tid = threadIdx.x;
    line_local = axis == 0 ? tid / L::R2 : tid % LINES;
    t = axis == 0 ? tid % L::R2 : tid / LINES;
    line = it.block * LINES + line_local;
  }
};

// Window offset of the item's site; an offset outside the screen volume is
// flagged (reported as MM_ERR_ARGUMENT) and replaced by the volume's corner.
__device__ __forceinline__ int2 site_offset(const Params& p, const Item& it) {
  const StageP& st = p.st[it.stage];
  int xo = __ldg(p.offsets + 2 * it.site), yo = __ldg(p.offsets + 2 * it.site + 1);
  if (xo < 0 || yo < 0 || xo + st.size > st.vol_h || yo + st.size > st.vol_w) {
    if (threadIdx.x == 0) atomicOr(p.error, 2);
    xo = 0;
    yo = 0;
  }
  return make_int2(xo, yo);
}

// One (site, segment, line block) work item.
template <class L, int LINES>
__device__ void process(const Params& p, const Item& it, float2* xa, float2* xb, const typename L::TF* twf,
                        const typename L::TI* twi, float* red) {
  constexpr int R1 = L::R1, R2 = L::R2;
  const StageP& st = p.st[it.stage];
  const int N = st.size;
  const Lane<L, LINES> ln(p, it);
  const int axis = ln.axis, line_local = ln.line_local, t = ln.t, line = ln.line;
  float2* xa_l = xa + line_local * L::XBUF;
  float2* xb_l = xa_l;  // one exchange buffer per line (see propagate<SINGLE>)
  // Radix-2 lines exactly fill their threads; the dense policy guards lines
  // and samples beyond the window (those threads still take every barrier).
  const bool live = L::kFft || line < N;
  auto in_line = [&](int e) { return L::kFft || (live && e < N); };

  // Element j of this thread: (row, col) = (row0, col0) + j * (drow, dcol).
  const int row0 = axis == 0 ? line : t, col0 = axis == 0 ? t : line;
  const int drow = axis == 0 ? 0 : R2, dcol = axis == 0 ? R2 : 0;
  const int jstep = axis == 0 ? R2 : R2 * N;  // linear step in an N x N buffer

  float2 v[R1];
  // ------------------------------------------------------------------ load
  {
    const size_t slot_a = (size_t)it.slot * p.n * p.n;
    const size_t slot_b = (size_t)it.slot * p.n2 * p.n2;
    if (it.k > 0 || it.stage == 0) {
      const float2* src = it.k == 0 ? p.base : (it.stage == 1 ? p.bufB + slot_b : p.bufA + slot_a);
      src += (size_t)row0 * N + col0;
#pragma unroll
      for (int j = 0; j < R1; ++j) {
        v[j] = make_float2(0.f, 0.f);
        if (!in_line(t + R2 * j)) continue;
        v[j] = it.k == 0 ? __ldg(src + (size_t)j * jstep) : __ldcg(src + (size_t)j * jstep);
      }
    } else if (it.stage == 1) {  // crop the n x n field of stage A to the n2 window
      const float2* src = p.bufA + slot_a + (size_t)(row0 + p.crop0) * p.n + (col0 + p.crop0);
      const int step_n = axis == 0 ? R2 : R2 * p.n;
#pragma unroll
      for (int j = 0; j < R1; ++j) {
        v[j] = make_float2(0.f, 0.f);
        if (in_line(t + R2 * j)) v[j] = __ldcg(src + (size_t)j * step_n);
      }
    } else {  // zero-pad the n2 field of stage B to the n window
#pragma unroll
      for (int j = 0; j < R1; ++j) {
        const int r2 = row0 + j * drow - p.crop0, c2 = col0 + j * dcol - p.crop0;
        v[j] = (in_line(t + R2 * j) && r2 >= 0 && r2 < p.n2 && c2 >= 0 && c2 < p.n2)
                   ? __ldcg(p.bufB + slot_b + (size_t)r2 * p.n2 + c2)
                   : make_float2(0.f, 0.f);
      }
    }
  }
  // Row layout keeps each line inside one warp: its exchanges need only warp barriers.
  const bool warp_local = L::kFft && axis == 0 && 32 % R2 == 0;
  // Two half-steps share one copy of the line propagator (half 0: second
  // half of step k-1; half 1: first half of step k), the screen and the
  // plane save between them: one unrolled transform in the instruction stream.
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
  if (half == 0 ? it.k > 0 : it.k < st.steps)
    L::template propagate<true>(v, t, st.kern + (size_t)(it.k - 1 + half) * N, N, xa_l, xb_l, twf, twi, warp_local);
  if (half == 1) break;
  // ------------------------------------------------------- screen of step k
  if (it.k < st.steps) {
    // the screen samples at the site's window offset, read straight from the
    // (Z, H, W) volume: issued together, consumed after all have arrived
    const float eline = live ? __ldg(st.edge + line) : 0.f;
    const int2 so = site_offset(p, it);
    const float2* scr = st.screens + (size_t)it.k * st.vol_h * st.vol_w + (size_t)(so.x + row0) * st.vol_w + (so.y + col0);
    const size_t sstep = axis == 0 ? size_t(R2) : size_t(R2) * st.vol_w;
    float2 sv[R1];
#pragma unroll
    for (int j = 0; j < R1; ++j) sv[j] = in_line(t + R2 * j) ? __ldg(scr + j * sstep) : make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < R1; ++j) {
      const int e = t + R2 * j;
      if (!in_line(e)) continue;
      const float w = axis == 0 ? eline * __ldg(st.edge + e) : __ldg(st.edge + e) * eline;
      float2 s = sv[j];
      s = make_float2(s.x * w, s.y * w);
      if constexpr (std::is_same_v<typename L::CF, cpk>) v[j] = to_f2(cmul(from_f2<cpk>(v[j]), s));  // packed
      else v[j] = cmul(v[j], s);
    }
  }
  // ------------------------------------------------------------ plane save
  {
    int tail = -1, pt = 0;
    if (it.stage == 0 && it.k >= p.cut) { tail = 0; pt = it.k - p.cut; }
    if (it.stage == 2) { tail = 1; pt = it.k; }
    if (tail >= 0) {
      const float wgt = __ldg(p.tail_w[tail] + pt);
      float* img = p.tail_img[tail] + (size_t)(p.tail_per_site ? it.site : it.slot) * p.n2 * p.n2;
      const bool init = p.tail_per_site && pt == 0;
      float psum = 0.f;
      // the line must cross the centred n2 crop; then test the in-line coordinate
      const int lc = line - p.crop0;
      if (live && lc >= 0 && lc < p.n2) {
        // the line's pixel j sits at img0 + ec * estep; the earlier sums of
        // a group of pixels are read together (one round trip per group),
        // then the new ones written
        float* img0 = img + (axis == 0 ? (size_t)lc * p.n2 : (size_t)lc);
        const size_t estep = axis == 0 ? 1 : (size_t)p.n2;
        constexpr int G = R1 < 4 ? R1 : 4;
#pragma unroll
        for (int g = 0; g < R1; g += G) {
          float prev[G];
#pragma unroll
          for (int i = 0; i < G; ++i) {
            const int ec = t + R2 * (g + i) - p.crop0;
            const bool in = in_line(t + R2 * (g + i)) && ec >= 0 && ec < p.n2;
            prev[i] = (in && !init) ? __ldcg(img0 + (size_t)ec * estep) : 0.f;
          }
#pragma unroll
          for (int i = 0; i < G; ++i) {
            const int ec = t + R2 * (g + i) - p.crop0;
            if (!in_line(t + R2 * (g + i)) || ec < 0 || ec >= p.n2) continue;
            const float pw = photon_power(v[g + i], p.order);
            psum += pw;
            __stcg(img0 + (size_t)ec * estep, prev[i] + wgt * pw);
          }
        }
      }
      // the plane's power: warp sums, one FP64 atomic per warp (no CTA barrier)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) psum += __shfl_xor_sync(0xffffffffu, psum, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(p.profile[tail] + (size_t)it.site * p.planes[tail] + pt, (double)psum);
    } else if (it.stage == 1 && it.k < st.steps) {
      float* dst = p.focal + ((size_t)it.site * st.steps + it.k) * p.fh * p.fw;
      const int lf = line - (axis == 0 ? p.fx0 : p.fy0);            // line inside the focal crop?
      const int lext = axis == 0 ? p.fh : p.fw, eorg = axis == 0 ? p.fy0 : p.fx0, eext = axis == 0 ? p.fw : p.fh;
      if (live && lf >= 0 && lf < lext) {
#pragma unroll
        for (int j = 0; j < R1; ++j) {
          const int ef = t + R2 * j - eorg;
          if (!in_line(t + R2 * j) || ef < 0 || ef >= eext) continue;
          const size_t off = axis == 0 ? (size_t)lf * p.fw + ef : (size_t)ef * p.fw + lf;
          __stcs(dst + off, photon_power(v[j], p.order));
        }
      }
    }
  }
  }
  // ------------------------------------------------------------------ store
  if (!(it.stage == 2 && it.k == st.steps)) {
    float2* dst = (it.stage == 1 ? p.bufB + (size_t)it.slot * p.n2 * p.n2 : p.bufA + (size_t)it.slot * p.n * p.n) +
                  (size_t)row0 * N + col0;
#pragma unroll
    for (int j = 0; j < R1; ++j)
      if (in_line(t + R2 * j)) __stcg(dst + (size_t)j * jstep, v[j]);
  }
}

// Dynamic shared memory of a propagation CTA: the exchange buffer, the
// twiddle tables and the reduction scratch.  More shared memory (a second
// exchange buffer, staged screens) measured slower: it comes out of L1.
template <class L, int LINES>
struct Smem {
  static constexpr size_t xbuf = (size_t)LINES * L::XBUF;  // exchange-buffer elements (L::XT)
  static constexpr size_t xbytes = (xbuf * sizeof(typename L::XT) + 15) / 16 * 16;
  static constexpr size_t bytes = xbytes + L::kTwiddleBytes + 32 * sizeof(float);
  struct Parts {
    typename L::XT* xa;
    typename L::TF* twf;
    typename L::TI* twi;
    float* red;
  };
  __device__ static Parts carve(void* base) {
    char* b = static_cast<char*>(base);
    Parts q;
    q.xa = reinterpret_cast<typename L::XT*>(b);
    q.twf = reinterpret_cast<typename L::TF*>(b + xbytes);
    q.twi = reinterpret_cast<typename L::TI*>(b + xbytes + (L::kConjTw ? 0 : L::N * sizeof(typename L::TF)));
    q.red = reinterpret_cast<float*>(b + xbytes + L::kTwiddleBytes);
    return q;
  }
};

template <class L, int LINES>
__global__ void __launch_bounds__(LINES * L::R2, L::kMinBlocks * 128 / (LINES * L::R2)) persistent_kernel(Params p) {
  extern __shared__ float4 smem_raw[];
  const auto sm = Smem<L, LINES>::carve(smem_raw);
  // The queue position and its decoded item live in shared memory: thread 0
  // claims, decodes (64-bit divisions) and waits for each item once for the
  // whole CTA, so an item costs two CTA barriers.
  __shared__ long long s_item;
  __shared__ Item s_it;
  __shared__ int s_live;
  __shared__ int s_abort;
  if (p.reserve_sms > 0) {
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if (smid < unsigned(p.reserve_sms)) return;  // uniform per CTA; no item claimed yet
  }
  L::fill_twiddles(sm.twf, sm.twi);
  // counter value that publishes the segment before item it
  auto needed = [&](const Item& it) {
    const StageP& st = p.st[it.stage];
    const unsigned held = (p.hold_site == it.site + 1) ? 0x40000000u : 0u;
    return unsigned(it.wave * p.blocks_per_site + st.cum0 + (long long)it.k * st.nblocks) + held;
  };
  // thread 0: wait (bounded) until the item's inputs are published
  auto wait_for = [&](const Item& it) {
    const unsigned need = needed(it);
    long long spins = 0;
    unsigned ns = 32;
    while (ld_acquire(p.counters + it.slot) < need) {
      if (++spins > p.spin_limit || (ld_acquire(reinterpret_cast<unsigned*>(p.error)) & 1u) != 0u) {
        atomicOr(p.error, 1);
        return 1;
      }
      __nanosleep(ns);
      ns = ns < 256 ? ns * 2 : 256;
    }
    return 0;
  };
  if (threadIdx.x == 0) {
    Item it{};
    s_item = (long long)atomicAdd(p.head, 1u);
    s_live = s_item < p.total_items ? decode(p, s_item, it) : 0;
    s_abort = s_live ? wait_for(it) : 0;
    s_it = it;
  }
  __syncthreads();
  while (true) {
    const long long item = s_item;
    if (item >= p.total_items || s_abort) break;
    // Claim the next item now; the value is only consumed at the end of this
    // one, so the atomic's round trip overlaps the work below.
    unsigned next = 0;
    if (threadIdx.x == 0) next = atomicAdd(p.head, 1u);
    const Item it = s_it;
    const bool live = s_live != 0;
    if (live) process<L, LINES>(p, it, sm.xa, sm.xa, sm.twf, sm.twi, sm.red);
    // thread 0 decodes the next item and looks once at its dependency while
    // the other warps finish
    Item nit{};
    int nlive = 0, ready = 0;
    if (threadIdx.x == 0) {
      nlive = (long long)next < p.total_items ? int(decode(p, next, nit)) : 0;
      ready = !nlive || ld_acquire(p.counters + nit.slot) >= needed(nit);
    }
    __syncthreads();  // the item's stores are issued and every thread has read s_*
    if (threadIdx.x == 0) {
      if (live) {
        // release: the CTA's field stores (ordered by the barrier) become
        // visible before the counter that publishes them
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

template <class L, int LINES>
__global__ void __launch_bounds__(LINES * L::R2, L::kMinBlocks * 128 / (LINES * L::R2)) batched_kernel(Params p) {
  extern __shared__ float4 smem_raw[];
  const auto sm = Smem<L, LINES>::carve(smem_raw);
  L::fill_twiddles(sm.twf, sm.twi);
  __syncthreads();
  const StageP& st = p.st[p.b_stage];
  Item it;
  it.stage = p.b_stage;
  it.k = p.b_k;
  it.slot = blockIdx.x / st.nblocks;
  it.block = blockIdx.x % st.nblocks;
  it.site = p.b_site0 + it.slot;
  it.wave = 0;
  if (it.site >= p.nsites) return;
  process<L, LINES>(p, it, sm.xa, sm.xa, sm.twf, sm.twi, sm.red);
}

// ------------------------------------------------------------------- host --
struct Config {
  int r1, r2, lines;
};

bool fft_size(int n) { return n == 64 || n == 128 || n == 256 || n == 512; }

// Lines per CTA for a window; dense windows use 8 lines of 16 threads.
bool line_config(int n, Config& c) {
  switch (n) {
    case 64: c = {8, 8, kLines64}; return true;
    case 128: c = {16, 8, kLines128}; return true;
    case 256: c = {16, 16, kLines256}; return true;
    case 512: c = {32, 16, kLines512}; return true;
    default:
      if (n >= 2 && n <= 512 && n % 2 == 0) {
        c = {n <= 128 ? 8 : 32, 16, kLinesDense};
        return true;
      }
      return false;
  }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Workspace {
  float2* bufA;
  float2* bufB;
  unsigned* counters;
  unsigned* head;
  int* error;
  size_t bytes;
};

Workspace carve(void* base, int n, int n2, int slots) {
  Workspace w{};
  char* p = static_cast<char*>(base);
  size_t off = 0;
  auto take = [&](size_t b) {
    char* q = p ? p + off : nullptr;
    off += align256(b);
    return q;
  };
  w.bufA = reinterpret_cast<float2*>(take((size_t)slots * n * n * sizeof(float2)));
  w.bufB = reinterpret_cast<float2*>(take((size_t)slots * n2 * n2 * sizeof(float2)));
  w.counters = reinterpret_cast<unsigned*>(take((size_t)slots * sizeof(unsigned)));
  w.head = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
  w.error = reinterpret_cast<int*>(take(sizeof(int)));
  w.bytes = off;
  return w;
}

template <class L, int LINES>
int launch_batched(Params& p, int stage, int k, int site0, int batch, cudaStream_t s) {
  const size_t smem = Smem<L, LINES>::bytes;
  MM_CHECK_CUDA(cudaFuncSetAttribute(batched_kernel<L, LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(batched)");
  p.b_stage = stage;
  p.b_k = k;
  p.b_site0 = site0;
  const int grid = batch * p.st[stage].nblocks;
  batched_kernel<L, LINES><<<grid, LINES * L::R2, smem, s>>>(p);
  MM_CHECK_LAUNCH("batched propagation kernel");
  return MM_OK;
}

template <class CF, class CI>
int launch_batched_fft(Params& p, int stage, int k, int site0, int batch, cudaStream_t s) {
  switch (p.st[stage].size) {
    case 64: return launch_batched<FftLine<8, 8, CF, CI>, kLines64>(p, stage, k, site0, batch, s);
    case 128: return launch_batched<FftLine<16, 8, CF, CI>, kLines128>(p, stage, k, site0, batch, s);
    case 256: return launch_batched<FftLine<16, 16, CF, CI>, kLines256>(p, stage, k, site0, batch, s);
    default: return launch_batched<FftLine<32, 16, CF, CI>, kLines512>(p, stage, k, site0, batch, s);
  }
}

int launch_batched_any(Params& p, int stage, int k, int site0, int batch, cudaStream_t s) {
  const int n = p.st[stage].size;
  switch (n) {
    case 64:
    case 128:
    case 256:
    case 512:
      if (p.precision == MM_PRECISION_FP64) return launch_batched_fft<double2, double2>(p, stage, k, site0, batch, s);
      if (p.precision == MM_PRECISION_MIXED) return launch_batched_fft<float2, double2>(p, stage, k, site0, batch, s);
      if (p.precision == MM_PRECISION_COMPENSATED) return launch_batched_fft<cpk, cpk>(p, stage, k, site0, batch, s);
      if (p.precision == MM_PRECISION_COMPENSATED_FULL) return launch_batched_fft<cfx, cfx>(p, stage, k, site0, batch, s);
      return launch_batched_fft<float2, float2>(p, stage, k, site0, batch, s);
    default:
      if (n <= 128) return launch_batched<DenseLine<8>, kLinesDense>(p, stage, k, site0, batch, s);
      return launch_batched<DenseLine<32>, kLinesDense>(p, stage, k, site0, batch, s);
  }
}

template <class L, int LINES>
int launch_persistent(Params& p, cudaStream_t s) {
  const size_t smem = Smem<L, LINES>::bytes;
  MM_CHECK_CUDA(cudaFuncSetAttribute(persistent_kernel<L, LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(persistent)");
  int dev = 0, sms = 0, per_sm = 0;
  MM_CHECK_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  MM_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  MM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel<L, LINES>, LINES * L::R2, smem),
                "occupancy");
  if (per_sm < 1) {
    set_error("persistent propagation kernel cannot be resident (smem %zu)", smem);
    return MM_ERR_UNSUPPORTED;
  }
  const long long grid = std::min<long long>((long long)sms * per_sm, p.total_items);
  persistent_kernel<L, LINES><<<(unsigned)grid, LINES * L::R2, smem, s>>>(p);
  MM_CHECK_LAUNCH("persistent propagation kernel");
  return MM_OK;
}

template <class CF, class CI>
int launch_persistent_fft(Params& p, cudaStream_t s) {
  switch (p.n) {
    case 64: return launch_persistent<FftLine<8, 8, CF, CI>, kLines64>(p, s);
    case 128: return launch_persistent<FftLine<16, 8, CF, CI>, kLines128>(p, s);
    case 256: return launch_persistent<FftLine<16, 16, CF, CI>, kLines256>(p, s);
    default: return launch_persistent<FftLine<32, 16, CF, CI>, kLines512>(p, s);
  }
}

int launch_persistent_any(Params& p, cudaStream_t s) {
  if (!fft_size(p.n) || p.n != p.n2) {
    if (std::max(p.n, p.n2) <= 128) return launch_persistent<DenseLine<8>, kLinesDense>(p, s);
    return launch_persistent<DenseLine<32>, kLinesDense>(p, s);
  }
  if (p.precision == MM_PRECISION_FP64) return launch_persistent_fft<double2, double2>(p, s);
  if (p.precision == MM_PRECISION_MIXED) return launch_persistent_fft<float2, double2>(p, s);
  if (p.precision == MM_PRECISION_COMPENSATED) return launch_persistent_fft<cpk, cpk>(p, s);
  if (p.precision == MM_PRECISION_COMPENSATED_FULL) return launch_persistent_fft<cfx, cfx>(p, s);
  return launch_persistent_fft<float2, float2>(p, s);
}

int build_params(const mm_stage_plan* plan, int slots, Params& p) {
  MM_CHECK_ARG(plan != nullptr, "plan is NULL");
  MM_CHECK_ARG(plan->nsites >= 1, "need at least one site (got %d)", plan->nsites);
  MM_CHECK_ARG(slots >= 1, "slots must be >= 1 (got %d)", slots);
  MM_CHECK_ARG(plan->order >= 1 && plan->order <= 3, "photon order must be 1, 2 or 3 (got %d)", plan->order);
  MM_CHECK_ARG(plan->n >= plan->n2 && plan->n2 >= 1 && (plan->n - plan->n2) % 2 == 0,
               "incompatible windows n=%d n2=%d", plan->n, plan->n2);
  MM_CHECK_ARG(plan->base && plan->offsets && plan->focal && plan->tail_image[0] && plan->tail_image[1] &&
                   plan->tail_profile[0] && plan->tail_profile[1] && plan->tail_weight[0] && plan->tail_weight[1],
               "plan has NULL buffers");
  p = Params{};
  long long cum = 0;
  int seg = 0;
  for (int s = 0; s < 3; ++s) {
    const mm_stage_desc& d = plan->stage[s];
    Config c;
    MM_CHECK_ARG(d.size == (s == 1 ? plan->n2 : plan->n), "stage %d window %d does not match the plan", s, d.size);
    if (!line_config(d.size, c)) {
      set_error("no propagation kernel for window %d (even sizes up to 512)", d.size);
      return MM_ERR_UNSUPPORTED;
    }
    MM_CHECK_ARG(d.steps >= 1 && d.screens && d.edge1d && d.kernels, "stage %d incomplete", s);
    MM_CHECK_ARG(d.vol_h >= d.size && d.vol_w >= d.size, "stage %d screens smaller than the window", s);
    StageP& st = p.st[s];
    st.size = d.size;
    st.steps = d.steps;
    st.nseg = d.steps + 1;
    st.nblocks = (d.size + c.lines - 1) / c.lines;
    st.screens = static_cast<const float2*>(d.screens);
    st.vol_h = d.vol_h;
    st.vol_w = d.vol_w;
    st.edge = d.edge1d;
    st.kern = static_cast<const float2*>(d.kernels);
    st.cum0 = cum;
    st.seg0 = seg;
    cum += (long long)st.nseg * st.nblocks;
    seg += st.nseg;
  }
  MM_CHECK_ARG(plan->cut >= 0 && plan->cut <= plan->stage[0].steps, "cut %d outside stage A", plan->cut);
  MM_CHECK_ARG(plan->focal_x0 >= 0 && plan->focal_y0 >= 0 && plan->focal_h >= 1 && plan->focal_w >= 1 &&
                   plan->focal_x0 + plan->focal_h <= plan->n2 && plan->focal_y0 + plan->focal_w <= plan->n2,
               "focal crop outside the stage-B window");
  p.base = static_cast<const float2*>(plan->base);
  p.n = plan->n;
  p.n2 = plan->n2;
  p.crop0 = (plan->n - plan->n2) / 2;
  p.order = plan->order;
  p.cut = plan->cut;
  p.fx0 = plan->focal_x0;
  p.fy0 = plan->focal_y0;
  p.fh = plan->focal_h;
  p.fw = plan->focal_w;
  p.tail_w[0] = plan->tail_weight[0];
  p.tail_w[1] = plan->tail_weight[1];
  p.focal = plan->focal;
  p.tail_img[0] = plan->tail_image[0];
  p.tail_img[1] = plan->tail_image[1];
  p.tail_per_site = plan->tail_per_site;
  p.profile[0] = plan->tail_profile[0];
  p.profile[1] = plan->tail_profile[1];
  p.planes[0] = plan->stage[0].steps + 1 - plan->cut;
  p.planes[1] = plan->stage[2].steps + 1;
  p.offsets = plan->offsets;
  p.nsites = plan->nsites;
  p.slots = slots;
  MM_CHECK_ARG(plan->precision == MM_PRECISION_FP32 || plan->precision == MM_PRECISION_FP64 ||
                   plan->precision == MM_PRECISION_MIXED || plan->precision == MM_PRECISION_COMPENSATED ||
                   plan->precision == MM_PRECISION_COMPENSATED_FULL,
               "unknown precision %d", plan->precision);
  p.precision = plan->precision;
  MM_CHECK_ARG(plan->reserve_sms >= 0 && plan->reserve_sms <= 64, "reserve_sms %d outside 0..64", plan->reserve_sms);
  p.reserve_sms = plan->reserve_sms;
  MM_CHECK_ARG(plan->hold_site >= 0 && plan->hold_site <= plan->nsites, "hold_site %d outside 0..%d",
               plan->hold_site, plan->nsites);
  MM_CHECK_ARG(plan->spin_limit >= 0, "spin_limit must be >= 0");
  p.hold_site = plan->hold_site;
  p.spin_limit = plan->spin_limit > 0 ? plan->spin_limit : kSpinLimit;
  p.blocks_per_site = cum;
  return MM_OK;
}

}  // namespace

int propagation_slots(int nsites, int slots, int schedule) {
  slots = std::min(slots, nsites);
  if (schedule == MM_SCHEDULE_PERSISTENT && slots > 0) {
    // Balance the sites over the slots so the last wave is (nearly) full.
    const int waves = (nsites + slots - 1) / slots;
    slots = (nsites + waves - 1) / waves;
  }
  return slots;
}

}  // namespace mm

extern "C" size_t mm_propagate_workspace_size(const mm_stage_plan* plan, int slots, int schedule) {
  (void)schedule;
  if (!plan || slots < 1) return 0;
  return mm::carve(nullptr, plan->n, plan->n2, slots).bytes;
}

extern "C" int mm_propagate_status(const mm_stage_plan* plan, int schedule, int slots, const void* workspace,
                                   void* stream) {
  using namespace mm;
  MM_CHECK_ARG(plan != nullptr && workspace != nullptr && slots >= 1, "bad propagation status arguments");
  MM_CHECK_ARG(schedule == MM_SCHEDULE_PERSISTENT || schedule == MM_SCHEDULE_BATCHED, "unknown schedule %d", schedule);
  MM_CHECK_ARG(reinterpret_cast<uintptr_t>(workspace) % 256 == 0, "workspace must be 256-byte aligned");
  const Workspace w =
      carve(const_cast<void*>(workspace), plan->n, plan->n2, propagation_slots(plan->nsites, slots, schedule));
  MM_CHECK_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "propagation");
  int err = 0;
  MM_CHECK_CUDA(cudaMemcpy(&err, w.error, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
  if (err & 2) {
    set_error("a site window lies outside the screen volume (offsets out of range)");
    return MM_ERR_ARGUMENT;
  }
  if (err) {
    set_error("persistent propagation: a dependency wait timed out");
    return MM_ERR_TIMEOUT;
  }
  return MM_OK;
}

extern "C" int mm_propagate_sites(const mm_stage_plan* plan, int schedule, int slots, void* workspace,
                                  size_t workspace_bytes, int check, void* stream) {
  using namespace mm;
  Params p;
  if (int rc = build_params(plan, slots, p)) return rc;
  MM_CHECK_ARG(schedule == MM_SCHEDULE_PERSISTENT || schedule == MM_SCHEDULE_BATCHED, "unknown schedule %d", schedule);
  slots = propagation_slots(plan->nsites, slots, schedule);
  p.slots = slots;
  Workspace w = carve(workspace, plan->n, plan->n2, slots);
  MM_CHECK_ARG(workspace != nullptr && workspace_bytes >= w.bytes,
               "workspace too small: %zu bytes given, %zu needed", workspace_bytes, w.bytes);
  MM_CHECK_ARG(reinterpret_cast<uintptr_t>(workspace) % 256 == 0, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p.bufA = w.bufA;
  p.bufB = w.bufB;
  p.counters = w.counters;
  p.head = w.head;
  p.error = w.error;
  for (int t = 0; t < 2; ++t)
    MM_CHECK_CUDA(cudaMemsetAsync(p.profile[t], 0, sizeof(double) * (size_t)p.planes[t] * plan->nsites, s),
                  "zero tail profiles");
  MM_CHECK_CUDA(cudaMemsetAsync(w.counters, 0, (char*)w.error + sizeof(int) - (char*)w.counters, s),
                "zero queue state");
  int rc = MM_OK;
  if (schedule == MM_SCHEDULE_PERSISTENT) {
    MM_CHECK_ARG(plan->n == plan->n2 || !(fft_size(plan->n) && fft_size(plan->n2)),
                 "the persistent schedule needs one kernel for both windows (got %d, %d); use the batched one",
                 plan->n, plan->n2);
    const int waves = (plan->nsites + slots - 1) / slots;
    p.total_items = (long long)waves * slots * p.blocks_per_site;
    rc = launch_persistent_any(p, s);
  } else {
    for (int site0 = 0; site0 < plan->nsites && rc == MM_OK; site0 += slots) {
      const int batch = std::min(slots, plan->nsites - site0);
      for (int stage = 0; stage < 3 && rc == MM_OK; ++stage)
        for (int k = 0; k <= p.st[stage].steps && rc == MM_OK; ++k)
          rc = launch_batched_any(p, stage, k, site0, batch, s);
    }
  }
  if (rc != MM_OK || !check) return rc;
  MM_CHECK_CUDA(cudaStreamSynchronize(s), "propagation");
  int err = 0;
  MM_CHECK_CUDA(cudaMemcpy(&err, w.error, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
  if (err & 2) {
    set_error("a site window lies outside the screen volume (offsets out of range)");
    return MM_ERR_ARGUMENT;
  }
  if (err) {
    set_error("persistent propagation: a dependency wait timed out");
    return MM_ERR_TIMEOUT;
  }
  return MM_OK;
}
