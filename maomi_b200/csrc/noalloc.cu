// Site propagation for callers that cannot allocate device memory.
//
// Some hosts of this library own the whole device heap (they reserve it at
// start-up for their own pool and hand out no scratch pointers), and some
// code paths must not call cudaMalloc once they are running (a real-time
// acquisition loop, or code that is recording a stream).  Those callers still
// own their inputs and outputs, but cannot provide the propagation
// workspace.  mm_propagate_sites_noalloc runs the same propagation with the
// workspace taken from a fixed file-scope device array instead.
//
// Limits and rules:
//  * The array holds kNoAllocScratchBytes (32 MiB) on every GPU that loads
//    the library, for the life of the process.  At n = n2 = 256 that is room
//    for 31 sites in flight (1 MiB each); calls needing more are rejected.
//  * The first call on a device looks up the array's device address (with
//    that device current) and caches it; make that first call before any
//    stream capture begins.  The cache assumes the device keeps one primary
//    context for the life of the process (as CUDA runtime and PyTorch
//    programs do); if the cached address no longer belongs to the current
//    context (after cudaDeviceReset, say) it is looked up again.
//  * Every call shares the array and it keeps the last call's contents; the
//    propagation clears its queue counters and error flag itself and writes
//    every field buffer before reading it.  Calls whose work overlaps on the
//    GPU (other streams, other host threads) race on the array: serialise them.
//  * No cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>

#include "common.cuh"

namespace mm {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
int noalloc_scratch(void** out) {
  int dev = 0;
  MM_CHECK_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  MM_CHECK_ARG(dev >= 0 && dev < kMaxDevices, "device ordinal %d beyond %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_addr[dev]) {
    // A context torn down and recreated (cudaDeviceReset) reloads the module;
    // an address that is no longer device memory of this context is stale.
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, g_noalloc_addr[dev]) != cudaSuccess || attr.type != cudaMemoryTypeDevice ||
        attr.device != dev) {
      (void)cudaGetLastError();
      g_noalloc_addr[dev] = nullptr;
    }
  }
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    MM_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return MM_OK;
}

}  // namespace
}  // namespace mm

extern "C" int mm_propagate_sites_noalloc(const mm_stage_plan* plan, int schedule, int slots, int check, void* stream) {
  using namespace mm;
  MM_CHECK_ARG(plan != nullptr, "plan is NULL");
  MM_CHECK_ARG(slots >= 1, "slots must be >= 1 (got %d)", slots);
  MM_CHECK_ARG(plan->nsites >= 1, "nsites must be >= 1 (got %d)", plan->nsites);
  // size the request as mm_propagate_sites will run it: clamped to the site
  // count and balanced over the waves
  slots = propagation_slots(plan->nsites, slots, schedule);
  const size_t need = mm_propagate_workspace_size(plan, slots, schedule);
  if (need > kNoAllocScratchBytes) {
    const size_t one = mm_propagate_workspace_size(plan, 1, schedule);
    set_error("no-alloc propagation needs %zu bytes of scratch for %d sites in flight; the static array holds %zu "
              "bytes (at most about %zu sites in flight for this plan)",
              need, slots, kNoAllocScratchBytes, one ? kNoAllocScratchBytes / one : size_t(0));
    return MM_ERR_ARGUMENT;
  }
  void* scratch = nullptr;
  if (int rc = noalloc_scratch(&scratch)) return rc;
  return mm_propagate_sites(plan, schedule, slots, scratch, kNoAllocScratchBytes, check, stream);
}
