// Library-level entry points: version, error reporting, device check.
#include <atomic>
#include <string>

#include "common.cuh"

namespace mm {

namespace {
thread_local std::string g_error;
std::atomic<unsigned long long> g_launches{0};
}

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
}

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  return MM_ERR_CUDA;
}

}  // namespace mm

extern "C" int mm_version(void) { return 100; }

extern "C" const char* mm_last_error(void) { return mm::g_error.c_str(); }

extern "C" unsigned long long mm_launch_count(void) { return mm::g_launches.load(std::memory_order_relaxed); }

extern "C" int mm_device_supported(void) {
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess) return 0;
  return major == 10 && minor == 0;
}

extern "C" size_t mm_struct_size(const char* name) {
  if (!name) return 0;
  const std::string n(name);
  if (n == "mm_pupil_desc") return sizeof(mm_pupil_desc);
  if (n == "mm_base_desc") return sizeof(mm_base_desc);
  if (n == "mm_stage_desc") return sizeof(mm_stage_desc);
  if (n == "mm_stage_plan") return sizeof(mm_stage_plan);
  if (n == "mm_item_class") return sizeof(mm_item_class);
  if (n == "mm_local_desc") return sizeof(mm_local_desc);
  if (n == "mm_surrogate_desc") return sizeof(mm_surrogate_desc);
  if (n == "mm_scan_planes") return sizeof(mm_scan_planes);
  if (n == "mm_scan_desc") return sizeof(mm_scan_desc);
  if (n == "mm_scan_conv") return sizeof(mm_scan_conv);
  return 0;
}
