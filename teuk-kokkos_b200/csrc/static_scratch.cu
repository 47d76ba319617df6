// Static slope storage for the allocation-free RK4 entry point.  The array
// lives in its own translation unit, so only processes that call that entry
// point load it onto a device.
#include <mutex>

#include "static_scratch.h"

namespace teuk_b200 {

// k1 / stage-4 input, k2, weighted slope sum: every element a step reads is
// written earlier in the same step, so nothing here needs to start at zero.
static __device__ __align__(256) double2
    g_static_slopes[3 * kStaticSlopeCapacity];

cudaError_t static_slope_buffers(double2** base) {
  constexpr int kMaxDevices = 64;
  static std::mutex mutex;
  static void* cached[kMaxDevices] = {};
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return err;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mutex);
  if (cached[device] == nullptr) {
    void* address = nullptr;
    err = cudaGetSymbolAddress(&address, g_static_slopes);
    if (err != cudaSuccess) return err;
    cached[device] = address;
  }
  *base = static_cast<double2*>(cached[device]);
  return cudaSuccess;
}

}  // namespace teuk_b200
