// Fixed device scratch for the allocation-free RK4 entry point
// (teuk_b200_step_static_scratch).
//
// Some callers cannot obtain device memory when they want to step: a host
// framework whose caching allocator has already reserved the device for its
// own tensors (a driver allocation then fails or forces it to release its
// cache), or a loop with a latency budget that rules out a driver
// allocation call.  For them the three RK slope buffers of the linear band
// pipeline come from one statically sized device array instead of memory
// owned by the pipeline.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace teuk_b200 {

// Complex values per slope buffer.  Three buffers of 2^19 complex128 values
// (8 MiB each, 24 MiB in all) hold a band state of up to 524,288 values,
// e.g. one solve of m = -4..4, ell <= 16 at up to 1354 radial points.
inline constexpr std::size_t kStaticSlopeCapacity = std::size_t{1} << 19;

// Device address of the static slope array on the current device
// (3 * kStaticSlopeCapacity complex values, 256-byte aligned).  The first
// call on each device resolves the symbol, which loads the module that owns
// the array; later calls return the cached address without any CUDA call
// other than cudaGetDevice.  The cached address outlives a cudaDeviceReset
// of that device, which frees the array: the entry point must not run on a
// device after the host process reset it.
cudaError_t static_slope_buffers(double2** base);

}  // namespace teuk_b200
