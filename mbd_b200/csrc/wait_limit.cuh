// Limit of the bounded device-side waits (flag polls, group barriers,
// mbarrier waits), in SM clock cycles.  A wait that runs longer sets
// MBD_ERR_TIMEOUT in the context's error flag and returns; every other wait
// sees the flag and returns too, so a stuck dependency ends the launch
// instead of hanging the GPU.
//
// The library is built without relocatable device code, so every
// translation unit that waits holds its own copy of the limit; each exports
// a setter (kernels.h) and mbd_rsscs_set_option(MBD_OPT_WAIT_LIMIT_S) calls
// all of them.  The value lives in device memory of the current device and
// is read when a wait starts, so captured CUDA graphs follow changes.
#pragma once

#include <cuda_runtime.h>

namespace mbd {

constexpr long long kDefaultWaitCycles = 4000000000LL;   // ~2 s at 1965 MHz

static __device__ long long g_wait_limit_cycles = kDefaultWaitCycles;

__device__ __forceinline__ long long wait_limit_cycles() { return *(volatile long long*)&g_wait_limit_cycles; }

}  // namespace mbd

#define MBD_WAIT_LIMIT_SETTER(fn)                                                  \
  cudaError_t fn(long long cycles) {                                               \
    return cudaMemcpyToSymbol(::mbd::g_wait_limit_cycles, &cycles, sizeof(cycles)); \
  }
