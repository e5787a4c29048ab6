// Allocation-free symmetric eigenvalue entry point, mbd_rsscs_eigvalsh_noalloc.
//
// Some callers cannot allocate device memory at the moment they need the
// eigenvalues: a host program that hands the GPU over to its own memory
// pool or arena and forbids other allocations, a real-time or signal-driven
// path where cudaMalloc's implicit device synchronisation and unbounded
// latency are not acceptable, or a process that has already used all device
// memory for its own data.  For them this file keeps the scratch of the
// tridiagonal reduction and of the eigenvalue multisection in one fixed
// file-scope device array; the caller passes only its matrix and output.
//
// The array is a __device__ variable: every GPU that loads this library
// holds kScratchBytes of it until the process exits.  Host code cannot use
// its name as a device address, so the first call on each device (with that
// device current) looks the address up once with cudaGetSymbolAddress.
// Every call ends by reading the error flag back and synchronising the
// caller's stream, so no call may be made while a stream is being captured.
// All calls share the one array and it keeps the last call's contents: the parts that
// must start at zero are cleared on every call, and calls that overlap on
// the GPU (different streams, or host threads on the same device) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "kernels.h"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int kNoAllocMaxN = MBD_NOALLOC_MAX_N;
constexpr size_t kScratchBytes = (size_t)4 << 20;   // 4 MiB: room for kNoAllocMaxN with 160 CTAs
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceSetup {
  bool done = false;
  char* base = nullptr;   // device address of g_noalloc_scratch on that device
  int sms = 0;
  int ctas_per_sm = 1;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

__global__ void store_job(TridiagJob* dst, TridiagJob job) { *dst = job; }

// Scratch layout: [err][job][d | e | e^2][tridiagonal-reduction workspace].
constexpr size_t kHeader = 512;

size_t scratch_need(int n, int G) {
  return kHeader + 3 * sizeof(double) * (size_t)((n + 31) / 32 * 32) + tridiag_workspace_bytes(n, G);
}

int setup_device(int dev, DeviceSetup** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  DeviceSetup& s = g_setup[dev];
  if (!s.done) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return MBD_ERR_DEVICE;
    if (cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MBD_ERR_DEVICE;
    s.ctas_per_sm = tridiag_max_ctas_per_sm();
    if (s.ctas_per_sm < 1) return MBD_ERR_DEVICE;
    if (init_eigval_attributes() != cudaSuccess) return MBD_ERR_DEVICE;
    s.base = static_cast<char*>(ptr);
    s.done = true;
  }
  *out = &s;
  return MBD_OK;
}

}  // namespace
}  // namespace mbd

using namespace mbd;

extern "C" int mbd_rsscs_eigvalsh_noalloc(double* H, int n, int ld, double* w, void* stream) {
  if (!H || !w || n < 1 || ld < n) return MBD_ERR_ARG;
  if (n > kNoAllocMaxN) return MBD_ERR_TOO_LARGE;
  // 16-byte row starts for the kernel's vector copies
  if ((ld % 2) != 0 || (reinterpret_cast<uintptr_t>(H) % 16) != 0) return MBD_ERR_ARG;
  // a launch error left behind by the caller's own earlier work is not this
  // call's: clear it so that the check after the launches sees only ours
  (void)cudaGetLastError();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MBD_ERR_DEVICE;
  DeviceSetup* ds = nullptr;
  int st = setup_device(dev, &ds);
  if (st != MBD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nt = (n + kTrdTile - 1) / kTrdTile;
  const int G = std::max(1, std::min(std::min(ds->sms * ds->ctas_per_sm, nt * (nt + 1) / 2), kTridiagMaxGroup));
  if (scratch_need(n, G) > kScratchBytes) return MBD_ERR_TOO_LARGE;
  char* base = ds->base;
  int* err = reinterpret_cast<int*>(base);
  TridiagJob* job = reinterpret_cast<TridiagJob*>(base + 256);
  const size_t npad = (size_t)(n + 31) / 32 * 32;
  double* d = reinterpret_cast<double*>(base + kHeader);
  double* e = d + npad;
  double* e2 = e + npad;
  char* ws = base + kHeader + 3 * sizeof(double) * npad;
  const size_t wsb = tridiag_workspace_bytes(n, G);
  if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return MBD_ERR_DEVICE;
  store_job<<<1, 1, 0, s>>>(job, TridiagJob{H, n, ld, d, e});
  if (launch_tridiag(job, 1, 1, G, ws, wsb, n, err, s) != cudaSuccess) return MBD_ERR_DEVICE;
  launch_tridiag_eigenvalues_scratch(d, e, n, w, e2, s);
  if (cudaGetLastError() != cudaSuccess) return MBD_ERR_DEVICE;
  // the error flag comes back on the caller's stream (a synchronous copy on
  // the legacy stream would also wait for unrelated work on the device)
  int herr = 0;
  if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MBD_ERR_DEVICE;
  if (cudaStreamSynchronize(s) != cudaSuccess) return MBD_ERR_DEVICE;
  return herr ? herr : MBD_OK;
}
