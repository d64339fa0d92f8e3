// s2b_inverse_noalloc: the spin inverse transform with its workspace taken
// from a fixed device array of this library instead of from the caller.
//
// For callers that cannot allocate device memory: a plugin inside a host
// application that owns every allocation and hands over only the input and
// output buffers, or a path on which an allocation would synchronise the
// device. The array below is S2B_NOALLOC_SCRATCH_BYTES (32 MiB) and lives on
// every GPU that loads the library until the process exits; all calls on a
// device share it, so calls that overlap on the GPU race.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/s2b.h"
#include "s2b_internal.h"

namespace {

// Device-side storage. In host code this name is only a stand-in for the
// symbol, never a device address: the address comes from
// cudaGetSymbolAddress, per device, below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[S2B_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up on
// the first call for that device (with it current) and cached afterwards.
// The cache holds for the life of the device's primary context: after a
// cudaDeviceReset the module is loaded again and the array may move, so a
// program that resets a device must not call s2b_inverse_noalloc on it again.
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return s2b::set_last_error(S2B_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return s2b::set_last_error(S2B_ERR_INVALID, "s2b_inverse_noalloc: device ordinal >= 64");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      char msg[256];
      std::snprintf(msg, sizeof msg,
                    "s2b_inverse_noalloc: cudaGetSymbolAddress of the scratch array failed: %s",
                    cudaGetErrorString(e));
      return s2b::set_last_error(S2B_ERR_CUDA, msg);
    }
    g_noalloc_addr[dev] = ptr;
  }
  *out = g_noalloc_addr[dev];
  return S2B_OK;
}

}  // namespace

extern "C" int s2b_inverse_noalloc(s2b_plan* plan, const void* flm, void* f, void* stream) {
  size_t need = 0;
  int rc = s2b_workspace_size(plan, 0, &need);
  if (rc != S2B_OK) return rc;
  // the scratch array used is the current device's, so that device must hold the plan
  if ((rc = s2b::check_plan_device(plan)) != S2B_OK) return rc;
  if (need > S2B_NOALLOC_SCRATCH_BYTES) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "s2b_inverse_noalloc: this plan needs %zu bytes of scratch but the fixed "
                  "array holds %zu (S2B_NOALLOC_SCRATCH_BYTES); use s2b_inverse with a "
                  "caller-provided workspace, or a smaller batch",
                  need, (size_t)S2B_NOALLOC_SCRATCH_BYTES);
    return s2b::set_last_error(S2B_ERR_WORKSPACE, msg);
  }
  void* scratch = nullptr;
  if ((rc = scratch_address(&scratch)) != S2B_OK) return rc;
  // s2b_inverse zeroes the accumulation rows it sums into (on `stream`) and
  // writes every other scratch byte before reading it, so whatever an earlier
  // call left in the array does not reach this result.
  return s2b_inverse(plan, flm, f, scratch, S2B_NOALLOC_SCRATCH_BYTES, stream);
}
