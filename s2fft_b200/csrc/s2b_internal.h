// Internal declarations shared by the host plan code and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "s2b_fft.h"

struct s2b_plan;

namespace s2b {

// Coefficient tables indexed by m are stored with kPadLo zero rows on both
// sides of 0 <= m < L (row = m + kPadLo), so that every R-step group of the
// latitudinal kernel is one fixed-size contiguous copy.
constexpr int kPadLo = 8;
__host__ __device__ inline int tab_rows(int L) { return L + 2 * kPadLo; }
__host__ __device__ inline int round4(int x) { return (x + 3) & ~3; }

// One recursed ring (pole rings are handled separately, in closed form).
struct RingInfo {
  double B;    // 2 cot(theta)
  double A;    // 2 / sin(theta)
  double lc;   // log2 cos(theta/2)
  double ls;   // log2 sin(theta/2)
};

cudaError_t launch_lambda(bool fp64, int L, int spin, int nhalf, const RingInfo* rings, int nrings,
                          int Ls, void* lam, cudaStream_t s);

// FFT descriptors (host copies, in the order of the requested lengths; their table
// offsets index tw / chirp / bf) and the device tables they refer to.
struct FFTSet {
  std::vector<FFTDesc> host;
  void* tw = nullptr;
  void* chirp = nullptr;
  void* bf = nullptr;
};
// Builds the set for `count` lengths (each >= 2) in float or double; every device
// allocation is appended to *allocs (the caller frees them).
int build_fft_set(const int* lengths, int count, bool fp64, std::vector<void*>* allocs,
                  FFTSet* out);

// Records msg as the calling thread's s2b_last_error() text and returns code.
int set_last_error(int code, const char* msg);

// S2B_OK when the current device is the one the plan was created on, else an
// S2B_ERR_INVALID status with the message set.
int check_plan_device(const s2b_plan* p);

// cudaMalloc through the library's allocation counter (s2b_device_alloc_count).
cudaError_t dev_malloc_void(void** ptr, size_t bytes);
template <typename T>
cudaError_t dev_malloc(T** ptr, size_t bytes) {
  return dev_malloc_void(reinterpret_cast<void**>(ptr), bytes);
}

}  // namespace s2b
