// Peak-rate probe used to state the FP32 / FP64 SIMT roofline denominators:
// eight independent FMA chains per thread, no memory traffic in the loop.
#include <cuda_runtime.h>

#include "../../include/s2b.h"

namespace {
template <typename Real>
__global__ void fma_chain(int iters, Real* out) {
  Real a[8];
  const Real x = (Real)(1.0 + 1e-7 * threadIdx.x), y = (Real)(0.999999);
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = (Real)(i + 1) * x;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = fma(a[i], y, x);
  }
  Real s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int s2b_fma_probe(int fp64, int blocks, int iters, void* out, void* stream) {
  if (!out || blocks < 1 || iters < 1) return S2B_ERR_INVALID;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (fp64)
    fma_chain<double><<<blocks, 256, 0, s>>>(iters, (double*)out);
  else
    fma_chain<float><<<blocks, 256, 0, s>>>(iters, (float*)out);
  return cudaGetLastError() == cudaSuccess ? S2B_OK : S2B_ERR_CUDA;
}
