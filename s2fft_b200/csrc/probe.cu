// Peak-rate probe used to state the FP32 / FP64 SIMT roofline denominators:
// eight independent FMA chains per thread, no memory traffic in the loop; mode 2 runs
// the chains as packed float pairs (fma.rn.f32x2, two FMAs per instruction).
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

__global__ void fma_chain_x2(int iters, float* out) {
  unsigned long long a[8];
  const float x = 1.0f + 1e-7f * threadIdx.x, y = 0.999999f;
  unsigned long long xx, yy;
  asm("mov.b64 %0, {%1, %1};" : "=l"(xx) : "f"(x));
  asm("mov.b64 %0, {%1, %1};" : "=l"(yy) : "f"(y));
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float u = (float)(2 * i + 1) * x, v = (float)(2 * i + 2) * x;
    asm("mov.b64 %0, {%1, %2};" : "=l"(a[i]) : "f"(u), "f"(v));
  }
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int i = 0; i < 8; ++i)
        asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[i]) : "l"(yy), "l"(xx));
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float u, v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(u), "=f"(v) : "l"(a[i]));
    s += u + v;
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int s2b_fma_probe(int fp64, int blocks, int iters, void* out, void* stream) {
  if (!out || blocks < 1 || iters < 1) return S2B_ERR_INVALID;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (fp64 == 2)
    fma_chain_x2<<<blocks, 256, 0, s>>>(iters, (float*)out);
  else if (fp64)
    fma_chain<double><<<blocks, 256, 0, s>>>(iters, (double*)out);
  else
    fma_chain<float><<<blocks, 256, 0, s>>>(iters, (float*)out);
  return cudaGetLastError() == cudaSuccess ? S2B_OK : S2B_ERR_CUDA;
}
