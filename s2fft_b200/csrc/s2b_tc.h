// Tensor-core (tcgen05, BF16x3) batched precompute forward contraction (tc.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace s2b {

struct TcParams {
  int L, nth, M, B;
  int nlt, ntc, nbg;      // filled by the launcher
  int mshift;             // flm column of mi = 0
  float sign;             // (-1)^s
  const __nv_bfloat16* Ap;  // packed kernel  [M][nlt][ntc][hi/lo][128 x 64]
  const __nv_bfloat16* Bp;  // packed spectra [M][nbg][ntc][hi/lo][128 x 64]
  float2* out;            // flm [B][L][2L-1]
  int* status;
};

size_t tc_packed_a_bytes(int nth, int L, int M);
size_t tc_packed_b_bytes(int nth, int B, int M);
cudaError_t launch_tc_pack_a(const float* K, int nth, int L, int M, void* out, cudaStream_t s);
cudaError_t launch_tc_pack_b(const void* X, int B, int nth, int M, void* out, cudaStream_t s);
cudaError_t launch_tc_forward(TcParams p, cudaStream_t s);

}  // namespace s2b
