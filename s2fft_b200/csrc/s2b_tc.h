// Tensor-core (tcgen05, BF16x3) batched precompute forward contraction (tc.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace s2b {

struct TcParams {
  int L, nth, M, B;
  int rows, kdim;         // output rows (l forward, t inverse) and summation length
  int cplx;               // complex kernel: K dimension doubled ([Re K | Im K])
  int nlt, ntc, nbg;      // filled by the launcher
  float sign;             // (-1)^s
  const __nv_bfloat16* Ap;  // packed kernel  [M][nlt][ntc][hi/lo][128 x 64]
  const __nv_bfloat16* Bp;  // packed data    [M][nbg][ntc][hi/lo][128 x 64]
  float2* out;            // out[b * out_map + row * out_row + out_col0 + mi]
  long out_map;
  int out_row, out_col0;
  int* status;
};

// kdim = summation length, rows = output rows (forward: kdim = nth, rows = L; inverse:
// kdim = L, rows = nth)
// cplx: complex kernel (HEALPix), packed with a doubled K dimension
size_t tc_packed_a_bytes(int kdim, int rows, int M, int cplx);
size_t tc_packed_b_bytes(int kdim, int B, int M, int cplx);
// K [nth][L][M] float -> packed A; transposed = 0: rows l, k = t (forward);
// transposed = 1: rows t, k = l (inverse)
cudaError_t launch_tc_pack_a(const float* K, int nth, int L, int M, int transposed, int cplx,
                             void* out, cudaStream_t s);
// data element (map b, summation index q, column mi) at X[b in_map + q in_row + in_col0 + mi]
cudaError_t launch_tc_pack_b(const void* X, int B, int kdim, int M, long in_map, int in_row,
                             int in_col0, int cplx, void* out, cudaStream_t s);
cudaError_t launch_tc_forward(TcParams p, cudaStream_t s);

}  // namespace s2b
