// Per-plan tables of the latitudinal recursion shared by the forward and inverse kernels:
// lambda(theta_r, m) for every recursed ring, and the l-class geometry used to size the
// coefficient and sum tables (l = j + C q, C classes of 64 slots).
#include <cuda_runtime.h>

#include "s2b_internal.h"

namespace s2b {

// lambda(theta_r, m) = 2 (n - m cos theta) / sin theta = n A_r - m B_r, evaluated in
// double and rounded once; layout [half][m + kPadLo][Ls], zero outside 0 <= m < L.
template <typename Real>
__global__ void lambda_kernel(int L, int spin, int nhalf, const RingInfo* __restrict__ rings,
                              int nrings, int Ls, Real* __restrict__ out) {
  const int TR = tab_rows(L);
  const long total = (long)nhalf * TR * Ls;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % Ls);
    const int mr = (int)((idx / Ls) % TR);
    const int half = (int)(idx / ((long)Ls * TR));
    const int m = mr - kPadLo;
    const int n = half == 0 ? -spin : spin;
    double v = 0.0;
    if (r < nrings && m >= 0 && m < L) v = fma(-(double)m, rings[r].B, (double)n * rings[r].A);
    out[idx] = (Real)v;
  }
}

cudaError_t launch_lambda(bool fp64, int L, int spin, int nhalf, const RingInfo* rings, int nrings,
                          int Ls, void* lam, cudaStream_t s) {
  const long total = (long)nhalf * tab_rows(L) * Ls;
  long blocks = (total + 255) / 256;
  if (blocks > 8192) blocks = 8192;
  if (fp64)
    lambda_kernel<double><<<(int)blocks, 256, 0, s>>>(L, spin, nhalf, rings, nrings, Ls, (double*)lam);
  else
    lambda_kernel<float><<<(int)blocks, 256, 0, s>>>(L, spin, nhalf, rings, nrings, Ls, (float*)lam);
  return cudaGetLastError();
}

}  // namespace s2b
