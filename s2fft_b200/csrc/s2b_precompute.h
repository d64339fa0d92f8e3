// Precompute-kernel path: parameter blocks and launchers (precompute.cu).
#pragma once

#include <cuda_runtime.h>

namespace s2b {

struct KernelTableParams {
  int L, spin, reality, forward, complex_out;
  int nth;               // rings of the table
  const double* theta;   // ring colatitudes
  const double* weights; // forward: transform quadrature weights (nullptr: 1)
  const double* phi0;    // HEALPix ring phase (nullptr: none)
  const double* lbin;    // log2 sqrt(binom(2l, l+|s|))
  void* out;             // K [nth][L][M], M = L (reality) or 2L-1
};

struct PreContractParams {
  int L, nth, M, batch;
  int mshift;            // flm column of mi = 0 (L-1+m0)
  int mo;                // inverse: ftm column of mi = 0
  int ncol;              // inverse: ftm row width
  double sign;           // (-1)^s
  int conj;              // complex kernels: use conj(K) (adjoint transforms)
  const void* K;
  const void* in;
  void* out;
};

cudaError_t launch_kernel_table(bool fp64, const KernelTableParams& p, cudaStream_t s);
cudaError_t launch_pre_contract(bool fp64, bool forward, bool cplx, const PreContractParams& p,
                                cudaStream_t s);
cudaError_t launch_reality_mirror(bool fp64, void* flm, int B, int L, cudaStream_t s);

}  // namespace s2b
