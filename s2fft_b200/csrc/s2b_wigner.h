// Wigner (SO(3)) stage launchers (wigner.cu).
#pragma once

#include <cuda_runtime.h>

namespace s2b {

// real0: slice n = 0 of a real signal (orders weighted 0 / 1 / 2 for m < 0 / = 0 / > 0)
cudaError_t launch_gather_n(bool fp64, const void* flmn, void* tmp, int B, int N, int L, int n,
                            int real0, cudaStream_t s);
cudaError_t launch_scatter_n(bool fp64, const void* tmp, void* flmn, int B, int N, int L, int n,
                             int L0, cudaStream_t s);
cudaError_t launch_wigner_mirror(bool fp64, void* flmn, int B, int N, int L, cudaStream_t s);
cudaError_t launch_gamma_inverse(bool fp64, const void* fban, void* f, int B, int N, long npix,
                                 int reality, cudaStream_t s);
cudaError_t launch_gamma_forward(bool fp64, const void* f, void* fban, int B, int N, long npix,
                                 int reality, cudaStream_t s);

}  // namespace s2b
