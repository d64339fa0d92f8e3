// Orders m < |spin| of the latitudinal step by the degree recursion (lowm.cu).
#pragma once

#include <cuda_runtime.h>

#include "s2b_internal.h"

namespace s2b {

// The latitudinal kernels leave out the orders m < mlo (mlo = |spin| for spin != 0);
// these two kernels add them, on the same rings and tables as the kernel they complete.
struct LowmParams {
  int L, spin, nhalf, batch, nrings, NB, mlo;
  const RingInfo* rings;   // the recursed rings, in the order of the kernel they complete
  const double* g;         // [m][l] monic scale (d = dt g)
  // synthesis (completes lat_inv2): ftm[b][ring_row[r]][L-1 +- m + mo] += sum_l dt F
  const void* F;           // [batch][nhalf][NB][tab_rows][32]
  void* ftm;
  const int* ring_row;
  int nrows, ncol, mo;
  // projection (completes lat_fwd2): acc[b][half][m][l] += sum_r dt G[b][half][m][r]
  const void* G;           // [batch][nhalf][tab_rows][Gs]
  int Gs;
  void* acc;               // [batch][nhalf][L][NB * 32]
};

cudaError_t launch_lowm_synth(bool fp64, const LowmParams& p, cudaStream_t s);
cudaError_t launch_lowm_project(bool fp64, const LowmParams& p, cudaStream_t s);

}  // namespace s2b
