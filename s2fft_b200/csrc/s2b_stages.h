// Parameters and launchers of the element-wise stages (stages.cu).
#pragma once

#include <cuda_runtime.h>

namespace s2b {

struct StageParams {
  int L, L0, spin, batch;
  int nclass, Q;        // l classes of the latitudinal tiling, l = j + C q (Q padded)
  int TR, Gs;           // table rows (m + kPadLo) and forward spectra row stride
  int nhalf, dual;
  int nrows, ncol, mo;  // ftm / G row count, ftm columns, column offset
  int pole_south, pole_north;  // rows of the closed-form pole rings (-1: none)
  int Lp;               // 0: class layouts (l = j + C q); > 0: blocked layouts, inverse table
                        // F [C blocks][m][Q = 32] with l = 32 j + q, forward sums [m][Lp] by l
  const double* g;      // [m][l] monic scale g_{l,m}
  const void* flm;      // inverse input  [b][L][2L-1]
  void* F;              // inverse recursion table
  void* ftm;            // inverse ring spectra
  const void* G;        // forward weighted spectra
  const void* acc;      // forward projected sums
  void* flm_out;        // forward output
  size_t ftm_zero_bytes;  // > 0: launch_prologue zeroes that many bytes of ftm first
  int pole_blocks;      // set by launch_prologue: the pole rows ride on the prologue's grid
  int zero_ftm;         // set by launch_prologue: the prologue's CTAs zero ftm themselves
};

// the inverse coefficient table and the closed-form pole rows (pole_south / pole_north)
cudaError_t launch_prologue(bool fp64, const StageParams& p, cudaStream_t s);
cudaError_t launch_epilogue(bool fp64, const StageParams& p, cudaStream_t s);
cudaError_t launch_axpy(bool fp64, long n, double a, const void* x, void* y, cudaStream_t s);
cudaError_t launch_sub(bool fp64, long n, const void* x, const void* y, void* z, cudaStream_t s);

}  // namespace s2b
