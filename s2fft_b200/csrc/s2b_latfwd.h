// Forward latitudinal step, restart formulation (latfwd.cu).
#pragma once

#include <cuda_runtime.h>

#include "s2b_internal.h"

namespace s2b {

// l is tiled in blocks of 32 consecutive degrees; a CTA takes the pair of blocks
// (p, NB-1-p), so that every CTA carries about the same number of (l, m) pairs.
constexpr int kFwdBlock = 32;
__host__ __device__ inline int fwd_nblocks(int L) { return 2 * ((L + 2 * kFwdBlock - 1) / (2 * kFwdBlock)); }

// Start table of the forward recursion.
//   Mst [nhalf][NB][nrings]      first m of the recursion for (ring, block), a group start,
//                                 -1 when no degree of the block is significant on the ring
//   Vst [nhalf][NB][nrings][32]  (dt_M, dt_{M+1}) of each degree of the block, monic form
struct FwdStartParams {
  int L, L0, spin, nhalf, nrings, NB;
  double floor_log2;        // |d| below 2^floor_log2 is dropped from the projection
  int group;                // steps per group of the main kernel (starts are group starts)
  const RingInfo* rings;
  const double* lbin;       // log2 sqrt(binom(2l, l+|s|))
  const double* g;          // [m][l] monic scale
  int* Mst;
  void* Vst;
};

struct Fwd2Params {
  int L, nrings, nhalf, batch, NB;
  const int* Mst;
  const void* Vst;
  const void* Hb;           // [NB][tab_rows][32] h_{l,m}, l = 32 block + lane; 0 for m > l
  const void* lam;          // [nhalf][tab_rows][Ls]
  int Ls;
  const void* G;            // [batch][nhalf][tab_rows][Gs] weighted ring spectra (Real4 when dual)
  int Gs;
  void* acc;                // [batch][nhalf][L (m)][NB*32 (l)] projected sums (Real4 when dual)
  int* status;
  int tile;                 // 0: default rings per warp, 1: half of it (more CTAs)
  int mlo;                  // orders m < mlo are left to the degree recursion (lowm.cu)
};

// Inverse latitudinal step, blocked layout (latinv.cu).
struct Inv2Params {
  int L, nrings, nhalf, batch, NB;
  const int* Mst;           // start tables of these rings (FwdStartParams layout)
  const void* Vst;
  const void* Hb;           // [NB][tab_rows][32]
  const void* lam;          // [nhalf][tab_rows][Ls]
  int Ls;
  const void* F;            // [batch][nhalf][NB][tab_rows][32] coefficients (Real4 when dual)
  void* ftm;                // [batch][nrows][ncol] ring spectra, accumulated with atomics
  const int* ring_row;
  int nrows, ncol, mo;
  int* status;
  int tile;                 // 0: default rings per lane, 1: one ring per lane (more CTAs)
  int mlo;                  // orders m < mlo are left to the degree recursion (lowm.cu)
};
cudaError_t launch_inv2(bool fp64, bool dual, const Inv2Params& p, cudaStream_t s);

cudaError_t launch_fwd_start(bool fp64, const FwdStartParams& p, cudaStream_t s);
cudaError_t launch_fwd2(bool fp64, bool dual, const Fwd2Params& p, cudaStream_t s);
size_t fwd_start_bytes(bool fp64, int L, int nhalf, int nrings);
int fwd_group(bool fp64);  // steps per group of the forward kernel

}  // namespace s2b
