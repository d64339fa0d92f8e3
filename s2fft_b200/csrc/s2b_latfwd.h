// Forward latitudinal step, restart formulation (latfwd.cu).
#pragma once

#include <cuda_runtime.h>

#include "s2b_internal.h"

namespace s2b {

// l is tiled in blocks of 32 consecutive degrees; a CTA takes the pair of blocks
// (p, NB-1-p), so that every CTA carries about the same number of (l, m) pairs.
constexpr int kFwdBlock = 32;
__host__ __device__ inline int fwd_nblocks(int L) { return 2 * ((L + 2 * kFwdBlock - 1) / (2 * kFwdBlock)); }

// Split of the inverse kernel along m: block pair q (blocks q and NB-1-q) runs as up to
// kInvSegMax segments with about the same number of block-steps each (m from the pair's top
// degree down: one block above the lower block's top degree, two below). Boundary k of
// kInvSegMax (k = 0..kInvSegMax, decreasing in k, boundary kInvSegMax = 0) is a multiple
// of 8, so every segment starts on a group boundary; a run with S segments (S dividing
// kInvSegMax) uses every (kInvSegMax / S)-th boundary. Segment k >= 1 restarts the states
// begun above its top boundary b from exact values at m = b - 1.
constexpr int kInvSegMax = 8;
__host__ __device__ inline int inv_mbound(int L, int NB, int q, int k) {
  int top = (NB - 1 - q) * 32 + 31;
  if (top > L - 1) top = L - 1;
  if (k <= 0) return top + 1;
  if (k >= kInvSegMax) return 0;
  int lo = q * 32 + 32;
  if (lo > top + 1) lo = top + 1;
  const int w1 = top + 1 - lo, W = w1 + 2 * lo, t = (int)((long)k * W / kInvSegMax);
  int b = t <= w1 ? top + 1 - t : lo - (t - w1) / 2;
  b &= ~7;
  return b < 0 ? 0 : b;
}

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
  // optional restart tables of the inverse kernel's m-split, [kInvSegMax - 1][table]: for
  // boundary k (inv_mbound) states with M >= b restart at b - 1 (b > 0), others keep M
  int* Mst1;
  void* Vst1;
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
  // equator-symmetric mode (spin 0): the nrings rings are the northern members of ring
  // pairs (theta, pi - theta) plus the equator, G holds per pair (E, O) = G(theta) +- G(pi -
  // theta) (E = G, O = 0 for the equator) and Gs counts pairs; d^l_{m,0}(pi - theta) =
  // (-1)^(l+m) d^l_{m,0}(theta), so degree l projects E where l + m is even, O where odd
  int sym;
  // with sym, spin != 0: d^l_{m,n}(pi - theta) = (-1)^(l+m) d^l_{m,-n}(theta), so this half's
  // recursion also serves the other half's mirrored ring: G holds per pair and parity the
  // Real4 {G_h(theta), +-G_{1-h}(pi - theta)} and both halves' sums are updated
  int cross;
  int tab_stride;           // ring stride of Mst / Vst (0: nrings)
  // split along m as in the inverse kernel (inv_mbound): restart tables
  // [kInvSegMax - 1][table] (nullptr: one segment) and the number of segments (1, 2, 4, 8)
  const int* Mst1;
  const void* Vst1;
  int nseg;
};

// Inverse latitudinal step, blocked layout (latinv.cu).
struct Inv2Params {
  int L, nrings, nhalf, batch, NB;
  const int* Mst;           // start tables of these rings (FwdStartParams layout)
  const void* Vst;
  const int* Mst1;          // restart tables of the m-split (nullptr: one segment)
  const void* Vst1;
  int nseg;                 // segments along m: 1, 2, 4 or 8 (with Mst1)
  // equator-symmetric mode (spin 0): the nrings rings are the northern members of ring
  // pairs (ring q and tab_stride - 1 - q) plus the equator; a lane sums the degrees with
  // l + m even (E) and odd (O) apart and adds E + O to ring q and E - O to its mirror
  int sym;
  int tab_stride;           // ring stride of the start tables and ring count (0: nrings)
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

// Persistent latitudinal launches over the plans of a batch (one kernel variant: the same
// precision, layout and symmetry): the plans' parameter blocks travel in the kernel
// arguments, and every CTA takes (plan, tile) items from a device counter until none are
// left. start[i] = tiles of plans 0..i-1; counter is zeroed by the launcher (stream-ordered).
constexpr int kBatchPlans = 48;
struct Inv2Batch {
  int nplans;
  int start[kBatchPlans + 1];
  int* counter;
  Inv2Params p[kBatchPlans];
};
struct Fwd2Batch {
  int nplans;
  int start[kBatchPlans + 1];
  int* counter;
  Fwd2Params p[kBatchPlans];
};
// kernel parameters are limited to 32764 bytes
static_assert(sizeof(Inv2Batch) <= 32000 && sizeof(Fwd2Batch) <= 32000, "batch parameters");

// nplans <= kBatchPlans plans of one variant; counter: one device int; per_sm: CTAs per SM
// of the launch (0: as many as fit)
cudaError_t launch_inv2_batch(bool fp64, bool dual, const Inv2Params* ps, int nplans,
                              int* counter, int per_sm, cudaStream_t s);
cudaError_t launch_fwd2_batch(bool fp64, bool dual, const Fwd2Params* ps, int nplans,
                              int* counter, int per_sm, cudaStream_t s);

cudaError_t launch_fwd_start(bool fp64, const FwdStartParams& p, cudaStream_t s);
cudaError_t launch_fwd2(bool fp64, bool dual, const Fwd2Params& p, cudaStream_t s);
size_t fwd_start_bytes(bool fp64, int L, int nhalf, int nrings);
int fwd_group(bool fp64);  // steps per group of the forward kernel

}  // namespace s2b
