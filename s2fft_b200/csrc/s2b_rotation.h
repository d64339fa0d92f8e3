// Rotation of spherical-harmonic coefficients (rotation.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace s2b {

// rows of a Wigner-d plane per row block (one CTA owns whole row blocks)
constexpr int kRotRowsMax = 8;
constexpr int kRotThreads = 256;
// upper bound on device waits on a neighbouring row block (each poll sleeps ~100 ns)
constexpr long kRotSpinLimit = 1L << 24;

struct RotParams {
  int L, batch;
  double alpha, beta, gamma;
  const void* flm;      // [batch][L][2L-1] coefficients (nullptr: planes only)
  void* out;            // [batch][L][2L-1] rotated coefficients
  const double* dl_in;  // caller planes [L][2L-1][2L-1] at beta (nullptr: Risbo on the device)
  double* dl_out;       // optional: the planes written in that layout
  // workspace (rotate_workspace_bytes):
  double* plane0;  // d^l for even l: row I = l+m, column K = l+n, row stride ld
  double* plane1;  // d^l for odd l
  int ld;          // 2L
  double* sq;      // sqrt(k), k in [0, 2L]
  double2* ea;     // exp(-i m alpha), m in [-(L-1), L-1]
  double2* eg;     // exp(-i n gamma)
  int* done;       // per row block: number of degrees completed
  int* err;        // nonzero when a wait on a neighbour ran out of its bound
  // row blocks: rows [rb * rows, (rb + 1) * rows) of each plane
  int rows, nrb;
};

size_t rotate_workspace_bytes(int L);
// carves the workspace into the planes, tables and flags
void rotate_bind_workspace(RotParams& p, void* ws);
cudaError_t launch_rotate(bool fp64, RotParams p, cudaStream_t s);

}  // namespace s2b
