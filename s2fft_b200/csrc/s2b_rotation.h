// Rotation of spherical-harmonic coefficients (rotation.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace s2b {

constexpr int kRotThreads = 256;     // threads per CTA at most (8 warps)
constexpr int kRotMaxCluster = 8;    // CTAs of a cluster (portable limit)
constexpr int kRotMaxL = 8192;       // largest band-limit of the recurrence path

// a double with a separate binary exponent: m * 2^e (m in [0.5, 1) or 0), or a start
// value v * 2^k of the recurrence (k < 0 only below 2^-960)
struct RotXD {
  double m;
  int e;
  int pad;
};

struct RotParams {
  int L, batch;
  double alpha, beta, gamma;
  const void* flm;      // [batch][L][2L-1] coefficients (nullptr: planes only)
  void* out;            // [batch][L][2L-1] rotated coefficients
  const double* dl_in;  // caller planes [L][2L-1][2L-1] at beta (nullptr: recurrence)
  double* dl_out;       // planes written in that layout (every entry, zeros included)
  // cos(beta), c^2, s^2, (cs)^2 with c = cos(beta/2), s = sin(beta/2), and the signs of c, s
  double cb, c2, s2, cs2;
  int c_neg, s_neg;
  // workspace (rotate_workspace_bytes):
  double2* T;      // [L][L] (1/sqrt((l+1)^2-k^2), sqrt(l^2-k^2)) for k <= l, else 0
  double4* UVQ;    // [L][L] ((l+1)(2l+1) T.x, T.y/(l(2l+1)), -m/(l(l+1)), 0) for m <= l, else 0
  RotXD* start;    // [L][2L-1] d^{l}_{l,a}(beta) at [l][L-1+a], |a| <= l
  RotXD* carry;    // [ceil(L/32)][2L-1] segment products of the start table
  double2* ea;     // exp(-i m alpha), m in [-(L-1), L-1]
  double2* eg;     // exp(-i n gamma)
  // launch shape of the recurrence kernel: warps per CTA and CTAs per cluster
  int nw, nr;
};

size_t rotate_workspace_bytes(int L);
// carves the workspace into the tables
void rotate_bind_workspace(RotParams& p, void* ws);
cudaError_t launch_rotate(bool fp64, RotParams p, cudaStream_t s);

}  // namespace s2b
