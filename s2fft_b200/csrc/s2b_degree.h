// Degree recursion for d^l_{m,n}(theta) at fixed (m, n) with |m| < |n| (double).
//
//   d^{l+1} = a_l (cos(theta) - c_l) d^l - b_l d^{l-1},   c_l = m n / (l (l + 1)),
//   a_l = (2l + 1)(l + 1) / q_l,  q_l = sqrt(((l + 1)^2 - m^2)((l + 1)^2 - n^2)),
//   b_l = (l + 1) sqrt((l^2 - m^2)(l^2 - n^2)) / (l q_l),
// from the closed form at l = |n|:
//   d^j_{m,j}  = sqrt(C(2j, j+m)) cos^{j+m}(theta/2) sin^{j-m}(theta/2),
//   d^j_{m,-j} = (-1)^{m+j} sqrt(C(2j, j-m)) cos^{j-m}(theta/2) sin^{j+m}(theta/2).
// For growing l it runs in the growing or oscillating direction at every theta, so it is
// stable where the m-recursion is not (the degree recursion of Kostelec & Rockmore,
// J. Fourier Anal. Appl. 14 (2008) 145-179). Used by lowm.cu and precompute.cu.
#pragma once

#include <cuda_runtime.h>

namespace s2b {

struct DegreeCoef {
  double a, c, b;
};

// coefficients of the step l -> l + 1 (l >= |n| >= 1)
__device__ __forceinline__ DegreeCoef degree_coef(int l, int m, int n) {
  const double ld = (double)l, l1 = ld + 1.0, mm = (double)m * m, nn = (double)n * n;
  const double q = sqrt((l1 * l1 - mm) * (l1 * l1 - nn));
  DegreeCoef k;
  k.a = (2.0 * ld + 1.0) * l1 / q;
  k.c = (double)m * (double)n / (ld * l1);
  k.b = l1 * sqrt((ld * ld - mm) * (ld * ld - nn)) / (ld * q);
  return k;
}

// d^{|n|}_{m,n}(theta) = v 2^E, from lc = log2 cos(theta/2) and ls = log2 sin(theta/2)
__device__ __forceinline__ void degree_seed(double lc, double ls, int m, int n, double& v,
                                            int& E) {
  const int j = n < 0 ? -n : n;
  const int kc = n > 0 ? j + m : j - m;  // power of cos(theta/2)
  const int ks = 2 * j - kc;             // power of sin(theta/2)
  const double lb = 0.5 * (lgamma(2.0 * j + 1.0) - lgamma(kc + 1.0) - lgamma(ks + 1.0)) *
                    1.4426950408889634;  // log2 sqrt(binom(2j, kc))
  const double lg = lb + (double)kc * lc + (double)ks * ls;
  E = (int)floor(lg);
  v = exp2(lg - (double)E);
  if (n < 0 && ((m + j) & 1)) v = -v;
}

// one step of the recursion on (cur, prv) = (d^l, d^{l-1}) 2^-E; values above 2^64 move
// into the exponent (sc = 2^E)
__device__ __forceinline__ void degree_step(double a, double c, double b, double ct,
                                            double& cur, double& prv, int& E, double& sc) {
  const double nx = a * (ct - c) * cur - b * prv;
  prv = cur;
  cur = nx;
  if (fabs(cur) > 0x1p64) {
    cur *= 0x1p-64;
    prv *= 0x1p-64;
    E += 64;
    sc = ldexp(1.0, E);
  }
}

}  // namespace s2b
