// Fourier-Wigner SO(3) transforms and the spin-subset lifting ops.
//
// Replaces upstream s2fft:
//   precompute_transforms/fourier_wigner.py:13-88    inverse_transform
//   precompute_transforms/fourier_wigner.py:177-333  forward_transform
//   precompute_transforms/construct.py:614-639       fourier_wigner_kernel (quadrature part;
//                                                    the Delta planes come from s2b_rotate_dls)
//   precompute_transforms/custom_ops.py:5-83         wigner_subset_to_s2
//   precompute_transforms/custom_ops.py:168-205      so3_to_wigner_subset
//   precompute_transforms/custom_ops.py:251-333      s2_to_wigner_subset
//
// Every operation is a chain over "slices": one slice is one azimuthal index n of one
// map (a spin -n field). With Delta^l = d^l(pi/2) and c_l = (2l+1)/(8 pi^2):
//
//   inverse: Y[a, m] = i^(n-m) e^{i a theta0} sum_l c_l Delta^l_{a,m} Delta^l_{a,n} F[l, m]
//            (fw_contract_kernel<INV>), a DFT over a keeping the sampled rings
//            (fw_cols_inv_kernel), a DFT over m per ring (fw_rows_inv_kernel); the full
//            transform then sums over n (gamma DFT, fw_gamma_kernel).
//   forward: the gamma DFT (fw_gamma_kernel, or fw_gamma_subset_kernel for a spin subset), a DFT
//            per ring (fw_rows_fwd_kernel), per column m the periodic extension of beta to
//            [0, 2pi), its DFT, and the quadrature: upstream multiplies by 4L-3 upsampled
//            weights between an inverse and a forward DFT of length 4L-3, a convolution
//            that runs here on a power-of-two length Q >= 4L-1 with weights converted
//            from the caller's (fw_cols_fwd_kernel, fw_quads_pow2_kernel), and
//            H[l, m] = (2pi)^2 i^(m-n) sum_b G[b, m] Delta^l_{b,m} Delta^l_{b,n}
//            (fw_contract_kernel<FWD>).
//
// Frequencies are stored "value mod length", which is what upstream's fftshift /
// ifftshift pairs amount to. The FFTs are the block DFTs of s2b_fft_dev.h (one CTA per
// row or column, radix-2 or Bluestein in shared memory).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "s2b.h"
#include "s2b_fft.h"
#include "s2b_dev.h"
#include "s2b_fft_dev.h"
#include "s2b_internal.h"
#include "s2b_wigner.h"  // launch_wigner_mirror

namespace s2b {

// Slice bookkeeping. Slice e belongs to group g = e / S and has slot k = e % S; its
// azimuthal index is n = nlist ? nsign * nlist[k] : n0 + k. In the coefficient array
// (flmn) the slice sits at slot Soff + k of a group of Stot slots.
struct FWSlices {
  int S, Stot, Soff, n0, nsign;
  const int* nlist;
};

__device__ __forceinline__ int fw_n(const FWSlices& s, int k) {
  return s.nlist ? s.nsign * __ldg(s.nlist + k) : s.n0 + k;
}
__device__ __forceinline__ long fw_coef_slice(const FWSlices& s, int e) {
  return (long)(e / s.S) * s.Stot + s.Soff + e % s.S;
}

// z * i^k
template <typename R2>
__device__ __forceinline__ R2 mul_ipow(R2 z, int k) {
  R2 o;
  switch (k & 3) {
    case 0: o = z; break;
    case 1: o.x = -z.y; o.y = z.x; break;
    case 2: o.x = -z.x; o.y = -z.y; break;
    default: o.x = z.y; o.y = -z.x; break;
  }
  return o;
}

constexpr int kFwLanes = 128;  // threads of a contraction CTA, one m column each
constexpr int kFwQ = 32;       // summation indices staged per shared-memory chunk

// Output rows (a for the inverse, l for the forward) and slices per thread.
template <typename Real>
struct FWTile {
  static constexpr int R = 4;
  static constexpr int E = 4;
  // summation indices a thread's copies run ahead (cp.async ring in shared memory)
  static constexpr int D = sizeof(Real) == 4 ? 4 : 3;
};

template <typename Real>
struct FWContractParams {
  int L, E;
  int mwss;
  FWSlices sl;
  const double* delta;  // [L][2L-1][2L-1]
  const void* in;       // INV: coefficients (slice layout fw_coef_slice); FWD: Gf [E][L][2L-1]
  void* out;            // INV: Y [E][2L-1][2L-1]; FWD: coefficients
  const double2* thW;   // e^{i pi r / (2L-1)} at [r + L], |r| <= L (plan table)
  // adjoints: INV with adj writes the rows a >= 0 only, [E][L][2L-1], times (2pi)^2 and
  // i^(n-m) (the adjoint of the forward's last step); FWD with adj scales row l by c_l
  // without phase (the adjoint of the inverse's first step; the phases come from
  // fw_cols_inv_adj_kernel)
  int adj;
};

// With D[l][x][y] = Delta^l_{x,y} (zero where |x| > l or |y| > l) and the reflection
// D[l][-x][y] = (-1)^(l+y) D[l][x][y] of the planes at pi/2, the products
// D[l][x][m] D[l][x][n] are even or odd in x with (-1)^(m+n). Hence
// INV: for a >= 0, P[e][a][m] = sum_l c_l D[l][a][m] D[l][a][n] F[e][l][m], and
//      Y[a] = i^(n-m) e^{+i a theta0} P[a], Y[-a] = (-1)^(m+n) i^(n-m) e^{-i a theta0} P[a];
// FWD: out[e][l][m] = (2pi)^2 i^(m-n) sum_{0 <= b <= l} D[l][b][m] D[l][b][n] Gf[e][b][m],
//      where Gf[b] = G[b] + (-1)^(m+n) G[-b] (b > 0), Gf[0] = G[0] (fw_cols_fwd_kernel).
// Lanes run along m; each thread keeps R x E complex sums. The n-column weights of a chunk
// of kFwQ summation indices are staged in shared memory and read as broadcasts; each
// thread's own operands of an index (E coefficients, R plane values) arrive by cp.async a
// few indices ahead. The slice tiles run along blockIdx.x, so the CTAs that read the same
// planes run together.
template <typename Real, bool FWD>
__global__ void __launch_bounds__(kFwLanes) fw_contract_kernel(FWContractParams<Real> p) {
  using R2 = typename C2<Real>::t;
  constexpr int R = FWTile<Real>::R, E = FWTile<Real>::E, D = FWTile<Real>::D;
  const int L = p.L, W = 2 * L - 1;
  const int ci = blockIdx.y * kFwLanes + threadIdx.x;  // column index m + L - 1
  const bool live = ci < W;
  const int m = ci - (L - 1);
  const int r0 = blockIdx.z * R;  // first output row (a >= 0, or l)
  const int e0 = blockIdx.x * E;

  __shared__ Real wn[kFwQ][R][E];
  __shared__ int nsh[E];
  if (threadIdx.x < E) {
    const int e = e0 + threadIdx.x;
    int n = e < p.E ? fw_n(p.sl, e % p.sl.S) : 0;
    if (n > L - 1 || n < -(L - 1)) n = L;  // out of range: weights zero below
    nsh[threadIdx.x] = n;
  }
  __syncthreads();

  // summation range of the tile
  int qlo, qhi;
  const int cl = blockIdx.y * kFwLanes - (L - 1);
  const int ch = min(cl + kFwLanes - 1, L - 1);
  const int mmin = (cl <= 0 && ch >= 0) ? 0 : min(abs(cl), abs(ch));  // least |m| of the CTA
  if (FWD) {
    qlo = 0;
    qhi = min(r0 + R - 1, L - 1);
    if (mmin > qhi) qhi = -1;  // every D[l][b][m] of the tile is zero: write zeros
  } else {
    int nmin = L;
    for (int s = 0; s < E; ++s)
      if (e0 + s < p.E) nmin = min(nmin, abs(nsh[s]));
    qlo = max(max(r0, nmin), mmin);
    qhi = L - 1;
  }

  R2 acc[R][E];
#pragma unroll
  for (int j = 0; j < R; ++j)
#pragma unroll
    for (int s = 0; s < E; ++s) acc[j][s] = czero<R2>();

  const R2* X = reinterpret_cast<const R2*>(p.in);
  long xoff[E];
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int e = min(e0 + s, p.E - 1);
    xoff[s] = (FWD ? (long)e : fw_coef_slice(p.sl, e)) * (long)L * W;
  }

  const double pi = 3.141592653589793;
  // each thread's operands of summation index q (its coefficients of the E slices and its
  // plane values of the R rows) reach shared memory by cp.async, D - 1 indices ahead of
  // their arithmetic; only the thread itself reads its slots
  __shared__ __align__(16) R2 xr[D][E][kFwLanes];
  __shared__ __align__(16) double wr[D][R][kFwLanes];
  auto issue = [&](int q, int st) {
    if (!live || q > qhi) return;
#pragma unroll
    for (int s = 0; s < E; ++s)
      cp_async<sizeof(R2)>(smem_u32(&xr[st][s][threadIdx.x]), X + xoff[s] + (long)q * W + ci,
                           true);
#pragma unroll
    for (int j = 0; j < R; ++j) {  // rows past L-1 read row L-1 and get weight 0
      const int r = min(r0 + j, L - 1);
      const double* src = FWD ? p.delta + ((long)r * W + (q + L - 1)) * W + ci
                              : p.delta + ((long)q * W + (r + L - 1)) * W + ci;
      cp_async<8>(smem_u32(&wr[st][j][threadIdx.x]), src, true);
    }
  };
#pragma unroll
  for (int k = 0; k < D - 1; ++k) {
    issue(qlo + k, k);
    cp_async_commit();
  }
  int rs = 0;  // ring stage of the current index
  for (int q0 = qlo; q0 <= qhi; q0 += kFwQ) {
    // stage the n-column weights of this chunk
    for (int t = threadIdx.x; t < kFwQ * R * E; t += kFwLanes) {
      const int qq = t / (R * E), j = (t / E) % R, s = t % E;
      const int q = q0 + qq, r = r0 + j, n = nsh[s];
      double w = 0.0;
      if (q <= qhi && r <= L - 1 && n < L && e0 + s < p.E) {
        if (FWD)  // D[l = r][b = q][n]
          w = __ldg(p.delta + ((long)r * W + (q + L - 1)) * W + (n + L - 1));
        else      // c_l D[l = q][a = r][n]  (adjoint: (2pi)^2 D[l = q][a = r][n])
          w = (p.adj ? 4.0 * pi * pi : (2.0 * q + 1.0) / (8.0 * pi * pi)) *
              __ldg(p.delta + ((long)q * W + (r + L - 1)) * W + (n + L - 1));
      }
      wn[qq][j][s] = (Real)w;
    }
    __syncthreads();
    const int qend = min(kFwQ, qhi - q0 + 1);
    for (int qq = 0; qq < qend; ++qq) {
      issue(q0 + qq + D - 1, rs == 0 ? D - 1 : rs - 1);
      cp_async_commit();
      cp_async_wait<D - 1>();  // this thread's copies of index q0 + qq
      if (live) {
        R2 x[E];
        Real w1[R];
#pragma unroll
        for (int s = 0; s < E; ++s) x[s] = xr[rs][s][threadIdx.x];
#pragma unroll
        for (int j = 0; j < R; ++j) w1[j] = (Real)wr[rs][j][threadIdx.x];
#pragma unroll
        for (int j = 0; j < R; ++j) {
#pragma unroll
          for (int s = 0; s < E; ++s) {
            const Real w = w1[j] * wn[qq][j][s];
            acc[j][s].x = fma(w, x[s].x, acc[j][s].x);
            acc[j][s].y = fma(w, x[s].y, acc[j][s].y);
          }
        }
      }
      rs = rs == D - 1 ? 0 : rs + 1;
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  if (!live) return;

  R2* O = reinterpret_cast<R2*>(p.out);
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int e = e0 + s;
    if (e >= p.E) continue;
    const int n = nsh[s] == L ? 0 : nsh[s];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int r = r0 + j;
      if (r > L - 1) continue;
      if (FWD) {
        R2 v;
        if (p.adj) {
          v = cscale(acc[j][s], (Real)((2.0 * r + 1.0) / (8.0 * pi * pi)));
        } else {
          const Real sc = (Real)(4.0 * pi * pi);
          v = mul_ipow(acc[j][s], m - n);
          v.x *= sc;
          v.y *= sc;
        }
        O[fw_coef_slice(p.sl, e) * (long)L * W + (long)r * W + ci] = v;
      } else if (p.adj) {
        O[(long)e * L * W + (long)r * W + ci] = mul_ipow(acc[j][s], n - m);
      } else {
        const R2 v = mul_ipow(acc[j][s], n - m);
        R2* Y = O + (long)e * W * W;
        if (p.mwss) {
          Y[(long)(r + L - 1) * W + ci] = v;
          if (r > 0) Y[(long)(L - 1 - r) * W + ci] = (((m + n) & 1) ? cscale(v, Real(-1)) : v);
        } else {  // e^{+-i a pi / (2L-1)}
          const double2 t = p.thW[r + L];
          const Real c = (Real)t.x, sv = (Real)t.y;
          R2 u;
          u.x = v.x * c - v.y * sv;
          u.y = v.x * sv + v.y * c;
          Y[(long)(r + L - 1) * W + ci] = u;
          if (r > 0) {
            const Real sg = ((m + n) & 1) ? Real(-1) : Real(1);
            u.x = sg * (v.x * c + v.y * sv);
            u.y = sg * (v.y * c - v.x * sv);
            Y[(long)(L - 1 - r) * W + ci] = u;
          }
        }
      }
    }
  }
}

template <typename Real>
struct FWFftParams {
  int L, mwss, ntheta, nphi, P, E;
  FWSlices sl;
  int nmajor, groups;  // map index of slice e: (Soff + e % S) * groups + e / S when nmajor
  double scale;
  FFTDesc dphi, dP;
  FFTTables<Real> tb;
  const void* quads;  // complex128 [P]: the beta-convolution weights (quadsQ)
  const void* wconv;  // complex128 [4L-3]: w[k], k = -(2L-2) .. 2L-2
  const double2* thW;  // e^{i pi r / (2L-1)} at [r + L], |r| <= L (plan table)
  const void* in;
  void* out;
};

template <typename Real>
__device__ __forceinline__ long fw_map_index(const FWFftParams<Real>& p, int e) {
  return p.nmajor ? (long)(p.sl.Soff + e % p.sl.S) * p.groups + e / p.sl.S : (long)e;
}

// Inverse, beta: column m of Y[e] -> T[e][t][m] = sum_a Y[a][m] e^{+i a beta_t}, t < ntheta
// (beta_t = 2 pi t / nphi; the theta0 shift is in Y).
template <typename Real>
__global__ void __launch_bounds__(512) fw_cols_inv_kernel(FWFftParams<Real> p) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  const int L = p.L, W = 2 * L - 1, col = blockIdx.x, e = blockIdx.y;
  const R2* Y = reinterpret_cast<const R2*>(p.in) + (long)e * W * W;
  const int na = p.nphi;
  dft_run<Real>(s, p.dphi, p.tb, true, [&](int k) {
    const int a = k <= L - 1 ? k : k - na;
    return a >= -(L - 1) ? Y[(long)(a + L - 1) * W + col] : czero<R2>();
  });
  R2* T = reinterpret_cast<R2*>(p.out) + (long)e * p.ntheta * W;
  for (int t = threadIdx.x; t < p.ntheta; t += blockDim.x)
    T[(long)t * W + col] = dft_get<Real>(s, p.dphi, p.tb, true, t);
}

// Inverse, alpha: ring t of T[e] -> map[t][p] = sum_m T[t][m] e^{+i m alpha_p}.
template <typename Real>
__global__ void __launch_bounds__(512) fw_rows_inv_kernel(FWFftParams<Real> p) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  const int L = p.L, W = 2 * L - 1, t = blockIdx.x, e = blockIdx.y;
  const R2* T = reinterpret_cast<const R2*>(p.in) + ((long)e * p.ntheta + t) * W;
  const int np = p.nphi;
  dft_run<Real>(s, p.dphi, p.tb, true, [&](int k) {
    const int m = k <= L - 1 ? k : k - np;
    return m >= -(L - 1) ? T[m + L - 1] : czero<R2>();
  });
  R2* o = reinterpret_cast<R2*>(p.out) + (fw_map_index(p, e) * p.ntheta + t) * np;
  const Real sc = (Real)p.scale;
  for (int j = threadIdx.x; j < np; j += blockDim.x)
    o[j] = cscale(dft_get<Real>(s, p.dphi, p.tb, true, j), sc);
}

// Forward, alpha: ring t of map e -> S[e][t][m] = scale sum_p map[t][p] e^{-i m alpha_p},
// |m| <= L-1.
template <typename Real>
__global__ void __launch_bounds__(512) fw_rows_fwd_kernel(FWFftParams<Real> p) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  const int L = p.L, W = 2 * L - 1, t = blockIdx.x, e = blockIdx.y;
  const int np = p.nphi;
  const R2* f = reinterpret_cast<const R2*>(p.in) + (fw_map_index(p, e) * p.ntheta + t) * np;
  dft_run<Real>(s, p.dphi, p.tb, false, [&](int k) { return f[k]; });
  R2* S = reinterpret_cast<R2*>(p.out) + ((long)e * p.ntheta + t) * W;
  const Real sc = (Real)p.scale;
  for (int c = threadIdx.x; c < W; c += blockDim.x) {
    const int m = c - (L - 1);
    S[c] = cscale(dft_get<Real>(s, p.dphi, p.tb, false, pmod(m, np)), sc);
  }
}

// Forward, beta: column m of S[e] -> G[b], |b| <= L-1 (fourier_wigner.py:258-292), stored
// folded as Gf[e][b][m], 0 <= b <= L-1 (see fw_contract_kernel).
// The quadrature is applied as a product between an inverse and a forward DFT of length
// p.P = Q (power of two, >= 4L-1) with the weights p.quads = quadsQ (fw_quads_pow2_kernel).
// Shared memory: the DFT buffer (padded working length) and a buffer of Q values.
template <typename Real>
__global__ void __launch_bounds__(512) fw_cols_fwd_kernel(FWFftParams<Real> p, int bufM) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  R2* tmp = s + padded_len(bufM);
  const int L = p.L, W = 2 * L - 1, col = blockIdx.x, e = blockIdx.y;
  const int m = col - (L - 1);
  const int n = fw_n(p.sl, e % p.sl.S);
  const Real sgn = ((abs(m) + abs(n)) & 1) ? Real(-1) : Real(1);
  const int nth = p.ntheta, nx = p.nphi, P = p.P;
  const R2* Sx = reinterpret_cast<const R2*>(p.in) + (long)e * nth * W;
  // periodic extension to [0, 2pi): rows nth-1+j = sgn * rows nth-1-j, 1 <= j <= L-1
  dft_run<Real>(s, p.dphi, p.tb, false, [&](int k) {
    if (k < nth) return Sx[(long)k * W + col];
    return cscale(Sx[(long)(2 * (nth - 1) - k) * W + col], sgn);
  });
  const int blo = p.mwss ? -L : -(L - 1);
  const Real inx = (Real)(1.0 / nx);
  for (int b = blo + (int)threadIdx.x; b <= L - 1; b += blockDim.x) {
    R2 v = cscale(dft_get<Real>(s, p.dphi, p.tb, false, pmod(b, nx)), inx);
    if (!p.mwss) {  // e^{-i b pi / (2L-1)}
      const double2 t = p.thW[L - b];  // e^{-i b pi / (2L-1)}
      const R2 u = v;
      v.x = u.x * (Real)t.x - u.y * (Real)t.y;
      v.y = u.x * (Real)t.y + u.y * (Real)t.x;
    }
    tmp[b - blo] = v;
  }
  __syncthreads();
  // mwss: on upstream's 4L-3 points the spectrum value at b = -L meets the weight at
  // k = -(2L-2) again at b = L-1 (their distance is exactly 4L-3); kept for parity
  R2 alias = czero<R2>();
  if (p.mwss) {
    const double2 w0 = reinterpret_cast<const double2*>(p.wconv)[0];  // w[-(2L-2)]
    R2 w;
    w.x = (Real)w0.x;
    w.y = (Real)w0.y;
    alias = cmul(tmp[0], w);
  }
  // zero-padded to Q and inverse DFT (the upsampled beta samples)
  const int half = (P - 1) / 2;
  dft_run<Real>(s, p.dP, p.tb, true, [&](int k) {
    const int v = k <= half ? k : k - P;
    return (v >= blo && v <= L - 1) ? tmp[v - blo] : czero<R2>();
  });
  const double2* qd = reinterpret_cast<const double2*>(p.quads);
  for (int j = threadIdx.x; j < P; j += blockDim.x) {
    const double2 q = qd[j];
    R2 w;
    w.x = (Real)q.x;
    w.y = (Real)q.y;
    tmp[j] = cmul(dft_get<Real>(s, p.dP, p.tb, true, j), w);
  }
  __syncthreads();
  dft_run<Real>(s, p.dP, p.tb, false, [&](int k) { return tmp[k]; });
  // folded rows b >= 0: Gf[b] = G[b] + (-1)^(m+n) G[-b] (b > 0), Gf[0] = G[0]
  const Real iP = (Real)(1.0 / P);
  R2* G = reinterpret_cast<R2*>(p.out) + (long)e * L * W;
  for (int b = threadIdx.x; b <= L - 1; b += blockDim.x) {
    R2 v = dft_get<Real>(s, p.dP, p.tb, false, b);
    if (b > 0) v = cadd(v, cscale(dft_get<Real>(s, p.dP, p.tb, false, P - b), sgn));
    v = cscale(v, iP);
    if (b == L - 1) v = cadd(v, alias);
    G[(long)b * W + col] = v;
  }
}

// Adjoint of fw_cols_inv_kernel and of the phases / mirror of the inverse contraction:
// column m of T[e] (ntheta rows) -> Y[a] = sum_t T[t] e^{-i a beta_t}, |a| <= L-1, then
// Pf[a] = conj(ph(a)) Y[a] + (-1)^(m+n) conj(ph(-a)) Y[-a] (a > 0), Pf[0] = conj(ph(0)) Y[0],
// ph(a) = i^(n-m) e^{i a theta0}; stored [E][L][2L-1] for the adjoint contraction.
template <typename Real>
__global__ void __launch_bounds__(512) fw_cols_inv_adj_kernel(FWFftParams<Real> p) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  const int L = p.L, W = 2 * L - 1, col = blockIdx.x, e = blockIdx.y;
  const int m = col - (L - 1);
  const int n = fw_n(p.sl, e % p.sl.S);
  const Real sgn = ((abs(m) + abs(n)) & 1) ? Real(-1) : Real(1);
  const R2* T = reinterpret_cast<const R2*>(p.in) + (long)e * p.ntheta * W;
  const int na = p.nphi;
  dft_run<Real>(s, p.dphi, p.tb, false, [&](int k) {
    return k < p.ntheta ? T[(long)k * W + col] : czero<R2>();
  });
  R2* Pf = reinterpret_cast<R2*>(p.out) + (long)e * L * W;
  for (int a = threadIdx.x; a <= L - 1; a += blockDim.x) {
    R2 yp = dft_get<Real>(s, p.dphi, p.tb, false, a);
    R2 ym = a > 0 ? dft_get<Real>(s, p.dphi, p.tb, false, na - a) : czero<R2>();
    if (!p.mwss) {  // e^{-i a theta0} on Y[a], e^{+i a theta0} on Y[-a]
      const double2 t = p.thW[a + L];
      const Real c = (Real)t.x, sv = (Real)t.y;
      const R2 u = yp, v = ym;
      yp.x = u.x * c + u.y * sv;
      yp.y = u.y * c - u.x * sv;
      ym.x = v.x * c - v.y * sv;
      ym.y = v.x * sv + v.y * c;
    }
    Pf[(long)a * W + col] = mul_ipow(cadd(yp, cscale(ym, sgn)), m - n);
  }
}

// Adjoint of fw_cols_fwd_kernel: column m of Gf[e] ([E][L][2L-1]) -> S[e][t][m], t < ntheta.
// Unfold (G[b] = Gf[b], G[-b] = (-1)^(m+n) Gf[b]), the convolution's adjoint (the same
// length-Q chain with conj(quadsQ), plus the mwss wrap-around term's adjoint), the MW phase's
// conjugate, (1/nx) times the inverse DFT of length nx, and the extension folded back.
template <typename Real>
__global__ void __launch_bounds__(512) fw_cols_fwd_adj_kernel(FWFftParams<Real> p, int bufM) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  R2* tmp = s + padded_len(bufM);
  const int L = p.L, W = 2 * L - 1, col = blockIdx.x, e = blockIdx.y;
  const int m = col - (L - 1);
  const int n = fw_n(p.sl, e % p.sl.S);
  const Real sgn = ((abs(m) + abs(n)) & 1) ? Real(-1) : Real(1);
  const int nth = p.ntheta, nx = p.nphi, P = p.P;
  const R2* Gf = reinterpret_cast<const R2*>(p.in) + (long)e * L * W;
  // G[b'] at b' mod P, |b'| <= L-1, zero elsewhere; inverse DFT of length P, times 1/P
  const int half = (P - 1) / 2;
  dft_run<Real>(s, p.dP, p.tb, true, [&](int k) {
    const int v = k <= half ? k : k - P;
    if (v >= 0 && v <= L - 1) return Gf[(long)v * W + col];
    if (v < 0 && v >= -(L - 1)) return cscale(Gf[(long)(-v) * W + col], sgn);
    return czero<R2>();
  });
  const double2* qd = reinterpret_cast<const double2*>(p.quads);
  const Real iP = (Real)(1.0 / P);
  for (int j = threadIdx.x; j < P; j += blockDim.x) {
    const double2 q = qd[j];
    R2 w;
    w.x = (Real)q.x;
    w.y = (Real)(-q.y);  // conj(quadsQ)
    tmp[j] = cscale(cmul(dft_get<Real>(s, p.dP, p.tb, true, j), w), iP);
  }
  __syncthreads();
  dft_run<Real>(s, p.dP, p.tb, false, [&](int k) { return tmp[k]; });
  // B_adj[v], v in [blo, L-1] -> tmp[v - blo] (with the MW phase's conjugate)
  const int blo = p.mwss ? -L : -(L - 1);
  for (int v = blo + (int)threadIdx.x; v <= L - 1; v += blockDim.x) {
    R2 x = dft_get<Real>(s, p.dP, p.tb, false, pmod(v, P));
    if (p.mwss && v == -L) {  // adjoint of the wrap-around term B[-L] w[-(2L-2)] -> G[L-1]
      const double2 w0 = reinterpret_cast<const double2*>(p.wconv)[0];
      R2 cw;
      cw.x = (Real)w0.x;
      cw.y = (Real)(-w0.y);
      x = cadd(x, cmul(Gf[(long)(L - 1) * W + col], cw));
    }
    if (!p.mwss) {  // conj(e^{-i v pi / (2L-1)})
      const double2 t = p.thW[v + L];
      const R2 u = x;
      x.x = u.x * (Real)t.x - u.y * (Real)t.y;
      x.y = u.x * (Real)t.y + u.y * (Real)t.x;
    }
    tmp[v - blo] = x;
  }
  __syncthreads();
  // (1/nx) inverse DFT of length nx over the bins v mod nx
  dft_run<Real>(s, p.dphi, p.tb, true, [&](int k) {
    const int v = k <= (nx - 1) / 2 ? k : k - nx;  // nx odd (mw): |v| <= L-1; even: -L..L-1
    return (v >= blo && v <= L - 1) ? tmp[v - blo] : czero<R2>();
  });
  const Real inx = (Real)(1.0 / nx);
  R2* S = reinterpret_cast<R2*>(p.out) + (long)e * nth * W;
  for (int t = threadIdx.x; t < nth; t += blockDim.x) {
    R2 x = dft_get<Real>(s, p.dphi, p.tb, true, t);
    const int t2 = 2 * (nth - 1) - t;  // the extension row that copied ring t
    if (t2 >= nth && t2 < nx) x = cadd(x, cscale(dft_get<Real>(s, p.dphi, p.tb, true, t2), sgn));
    S[(long)t * W + col] = cscale(x, inx);
  }
}

// Gamma DFT of the full transform: one thread per (map, pixel) and block of kGamK outputs
// (blockIdx.y). The sums below are multiplied by `scale` (1 for the inverse, 1/G for the
// forward in the transforms; the adjoints use G and 1/G).
//   inverse: f[b][g][px] = sum_n x[N-1+n][b][px] e^{+2 pi i n g / G}, n in [-(N-1), N-1];
//            reality: real output from n >= 0 (irfft: n = 0 real part, n > 0 doubled)
//   forward: x[N-1+n][b][px] = sum_g f[b][g][px] e^{-2 pi i n g / G}, n in [n0, N-1]
// (fourier_wigner.py:80-87 and 241-248). A table of the G roots e^{2 pi i j / G} sits in
// shared memory; the exponent n g is reduced mod G exactly. The sums run in the transform's
// precision (at most 2N-1 < 24 terms).
constexpr int kGamK = 8;

template <typename Real, bool FWD>
__global__ void fw_gamma_kernel(const void* in, void* out, int B, int N, long npix, int reality,
                                double scale) {
  using R2 = typename C2<Real>::t;
  extern __shared__ __align__(16) unsigned char groots_raw[];
  R2* const roots = reinterpret_cast<R2*>(groots_raw);
  const int G = 2 * N - 1;
  for (int j = threadIdx.x; j < G; j += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * (double)j / (double)G, &sn, &cs);
    roots[j].x = (Real)cs;
    roots[j].y = (Real)sn;
  }
  __syncthreads();
  const long total = (long)B * npix;
  const int nlo = reality ? 0 : -(N - 1);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long b = i / npix, px = i % npix;
    if (!FWD) {
      const R2* x = reinterpret_cast<const R2*>(in);
      {
        const int g0 = blockIdx.y * kGamK;
        Real re[kGamK], im[kGamK];
#pragma unroll
        for (int u = 0; u < kGamK; ++u) re[u] = im[u] = Real(0);
        for (int n = nlo; n < N; ++n) {
          const R2 v = x[((long)(N - 1 + n) * B + b) * npix + px];
          Real vr = v.x, vi = v.y;
          if (reality) {
            if (n == 0) vi = Real(0);
            else { vr *= Real(2); vi *= Real(2); }
          }
          const int step = ((n % G) + G) % G;
          int r = (int)(((long)step * g0) % G);
#pragma unroll
          for (int u = 0; u < kGamK; ++u) {
            const R2 w = roots[r];
            re[u] += vr * w.x - vi * w.y;
            im[u] += vr * w.y + vi * w.x;
            r += step;
            if (r >= G) r -= G;
          }
        }
#pragma unroll
        for (int u = 0; u < kGamK; ++u) {
          const int g = g0 + u;
          if (g >= G) break;
          const long o = (b * G + g) * npix + px;
          if (reality) {
            reinterpret_cast<Real*>(out)[o] = (Real)(re[u] * scale);
          } else {
            R2 w;
            w.x = (Real)(re[u] * scale);
            w.y = (Real)(im[u] * scale);
            reinterpret_cast<R2*>(out)[o] = w;
          }
        }
      }
    } else {
      R2* x = reinterpret_cast<R2*>(out);
      {
        const int n0 = nlo + (int)blockIdx.y * kGamK;
        Real re[kGamK], im[kGamK];
#pragma unroll
        for (int u = 0; u < kGamK; ++u) re[u] = im[u] = Real(0);
        for (int g = 0; g < G; ++g) {
          Real vr, vi;
          const long o = (b * G + g) * npix + px;
          if (reality) {
            vr = reinterpret_cast<const Real*>(in)[o];
            vi = Real(0);
          } else {
            const R2 v = reinterpret_cast<const R2*>(in)[o];
            vr = v.x;
            vi = v.y;
          }
          // e^{-2 pi i n g / G} = roots[(-n g) mod G]
          const int step = (G - g % G) % G;  // (-g) mod G, advances with n
          int r = (int)(((long)step * (((n0 % G) + G) % G)) % G);
#pragma unroll
          for (int u = 0; u < kGamK; ++u) {
            const R2 w = roots[r];
            re[u] += vr * w.x - vi * w.y;
            im[u] += vr * w.y + vi * w.x;
            r += step;
            if (r >= G) r -= G;
          }
        }
        const double sc = scale;
#pragma unroll
        for (int u = 0; u < kGamK; ++u) {
          const int n = n0 + u;
          if (n >= N) break;
          R2 w;
          w.x = (Real)(re[u] * sc);
          w.y = (Real)(im[u] * sc);
          x[((long)(N - 1 + n) * B + b) * npix + px] = w;
        }
      }
    }
  }
}

// Gamma DFT by the block FFT (2N-1 >= kGamFFTMin): one CTA per (pixel, map), the
// 2N-1 values of the pixel gathered with stride (map count x pixels). Same sums as
// fw_gamma_kernel.
constexpr int kGamFFTMin = 24;

template <typename Real, bool FWD>
__global__ void __launch_bounds__(512) fw_gamma_fft_kernel(const void* in, void* out, int B,
                                                           int N, long npix, int reality,
                                                           double scale, FFTDesc dg,
                                                           FFTTables<Real> tb) {
  using R2 = typename C2<Real>::t;
  extern __shared__ unsigned char fw_smem[];
  R2* s = reinterpret_cast<R2*>(fw_smem);
  const long px = blockIdx.x;
  const long b = blockIdx.y;
  const int G = 2 * N - 1;
  if (!FWD) {
    const R2* x = reinterpret_cast<const R2*>(in);
    dft_run<Real>(s, dg, tb, true, [&](int k) {
      const int n = k <= N - 1 ? k : k - G;
      if (!reality) return x[((long)(N - 1 + n) * B + b) * npix + px];
      // Hermitian: x_{-n} = conj(x_n), the imaginary part of x_0 dropped (irfft)
      R2 v = x[((long)(N - 1 + (n < 0 ? -n : n)) * B + b) * npix + px];
      if (n < 0) v.y = -v.y;
      if (n == 0) v.y = Real(0);
      return v;
    });
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
      const R2 v = cscale(dft_get<Real>(s, dg, tb, true, g), (Real)scale);
      const long o = (b * G + g) * npix + px;
      if (reality)
        reinterpret_cast<Real*>(out)[o] = v.x;
      else
        reinterpret_cast<R2*>(out)[o] = v;
    }
  } else {
    dft_run<Real>(s, dg, tb, false, [&](int k) {
      const long o = (b * G + k) * npix + px;
      if (reality) {
        R2 v;
        v.x = reinterpret_cast<const Real*>(in)[o];
        v.y = Real(0);
        return v;
      }
      return reinterpret_cast<const R2*>(in)[o];
    });
    R2* x = reinterpret_cast<R2*>(out);
    const Real sc = (Real)scale;
    for (int n = (reality ? 0 : -(N - 1)) + (int)threadIdx.x; n < N; n += blockDim.x)
      x[((long)(N - 1 + n) * B + b) * npix + px] =
          cscale(dft_get<Real>(s, dg, tb, false, n < 0 ? n + G : n), sc);
  }
}

// quads[j] = sum_{|k| <= 2L-2} w(-k) e^{+2 pi i k j / (4L-3)}, w the MW weights
// (w(+-1) = +-i pi/2, w(even k) = 2/(1-k^2), else 0); construct.py:629-634.
// roots[r] = e^{2 pi i r / n}, r in [0, n)
__global__ void fw_roots_kernel(int n, double2* roots) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi(2.0 * (double)r / (double)n, &sn, &cs);
    roots[r] = make_double2(cs, sn);
  }
}

// tab[i] = e^{i pi (i - L) / (2L-1)}, i in [0, 2L]: the MW theta0 phases of the column chains
__global__ void fw_theta_phase_kernel(int L, double2* tab) {
  const int W = 2 * L - 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= 2 * L; i += gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi((double)(i - L) / (double)W, &sn, &cs);
    tab[i] = make_double2(cs, sn);
  }
}

// exponent index (a b) mod n (n > 0), for any signs of a and b
__device__ __forceinline__ int fw_mulmod(long a, long b, int n) {
  return (int)(((a * b) % n + n) % n);
}

__global__ void fw_quads_kernel(int L, double2* quads, const double2* __restrict__ rootsP) {
  // one warp per output j, the 4L-3 terms split over the lanes and summed by shuffles; the
  // exponent index of term k = k0 + 32 t advances by 32 j (mod P)
  const int P = 4 * L - 3;
  const int j = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= P) return;  // whole warps leave together (blockDim is a multiple of 32)
  double re = 0.0, im = 0.0;
  int r = fw_mulmod(-(2 * L - 2) + lane, j, P);
  const int dr = fw_mulmod(32, j, P);
  for (int k = -(2 * L - 2) + lane; k <= 2 * L - 2; k += 32) {
    const int mk = -k;
    const int rk = r;
    r += dr;
    if (r >= P) r -= P;
    double wr = 0.0, wi = 0.0;
    if (mk == 1)
      wi = 1.5707963267948966;
    else if (mk == -1)
      wi = -1.5707963267948966;
    else if ((mk & 1) == 0)
      wr = 2.0 / (1.0 - (double)mk * (double)mk);
    else
      continue;
    const double2 e = rootsP[rk];
    re += wr * e.x - wi * e.y;
    im += wr * e.y + wi * e.x;
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (lane == 0) quads[j] = make_double2(re, im);
}

// The beta convolution of the forward runs on a power-of-two length Q >= 4L-1 instead of
// the 4L-3 points of the weights: the product of the upsampled samples with quads between
// an inverse and a forward DFT of length 4L-3 is the convolution of the beta spectrum with
// w[k] = (1/(4L-3)) sum_j quads[j] e^{-2 pi i j k / (4L-3)}, |k| <= 2L-2, and on Q points the
// same convolution needs quadsQ[j] = sum_k w[k] e^{+2 pi i k j / Q}. Q >= 4L-1 keeps the
// wrapped terms off the 2L-1 kept outputs (the spectrum spans at most 2L values).
// One warp per output; exponents reduced exactly.
__global__ void fw_weights_from_quads_kernel(int L, const double2* __restrict__ quads,
                                             double2* __restrict__ w,
                                             const double2* __restrict__ rootsP) {
  const int P = 4 * L - 3;
  const int o = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (o >= P) return;
  const int k = o - (2 * L - 2);
  double re = 0.0, im = 0.0;
  int r = fw_mulmod(-lane, k, P);  // (-j k) mod P, advancing by (-32 k) mod P
  const int dr = fw_mulmod(-32, k, P);
  for (int j = lane; j < P; j += 32) {
    const double2 e = rootsP[r];
    const double2 q = quads[j];
    re += q.x * e.x - q.y * e.y;
    im += q.x * e.y + q.y * e.x;
    r += dr;
    if (r >= P) r -= P;
  }
  for (int sh = 16; sh > 0; sh >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, sh);
    im += __shfl_xor_sync(0xffffffffu, im, sh);
  }
  if (lane == 0) w[o] = make_double2(re / P, im / P);
}

__global__ void fw_quads_pow2_kernel(int L, int Q, const double2* __restrict__ w,
                                     double2* __restrict__ quadsQ,
                                     const double2* __restrict__ rootsQ) {
  const int P = 4 * L - 3;
  const int j = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= Q) return;
  double re = 0.0, im = 0.0;
  int r = fw_mulmod(lane - (2 * L - 2), j, Q);  // (k j) mod Q, advancing by 32 j (Q = 2^q)
  const int dr = fw_mulmod(32, j, Q);
  for (int o = lane; o < P; o += 32) {
    const double2 e = rootsQ[r];
    const double2 v = w[o];
    re += v.x * e.x - v.y * e.y;
    im += v.x * e.y + v.y * e.x;
    r = (r + dr) & (Q - 1);
  }
  for (int sh = 16; sh > 0; sh >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, sh);
    im += __shfl_xor_sync(0xffffffffu, im, sh);
  }
  if (lane == 0) quadsQ[j] = make_double2(re, im);
}

// Gamma DFT at a spin subset: x[g][k][px] = (1/G) sum_c f[g][c][px] e^{-2 pi i c n_k / G}
// (n_k = -spin_k; custom_ops.py:200-204), f [O][G][npix], x [O][S][npix].
template <typename Real>
__global__ void fw_gamma_subset_kernel(const void* fin, void* xout, int O, int G, int S,
                                       long npix, FWSlices sl) {
  using R2 = typename C2<Real>::t;
  const R2* f = reinterpret_cast<const R2*>(fin);
  R2* x = reinterpret_cast<R2*>(xout);
  const long total = (long)O * npix;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long o = i / npix, px = i % npix;
    for (int k = 0; k < S; ++k) {
      const int nm = ((fw_n(sl, k) % G) + G) % G;  // n mod G, so that c * nm < G^2 fits an int
      double re = 0.0, im = 0.0;
      for (int c = 0; c < G; ++c) {
        const R2 v = f[(o * G + c) * npix + px];
        const int r = (G - (c * nm) % G) % G;  // (-c n) mod G
        double sn, cs;
        sincospi(2.0 * (double)r / (double)G, &sn, &cs);
        re += (double)v.x * cs - (double)v.y * sn;
        im += (double)v.x * sn + (double)v.y * cs;
      }
      R2 out;
      out.x = (Real)(re / G);
      out.y = (Real)(im / G);
      x[(o * S + k) * npix + px] = out;
    }
  }
}

// Adjoint of fw_gamma_subset_kernel: f[o][c][px] = (1/G) sum_k x[o][k][px] e^{+2 pi i c n_k / G}
// for the G gamma samples c.
template <typename Real>
__global__ void fw_gamma_subset_adj_kernel(const void* xin, void* fout, int O, int G, int S,
                                           long npix, FWSlices sl) {
  using R2 = typename C2<Real>::t;
  const R2* x = reinterpret_cast<const R2*>(xin);
  R2* f = reinterpret_cast<R2*>(fout);
  const long total = (long)O * npix;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long o = i / npix, px = i % npix;
    for (int c = 0; c < G; ++c) {
      double re = 0.0, im = 0.0;
      for (int k = 0; k < S; ++k) {
        const int nm = ((fw_n(sl, k) % G) + G) % G;  // n mod G: c * nm < G^2 fits an int
        const R2 v = x[(o * S + k) * npix + px];
        const int r = (c * nm) % G;
        double sn, cs;
        sincospi(2.0 * (double)r / (double)G, &sn, &cs);
        re += (double)v.x * cs - (double)v.y * sn;
        im += (double)v.x * sn + (double)v.y * cs;
      }
      R2 out;
      out.x = (Real)(re / G);
      out.y = (Real)(im / G);
      f[(o * G + c) * npix + px] = out;
    }
  }
}

}  // namespace s2b

using namespace s2b;

struct s2b_fw_plan {
  int L, N, mwss, ntheta, nphi, P, Q;  // P = 4L-3 weights, Q = pow2 >= 4L-1 beta convolution
  bool gamma_fft;  // fft.host[2] is the length-(2N-1) descriptor
  bool fp64;
  int device;
  std::vector<void*> allocs;
  FFTSet fft;  // host[0]: length nphi, host[1]: length Q, host[2]: 2N-1 (gamma_fft)
  double2* rootsP = nullptr;  // e^{2 pi i r / P}, r in [0, P)
  double2* rootsQ = nullptr;  // e^{2 pi i r / Q}, r in [0, Q)
  double2* thW = nullptr;     // e^{i pi r / (2L-1)} at [r + L], |r| <= L
  ~s2b_fw_plan() {
    for (void* a : allocs) cudaFree(a);
  }
};

namespace {

int fw_fail(int code, const std::string& msg) { return s2b::set_last_error(code, msg.c_str()); }

#define FW_CK(call)                                                                       \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return fw_fail(S2B_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));   \
  } while (0)

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

bool aligned16(const void* p) { return p && ((uintptr_t)p & 15) == 0; }

// Workspace regions: A (Y, G, or the gamma maps), B (T or S), C (spin-subset gamma maps).
// D: the beta-convolution weights of the forward (w [4L-3], quadsQ [Q], complex double).
struct FWLayout {
  size_t a, b, c, d;
  size_t total() const { return a + b + c + d; }
};

FWLayout fw_layout(const s2b_fw_plan* p, long E, long nmaps_gamma, long E_subset_gamma) {
  const size_t cs = p->fp64 ? 16 : 8;
  const long W = 2L * p->L - 1;
  const long npix = (long)p->ntheta * p->nphi;
  FWLayout l;
  l.a = al256(cs * (size_t)std::max(E * W * W, nmaps_gamma * npix));
  l.b = al256(cs * (size_t)(E * p->ntheta * W));
  l.c = al256(cs * (size_t)(E_subset_gamma * npix));
  l.d = al256(sizeof(double2) * (size_t)(p->P + p->Q));
  return l;
}

template <typename Real>
FFTTables<Real> tables(const s2b_fw_plan* p) {
  FFTTables<Real> t;
  t.tw = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->fft.tw);
  t.chirp = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->fft.chirp);
  t.bfilt = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->fft.bf);
  return t;
}

int fft_threads_for(int M) {
  int t = M / 8;
  if (t > 512) t = 512;
  if (t < 32) t = 32;
  return t;
}

template <typename Real>
FWFftParams<Real> fft_params(const s2b_fw_plan* p, int E, const FWSlices& sl) {
  FWFftParams<Real> f{};
  f.L = p->L;
  f.mwss = p->mwss;
  f.ntheta = p->ntheta;
  f.nphi = p->nphi;
  f.P = p->Q;  // length of the beta convolution (dP)
  f.E = E;
  f.sl = sl;
  f.nmajor = 0;
  f.groups = 1;
  f.scale = 1.0;
  f.dphi = p->fft.host[0];
  f.dP = p->fft.host[1];
  f.tb = tables<Real>(p);
  f.thW = p->thW;
  return f;
}

template <typename Real, typename K>
cudaError_t launch_fft(K kernel, dim3 grid, int M, size_t smem, cudaStream_t st,
                       const FWFftParams<Real>& f) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  kernel<<<grid, fft_threads_for(M), smem, st>>>(f);
  return cudaGetLastError();
}

template <typename Real>
int contract(const s2b_fw_plan* p, bool fwd, int E, const FWSlices& sl, const double* delta,
             const void* in, void* out, cudaStream_t st, int adj = 0) {
  FWContractParams<Real> c{};
  c.adj = adj;
  c.thW = p->thW;
  c.L = p->L;
  c.E = E;
  c.mwss = p->mwss;
  c.sl = sl;
  c.delta = delta;
  c.in = in;
  c.out = out;
  const int W = 2 * p->L - 1;
  constexpr int R = FWTile<Real>::R, Et = FWTile<Real>::E;
  dim3 grid((E + Et - 1) / Et, (W + kFwLanes - 1) / kFwLanes, (p->L + R - 1) / R);
  if (fwd)
    fw_contract_kernel<Real, true><<<grid, kFwLanes, 0, st>>>(c);
  else
    fw_contract_kernel<Real, false><<<grid, kFwLanes, 0, st>>>(c);
  FW_CK(cudaGetLastError());
  return S2B_OK;
}

// sphere-side inverse chain: Y (region A) -> T (region B) -> maps
template <typename Real>
int inverse_chain(const s2b_fw_plan* p, int E, const FWSlices& sl, const double* delta,
                  const void* coef, void* maps, int nmajor, int groups, char* ws,
                  const FWLayout& lay, cudaStream_t st) {
  using R2 = typename C2<Real>::t;
  void* A = ws;
  void* B = ws + lay.a;
  int rc = contract<Real>(p, false, E, sl, delta, coef, A, st);
  if (rc) return rc;
  FWFftParams<Real> f = fft_params<Real>(p, E, sl);
  const int M = f.dphi.M;
  const size_t smem = (size_t)padded_len(M) * sizeof(R2);
  f.in = A;
  f.out = B;
  FW_CK(launch_fft<Real>(fw_cols_inv_kernel<Real>, dim3(2 * p->L - 1, E), M, smem, st, f));
  f.in = B;
  f.out = maps;
  f.nmajor = nmajor;
  f.groups = groups;
  FW_CK(launch_fft<Real>(fw_rows_inv_kernel<Real>, dim3(p->ntheta, E), M, smem, st, f));
  return S2B_OK;
}

// sphere-side forward chain: maps -> S (region B) -> G (region A) -> coefficients
template <typename Real>
int forward_chain(const s2b_fw_plan* p, int E, const FWSlices& sl, const double* delta,
                  const void* quads, const void* maps, void* coef, int nmajor, int groups,
                  double scale, char* ws, const FWLayout& lay, cudaStream_t st) {
  using R2 = typename C2<Real>::t;
  void* A = ws;
  void* B = ws + lay.a;
  double2* wk = reinterpret_cast<double2*>(ws + lay.a + lay.b + lay.c);
  double2* qQ = wk + p->P;
  fw_weights_from_quads_kernel<<<(p->P + 3) / 4, 128, 0, st>>>(
      p->L, reinterpret_cast<const double2*>(quads), wk, p->rootsP);
  FW_CK(cudaGetLastError());
  fw_quads_pow2_kernel<<<(p->Q + 3) / 4, 128, 0, st>>>(p->L, p->Q, wk, qQ, p->rootsQ);
  FW_CK(cudaGetLastError());
  FWFftParams<Real> f = fft_params<Real>(p, E, sl);
  f.quads = qQ;
  f.wconv = wk;
  const int M = f.dphi.M;
  f.in = maps;
  f.out = B;
  f.nmajor = nmajor;
  f.groups = groups;
  f.scale = scale;
  FW_CK(launch_fft<Real>(fw_rows_fwd_kernel<Real>, dim3(p->ntheta, E), M,
                         (size_t)padded_len(M) * sizeof(R2), st, f));
  f.in = B;
  f.out = A;
  f.nmajor = 0;
  f.scale = 1.0;
  const int bufM = std::max(f.dphi.M, f.dP.M);
  const size_t smem = (size_t)(padded_len(bufM) + p->Q) * sizeof(R2);
  FW_CK(cudaFuncSetAttribute(fw_cols_fwd_kernel<Real>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fw_cols_fwd_kernel<Real><<<dim3(2 * p->L - 1, E), fft_threads_for(bufM), smem, st>>>(f, bufM);
  FW_CK(cudaGetLastError());
  return contract<Real>(p, true, E, sl, delta, A, coef, st);
}

// Adjoint of inverse_chain (maps -> coefficients): alpha DFTs (rows_fwd, scale 1), the
// beta adjoint with the phases and mirror (cols_inv_adj), the adjoint contraction.
template <typename Real>
int inverse_adjoint_chain(const s2b_fw_plan* p, int E, const FWSlices& sl, const double* delta,
                          const void* maps, void* coef, int nmajor, int groups, char* ws,
                          const FWLayout& lay, cudaStream_t st) {
  using R2 = typename C2<Real>::t;
  void* A = ws;
  void* B = ws + lay.a;
  FWFftParams<Real> f = fft_params<Real>(p, E, sl);
  const int M = f.dphi.M;
  const size_t smem = (size_t)padded_len(M) * sizeof(R2);
  f.in = maps;
  f.out = B;
  f.nmajor = nmajor;
  f.groups = groups;
  f.scale = 1.0;
  FW_CK(launch_fft<Real>(fw_rows_fwd_kernel<Real>, dim3(p->ntheta, E), M, smem, st, f));
  f.in = B;
  f.out = A;
  f.nmajor = 0;
  FW_CK(launch_fft<Real>(fw_cols_inv_adj_kernel<Real>, dim3(2 * p->L - 1, E), M, smem, st, f));
  return contract<Real>(p, true, E, sl, delta, A, coef, st, 1);
}

// Adjoint of forward_chain (coefficients -> maps): the adjoint contraction, the beta-chain
// adjoint (cols_fwd_adj) and inverse alpha DFTs times 1/nphi.
template <typename Real>
int forward_adjoint_chain(const s2b_fw_plan* p, int E, const FWSlices& sl, const double* delta,
                          const void* quads, const void* coef, void* maps, int nmajor,
                          int groups, char* ws, const FWLayout& lay, cudaStream_t st) {
  using R2 = typename C2<Real>::t;
  void* A = ws;
  void* B = ws + lay.a;
  double2* wk = reinterpret_cast<double2*>(ws + lay.a + lay.b + lay.c);
  double2* qQ = wk + p->P;
  fw_weights_from_quads_kernel<<<(p->P + 3) / 4, 128, 0, st>>>(
      p->L, reinterpret_cast<const double2*>(quads), wk, p->rootsP);
  FW_CK(cudaGetLastError());
  fw_quads_pow2_kernel<<<(p->Q + 3) / 4, 128, 0, st>>>(p->L, p->Q, wk, qQ, p->rootsQ);
  FW_CK(cudaGetLastError());
  int rc = contract<Real>(p, false, E, sl, delta, coef, A, st, 1);
  if (rc) return rc;
  FWFftParams<Real> f = fft_params<Real>(p, E, sl);
  f.quads = qQ;
  f.wconv = wk;
  f.in = A;
  f.out = B;
  const int bufM = std::max(f.dphi.M, f.dP.M);
  const size_t smem = (size_t)(padded_len(bufM) + p->Q) * sizeof(R2);
  FW_CK(cudaFuncSetAttribute(fw_cols_fwd_adj_kernel<Real>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fw_cols_fwd_adj_kernel<Real><<<dim3(2 * p->L - 1, E), fft_threads_for(bufM), smem, st>>>(f,
                                                                                        bufM);
  FW_CK(cudaGetLastError());
  f.in = B;
  f.out = maps;
  f.nmajor = nmajor;
  f.groups = groups;
  f.scale = 1.0 / p->nphi;
  const int M = f.dphi.M;
  FW_CK(launch_fft<Real>(fw_rows_inv_kernel<Real>, dim3(p->ntheta, E), M,
                         (size_t)padded_len(M) * sizeof(R2), st, f));
  return S2B_OK;
}

template <typename Real>
int gamma_dft(const s2b_fw_plan* p, bool fwd, const void* in, void* out, int B, int N,
              long npix, int reality, cudaStream_t st, double scale = -1.0) {
  const int G = 2 * N - 1;
  if (scale < 0) scale = fwd ? 1.0 / G : 1.0;  // the transforms' own normalisation
  if (p->gamma_fft && N == p->N) {
    using R2 = typename C2<Real>::t;
    const FFTDesc& dg = p->fft.host[2];
    const size_t smem = (size_t)padded_len(dg.M) * sizeof(R2);
    if (npix > 2147483647L || B > 65535)
      return fw_fail(S2B_ERR_INVALID, "too many pixels or maps for the gamma FFT");
    dim3 grid((unsigned)npix, B);
    if (fwd) {
      FW_CK(cudaFuncSetAttribute(fw_gamma_fft_kernel<Real, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      fw_gamma_fft_kernel<Real, true><<<grid, fft_threads_for(dg.M), smem, st>>>(
          in, out, B, N, npix, reality, scale, dg, tables<Real>(p));
    } else {
      FW_CK(cudaFuncSetAttribute(fw_gamma_fft_kernel<Real, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      fw_gamma_fft_kernel<Real, false><<<grid, fft_threads_for(dg.M), smem, st>>>(
          in, out, B, N, npix, reality, scale, dg, tables<Real>(p));
    }
    FW_CK(cudaGetLastError());
    return S2B_OK;
  }
  const long tot = (long)B * npix;
  const int nout = fwd ? (reality ? N : G) : G;
  const int chunks = (nout + kGamK - 1) / kGamK;
  const int blocks = (int)std::min<long>((tot + 255) / 256, 4L * 148 * 8);
  const size_t smem = (size_t)G * sizeof(double2);
  if (chunks > 65535) return fw_fail(S2B_ERR_INVALID, "N too large for the gamma DFT");
  if (fwd)
    fw_gamma_kernel<Real, true><<<dim3(blocks, chunks), 256, smem, st>>>(in, out, B, N, npix,
                                                                        reality, scale);
  else
    fw_gamma_kernel<Real, false><<<dim3(blocks, chunks), 256, smem, st>>>(in, out, B, N, npix,
                                                                         reality, scale);
  FW_CK(cudaGetLastError());
  return S2B_OK;
}

int check_plan(const s2b_fw_plan* p) {
  if (!p) return fw_fail(S2B_ERR_INVALID, "NULL Fourier-Wigner plan");
  int dev = -1;
  FW_CK(cudaGetDevice(&dev));
  if (dev != p->device)
    return fw_fail(S2B_ERR_INVALID, "the current device is not the plan's device");
  return S2B_OK;
}

int check_ptrs(std::initializer_list<const void*> ptrs) {
  for (const void* q : ptrs)
    if (!aligned16(q)) return fw_fail(S2B_ERR_ALIGN, "NULL or misaligned (16-byte) pointer");
  return S2B_OK;
}

// slices run along gridDim.y of the FFT kernels
int check_slices(long E) {
  if (E > 65535) return fw_fail(S2B_ERR_INVALID, "more than 65535 slices in one call");
  return S2B_OK;
}

int check_ws(const FWLayout& lay, const void* ws, size_t bytes) {
  if (bytes < lay.total())
    return fw_fail(S2B_ERR_WORKSPACE, "Fourier-Wigner workspace too small: need " +
                                          std::to_string(lay.total()) + " bytes");
  if (lay.total() && ((uintptr_t)ws & 255))
    return fw_fail(S2B_ERR_ALIGN, "Fourier-Wigner workspace must be 256-byte aligned");
  return S2B_OK;
}

FWSlices full_slices(int N, int reality) {
  FWSlices s{};
  s.S = reality ? N : 2 * N - 1;
  s.Stot = 2 * N - 1;
  s.Soff = reality ? N - 1 : 0;
  s.n0 = reality ? 0 : -(N - 1);
  s.nsign = 1;
  s.nlist = nullptr;
  return s;
}

FWSlices spin_slices(int nspins, const int* spins) {
  FWSlices s{};
  s.S = nspins;
  s.Stot = nspins;
  s.Soff = 0;
  s.n0 = 0;
  s.nsign = -1;  // slice n = -spin
  s.nlist = spins;
  return s;
}

}  // namespace

extern "C" {

int s2b_fw_plan_create(int L, int N, int sampling, int precision, s2b_fw_plan** plan) {
  if (!plan) return fw_fail(S2B_ERR_INVALID, "plan is NULL");
  *plan = nullptr;
  if (L < 2) return fw_fail(S2B_ERR_INVALID, "Fourier-Wigner transforms need L >= 2");
  if (N < 1 || N > L) return fw_fail(S2B_ERR_INVALID, "need 1 <= N <= L");
  if (sampling != S2B_MW && sampling != S2B_MWSS)
    return fw_fail(S2B_ERR_INVALID, "Fourier-Wigner algorithm supports mw and mwss sampling only");
  if (precision != S2B_F64 && precision != S2B_F32)
    return fw_fail(S2B_ERR_INVALID, "Fourier-Wigner precision must be S2B_F64 or S2B_F32");
  auto* p = new s2b_fw_plan();
  p->L = L;
  p->mwss = sampling == S2B_MWSS;
  p->ntheta = p->mwss ? L + 1 : L;
  p->nphi = p->mwss ? 2 * L : 2 * L - 1;
  p->P = 4 * L - 3;
  p->Q = 1;
  while (p->Q < 4 * L - 1) p->Q <<= 1;
  p->fp64 = precision == S2B_F64;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e != cudaSuccess) {
    delete p;
    return fw_fail(S2B_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  }
  p->N = N;
  p->gamma_fft = 2 * N - 1 >= kGamFFTMin;
  const int lens[3] = {p->nphi, p->Q, 2 * N - 1};
  const int rc = build_fft_set(lens, p->gamma_fft ? 3 : 2, p->fp64, &p->allocs, &p->fft);
  if (rc) {
    delete p;
    return rc;
  }
  // root tables of the quadrature weights (built once; the weights are recomputed from the
  // caller's quads on every forward call)
  for (int t = 0; t < 3; ++t) {
    const int n = t == 0 ? p->P : t == 1 ? p->Q : 2 * L + 1;
    void* d = nullptr;
    e = cudaMalloc(&d, (size_t)n * sizeof(double2));
    if (e == cudaSuccess) {
      p->allocs.push_back(d);
      if (t < 2)
        fw_roots_kernel<<<(n + 255) / 256, 256>>>(n, reinterpret_cast<double2*>(d));
      else
        fw_theta_phase_kernel<<<(n + 255) / 256, 256>>>(L, reinterpret_cast<double2*>(d));
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      delete p;
      return fw_fail(S2B_ERR_CUDA, std::string("phase tables: ") + cudaGetErrorString(e));
    }
    (t == 0 ? p->rootsP : t == 1 ? p->rootsQ : p->thW) = reinterpret_cast<double2*>(d);
  }
  // the column chain keeps a DFT buffer and Q values in shared memory
  const size_t cs = p->fp64 ? 16 : 8;
  const int bufM = std::max(p->fft.host[0].M, p->fft.host[1].M);
  if ((padded_len(bufM) + (size_t)p->Q) * cs > 227 * 1024) {
    delete p;
    return fw_fail(S2B_ERR_INVALID, "band-limit too large for the Fourier-Wigner beta chain");
  }
  *plan = p;
  return S2B_OK;
}

int s2b_fw_plan_destroy(s2b_fw_plan* plan) {
  delete plan;
  return S2B_OK;
}

int s2b_fw_quads(s2b_fw_plan* plan, void* quads, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if ((rc = check_ptrs({quads}))) return rc;
  fw_quads_kernel<<<(plan->P + 3) / 4, 128, 0, (cudaStream_t)stream>>>(
      plan->L, (double2*)quads, plan->rootsP);
  FW_CK(cudaGetLastError());
  return S2B_OK;
}

size_t s2b_fw_workspace_size(const s2b_fw_plan* plan, int op, int batch, int reality,
                             int nspins) {
  if (!plan || batch < 1) return 0;
  const int N = plan->N;
  switch (op) {
    case S2B_FW_INVERSE:
    case S2B_FW_FORWARD: {
      const long S = reality ? N : 2L * N - 1;
      return fw_layout(plan, (long)batch * S, (long)batch * (2L * N - 1), 0).total();
    }
    case S2B_FW_SUBSET_TO_S2:
    case S2B_FW_S2_TO_SUBSET:
      return fw_layout(plan, (long)batch * nspins, 0, 0).total();
    case S2B_FW_SO3_TO_SUBSET:
      return fw_layout(plan, (long)batch * nspins, 0, (long)batch * nspins).total();
    default:
      return 0;
  }
}

int s2b_fw_inverse(s2b_fw_plan* plan, int batch, int reality, const double* delta,
                   const void* flmn, void* f, void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1");
  const int N = plan->N;
  if ((rc = check_ptrs({delta, flmn, f}))) return rc;
  const FWSlices sl = full_slices(N, reality);
  const int E = batch * sl.S;
  if ((rc = check_slices((long)batch * sl.S))) return rc;
  const FWLayout lay = fw_layout(plan, E, (long)batch * (2L * N - 1), 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)ws;
  // the per-n maps go to region A (after Y is consumed), n-major for the gamma DFT
  if (plan->fp64)
    rc = inverse_chain<double>(plan, E, sl, delta, flmn, w, 1, batch, w, lay, st);
  else
    rc = inverse_chain<float>(plan, E, sl, delta, flmn, w, 1, batch, w, lay, st);
  if (rc) return rc;
  const long npix = (long)plan->ntheta * plan->nphi;
  return plan->fp64 ? gamma_dft<double>(plan, false, w, f, batch, N, npix, reality, st)
                    : gamma_dft<float>(plan, false, w, f, batch, N, npix, reality, st);
}

int s2b_fw_forward(s2b_fw_plan* plan, int batch, int reality, const double* delta,
                   const void* quads, const void* f, void* flmn, void* ws, size_t ws_bytes,
                   void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1");
  const int N = plan->N;
  if ((rc = check_ptrs({delta, quads, f, flmn}))) return rc;
  const FWSlices sl = full_slices(N, reality);
  const int E = batch * sl.S;
  if ((rc = check_slices((long)batch * sl.S))) return rc;
  const FWLayout lay = fw_layout(plan, E, (long)batch * (2L * N - 1), 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)ws;
  const long npix = (long)plan->ntheta * plan->nphi;
  // gamma DFT into region A, n-major
  rc = plan->fp64 ? gamma_dft<double>(plan, true, f, w, batch, N, npix, reality, st)
                  : gamma_dft<float>(plan, true, f, w, batch, N, npix, reality, st);
  if (rc) return rc;
  const double scale = 1.0 / plan->nphi;
  if (plan->fp64)
    rc = forward_chain<double>(plan, E, sl, delta, quads, w, flmn, 1, batch, scale, w, lay, st);
  else
    rc = forward_chain<float>(plan, E, sl, delta, quads, w, flmn, 1, batch, scale, w, lay, st);
  if (rc) return rc;
  if (reality) FW_CK(launch_wigner_mirror(plan->fp64, flmn, batch, N, plan->L, st));
  return S2B_OK;
}

int s2b_fw_inverse_adjoint(s2b_fw_plan* plan, int batch, const double* delta, const void* g_f,
                           void* g_flmn, void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1");
  const int N = plan->N;
  if ((rc = check_ptrs({delta, g_f, g_flmn}))) return rc;
  const FWSlices sl = full_slices(N, 0);
  const int E = batch * sl.S;
  if ((rc = check_slices((long)batch * sl.S))) return rc;
  const FWLayout lay = fw_layout(plan, E, (long)batch * (2L * N - 1), 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)ws;
  const long npix = (long)plan->ntheta * plan->nphi;
  // adjoint of the inverse gamma DFT: the forward DFT without its 1/G, into region A
  rc = plan->fp64 ? gamma_dft<double>(plan, true, g_f, w, batch, N, npix, 0, st, 1.0)
                  : gamma_dft<float>(plan, true, g_f, w, batch, N, npix, 0, st, 1.0);
  if (rc) return rc;
  return plan->fp64
             ? inverse_adjoint_chain<double>(plan, E, sl, delta, w, g_flmn, 1, batch, w, lay, st)
             : inverse_adjoint_chain<float>(plan, E, sl, delta, w, g_flmn, 1, batch, w, lay, st);
}

int s2b_fw_forward_adjoint(s2b_fw_plan* plan, int batch, const double* delta, const void* quads,
                           const void* g_flmn, void* g_f, void* ws, size_t ws_bytes,
                           void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1");
  const int N = plan->N;
  if ((rc = check_ptrs({delta, quads, g_flmn, g_f}))) return rc;
  const FWSlices sl = full_slices(N, 0);
  const int E = batch * sl.S;
  if ((rc = check_slices((long)batch * sl.S))) return rc;
  const FWLayout lay = fw_layout(plan, E, (long)batch * (2L * N - 1), 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)ws;
  const long npix = (long)plan->ntheta * plan->nphi;
  rc = plan->fp64 ? forward_adjoint_chain<double>(plan, E, sl, delta, quads, g_flmn, w, 1, batch,
                                                  w, lay, st)
                  : forward_adjoint_chain<float>(plan, E, sl, delta, quads, g_flmn, w, 1, batch,
                                                 w, lay, st);
  if (rc) return rc;
  // adjoint of the forward gamma DFT (with its 1/G): the inverse DFT times 1/G
  const double G = 2.0 * N - 1.0;
  return plan->fp64 ? gamma_dft<double>(plan, false, w, g_f, batch, N, npix, 0, st, 1.0 / G)
                    : gamma_dft<float>(plan, false, w, g_f, batch, N, npix, 0, st, 1.0 / G);
}

int s2b_fw_subset_to_s2(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                        const double* delta, const void* flmn, void* f, void* ws,
                        size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1 || nspins < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1 and nspins >= 1");
  if (!spins) return fw_fail(S2B_ERR_INVALID, "spins is NULL");
  if ((rc = check_ptrs({delta, flmn, f}))) return rc;
  const FWSlices sl = spin_slices(nspins, spins);
  const int E = batch * nspins;
  if ((rc = check_slices((long)batch * nspins))) return rc;
  const FWLayout lay = fw_layout(plan, E, 0, 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->fp64)
    return inverse_chain<double>(plan, E, sl, delta, flmn, f, 0, 1, (char*)ws, lay, st);
  return inverse_chain<float>(plan, E, sl, delta, flmn, f, 0, 1, (char*)ws, lay, st);
}

int s2b_fw_s2_to_subset(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                        const double* delta, const void* quads, const void* f, void* flmn,
                        void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1 || nspins < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1 and nspins >= 1");
  if (!spins) return fw_fail(S2B_ERR_INVALID, "spins is NULL");
  if ((rc = check_ptrs({delta, quads, f, flmn}))) return rc;
  const FWSlices sl = spin_slices(nspins, spins);
  const int E = batch * nspins;
  if ((rc = check_slices((long)batch * nspins))) return rc;
  const FWLayout lay = fw_layout(plan, E, 0, 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const double scale = 1.0 / plan->nphi;
  if (plan->fp64)
    return forward_chain<double>(plan, E, sl, delta, quads, f, flmn, 0, 1, scale, (char*)ws,
                                 lay, st);
  return forward_chain<float>(plan, E, sl, delta, quads, f, flmn, 0, 1, scale, (char*)ws, lay,
                              st);
}

int s2b_fw_so3_to_subset(s2b_fw_plan* plan, int batch, int ngamma, int nspins, const int* spins,
                         const double* delta, const void* quads, const void* f, void* flmn,
                         void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1 || nspins < 1 || ngamma < 1)
    return fw_fail(S2B_ERR_INVALID, "need batch, ngamma, nspins >= 1");
  if (ngamma > 46340)  // the gamma DFT's phase index c * n mod ngamma stays below 2^31
    return fw_fail(S2B_ERR_INVALID, "ngamma must be <= 46340");
  if (!spins) return fw_fail(S2B_ERR_INVALID, "spins is NULL");
  if ((rc = check_ptrs({delta, quads, f, flmn}))) return rc;
  const FWSlices sl = spin_slices(nspins, spins);
  const int E = batch * nspins;
  if ((rc = check_slices((long)batch * nspins))) return rc;
  const FWLayout lay = fw_layout(plan, E, 0, E);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)ws;
  void* C = w + lay.a + lay.b;
  const long npix = (long)plan->ntheta * plan->nphi;
  const long tot = (long)batch * npix;
  const int blocks = (int)std::min<long>((tot + 255) / 256, 65535L);
  if (plan->fp64)
    fw_gamma_subset_kernel<double><<<blocks, 256, 0, st>>>(f, C, batch, ngamma, nspins, npix, sl);
  else
    fw_gamma_subset_kernel<float><<<blocks, 256, 0, st>>>(f, C, batch, ngamma, nspins, npix, sl);
  FW_CK(cudaGetLastError());
  const double scale = 1.0 / plan->nphi;
  if (plan->fp64)
    return forward_chain<double>(plan, E, sl, delta, quads, C, flmn, 0, 1, scale, w, lay, st);
  return forward_chain<float>(plan, E, sl, delta, quads, C, flmn, 0, 1, scale, w, lay, st);
}

// Adjoints of the spin-subset ops (same arguments, workspace and layouts as the op they
// adjoin, with input and output exchanged).
int s2b_fw_subset_to_s2_adjoint(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                                const double* delta, const void* g_f, void* g_flmn, void* ws,
                                size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1 || nspins < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1 and nspins >= 1");
  if (!spins) return fw_fail(S2B_ERR_INVALID, "spins is NULL");
  if ((rc = check_ptrs({delta, g_f, g_flmn}))) return rc;
  const FWSlices sl = spin_slices(nspins, spins);
  const int E = batch * nspins;
  if ((rc = check_slices((long)batch * nspins))) return rc;
  const FWLayout lay = fw_layout(plan, E, 0, 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->fp64)
    return inverse_adjoint_chain<double>(plan, E, sl, delta, g_f, g_flmn, 0, 1, (char*)ws, lay, st);
  return inverse_adjoint_chain<float>(plan, E, sl, delta, g_f, g_flmn, 0, 1, (char*)ws, lay, st);
}

int s2b_fw_s2_to_subset_adjoint(s2b_fw_plan* plan, int batch, int nspins, const int* spins,
                                const double* delta, const void* quads, const void* g_flmn,
                                void* g_f, void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1 || nspins < 1) return fw_fail(S2B_ERR_INVALID, "need batch >= 1 and nspins >= 1");
  if (!spins) return fw_fail(S2B_ERR_INVALID, "spins is NULL");
  if ((rc = check_ptrs({delta, quads, g_flmn, g_f}))) return rc;
  const FWSlices sl = spin_slices(nspins, spins);
  const int E = batch * nspins;
  if ((rc = check_slices((long)batch * nspins))) return rc;
  const FWLayout lay = fw_layout(plan, E, 0, 0);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->fp64)
    return forward_adjoint_chain<double>(plan, E, sl, delta, quads, g_flmn, g_f, 0, 1,
                                         (char*)ws, lay, st);
  return forward_adjoint_chain<float>(plan, E, sl, delta, quads, g_flmn, g_f, 0, 1, (char*)ws,
                                      lay, st);
}

int s2b_fw_so3_to_subset_adjoint(s2b_fw_plan* plan, int batch, int ngamma, int nspins,
                                 const int* spins, const double* delta, const void* quads,
                                 const void* g_flmn, void* g_f, void* ws, size_t ws_bytes,
                                 void* stream) {
  int rc;
  if ((rc = check_plan(plan))) return rc;
  if (batch < 1 || nspins < 1 || ngamma < 1)
    return fw_fail(S2B_ERR_INVALID, "need batch, ngamma, nspins >= 1");
  if (ngamma > 46340)  // the gamma DFT's phase index c * n mod ngamma stays below 2^31
    return fw_fail(S2B_ERR_INVALID, "ngamma must be <= 46340");
  if (!spins) return fw_fail(S2B_ERR_INVALID, "spins is NULL");
  if ((rc = check_ptrs({delta, quads, g_flmn, g_f}))) return rc;
  const FWSlices sl = spin_slices(nspins, spins);
  const int E = batch * nspins;
  if ((rc = check_slices((long)batch * nspins))) return rc;
  const FWLayout lay = fw_layout(plan, E, 0, E);
  if ((rc = check_ws(lay, ws, ws_bytes))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)ws;
  void* C = w + lay.a + lay.b;
  rc = plan->fp64 ? forward_adjoint_chain<double>(plan, E, sl, delta, quads, g_flmn, C, 0, 1, w,
                                                  lay, st)
                  : forward_adjoint_chain<float>(plan, E, sl, delta, quads, g_flmn, C, 0, 1, w,
                                                 lay, st);
  if (rc) return rc;
  const long npix = (long)plan->ntheta * plan->nphi;
  const long tot = (long)batch * npix;
  const int blocks = (int)std::min<long>((tot + 255) / 256, 65535L);
  if (plan->fp64)
    fw_gamma_subset_adj_kernel<double><<<blocks, 256, 0, st>>>(C, g_f, batch, ngamma, nspins,
                                                               npix, sl);
  else
    fw_gamma_subset_adj_kernel<float><<<blocks, 256, 0, st>>>(C, g_f, batch, ngamma, nspins,
                                                              npix, sl);
  FW_CK(cudaGetLastError());
  return S2B_OK;
}

}  // extern "C"
