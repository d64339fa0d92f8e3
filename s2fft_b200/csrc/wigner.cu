// Wigner (SO(3)) transform stages: the gamma-axis DFT and the per-n gather /
// scatter of the coefficient slices around the 2N-1 spin transforms.
// Follows s2fft/transforms/wigner.py:110-196 (inverse_numpy) and 442-533
// (forward_numpy): flmn[n] * sqrt((2l+1)/(16 pi^3)) -> spin -n inverse SHTs,
// (-1)^n, then an inverse DFT over gamma; forward: DFT over gamma times
// 2pi/(2N-1), spin -n forward SHTs, (-1)^n, times sqrt(4pi/(2l+1)).
#include <cuda_runtime.h>

#include <type_traits>

#include "s2b_wigner.h"

namespace s2b {

template <typename Real>
using W2 = std::conditional_t<sizeof(Real) == 4, float2, double2>;

static int wgrid(long n) {
  long b = (n + 255) / 256;
  if (b > 65535) b = 65535;
  return b < 1 ? 1 : (int)b;
}

// tmp[b][l][c] = flmn[b][N-1+n][l][c] * (-1)^n sqrt((2l+1)/(16 pi^3)); the spin
// transform that follows applies its own sqrt((2l+1)/4pi) on top, as upstream does.
// real0 (real signals, slice n = 0): upstream runs that slice as a real spin-0 inverse,
// which reads the orders m >= 0 only and takes the real part of their Hermitian extension
// (wigner.py:176-187, spherical.py:176-208); the complex transform that follows does the
// same when the orders are weighted by 0 (m < 0), 1 (m = 0) and 2 (m > 0) and the gamma DFT
// keeps the real part of the slice.
template <typename Real>
__global__ void gather_n_kernel(const W2<Real>* flmn, W2<Real>* tmp, int B, int N, int L, int n,
                                int real0) {
  const long per = (long)L * (2 * L - 1);
  const long total = per * B;
  const double pi = 3.141592653589793;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long b = i / per, r = i % per;
    const int l = (int)(r / (2 * L - 1));
    const int m = (int)(r % (2 * L - 1)) - (L - 1);
    double f = ((n & 1) ? -1.0 : 1.0) * sqrt((2.0 * l + 1.0) / (16.0 * pi * pi * pi));
    if (real0) f *= m < 0 ? 0.0 : (m == 0 ? 1.0 : 2.0);
    W2<Real> v = flmn[(b * (2 * N - 1) + (N - 1 + n)) * per + r];
    v.x = (Real)(v.x * f);
    v.y = (Real)(v.y * f);
    tmp[i] = v;
  }
}

// flmn[b][N-1+n][l][c] = (-1)^n sqrt(4pi/(2l+1)) tmp[b][l][c]  (l >= L0; else 0)
template <typename Real>
__global__ void scatter_n_kernel(const W2<Real>* tmp, W2<Real>* flmn, int B, int N, int L, int n,
                                 int L0) {
  const long per = (long)L * (2 * L - 1);
  const long total = per * B;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long b = i / per, r = i % per;
    const int l = (int)(r / (2 * L - 1));
    W2<Real> v = tmp[i];
    double f = 0.0;
    if (l >= L0) f = ((n & 1) ? -1.0 : 1.0) * sqrt(4.0 * 3.141592653589793 / (2.0 * l + 1.0));
    v.x = (Real)(v.x * f);
    v.y = (Real)(v.y * f);
    flmn[(b * (2 * N - 1) + (N - 1 + n)) * per + r] = v;
  }
}

// reality: flmn[N-1-n][l][L-1-m] = conj(flmn[N-1+n][l][L-1+m]) (-1)^(m+n), n >= 1
template <typename Real>
__global__ void wigner_mirror_kernel(W2<Real>* flmn, int B, int N, int L) {
  const long per = (long)L * (2 * L - 1);
  const long total = per * B * (N - 1);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long r = i % per;
    const long rest = i / per;
    const int n = 1 + (int)(rest % (N - 1));
    const long b = rest / (N - 1);
    const int l = (int)(r / (2 * L - 1));
    const int c = (int)(r % (2 * L - 1));
    const int m = c - (L - 1);
    W2<Real> v = flmn[(b * (2 * N - 1) + (N - 1 + n)) * per + (long)l * (2 * L - 1) + (L - 1 + m)];
    const int am = m < 0 ? -m : m;
    const double s = ((am + n) & 1) ? -1.0 : 1.0;
    W2<Real> o;
    o.x = (Real)(s * v.x);
    o.y = (Real)(-s * v.y);
    flmn[(b * (2 * N - 1) + (N - 1 - n)) * per + (long)l * (2 * L - 1) + (L - 1 - m)] = o;
  }
}

// exp(sign 2 pi i ((j * k) mod G) / G) for j, k < G, one table per CTA in shared memory
// (G = 2N - 1 <= 2L - 1; computed in double, kept in double)
__device__ inline void gamma_phases(double2* tab, int G, double sign) {
  for (int x = threadIdx.x; x < G * G; x += blockDim.x) {
    const int j = x / G, k = x % G;
    double sn, cs;
    sincospi(sign * 2.0 * (double)((j * k) % G) / (double)G, &sn, &cs);
    tab[x] = make_double2(cs, sn);
  }
  __syncthreads();
}

// Inverse gamma DFT: f[b][k][p] = sum_n fban[n][b][p] exp(+2 pi i n k / (2N-1)),
// n in [-(N-1), N-1]; reality: real output from n >= 0 (irfft semantics).
template <typename Real>
__global__ void gamma_inverse_kernel(const W2<Real>* fban, void* f, int B, int N, long npix,
                                     int reality) {
  extern __shared__ double2 tab[];  // [n mod G][k]
  const int G = 2 * N - 1;
  gamma_phases(tab, G, 1.0);
  const long total = (long)B * npix;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long b = i / npix, px = i % npix;
    for (int k = 0; k < G; ++k) {
      double re = 0.0, im = 0.0;
      for (int n = reality ? 0 : -(N - 1); n < N; ++n) {
        const W2<Real> x = fban[((long)(N - 1 + n) * B + b) * npix + px];
        const double2 e = tab[((n + G) % G) * G + k];
        double xr = x.x, xi = x.y;
        if (reality && n == 0) xi = 0.0;
        const double w = (reality && n > 0) ? 2.0 : 1.0;
        re += w * (xr * e.x - xi * e.y);
        im += w * (xr * e.y + xi * e.x);
      }
      if (reality) {
        reinterpret_cast<Real*>(f)[(b * G + k) * npix + px] = (Real)re;
      } else {
        W2<Real> o;
        o.x = (Real)re;
        o.y = (Real)im;
        reinterpret_cast<W2<Real>*>(f)[(b * G + k) * npix + px] = o;
      }
    }
  }
}

// Forward gamma DFT: fban[n][b][p] = 2pi/(2N-1) sum_k f[b][k][p] exp(-2 pi i n k/(2N-1)),
// n in [n0, N-1] (n0 = 0 for real input).
template <typename Real>
__global__ void gamma_forward_kernel(const void* f, W2<Real>* fban, int B, int N, long npix,
                                     int reality) {
  extern __shared__ double2 tab[];
  const int G = 2 * N - 1;
  gamma_phases(tab, G, -1.0);
  const long total = (long)B * npix;
  const double sc = 2.0 * 3.141592653589793 / (double)G;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long b = i / npix, px = i % npix;
    for (int n = reality ? 0 : -(N - 1); n < N; ++n) {
      double re = 0.0, im = 0.0;
      for (int k = 0; k < G; ++k) {
        double xr, xi;
        if (reality) {
          xr = reinterpret_cast<const Real*>(f)[(b * G + k) * npix + px];
          xi = 0.0;
        } else {
          const W2<Real> x = reinterpret_cast<const W2<Real>*>(f)[(b * G + k) * npix + px];
          xr = x.x;
          xi = x.y;
        }
        const double2 e = tab[((n + G) % G) * G + k];
        re += xr * e.x - xi * e.y;
        im += xr * e.y + xi * e.x;
      }
      W2<Real> o;
      o.x = (Real)(sc * re);
      o.y = (Real)(sc * im);
      fban[((long)(N - 1 + n) * B + b) * npix + px] = o;
    }
  }
}

cudaError_t launch_gather_n(bool fp64, const void* flmn, void* tmp, int B, int N, int L, int n,
                            int real0, cudaStream_t s) {
  const long tot = (long)B * L * (2 * L - 1);
  if (fp64)
    gather_n_kernel<double><<<wgrid(tot), 256, 0, s>>>((const double2*)flmn, (double2*)tmp, B, N, L, n,
                                                       real0);
  else
    gather_n_kernel<float><<<wgrid(tot), 256, 0, s>>>((const float2*)flmn, (float2*)tmp, B, N, L, n,
                                                      real0);
  return cudaGetLastError();
}

cudaError_t launch_scatter_n(bool fp64, const void* tmp, void* flmn, int B, int N, int L, int n,
                             int L0, cudaStream_t s) {
  const long tot = (long)B * L * (2 * L - 1);
  if (fp64)
    scatter_n_kernel<double><<<wgrid(tot), 256, 0, s>>>((const double2*)tmp, (double2*)flmn, B, N, L, n, L0);
  else
    scatter_n_kernel<float><<<wgrid(tot), 256, 0, s>>>((const float2*)tmp, (float2*)flmn, B, N, L, n, L0);
  return cudaGetLastError();
}

cudaError_t launch_wigner_mirror(bool fp64, void* flmn, int B, int N, int L, cudaStream_t s) {
  if (N < 2) return cudaSuccess;
  const long tot = (long)B * (N - 1) * L * (2 * L - 1);
  if (fp64)
    wigner_mirror_kernel<double><<<wgrid(tot), 256, 0, s>>>((double2*)flmn, B, N, L);
  else
    wigner_mirror_kernel<float><<<wgrid(tot), 256, 0, s>>>((float2*)flmn, B, N, L);
  return cudaGetLastError();
}

cudaError_t launch_gamma_inverse(bool fp64, const void* fban, void* f, int B, int N, long npix,
                                 int reality, cudaStream_t s) {
  const size_t sm = (size_t)(2 * N - 1) * (2 * N - 1) * sizeof(double2);
  if (fp64)
    gamma_inverse_kernel<double><<<wgrid((long)B * npix), 256, sm, s>>>((const double2*)fban, f, B, N, npix, reality);
  else
    gamma_inverse_kernel<float><<<wgrid((long)B * npix), 256, sm, s>>>((const float2*)fban, f, B, N, npix, reality);
  return cudaGetLastError();
}

cudaError_t launch_gamma_forward(bool fp64, const void* f, void* fban, int B, int N, long npix,
                                 int reality, cudaStream_t s) {
  const size_t sm = (size_t)(2 * N - 1) * (2 * N - 1) * sizeof(double2);
  if (fp64)
    gamma_forward_kernel<double><<<wgrid((long)B * npix), 256, sm, s>>>(f, (double2*)fban, B, N, npix, reality);
  else
    gamma_forward_kernel<float><<<wgrid((long)B * npix), 256, sm, s>>>(f, (float2*)fban, B, N, npix, reality);
  return cudaGetLastError();
}

}  // namespace s2b
