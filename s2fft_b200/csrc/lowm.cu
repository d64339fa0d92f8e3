// Orders m < |spin| of the latitudinal step by the degree recursion.
//
// For spin s != 0 the latitudinal kernels generate d^l_{m,n}(theta) (n = -s in half 0,
// n = +s in half 1) by the m-recursion from m = l down to m = 0, the order of upstream
// s2fft (s2fft/transforms/otf_recursions.py:134-171). On rings with n cos(theta) > 0 that
// recursion crosses, below m = n cos(theta) - sin(theta) sqrt(l^2 - n^2), a range where
// d^l_{m,n} decays as m decreases; a downward three-term recursion is unstable there and
// rounding errors grow like the dominant solution (first MW ring at L = 512, n = 7:
// d^7_{0,7} = 1.2e-18 comes out as 6.0 in double). The range lies inside m < |s| on every
// ring, so the latitudinal kernels leave the orders m < |s| out and the kernels below add
// them by the degree recursion at fixed (m, n) (s2b_degree.h), which is stable for every
// theta. All arithmetic is double, with a running power-of-two exponent for the small
// values near the poles; the values enter the sums in the monic form dt = d / g_{l,m} of
// the tables they complete.
//
// Cost: |s| orders out of L, one thread per (ring, order, half, map); the degree loop is
// sequential per thread, its coefficients are shared per CTA in shared memory.
#include <cuda_runtime.h>

#include <cstdint>

#include "s2b_degree.h"
#include "s2b_dev.h"
#include "s2b_lowm.h"

namespace s2b {
namespace {

constexpr int kLowmRings = 128;  // rings (threads) per CTA
constexpr int kLowmChunk = 256;  // degrees per coefficient chunk
static_assert(kLowmChunk % 32 == 0, "the projection reduces 32 degrees at a time");

struct LowmChunk {
  double a[kLowmChunk];   // a_l
  double c[kLowmChunk];   // m n / (l (l + 1))
  double b[kLowmChunk];   // b_l
  double ig[kLowmChunk];  // 1 / g_{l,m}
};

// Degree-recursion coefficients of order m for degrees [l0, l0 + kLowmChunk).
__device__ void lowm_fill(LowmChunk& ch, const double* __restrict__ g, int L, int m, int n,
                          int l0) {
  for (int i = threadIdx.x; i < kLowmChunk; i += blockDim.x) {
    const int l = l0 + i;
    double a = 0.0, c = 0.0, b = 0.0, ig = 0.0;
    if (l < L) {
      const DegreeCoef k = degree_coef(l, m, n);
      a = k.a;
      c = k.c;
      b = k.b;
      ig = 1.0 / g[(size_t)m * L + l];
    }
    ch.a[i] = a;
    ch.c[i] = c;
    ch.b[i] = b;
    ch.ig[i] = ig;
  }
}

// one degree step with the chunk's coefficients
__device__ __forceinline__ void lowm_step(const LowmChunk& ch, int i, double ct, double& cur,
                                          double& prv, int& E, double& sc) {
  degree_step(ch.a[i], ch.c[i], ch.b[i], ct, cur, prv, E, sc);
}

template <typename Real>
__global__ void __launch_bounds__(kLowmRings) lowm_synth_kernel(const LowmParams p) {
  using R2 = typename Vec<Real>::t2;
  __shared__ LowmChunk ch;
  __shared__ double2 fc[kLowmChunk];
  const int m = (int)blockIdx.y;
  const int half = (int)(blockIdx.z % p.nhalf);
  const int b = (int)(blockIdx.z / p.nhalf);
  if (half == 1 && m == 0) return;  // column m = 0 belongs to half 0 (uniform per CTA)
  const int n = half == 0 ? -p.spin : p.spin;
  const int j = n < 0 ? -n : n;
  const int L = p.L, TR = tab_rows(L);
  const int r = (int)blockIdx.x * kLowmRings + (int)threadIdx.x;
  const bool live = r < p.nrings;
  const RingInfo ri = p.rings[live ? r : 0];
  const double ct = ri.B / ri.A;  // cos(theta)
  double cur = 0.0, prv = 0.0, sx = 0.0, sy = 0.0;
  int E = 0;
  if (live) degree_seed(ri.lc, ri.ls, m, n, cur, E);
  double sc = ldexp(1.0, E);
  const R2* __restrict__ F =
      reinterpret_cast<const R2*>(p.F) + (size_t)(b * p.nhalf + half) * p.NB * TR * 32;
  for (int l0 = j; l0 < L; l0 += kLowmChunk) {
    __syncthreads();
    lowm_fill(ch, p.g, L, m, n, l0);
    for (int i = threadIdx.x; i < kLowmChunk; i += blockDim.x) {
      const int l = l0 + i;
      double2 f = make_double2(0.0, 0.0);
      if (l < L) {
        const R2 x = F[((size_t)(l >> 5) * TR + m + kPadLo) * 32 + (l & 31)];
        f = make_double2((double)x.x, (double)x.y);
      }
      fc[i] = f;
    }
    __syncthreads();
    const int cnt = min(kLowmChunk, L - l0);
    for (int i = 0; i < cnt; ++i) {
      const double t = cur * sc * ch.ig[i];
      sx = fma(t, fc[i].x, sx);
      sy = fma(t, fc[i].y, sy);
      lowm_step(ch, i, ct, cur, prv, E, sc);
    }
  }
  if (live) {
    R2* ftm = reinterpret_cast<R2*>(p.ftm) + ((size_t)b * p.nrows + p.ring_row[r]) * p.ncol;
    R2 o;
    o.x = (Real)sx;
    o.y = (Real)sy;
    red_add(ftm + (L - 1 + (half == 0 ? m : -m) + p.mo), o);
  }
}

template <typename Real>
__global__ void __launch_bounds__(kLowmRings) lowm_project_kernel(const LowmParams p) {
  using R2 = typename Vec<Real>::t2;
  constexpr int NW = kLowmRings / 32;
  __shared__ LowmChunk ch;
  __shared__ double2 ws[NW][kLowmChunk];
  const int m = (int)blockIdx.y;
  const int half = (int)(blockIdx.z % p.nhalf);
  const int b = (int)(blockIdx.z / p.nhalf);
  if (half == 1 && m == 0) return;  // order 0 is projected by half 0 only (uniform per CTA)
  const int n = half == 0 ? -p.spin : p.spin;
  const int j = n < 0 ? -n : n;
  const int L = p.L, TR = tab_rows(L), Lp = p.NB * 32;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int r = (int)blockIdx.x * kLowmRings + (int)threadIdx.x;
  const bool live = r < p.nrings;
  const RingInfo ri = p.rings[live ? r : 0];
  const double ct = ri.B / ri.A;
  double gx = 0.0, gy = 0.0, cur = 0.0, prv = 0.0;
  int E = 0;
  if (live) {
    const R2 x = reinterpret_cast<const R2*>(
        p.G)[(((size_t)b * p.nhalf + half) * TR + m + kPadLo) * p.Gs + r];
    gx = x.x;
    gy = x.y;
    degree_seed(ri.lc, ri.ls, m, n, cur, E);
  }
  double sc = ldexp(1.0, E);
  R2* __restrict__ acc =
      reinterpret_cast<R2*>(p.acc) + (((size_t)b * p.nhalf + half) * L + m) * Lp;
  for (int l0 = j; l0 < L; l0 += kLowmChunk) {
    __syncthreads();
    lowm_fill(ch, p.g, L, m, n, l0);
    __syncthreads();
    const int cnt = min(kLowmChunk, L - l0);
    for (int i0 = 0; i0 < cnt; i0 += 32) {  // uniform; degrees past L have zero coefficients
      double vx[32], vy[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const double t = cur * sc * ch.ig[i0 + i];
        vx[i] = t * gx;
        vy[i] = t * gy;
        lowm_step(ch, i0 + i, ct, cur, prv, E, sc);
      }
      // transpose reduction over the warp's rings: at the level of stride `off` a lane keeps
      // the degrees whose bit `off` equals its own and adds its partner's; lane k ends with
      // the warp sum of degree l0 + i0 + k (31 shuffles per component for 32 degrees)
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) {
        const bool up = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < off; ++i) {
          const double sx = up ? vx[i] : vx[i + off];
          const double sy = up ? vy[i] : vy[i + off];
          const double kx = up ? vx[i + off] : vx[i];
          const double ky = up ? vy[i + off] : vy[i];
          vx[i] = kx + __shfl_xor_sync(0xffffffffu, sx, off);
          vy[i] = ky + __shfl_xor_sync(0xffffffffu, sy, off);
        }
      }
      ws[wp][i0 + lane] = make_double2(vx[0], vy[0]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      double2 s = ws[0][i];
#pragma unroll
      for (int w = 1; w < NW; ++w) {
        s.x += ws[w][i].x;
        s.y += ws[w][i].y;
      }
      R2 o;
      o.x = (Real)s.x;
      o.y = (Real)s.y;
      red_add(acc + l0 + i, o);
    }
  }
}

template <typename Real>
cudaError_t lowm_launch(bool project, const LowmParams& p, cudaStream_t s) {
  if (p.mlo <= 0 || p.nrings <= 0 || p.batch <= 0) return cudaSuccess;
  if (p.nhalf < 1 || p.nhalf > 2 || (long)p.batch * p.nhalf > 65535 || p.mlo > 65535)
    return cudaErrorInvalidValue;
  dim3 grid((p.nrings + kLowmRings - 1) / kLowmRings, p.mlo, p.batch * p.nhalf);
  if (project)
    lowm_project_kernel<Real><<<grid, kLowmRings, 0, s>>>(p);
  else
    lowm_synth_kernel<Real><<<grid, kLowmRings, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_lowm_synth(bool fp64, const LowmParams& p, cudaStream_t s) {
  return fp64 ? lowm_launch<double>(false, p, s) : lowm_launch<float>(false, p, s);
}

cudaError_t launch_lowm_project(bool fp64, const LowmParams& p, cudaStream_t s) {
  return fp64 ? lowm_launch<double>(true, p, s) : lowm_launch<float>(true, p, s);
}

}  // namespace s2b
