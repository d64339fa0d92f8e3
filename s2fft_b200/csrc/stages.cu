// Element-wise stages around the latitudinal kernel:
//  * inverse prologue: flm -> recursion-ready coefficient table F
//    (harmonic normalisation sqrt((2l+1)/4pi), (-1)^s, the monic scale g_{l,m}
//    and the m < 0 symmetry sign; s2fft/transforms/spherical.py:165-168, 192);
//  * inverse pole rows in closed form (spherical.py:175-184);
//  * forward epilogue: projected sums -> flm (g_{l,m}, pole terms, normalisation,
//    reality mirror, spin/L_lower mask, (-1)^s; spherical.py:566-588).
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "s2b_dev.h"
#include "s2b_internal.h"
#include "s2b_stages.h"

namespace s2b {

template <typename Real>
using R2_t = std::conditional_t<sizeof(Real) == 4, float2, double2>;
template <typename Real>
using R4_t = std::conditional_t<sizeof(Real) == 4, float4, double4>;

__device__ __forceinline__ double lnorm(int l) { return sqrt((2.0 * l + 1.0) / (4.0 * 3.141592653589793)); }

// F [b][half][j][m + kPadLo][q] (Real2, or Real4 when dual) from flm [b][l][L-1+m];
// the pad rows (m < 0, m = L) are written as zeros.
// Idx is the flat index type: 32-bit whenever the whole table fits, since 64-bit
// division by a runtime divisor costs several times the 32-bit one and these
// kernels are bound by their index arithmetic.
template <typename Real, typename Idx>
__global__ void prologue_kernel(StageParams p) {
  using R2 = R2_t<Real>;
  using R4 = R4_t<Real>;
  const int L = p.L, C = p.nclass, Q = p.Q, TR = p.TR;
  const Idx total = (Idx)p.nhalf * C * TR * Q * p.batch;
  const R2* flm = reinterpret_cast<const R2*>(p.flm);
  for (Idx idx = blockIdx.x * (Idx)blockDim.x + threadIdx.x; idx < total;
       idx += (Idx)gridDim.x * blockDim.x) {
    Idx r = idx;
    const int q = (int)(r % (Idx)Q);
    r /= (Idx)Q;
    const int m = (int)(r % (Idx)TR) - kPadLo;
    r /= (Idx)TR;
    const int j = (int)(r % (Idx)C);
    r /= (Idx)C;
    const int half = (int)(r % (Idx)p.nhalf);
    const int b = (int)(r / (Idx)p.nhalf);
    const int l = p.Lp > 0 ? j * Q + q : j + C * q;  // blocked: l = 32 block + column
    const int as = p.spin < 0 ? -p.spin : p.spin;
    const bool ok = m >= 0 && m < L && l < L && l >= m && l >= p.L0 && l >= as;
    double g = 0.0;
    if (ok) g = p.g[(size_t)m * L + l] * lnorm(l);
    const R2* row = flm + ((size_t)b * L + (ok ? l : 0)) * (2 * L - 1) + (ok ? 0 : (L - 1));
    const int mm = ok ? m : 0;
    const double sgn_s = (p.spin & 1) ? -1.0 : 1.0;
    const double sgn_m = (m & 1) ? -1.0 : 1.0;
    if (p.dual) {
      R4 o;
      R2 a = row[L - 1 + mm], c = row[L - 1 - mm];
      const double gp = ok ? g : 0.0;
      const double gn = (ok && m > 0) ? g * sgn_m : 0.0;
      o.x = (Real)(gp * a.x);
      o.y = (Real)(gp * a.y);
      o.z = (Real)(gn * c.x);
      o.w = (Real)(gn * c.y);
      reinterpret_cast<R4*>(p.F)[idx] = o;
    } else {
      R2 o;
      if (half == 0) {
        const R2 a = row[L - 1 + mm];
        const double f = ok ? g * sgn_s : 0.0;
        o.x = (Real)(f * a.x);
        o.y = (Real)(f * a.y);
      } else {
        const R2 a = row[L - 1 - mm];
        const double f = (ok && m > 0) ? g * sgn_m : 0.0;
        o.x = (Real)(f * a.x);
        o.y = (Real)(f * a.y);
      }
      reinterpret_cast<R2*>(p.F)[idx] = o;
    }
  }
}

// Pole rows of the inverse: ftm[pole][L-1+ms+mo] = (-1)^s sum_l sign_l N_l flm[l][L-1+ms],
// south (theta = pi): ms = s, sign_l = (-1)^(l-s); north (theta = 0): ms = -s, sign 1.
// One CTA of 256 threads per (pole, map); red holds 2 x 256 doubles of shared memory.
template <typename Real>
__device__ __forceinline__ void poles_block(const StageParams& p, int which, int b, int tid,
                                            double* red) {
  using R2 = R2_t<Real>;
  const int L = p.L;
  const int row = which == 0 ? p.pole_south : p.pole_north;
  if (row < 0) return;
  const int ms = which == 0 ? p.spin : -p.spin;
  const R2* flm = reinterpret_cast<const R2*>(p.flm) + (size_t)b * L * (2 * L - 1);
  R2* ftm = reinterpret_cast<R2*>(p.ftm) + ((size_t)b * p.nrows + row) * p.ncol;
  if (p.zero_ftm) {
    // the pole row is this CTA's to clear; the reduction's barriers order it before the store
    R2 z;
    z.x = z.y = 0;
    for (int c = tid; c < p.ncol; c += 256) ftm[c] = z;
  }
  double sx = 0.0, sy = 0.0;
#pragma unroll 1
  for (int l = p.L0 + tid; l < L; l += 256) {
    double f = lnorm(l);
    if (which == 0 && (((l - p.spin) % 2 + 2) % 2)) f = -f;
    const R2 a = flm[(size_t)l * (2 * L - 1) + L - 1 + ms];
    sx += f * a.x;
    sy += f * a.y;
  }
  red[tid] = sx;
  red[256 + tid] = sy;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (tid < st) {
      red[tid] += red[tid + st];
      red[256 + tid] += red[256 + tid + st];
    }
    __syncthreads();
  }
  if (tid == 0) {
    const double sg = (p.spin & 1) ? -1.0 : 1.0;
    R2 o;
    o.x = (Real)(sg * red[0]);
    o.y = (Real)(sg * red[256]);
    ftm[L - 1 + ms + p.mo] = o;
  }
}

// grid (2, batch), 256 threads
template <typename Real>
__global__ void __launch_bounds__(256) poles_kernel(StageParams p) {
  __shared__ double red[2 * 256];
  poles_block<Real>(p, blockIdx.x, blockIdx.y, threadIdx.x, red);
}

// Zeroes ftm [batch][nrows][ncol] before the latitudinal kernel accumulates into it, in units
// of 256 entries of one row spread over the prologue's tile CTAs (cta of ncta); with
// pole_blocks the pole rows are left to their pole CTAs.
template <typename Real>
__device__ __forceinline__ void zero_ftm_rows(const StageParams& p, int cta, int ncta, int tid) {
  using R2 = R2_t<Real>;
  const int nseg = (p.ncol + 255) / 256;
  const int units = p.batch * p.nrows * nseg;  // below 2^31 (launch_prologue)
  R2 z;
  z.x = z.y = 0;
  for (int u = cta; u < units; u += ncta) {
    const int rg = u / nseg, c = (u - rg * nseg) * 256 + tid;
    const int row = rg % p.nrows;
    if (p.pole_blocks && (row == p.pole_south || row == p.pole_north)) continue;
    if (c < p.ncol) reinterpret_cast<R2*>(p.ftm)[(size_t)rg * p.ncol + c] = z;
  }
}

// Blocked layout (p.Lp > 0, Q = 32): the same table, a 32 (m) x 32 (l) tile per CTA through
// shared memory, since flm is [l][m] and F is [m][l]: the coefficients are read with
// consecutive threads on consecutive m, the table (and g) with consecutive threads on
// consecutive l. grid (ceil(TR / 32) + pole_blocks, C, batch * nhalf), 32 x 8 threads; with
// pole_blocks the last column of CTAs computes the pole rows instead (y = 0 south, 1 north),
// with zero_ftm the tile CTAs also clear ftm.
template <typename Real>
__global__ void __launch_bounds__(256) prologue_tiled_kernel(StageParams p) {
  chain_enter();
  using R2 = R2_t<Real>;
  using R4 = R4_t<Real>;
  __shared__ R2 ta[32][33], tc[32][33];  // [q][m]: flm at +m and at -m, padded
  const int L = p.L, C = p.nclass, TR = p.TR;
  const int m0 = (int)blockIdx.x * 32 - kPadLo, j = blockIdx.y;
  const int half = (int)(blockIdx.z % p.nhalf), b = (int)(blockIdx.z / p.nhalf);
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (p.pole_blocks && blockIdx.x == gridDim.x - 1) {
    static_assert(sizeof(ta) >= 2 * 256 * sizeof(double), "pole reduction fits the tile");
    if (j < 2 && half == 0)
      poles_block<Real>(p, j, b, ty * 32 + tx, reinterpret_cast<double*>(&ta[0][0]));
    return;
  }
  if (p.zero_ftm) {
    const int gx = (int)gridDim.x - p.pole_blocks;
    zero_ftm_rows<Real>(p, (int)blockIdx.x + gx * (j + (int)gridDim.y * (int)blockIdx.z),
                        gx * (int)gridDim.y * (int)gridDim.z, ty * 32 + tx);
  }
  const R2* flm = reinterpret_cast<const R2*>(p.flm) + (size_t)b * L * (2 * L - 1);
  // a thread keeps one l in the second pass: its four weights are loaded here, beside the
  // coefficients, so that both wait on memory together
  const int as = p.spin < 0 ? -p.spin : p.spin;
  const int lt = 32 * j + tx;
  double gk[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int m = m0 + ty + 8 * k;
    const bool ok = m >= 0 && m < L && lt < L && lt >= m && lt >= p.L0 && lt >= as;
    gk[k] = ok ? p.g[(size_t)m * L + lt] : 0.0;
  }
#pragma unroll
  for (int qq = ty; qq < 32; qq += 8) {
    const int l = 32 * j + qq, m = m0 + tx;
    R2 a, c;
    a.x = a.y = c.x = c.y = 0;
    if (m >= 0 && m < L && l < L && l >= m) {
      const R2* row = flm + (size_t)l * (2 * L - 1) + (L - 1);
      if (p.dual || half == 0) a = row[m];
      if (p.dual || half == 1) c = row[-m];
    }
    ta[qq][tx] = a;
    tc[qq][tx] = c;
  }
  __syncthreads();
  const double sgn_s = (p.spin & 1) ? -1.0 : 1.0;
  const double nl = lnorm(lt);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int mm = ty + 8 * k;
    const int m = m0 + mm, mrow = m + kPadLo;
    if (mrow >= TR) continue;
    const double g = gk[k] * nl;
    const double sgn_m = (m & 1) ? -1.0 : 1.0;
    const size_t idx = ((((size_t)b * p.nhalf + half) * C + j) * TR + mrow) * 32 + tx;
    if (p.dual) {
      const R2 a = ta[tx][mm], c = tc[tx][mm];
      const double gn = m > 0 ? g * sgn_m : 0.0;
      R4 o;
      o.x = (Real)(g * a.x);
      o.y = (Real)(g * a.y);
      o.z = (Real)(gn * c.x);
      o.w = (Real)(gn * c.y);
      reinterpret_cast<R4*>(p.F)[idx] = o;
    } else {
      const R2 a = half == 0 ? ta[tx][mm] : tc[tx][mm];
      const double f = half == 0 ? g * sgn_s : (m > 0 ? g * sgn_m : 0.0);
      R2 o;
      o.x = (Real)(f * a.x);
      o.y = (Real)(f * a.y);
      reinterpret_cast<R2*>(p.F)[idx] = o;
    }
  }
}

// Weighted ring spectrum at (row, m) from the forward spectra array G.
template <typename Real>
__device__ __forceinline__ R2_t<Real> spectrum_at(const StageParams& p, int b, int row, int m) {
  using R2 = R2_t<Real>;
  const int am = m < 0 ? -m : m;
  const R2* G = reinterpret_cast<const R2*>(p.G);
  const size_t mr = (size_t)(am + kPadLo);
  if (p.dual) return G[(((size_t)b * p.TR + mr) * p.Gs + row) * 2 + (m < 0 ? 1 : 0)];
  if (m >= 0) return G[(((size_t)b * p.nhalf + 0) * p.TR + mr) * p.Gs + row];
  if (p.nhalf > 1) return G[(((size_t)b * p.nhalf + 1) * p.TR + mr) * p.Gs + row];
  R2 z;
  z.x = 0;
  z.y = 0;
  return z;
}

// The loads behind one flm[b][l][L-1+m]: the projected sum at (|m|, l) of the half that
// holds m, and the projection weight g[|m|][l]; ok is false outside l >= max(|s|, L0),
// |m| <= l (the value is zero there), mirror marks a reality -m taken from +m.
struct EpiCell {
  double ar, ai, g;
  bool ok, mirror;
};

template <typename Real>
__device__ __forceinline__ EpiCell epi_fetch(const StageParams& p, int b, int l, int m) {
  using R2 = R2_t<Real>;
  const int L = p.L, C = p.nclass, Q = p.Q;
  const int as = p.spin < 0 ? -p.spin : p.spin;
  const int lmin = as > p.L0 ? as : p.L0;
  const int am = m < 0 ? -m : m;
  EpiCell e;
  e.ar = e.ai = e.g = 0.0;
  e.ok = l >= lmin && am <= l;
  e.mirror = !p.dual && m < 0 && p.nhalf <= 1;
  if (e.ok) {
    const int j = l % C, q = l / C;
    // offset of (m, l) in one [batch][half] slice of the forward sums, in R2/R4 units
    const size_t cell = p.Lp > 0 ? (size_t)am * p.Lp + l : ((size_t)j * L + am) * Q + q;
    const size_t slice = p.Lp > 0 ? (size_t)L * p.Lp : (size_t)C * L * Q;
    const R2* A = reinterpret_cast<const R2*>(p.acc);
    size_t at;
    if (p.dual)
      at = ((size_t)b * slice + cell) * 2 + (m < 0 ? 1 : 0);
    else if (!e.mirror)
      at = ((size_t)b * p.nhalf + (m >= 0 ? 0 : 1)) * slice + cell;
    else  // reality: flm[l, -m] = (-1)^m conj(flm[l, m])
      at = (size_t)b * slice + cell;
    const R2 a = A[at];
    e.ar = a.x;
    e.ai = a.y;
    e.g = p.g[(size_t)am * L + l];
  }
  return e;
}

// flm[b][l][L-1+m] from its fetched cell; nl = N_l (-1)^s, the degree's normalisation.
template <typename Real>
__device__ __forceinline__ R2_t<Real> epi_finish(const StageParams& p, int b, int l, int m,
                                                 const EpiCell& e, double nl) {
  using R2 = R2_t<Real>;
  const int am = m < 0 ? -m : m;
  double re = 0.0, im = 0.0;
  if (e.ok) {
    // d-projection with the m < 0 symmetry sign (-1)^(m+s) (spin folded below)
    double f = e.g;
    if (m < 0 && !e.mirror) f *= ((am + p.spin) % 2 + 2) % 2 ? -1.0 : 1.0;
    re = f * e.ar;
    im = f * e.ai;
    // closed-form pole rings (each present pole: theta = pi contributes at m = s, theta = 0 at
    // m = -s)
    if (!e.mirror) {
      if (p.pole_south >= 0 && m == p.spin) {
        const R2 s = spectrum_at<Real>(p, b, p.pole_south, m);
        const double sg = ((l - p.spin) % 2 + 2) % 2 ? -1.0 : 1.0;
        re += sg * s.x;
        im += sg * s.y;
      }
      if (p.pole_north >= 0 && m == -p.spin) {
        const R2 s = spectrum_at<Real>(p, b, p.pole_north, m);
        re += s.x;
        im += s.y;
      }
    }
    re *= nl;
    im *= nl;
    if (e.mirror) {
      // value above is flm[l, |m|]; mirror (-1)^m conj(.)
      const double sm = (am & 1) ? -1.0 : 1.0;
      im = -im;
      re *= sm;
      im *= sm;
    }
  }
  R2 o;
  o.x = (Real)re;
  o.y = (Real)im;
  return o;
}

__device__ __forceinline__ double epi_norm(const StageParams& p, int l) {
  return lnorm(l) * ((p.spin & 1) ? -1.0 : 1.0);
}

// flm[b][l][L-1+m] from the projected sums acc [b][half][j][m][q] (one element).
template <typename Real>
__device__ __forceinline__ R2_t<Real> epi_value(const StageParams& p, int b, int l, int m) {
  return epi_finish<Real>(p, b, l, m, epi_fetch<Real>(p, b, l, m), epi_norm(p, l));
}

// flm [b][l][L-1+m] from the projected sums, one element per thread (any layout).
template <typename Real, typename Idx>
__global__ void epilogue_kernel(StageParams p) {
  const int L = p.L;
  const int W = 2 * L - 1;
  const Idx total = (Idx)p.batch * L * W;
  for (Idx idx = blockIdx.x * (Idx)blockDim.x + threadIdx.x; idx < total;
       idx += (Idx)gridDim.x * blockDim.x) {
    const Idx lw = idx / (Idx)W;
    const int c = (int)(idx - lw * (Idx)W);
    const Idx bl = lw / (Idx)L;
    const int l = (int)(lw - bl * (Idx)L);
    reinterpret_cast<R2_t<Real>*>(p.flm_out)[idx] = epi_value<Real>(p, (int)bl, l, c - (L - 1));
  }
}

// Blocked layouts: the sums are [m][l] and flm is [l][m], so a CTA transposes a 32 x 32
// tile through shared memory: it computes the tile with consecutive threads on
// consecutive l (coalesced reads of the sums and of g) and writes it with consecutive
// threads on consecutive m. grid (ceil((2L-1)/32), ceil(L/32), batch), 32 x 8 threads.
template <typename Real>
__global__ void __launch_bounds__(256) epilogue_tiled_kernel(StageParams p) {
  chain_enter();
  using R2 = R2_t<Real>;
  __shared__ R2 tile[32][33];  // [c][l], padded
  const int L = p.L, W = 2 * L - 1;
  const int c0 = blockIdx.x * 32, l0 = blockIdx.y * 32, b = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  // a thread keeps one l: all four cells' loads are issued before any is used, and the
  // degree's normalisation is computed once
  const int l = l0 + tx;
  EpiCell e[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c = c0 + ty + 8 * k;
    e[k].ok = false;
    e[k].mirror = false;
    if (c < W && l < L) e[k] = epi_fetch<Real>(p, b, l, c - (L - 1));
  }
  const double nl = epi_norm(p, l);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c = c0 + ty + 8 * k;
    tile[ty + 8 * k][tx] = epi_finish<Real>(p, b, l, c - (L - 1), e[k], nl);
  }
  __syncthreads();
  R2* out = reinterpret_cast<R2*>(p.flm_out) + (size_t)b * L * W;
  for (int ll = ty; ll < 32; ll += 8) {
    const int l = l0 + ll, c = c0 + tx;
    if (l < L && c < W) out[(size_t)l * W + c] = tile[tx][ll];
  }
}

// y += a * x over n complex elements (iterative refinement update)
template <typename Real>
__global__ void axpy_kernel(long n, Real a, const R2_t<Real>* x, R2_t<Real>* y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    R2_t<Real> v = y[i];
    v.x += a * x[i].x;
    v.y += a * x[i].y;
    y[i] = v;
  }
}

// z = x - y over n real elements
template <typename Real>
__global__ void sub_kernel(long n, const Real* x, const Real* y, Real* z) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    z[i] = x[i] - y[i];
}

static int grid_for(long n) {
  long b = (n + 255) / 256;
  if (b > 65535) b = 65535;
  if (b < 1) b = 1;
  return (int)b;
}

// A flat index fits 32 bits when the last grid-stride step (index + grid size, at most
// 65535 x 256 beyond the end) stays below 2^32.
static bool fits32(long n) { return n + 65535L * 256 < (1L << 32); }

static cudaError_t launch_poles(bool fp64, const StageParams& p, cudaStream_t s) {
  if (p.pole_south < 0 && p.pole_north < 0) return cudaSuccess;
  if (fp64)
    poles_kernel<double><<<dim3(2, p.batch), 256, 0, s>>>(p);
  else
    poles_kernel<float><<<dim3(2, p.batch), 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_prologue(bool fp64, const StageParams& p, cudaStream_t s) {
  if (p.Lp > 0 && p.Q == 32 && (long)p.batch * p.nhalf <= 65535 && p.nclass <= 65535) {
    StageParams q = p;
    const bool poles = p.pole_south >= 0 || p.pole_north >= 0;
    // the pole rows ride on one extra column of CTAs when there are two classes for them
    q.pole_blocks = poles && p.nclass >= 2 ? 1 : 0;
    // ftm is cleared by the same CTAs when it is exactly the [batch][nrows][ncol] table
    const long units = (long)p.batch * p.nrows * ((p.ncol + 255) / 256);
    q.zero_ftm = p.ftm_zero_bytes > 0 && units < (1L << 31) &&
                 p.ftm_zero_bytes == (size_t)p.batch * p.nrows * p.ncol * (fp64 ? 16 : 8);
    if (p.ftm_zero_bytes > 0 && !q.zero_ftm) {
      const cudaError_t e = cudaMemsetAsync(p.ftm, 0, p.ftm_zero_bytes, s);
      if (e != cudaSuccess) return e;
    }
    const dim3 grid((p.TR + 31) / 32 + q.pole_blocks, p.nclass, p.batch * p.nhalf);
    cudaError_t e = fp64 ? launch_chained(prologue_tiled_kernel<double>, grid, dim3(32, 8), 0, s, q)
                         : launch_chained(prologue_tiled_kernel<float>, grid, dim3(32, 8), 0, s, q);
    if (e == cudaSuccess && poles && !q.pole_blocks) e = launch_poles(fp64, p, s);
    return e;
  }
  if (p.ftm_zero_bytes > 0) {
    const cudaError_t e = cudaMemsetAsync(p.ftm, 0, p.ftm_zero_bytes, s);
    if (e != cudaSuccess) return e;
  }
  const long total = (long)p.batch * p.nhalf * p.nclass * p.TR * p.Q;
  const bool i32 = fits32(total);
  if (fp64 && i32)
    prologue_kernel<double, uint32_t><<<grid_for(total), 256, 0, s>>>(p);
  else if (fp64)
    prologue_kernel<double, uint64_t><<<grid_for(total), 256, 0, s>>>(p);
  else if (i32)
    prologue_kernel<float, uint32_t><<<grid_for(total), 256, 0, s>>>(p);
  else
    prologue_kernel<float, uint64_t><<<grid_for(total), 256, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_poles(fp64, p, s);
  return e;
}

cudaError_t launch_epilogue(bool fp64, const StageParams& p, cudaStream_t s) {
  if (p.Lp > 0 && p.batch <= 65535) {
    const dim3 grid((2 * p.L - 1 + 31) / 32, (p.L + 31) / 32, p.batch);
    return fp64 ? launch_chained(epilogue_tiled_kernel<double>, grid, dim3(32, 8), 0, s, p)
                : launch_chained(epilogue_tiled_kernel<float>, grid, dim3(32, 8), 0, s, p);
  }
  const long total = (long)p.batch * p.L * (2 * p.L - 1);
  const bool i32 = fits32(total);
  if (fp64 && i32)
    epilogue_kernel<double, uint32_t><<<grid_for(total), 256, 0, s>>>(p);
  else if (fp64)
    epilogue_kernel<double, uint64_t><<<grid_for(total), 256, 0, s>>>(p);
  else if (i32)
    epilogue_kernel<float, uint32_t><<<grid_for(total), 256, 0, s>>>(p);
  else
    epilogue_kernel<float, uint64_t><<<grid_for(total), 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_axpy(bool fp64, long n, double a, const void* x, void* y, cudaStream_t s) {
  if (fp64)
    axpy_kernel<double><<<grid_for(n), 256, 0, s>>>(n, a, (const double2*)x, (double2*)y);
  else
    axpy_kernel<float><<<grid_for(n), 256, 0, s>>>(n, (float)a, (const float2*)x, (float2*)y);
  return cudaGetLastError();
}

cudaError_t launch_sub(bool fp64, long n, const void* x, const void* y, void* z, cudaStream_t s) {
  if (fp64)
    sub_kernel<double><<<grid_for(n), 256, 0, s>>>(n, (const double*)x, (const double*)y,
                                                    (double*)z);
  else
    sub_kernel<float><<<grid_for(n), 256, 0, s>>>(n, (const float*)x, (const float*)y, (float*)z);
  return cudaGetLastError();
}

}  // namespace s2b
