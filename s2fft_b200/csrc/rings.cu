// Ring FFTs and the element-wise stages around the latitudinal kernel.
//
// Replaces the longitudinal steps of upstream s2fft:
//   equiangular rows: np.fft.fft / ifft / rfft / irfft in
//     s2fft/transforms/spherical.py:191-208 (inverse) and 527-541 (forward);
//   MW -> MWSS resampling and x2 upsampling (s2fft/utils/resampling.py:104-355),
//     folded into one per-column chain in the phi-Fourier domain;
//   HEALPix ring FFTs with spectral extension / folding and phi0 phase shifts
//     (s2fft/utils/healpix_ffts.py:19-117, 187-226, 335-371, 482-509) and the
//     native cuFFT path (lib/src/s2fft.cu:119-154, lib/src/s2fft_kernels.cu:46-235).
//
// One CTA per transform (ring, row or column). Lengths that are powers of two
// use a radix-2 decimation-in-frequency pass; other lengths use Bluestein's
// chirp-z algorithm with a power-of-two convolution (forward DIF, pointwise
// product with the pre-transformed chirp filter in bit-reversed order, inverse
// DIT), so no permutation pass is ever needed. Shifts, scalings, weights,
// phase factors, spectral extension and folding are fused into the load/store
// of each transform.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "s2b_fft.h"
#include "s2b_internal.h"
#include "s2b_fft_dev.h"
#include "s2b_fft_reg.h"
#include "s2b_dev.h"

namespace s2b {

// CTAs per SM the register-engine kernels are compiled for (launch bounds): 32 warps per SM
// in float (the points of a 2^LOGM transform take 2^(LOGM-4) threads; 64 registers, a few
// bytes of spills at most), 16 in double (twice the registers per point); one CTA of 512
// threads for 8192 points. The shared-memory passes (LOGM = 0): two in float, one in double.
template <typename Real>
__host__ __device__ constexpr int reg_min_blocks(int logm) {
  // (registers are allocated per warp: a CTA of fewer than 32 threads counts as one warp;
  // 256 points, whose 16 threads do the work of a warp, get half the warps per SM)
  return logm == 0    ? (sizeof(Real) == 4 ? 2 : 1)
         : logm >= 13 ? 1
                      : (((sizeof(Real) == 4 ? 1024 : 512) >> (logm <= 8 ? 1 : 0)) >>
                         (logm - 4 > 5 ? logm - 4 : 5));
}

// Any-length DFT of one CTA on the register engine (M = 2^LOGM, blockDim.x = M / 16; d.M
// must be M): inputs load(k), k < d.n; every output X_k (k < d.n, conjugated when inv,
// times the Bluestein output chirp unless chirp_out is false) goes to emit(k, X_k) once,
// from the thread that holds it (natural order k = j + T a for Bluestein lengths, the
// bit-reversed positions of a power-of-two length). buf: RegFFT<LOGM, NBUF>::SMEM_ELEMS
// elements. With sync_emit a barrier precedes the emits, so that emit may write buf.
template <typename Real, int LOGM, int NBUF, typename Load, typename Emit>
__device__ __forceinline__ void reg_dft(typename C2<Real>::t* buf, const FFTDesc& d,
                                        const FFTTables<Real>& tb, bool inv, bool chirp_out,
                                        bool sync_emit, Load load, Emit emit) {
  using R2 = typename C2<Real>::t;
  using RF = RegFFT<LOGM, NBUF>;
  const int j = threadIdx.x;
  const R2* tw = tb.rtw + d.rtw_off;
  int ping = 0;
  R2 x[16];
  if (d.bluestein) {
    const R2* __restrict__ ch = tb.chirp + d.chirp_off;
    const R2* __restrict__ bf = tb.rbf + d.rbf_off;  // position 16 j + a at [a T + j]
    // the filter is read after the forward passes: its lines into L1 now, so that those
    // reads do not wait on L2
#pragma unroll
    for (int a = 0; a < 16; ++a) prefetch_l1(bf + a * RF::T + j);
#pragma unroll
    for (int a = 0; a < 16; ++a) {
      const int k = j + RF::T * a;
      R2 v = czero<R2>();
      if (k < d.n) {
        v = load(k);
        if (inv) v = cconj(v);
        v = cmul(v, ch[k]);
      }
      x[a] = v;
    }
    RF::dif(x, buf, tw, false, ping);
#pragma unroll
    for (int a = 0; a < 16; ++a) x[a] = cmul(x[a], bf[a * RF::T + j]);
    RF::dit(x, buf, tw, true, ping);
    if (sync_emit) __syncthreads();
#pragma unroll
    for (int a = 0; a < 16; ++a) {
      const int k = j + RF::T * a;
      if (k < d.n) {
        R2 v = chirp_out ? cmul(x[a], ch[k]) : x[a];
        emit(k, inv ? cconj(v) : v);
      }
    }
  } else {
#pragma unroll
    for (int a = 0; a < 16; ++a) {
      R2 v = load(j + RF::T * a);
      x[a] = inv ? cconj(v) : v;
    }
    RF::dif(x, buf, tw, false, ping);
    if (sync_emit) __syncthreads();
#pragma unroll
    for (int a = 0; a < 16; ++a) emit(bitrev(RF::point(j, a, 0), LOGM), inv ? cconj(x[a]) : x[a]);
  }
}

// ---------------------------------------------------------------------------
// Inverse rows: ftm [B][nrows][ncol] -> f (equiangular rows or HEALPix rings).
// One CTA per (ring, map). Column c of ftm holds m = c - (L-1) - mo.
// ---------------------------------------------------------------------------
// LOGM > 0: the register engine for uniform rings of one power-of-two working length 2^LOGM
// (equiangular samplings; blockDim.x = 2^LOGM / 16); LOGM = 0: the shared-memory passes.
template <typename Real, int LOGM, int NBUF>
__global__ void __launch_bounds__(LOGM ? (1 << LOGM) / 16 : 512, reg_min_blocks<Real>(LOGM))
    inv_rows_kernel(RowsParams<Real> p) {
  chain_enter();
  using R2 = typename C2<Real>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R2* s = reinterpret_cast<R2*>(smem_raw);
  const int t = blockIdx.x;
  const int b = blockIdx.y;
  const FFTDesc d = p.desc[p.ring_desc ? p.ring_desc[t] : 0];
  const int n = d.n;
  const R2* row = reinterpret_cast<const R2*>(p.in) + ((size_t)b * p.nrows + t) * p.ncol;
  const int L = p.L;
  const double phi0 = p.phi0 ? p.phi0[t] : 0.0;
  // the Hermitian mirror applies on every ring, or (rings_real_2L) only on rings of 2L
  // pixels, where the rows hold the rfft half spectrum; other rings then use the full row
  const bool mirror = p.reality && (!p.rings_real_2L || n == 2 * p.L);
  // coefficient C_m with the HEALPix phase exp(+i m phi0) and reality mirror
  auto coef = [&](int m) -> R2 {
    R2 c;
    if (mirror && m < 0) {
      c = cconj(row[L - 1 - m + p.mo]);
      if (p.phi0) {
        double sn, cs;
        sincos((double)(-m) * phi0, &sn, &cs);
        R2 e;
        e.x = (Real)cs;
        e.y = (Real)sn;
        c = cconj(cmul(cconj(c), e));
      }
      return c;
    }
    c = row[L - 1 + m + p.mo];
    if (p.phi0) {
      double sn, cs;
      sincos((double)m * phi0, &sn, &cs);
      R2 e;
      e.x = (Real)cs;
      e.y = (Real)sn;
      c = cmul(c, e);
    }
    return c;
  };
  const int mlo = mirror ? -(L - 1) : -(L - 1) - p.mo;  // lowest m present
  const int mhi = L - 1;
  auto load = [&](int k) -> R2 {
    // X_k = sum of C_m over m == k (mod n), m in [mlo, mhi]
    R2 acc = czero<R2>();
    if (n >= p.ncol) {
      // no aliasing: unique m with m mod n == k, |m| small
      int m = k;
      if (m > mhi) m -= n;
      if (m >= mlo && m <= mhi) acc = coef(m);
      return acc;
    }
    int m = k;
    while (m - n >= mlo) m -= n;
    for (; m <= mhi; m += n) acc = cadd(acc, coef(m));
    return acc;
  };
  const Real scale = (Real)(p.scale * (p.weights ? p.weights[t] : 1.0));
  if constexpr (LOGM > 0) {
    // uniform rings without phases or aliasing (n >= ncol): X_k is the one C_m with
    // m = k or k - n
    auto load_eq = [&](int k) -> R2 {
      const int m = k > mhi ? k - n : k;
      if (m < mlo) return czero<R2>();
      return (mirror && m < 0) ? cconj(row[L - 1 - m + p.mo]) : row[L - 1 + m + p.mo];
    };
    R2* outc = reinterpret_cast<R2*>(p.out) + (size_t)b * p.out_batch_stride + p.ring_off[t];
    Real* outr = reinterpret_cast<Real*>(p.out) + (size_t)b * p.out_batch_stride + p.ring_off[t];
    if (d.bluestein) {  // outputs in natural order: coalesced stores from the registers
      reg_dft<Real, LOGM, NBUF>(s, d, p.tb, true, true, false, load_eq, [&](int k, R2 v) {
        if (p.real_out)
          outr[k] = v.x * scale;
        else
          outc[k] = cscale(v, scale);
      });
    } else {  // bit-reversed positions: through shared memory to natural order
      reg_dft<Real, LOGM, NBUF>(s, d, p.tb, true, true, true, load_eq,
                                [&](int k, R2 v) { s[ridx(k)] = v; });
      __syncthreads();
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        if (p.real_out)
          outr[k] = s[ridx(k)].x * scale;
        else
          outc[k] = cscale(s[ridx(k)], scale);
      }
    }
  } else {
    // rings with fewer pixels than columns (HEALPix polar rings): the aliased sums X_k are
    // spread over the CTA (thread = bin k and chunk c of its aliases) and combined in a
    // fixed order, instead of one thread per bin walking all ncol / n aliases
    R2* xs = p.alias_off ? s + p.alias_off : nullptr;
    const bool pre = xs != nullptr && n < p.ncol;
    if (pre) {
      const int nc = n < (int)blockDim.x ? (int)blockDim.x / n : 1;
      for (int u = threadIdx.x; u < n * nc; u += blockDim.x) {
        const int k = u % n, c = u / n;
        const int mk = mlo + pmod(k - mlo, n);  // lowest m == k (mod n) in range
        R2 acc = czero<R2>();
        for (int m = mk + c * n; m <= mhi; m += n * nc) acc = cadd(acc, coef(m));
        xs[u] = acc;
      }
      __syncthreads();
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        R2 acc = xs[k];
        for (int c = 1; c < nc; ++c) acc = cadd(acc, xs[c * n + k]);
        xs[k] = acc;  // the chunks c >= 1 of bin k lie above n: no other bin reads slot k
      }
      __syncthreads();
    }
    dft_run<Real>(s, d, p.tb, true, [&](int k) -> R2 { return pre ? xs[k] : load(k); });
    if (p.real_out) {
      Real* out = reinterpret_cast<Real*>(p.out) + (size_t)b * p.out_batch_stride + p.ring_off[t];
      for (int j = threadIdx.x; j < n; j += blockDim.x)
        out[j] = dft_get<Real>(s, d, p.tb, true, j).x * scale;
    } else {
      R2* out = reinterpret_cast<R2*>(p.out) + (size_t)b * p.out_batch_stride + p.ring_off[t];
      for (int j = threadIdx.x; j < n; j += blockDim.x)
        out[j] = cscale(dft_get<Real>(s, d, p.tb, true, j), scale);
    }
  }
}

template <typename Real, typename Val>
__device__ __forceinline__ void store_spectra(const RowsParams<Real>& p, int b, int t, Val val) {
  // G [b][half][m + kPadLo][Gs]: rows m outside [0, L) and columns >= nrows are zero
  using R2 = typename C2<Real>::t;
  const int L = p.L;
  const int col = p.col_of_ring ? p.col_of_ring[t] : t;
  if (t == p.nrows - 1 && p.Gs > p.nrows) {
    const int halves = p.dual ? 1 : p.nhalf, per = p.dual ? 2 : 1;
    R2* o2 = reinterpret_cast<R2*>(p.out);
    const int padc = p.Gs - p.nrows;
    for (int x = threadIdx.x; x < halves * p.TR * padc * per; x += blockDim.x) {
      const int c = x % (padc * per);
      const int rowi = x / (padc * per);
      o2[(((size_t)b * halves * p.TR + rowi) * p.Gs + p.nrows) * per + c] = czero<R2>();
    }
  }
  if (p.dual) {
    using R4 = std::conditional_t<sizeof(Real) == 4, float4, double4>;
    R4* out = reinterpret_cast<R4*>(p.out);
    for (int mr = threadIdx.x; mr < p.TR; mr += blockDim.x) {
      const int m = mr - kPadLo;
      R2 a = czero<R2>(), c = czero<R2>();
      if (m >= 0 && m < L) {
        a = val(m);
        if (m > 0) c = val(-m);
      }
      R4 o;
      o.x = a.x;
      o.y = a.y;
      o.z = c.x;
      o.w = c.y;
      out[((size_t)b * p.TR + mr) * p.Gs + col] = o;
    }
  } else {
    R2* out = reinterpret_cast<R2*>(p.out);
    for (int mr = threadIdx.x; mr < p.TR; mr += blockDim.x) {
      const int m = mr - kPadLo;
      const bool ok = m >= 0 && m < L;
      out[(((size_t)b * p.nhalf + 0) * p.TR + mr) * p.Gs + col] = ok ? val(m) : czero<R2>();
      if (p.nhalf > 1)
        out[(((size_t)b * p.nhalf + 1) * p.TR + mr) * p.Gs + col] =
            (ok && m > 0) ? val(-m) : czero<R2>();
    }
  }
}

// ---------------------------------------------------------------------------
// Forward rows: f rows/rings -> weighted spectra G [B][half][m][nrows]
// (dual: Real4 {+m, -m}; single: half 0 holds +m, half 1 holds -m), or, for
// the MW/MWSS resampling chain, the transposed raw spectra Fc [B][ncolm][nrows].
// ---------------------------------------------------------------------------
template <typename Real, int LOGM, int NBUF>
__global__ void __launch_bounds__(LOGM ? (1 << LOGM) / 16 : 512, reg_min_blocks<Real>(LOGM))
    fwd_rows_kernel(RowsParams<Real> p) {
  chain_enter();
  using R2 = typename C2<Real>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R2* s = reinterpret_cast<R2*>(smem_raw);
  const int t = blockIdx.x;
  const int b = blockIdx.y;
  if (p.zero) {
    // the latitudinal kernel's accumulators, cleared here instead of by a memset of their own
    const long nth = (long)gridDim.x * gridDim.y * blockDim.x;
    for (long i = ((long)b * gridDim.x + t) * blockDim.x + threadIdx.x; i < p.zero16; i += nth)
      reinterpret_cast<float4*>(p.zero)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  const FFTDesc d = p.desc[p.ring_desc ? p.ring_desc[t] : 0];
  const int n = d.n;
  const int L = p.L;
  const size_t off = (size_t)b * p.out_batch_stride + p.ring_off[t];
  auto load = [&](int k) -> R2 {
    R2 x;
    if (p.real_in) {
      x.x = reinterpret_cast<const Real*>(p.in)[off + k];
      x.y = 0;
    } else {
      x = reinterpret_cast<const R2*>(p.in)[off + k];
    }
    return x;
  };
  if constexpr (LOGM > 0) {
    if (p.mode == FWD_TO_COLS) {
      // Fc[b][m + mshift][t] = scale * X_m for m in [mlo, L-1], straight from the registers
      R2* out = reinterpret_cast<R2*>(p.out);
      const int mlo = -(L - 1) - p.mo;
      const int ncm = L - mlo;
      reg_dft<Real, LOGM, NBUF>(s, d, p.tb, false, true, false, load, [&](int k, R2 v) {
        const int m = k <= L - 1 ? k : k - n;
        if (m >= mlo && m <= L - 1)
          out[((size_t)b * ncm + (m - mlo)) * p.nrows + t] = cscale(v, (Real)p.scale);
      });
      return;
    }
    reg_dft<Real, LOGM, NBUF>(s, d, p.tb, false, true, true, load,
                              [&](int k, R2 v) { s[ridx(k)] = v; });
    __syncthreads();
  } else {
    dft_run<Real>(s, d, p.tb, false, load);
  }
  // X_k of this ring, k < n
  auto get = [&](int k) -> R2 {
    if constexpr (LOGM > 0)
      return s[ridx(k)];
    else
      return dft_get<Real>(s, d, p.tb, false, k);
  };
  const double w = p.weights ? p.weights[t] : 1.0;
  const double phi0 = p.phi0 ? p.phi0[t] : 0.0;
  if (p.mode == FWD_TO_RAW) {
    R2* out = reinterpret_cast<R2*>(p.out);
    for (int mi = threadIdx.x; mi < p.M; mi += blockDim.x) {
      const int m = p.m0 + mi;
      R2 x = get(pmod(m, n));
      // real input on a ring of 2L pixels keeps m >= 0 only (the rfft half spectrum,
      // s2fft/utils/healpix_ffts.py:212-216)
      if (p.real_in && p.reality && n == 2 * L && m < 0) x = czero<R2>();
      out[((size_t)b * p.nrows + t) * p.M + mi] = cscale(x, (Real)p.scale);
    }
    return;
  }
  if (p.mode == FWD_TO_COLS) {
    // Fc[b][m + mshift][t] = scale * X_m for m in [mlo, L-1]
    R2* out = reinterpret_cast<R2*>(p.out);
    const int mlo = -(L - 1) - p.mo;
    const int ncm = L - mlo;
    for (int mi = threadIdx.x; mi < ncm; mi += blockDim.x) {
      const int m = mlo + mi;
      R2 x = get(pmod(m, n));
      out[((size_t)b * ncm + mi) * p.nrows + t] = cscale(x, (Real)p.scale);
    }
    return;
  }
  // weighted, phase-shifted spectrum for m in [-(L-1), L-1] (periodic in n)
  auto val = [&](int m) -> R2 {
    R2 x = get(pmod(m, n));
    double re = (double)x.x * w, im = (double)x.y * w;
    if (p.phi0) {
      double sn, cs;
      sincos(-(double)m * phi0, &sn, &cs);
      const double r2 = re * cs - im * sn;
      im = re * sn + im * cs;
      re = r2;
    }
    R2 o;
    o.x = (Real)re;
    o.y = (Real)im;
    return o;
  };
  store_spectra<Real>(p, b, t, val);
}


// ---------------------------------------------------------------------------
// MW / MWSS forward resampling, per phi-frequency column m (one CTA per column):
//   theta periodic extension with parity (-1)^(m+s) (resampling.py:6-61, 64-101),
//   DFT over the extended circle, MW half-sample shift exp(-i p pi/(2L-1))
//   (resampling.py:284-326), zero-padding to 4L and inverse DFT
//   (resampling.py:104-160), evaluation on the 2L+1 MWSS(2L) rings, times the
//   quadrature weights. The phi resampling 2L-1 -> 2L (resampling.py:248-281)
//   reduces to the overall factor 2L/(2L-1) in the phi-Fourier domain.
// ---------------------------------------------------------------------------
// The column chain's output for column m of map b: chain(t) = the inverse-DFT value on
// MWSS(2L) ring t (t = 0..2L) with the pole and Nyquist corrections, before the overall
// factor and the weights; writes it in the layout ColsParams describes (raw, ring pairs,
// or rows), and the zero padding once per map (column m = 0).
template <typename Real, typename Chain>
__device__ __forceinline__ void cols_emit(const ColsParams<Real>& p, int b, int m, Chain chain) {
  using R2 = typename C2<Real>::t;
  const int L = p.L;
  const int nout = 2 * L + 1;
  const int am = m < 0 ? -m : m;
  R2* out = reinterpret_cast<R2*>(p.out);
  if (p.raw) {
    if (m < p.m0) return;
    for (int t = threadIdx.x; t < nout; t += blockDim.x) {
      R2 u = chain(t);
      u.x = (Real)((double)u.x * p.scale);
      u.y = (Real)((double)u.y * p.scale);
      out[((size_t)b * nout + t) * p.M + (m - p.m0)] = u;
    }
    return;
  }
  auto weighted = [&](int t) -> R2 {
    R2 u = chain(t);
    const double f = p.scale * p.weights[t];
    u.x = (Real)((double)u.x * f);
    u.y = (Real)((double)u.y * f);
    return u;
  };
  if (p.out2) {
    // ring pairs (t, 2L - t) as (E, O), in the layout of out with a trailing pair axis
    R2* o2 = reinterpret_cast<R2*>(p.out2);
    const size_t mr = (size_t)(am + kPadLo);
    const int per = p.dual ? 2 : 1;
    const size_t rowbase =
        p.dual ? ((size_t)b * p.TR + mr) * p.Gs2 : ((size_t)b * p.nhalf * p.TR + mr) * p.Gs2;
    if (p.dual || m >= 0) {
      for (int q = threadIdx.x; q < L; q += blockDim.x) {
        const R2 un = weighted(q + 1);
        R2 e = un, o = czero<R2>();
        if (q < L - 1) {
          const R2 us = weighted(2 * L - 1 - q);
          e.x = un.x + us.x;
          e.y = un.y + us.y;
          o.x = un.x - us.x;
          o.y = un.y - us.y;
        }
        o2[((rowbase + q) * 2 + 0) * per + (m < 0 ? 1 : 0)] = e;
        o2[((rowbase + q) * 2 + 1) * per + (m < 0 ? 1 : 0)] = o;
      }
    }
    // the pole rows stay in out (read by the epilogue)
    if (threadIdx.x < 2) {
      const int t = threadIdx.x == 0 ? 0 : 2 * L;
      const int row = t == 0 ? 2 * L - 1 : 2 * L;
      const R2 u = weighted(t);
      if (p.dual)
        out[(((size_t)b * p.TR + mr) * p.Gs + row) * 2 + (m < 0 ? 1 : 0)] = u;
      else if (m >= 0)
        out[(((size_t)b * p.nhalf + 0) * p.TR + mr) * p.Gs + row] = u;
    }
    if (m == 0) {
      // zero pad rows (m outside [0, L)), pad pair columns (>= L) and, in the dual layout,
      // the unused -m half of m = 0 (spin 0: one half)
      const int rowlen = p.Gs2 * 2 * per;  // R2 entries per m row
      R2* ob = o2 + (size_t)b * p.TR * rowlen;
      for (int x = threadIdx.x; x < 2 * kPadLo * rowlen; x += blockDim.x) {
        const int pr = x / rowlen;
        const int mrow = pr < kPadLo ? pr : L + pr;
        ob[(size_t)mrow * rowlen + x % rowlen] = czero<R2>();
      }
      const int padq = p.Gs2 - L;
      for (int x = threadIdx.x; x < L * padq * 2 * per; x += blockDim.x) {
        const int mrow = kPadLo + x / (padq * 2 * per);
        ob[(size_t)mrow * rowlen + L * 2 * per + x % (padq * 2 * per)] = czero<R2>();
      }
      if (p.dual)
        for (int x = threadIdx.x; x < L * 2; x += blockDim.x)
          ob[(size_t)kPadLo * rowlen + x * 2 + 1] = czero<R2>();
    }
    return;
  }
  for (int t = threadIdx.x; t < nout; t += blockDim.x) {
    const R2 u = weighted(t);
    const int row = t == 0 ? 2 * L - 1 : (t == 2 * L ? 2 * L : t - 1);  // poles after the recursed rings
    const size_t mr = (size_t)(am + kPadLo);
    if (p.dual) {
      // Real4 {+m, -m} viewed as pairs of Real2
      out[(((size_t)b * p.TR + mr) * p.Gs + row) * 2 + (m < 0 ? 1 : 0)] = u;
    } else if (m >= 0) {
      out[(((size_t)b * p.nhalf + 0) * p.TR + mr) * p.Gs + row] = u;
    } else if (p.nhalf > 1) {
      out[(((size_t)b * p.nhalf + 1) * p.TR + mr) * p.Gs + row] = u;
    }
  }
  // zero pad rows (m outside [0, L)) and pad columns (>= 2L+1), once per map (m = 0 CTA)
  if (m == 0) {
    const int per = p.dual ? 2 : 1;
    const int halves = p.dual ? 1 : p.nhalf;
    const int padc = p.Gs - nout;
    for (int x = threadIdx.x; x < halves * p.TR * padc * per; x += blockDim.x) {
      const int c = x % (padc * per);
      const int rowi = x / (padc * per);
      out[(((size_t)b * halves * p.TR + rowi) * p.Gs + nout) * per + c] = czero<R2>();
    }
    for (int h = 0; h < halves; ++h)
      for (int pr = 0; pr < 2 * kPadLo; ++pr) {
        const int mr = pr < kPadLo ? pr : L + pr;  // rows m < 0 and m >= L
        R2* base = out + (((size_t)b * halves + h) * p.TR + mr) * p.Gs * per;
        for (int x = threadIdx.x; x < p.Gs * per; x += blockDim.x) base[x] = czero<R2>();
      }
    if (p.dual || p.nhalf > 1) {
      // the unused half of m = 0 in the dual layout is zero as well
      if (p.dual)
        for (int t = threadIdx.x; t < nout; t += blockDim.x) {
          const int row = t == 0 ? 2 * L - 1 : (t == 2 * L ? 2 * L : t - 1);
          out[(((size_t)b * p.TR + kPadLo) * p.Gs + row) * 2 + 1] = czero<R2>();
        }
      else
        for (int t = threadIdx.x; t < nout; t += blockDim.x) {
          const int row = t == 0 ? 2 * L - 1 : (t == 2 * L ? 2 * L : t - 1);
          out[(((size_t)b * p.nhalf + 1) * p.TR + kPadLo) * p.Gs + row] = czero<R2>();
        }
    }
  }
}

// LOGM > 0: both transforms on the register engine (d1.M = d2.M = 2^LOGM, the inverse DFT
// of power-of-two length 4L; blockDim.x = 2^LOGM / 16); LOGM = 0: the shared-memory passes.
template <typename Real, int LOGM, int NBUF>
__global__ void __launch_bounds__(LOGM ? (1 << LOGM) / 16 : 512, reg_min_blocks<Real>(LOGM))
    mw_cols_kernel(ColsParams<Real> p) {
  chain_enter();
  using R2 = typename C2<Real>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const FFTDesc d1 = *p.d1;
  const FFTDesc d2 = *p.d2;
  // one DFT buffer for both transforms; the 2L-1 (2L) bins of the first that feed the
  // second are kept, phase-multiplied, in tmp in between
  R2* s1 = reinterpret_cast<R2*>(smem_raw);
  R2* s2 = s1;
  R2* tmp = s1 + (LOGM > 0 ? RegFFT<(LOGM > 0 ? LOGM : 8), NBUF>::SMEM_ELEMS
                           : padded_len(d1.M > d2.M ? d1.M : d2.M));
  const int L = p.L;
  const int mlo = p.mw ? -(L - 1) : -L;
  const int ncm = L - mlo;
  const int mi = blockIdx.x;
  const int b = blockIdx.y;
  const int m = mlo + mi;
  if (m < -(L - 1)) return;  // MWSS m = -L never reaches the recursion
  const R2* c = reinterpret_cast<const R2*>(p.in) + ((size_t)b * ncm + mi) * p.nin;
  const int par = ((m + p.spin) % 2 + 2) % 2;
  const Real sgn = par ? Real(-1) : Real(1);
  const int n1 = d1.n;
  auto load1 = [&](int t) -> R2 {
    if (p.mw) {
      if (t < L) return c[t];
      return cscale(c[2 * L - 2 - t], sgn);  // t = L + jj -> c[L-2-jj]
    }
    if (t <= L) return c[t];
    return cscale(c[2 * L - t], sgn);  // t = L+1+jj -> c[L-1-jj]
  };
  const int plo = p.mw ? -(L - 1) : -L;
  const int phi = L - 1;
  const int n2 = d2.n;  // 4L
  const R2* __restrict__ ph = reinterpret_cast<const R2*>(p.ph);
  if constexpr (LOGM > 0) {
    // bin k of the theta DFT is p = k (k <= L-1) or k - n1; ph carries the Bluestein chirp
    reg_dft<Real, LOGM, NBUF>(s1, d1, p.tb, false, false, false, load1, [&](int k, R2 v) {
      const int pp = k <= phi ? k : k - n1;
      if (pp >= plo) tmp[pp - plo] = cmul(v, ph[(pp + n2) % n2]);
    });
  } else {
    dft_run<Real>(s1, d1, p.tb, false, load1);
    for (int pp = plo + (int)threadIdx.x; pp <= phi; pp += blockDim.x) {
      const int j = pmod(pp, n1);
      const R2 g = d1.bluestein ? s1[pidx(j)] : s1[pidx(bitrev(j, d1.logM))];
      tmp[pp - plo] = cmul(g, ph[(pp + n2) % n2]);
    }
  }
  __syncthreads();
  auto load2 = [&](int k) -> R2 {
    // k = pp mod 4L for pp in [plo, phi]; zero outside
    const int pp = k <= phi ? k : k - n2;
    return (pp < plo || pp > phi) ? czero<R2>() : tmp[pp - plo];
  };
  // upstream's MWSS(L) detour (corrections described in ColsParams): the MW pole ring's odd
  // (m + s) part, and for real MWSS maps the split theta-Nyquist bin (p = -L, tmp[0])
  const R2* __restrict__ pole = (p.mw && par) ? reinterpret_cast<const R2*>(p.pole) : nullptr;
  const R2 xpole = pole ? c[L - 1] : czero<R2>();
  const R2 nyq = (!p.mw && p.nyq_split) ? tmp[0] : czero<R2>();
  if constexpr (LOGM > 0) {
    // the 4L outputs in natural order in shared memory (after a barrier: the transform's
    // last exchange may still be read)
    reg_dft<Real, LOGM, NBUF>(s2, d2, p.tb, true, true, true, load2,
                              [&](int k, R2 v) { s2[ridx(k)] = v; });
    __syncthreads();
  } else {
    dft_run<Real>(s2, d2, p.tb, true, load2);
  }
  auto chain = [&](int t) -> R2 {
    R2 u;
    if constexpr (LOGM > 0)
      u = s2[ridx(t)];
    else
      u = dft_get<Real>(s2, d2, p.tb, true, t);
    if (pole) u = cadd(u, cmul(xpole, pole[t]));
    if (t & 1) {  // i N sin(pi t / 2)
      const Real sg = (t & 2) ? Real(-1) : Real(1);
      u.x -= sg * nyq.y;
      u.y += sg * nyq.x;
    }
    return u;
  };
  cols_emit(p, b, m, chain);
}

// Two columns per CTA on the register engine: m and m + 1 have opposite parities
// (-1)^(m+s), so their theta extensions x_A, x_B are mirror-symmetric with opposite signs
// (MW: x[n1-1-t] = s x[t]; MWSS: x[n1-t] = s x[t]), and so are the inverse-DFT outputs
// u_A, u_B on the 4L circle (u[-t] = s u[t]: the half-sample phase keeps the symmetry). The
// chain is linear and the same for both columns, so it runs once on z = x_A + i x_B and
// u_A = (z'_t + s_A z'_-t) / 2, u_B = (z'_t - s_A z'_-t) / 2i separate the outputs. Parts
// that break the symmetry stay out of z and are added per column:
//   * the samples that are their own mirror (MW: the pole t = L-1; MWSS: t = 0 and L) of
//     the odd column, through the chain's response to a unit impulse there
//     (ColsParams::imp, which includes the pole and Nyquist corrections);
//   * MWSS: the theta-Nyquist bin p = -L, which only the even column has (u gets
//     N (-i)^t, and the split correction for real maps).
// The last column of the odd count 2L-1 runs alone (x_B = 0).
template <typename Real, int LOGM, int NBUF>
__global__ void __launch_bounds__((1 << LOGM) / 16, reg_min_blocks<Real>(LOGM))
    mw_cols_pair_kernel(ColsParams<Real> p) {
  chain_enter();
  using R2 = typename C2<Real>::t;
  using RF = RegFFT<LOGM, NBUF>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const FFTDesc d1 = *p.d1;
  const FFTDesc d2 = *p.d2;
  R2* s = reinterpret_cast<R2*>(smem_raw);
  R2* tmp = s + RF::SMEM_ELEMS;
  const int L = p.L;
  const int mlo = p.mw ? -(L - 1) : -L;
  const int ncm = L - mlo;
  const int b = blockIdx.y;
  const int mA = -(L - 1) + 2 * (int)blockIdx.x;
  const bool hasB = mA + 1 <= L - 1;
  const R2* cA = reinterpret_cast<const R2*>(p.in) + ((size_t)b * ncm + (mA - mlo)) * p.nin;
  const R2* cB = cA + p.nin;
  const bool oddA = (((mA + p.spin) % 2) + 2) % 2 == 1;
  const Real sA = oddA ? Real(-1) : Real(1);
  // extended sequence of a column, its self-mirrored samples left out when it is odd
  auto xcol = [&](const R2* c, bool odd, int t) -> R2 {
    const Real sg = odd ? Real(-1) : Real(1);
    if (p.mw) {
      if (t < L) return (odd && t == L - 1) ? czero<R2>() : c[t];
      return cscale(c[2 * L - 2 - t], sg);
    }
    if (t <= L) return (odd && (t == 0 || t == L)) ? czero<R2>() : c[t];
    return cscale(c[2 * L - t], sg);
  };
  auto load1 = [&](int t) -> R2 {
    R2 v = xcol(cA, oddA, t);
    if (hasB) {
      const R2 w = xcol(cB, !oddA, t);
      v.x -= w.y;
      v.y += w.x;
    }
    return v;
  };
  const int plo = p.mw ? -(L - 1) : -L;
  const int phi = L - 1;
  const int n1 = d1.n;
  const int n2 = d2.n;  // 4L
  const R2* __restrict__ ph = reinterpret_cast<const R2*>(p.ph);
  reg_dft<Real, LOGM, NBUF>(s, d1, p.tb, false, false, false, load1, [&](int k, R2 v) {
    const int pp = k <= phi ? k : k - n1;
    if (pp >= plo) tmp[pp - plo] = cmul(v, ph[(pp + n2) % n2]);
  });
  __syncthreads();
  // MWSS: the Nyquist bin (tmp[0]) belongs to the even column alone
  const R2 nyqZ = p.mw ? czero<R2>() : tmp[0];
  auto load2 = [&](int k) -> R2 {
    const int pp = k <= phi ? k : k - n2;
    return (pp < plo || pp > phi || (!p.mw && pp == -L)) ? czero<R2>() : tmp[pp - plo];
  };
  reg_dft<Real, LOGM, NBUF>(s, d2, p.tb, true, true, true, load2,
                            [&](int k, R2 v) { s[ridx(k)] = v; });
  __syncthreads();
  const R2* __restrict__ imp = reinterpret_cast<const R2*>(p.imp);
  const int nout = 2 * L + 1;
  // column A (B): sym = +1 (-1) picks u_A (u_B) out of z'
  auto chain = [&](bool colA, int t) -> R2 {
    const R2 zp = s[ridx(t)], zm = s[ridx(t == 0 ? 0 : n2 - t)];
    R2 d;
    d.x = (Real)0.5 * (colA ? zp.x + sA * zm.x : zp.x - sA * zm.x);
    d.y = (Real)0.5 * (colA ? zp.y + sA * zm.y : zp.y - sA * zm.y);
    R2 u = d;
    if (!colA) {  // divide by i
      u.x = d.y;
      u.y = -d.x;
    }
    const bool odd = colA == oddA;
    const R2* c = colA ? cA : cB;
    if (odd) {
      if (p.mw) {
        u = cadd(u, cmul(c[L - 1], imp[t]));
      } else {
        u = cadd(u, cmul(c[0], imp[t]));
        u = cadd(u, cmul(c[L], imp[nout + t]));
      }
    } else if (!p.mw) {
      // N (-i)^t from the Nyquist bin, N = the even column's bin -L
      R2 N = nyqZ;
      if (!colA) {  // nyqZ = i N_B
        N.x = nyqZ.y;
        N.y = -nyqZ.x;
      }
      R2 e = N;
      switch (t & 3) {
        case 1: e.x = N.y; e.y = -N.x; break;    // -i N
        case 2: e.x = -N.x; e.y = -N.y; break;   // -N
        case 3: e.x = -N.y; e.y = N.x; break;    // i N
        default: break;
      }
      u = cadd(u, e);
      if (p.nyq_split && (t & 1)) {  // i N sin(pi t / 2)
        const Real sg = (t & 2) ? Real(-1) : Real(1);
        u.x -= sg * N.y;
        u.y += sg * N.x;
      }
    }
    return u;
  };
  cols_emit(p, b, mA, [&](int t) { return chain(true, t); });
  if (hasB) cols_emit(p, b, mA + 1, [&](int t) { return chain(false, t); });
}

// ---------------------------------------------------------------------------
// Adjoint of the MW / MWSS column chain (one CTA per (m column, map)): the
// conjugate transpose of mw_cols_kernel, step by step in reverse order:
//   y (2L+1 MWSS(2L) ring values) * scale * weights -> zero-padded DFT over 4L
//   -> bins p in [plo, phi] times conj(half-sample phase) / n1 -> unnormalised
//   inverse DFT over the n1-point extended circle -> fold the extension back
//   onto the input rings with the parity (-1)^(m+s).
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(512, sizeof(Real) == 4 ? 2 : 1) mw_cols_adj_kernel(ColsParams<Real> p, int ncol_out, int mo_out) {
  using R2 = typename C2<Real>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const FFTDesc d1 = *p.d1;
  const FFTDesc d2 = *p.d2;
  // one DFT buffer for both transforms; the n1 inputs of the second, phase-multiplied,
  // are kept in tmp in between
  R2* s1 = reinterpret_cast<R2*>(smem_raw);
  R2* s2 = s1;
  R2* tmp = s1 + padded_len(d1.M > d2.M ? d1.M : d2.M);
  const int L = p.L;
  const int mlo = p.mw ? -(L - 1) : -L;
  const int mi = blockIdx.x;
  const int b = blockIdx.y;
  const int m = mlo + mi;
  R2* out = reinterpret_cast<R2*>(p.out) + (size_t)b * p.nin * ncol_out + (L - 1 + m + mo_out);
  if (m < -(L - 1)) {  // MWSS m = -L: the forward chain output of this column is never used
    for (int t = threadIdx.x; t < p.nin; t += blockDim.x) out[(size_t)t * ncol_out] = czero<R2>();
    return;
  }
  const int nout = 2 * L + 1;
  const R2* y = reinterpret_cast<const R2*>(p.in) + (size_t)b * nout * (2 * L - 1) + (L - 1 + m);
  auto load2 = [&](int t) -> R2 {
    if (t >= nout) return czero<R2>();
    // raw: rings in natural order and no weights (adjoint of the raw chain of the precompute
    // path, whose kernel tables carry the weights)
    const int row = p.raw ? t : (t == 0 ? 2 * L - 1 : (t == 2 * L ? 2 * L : t - 1));
    const R2 v = y[(size_t)row * (2 * L - 1)];
    const double f = p.raw ? p.scale : p.scale * p.weights[t];
    R2 o;
    o.x = (Real)((double)v.x * f);
    o.y = (Real)((double)v.y * f);
    return o;
  };
  dft_run<Real>(s2, d2, p.tb, false, load2);  // DFT over 4L
  const int plo = p.mw ? -(L - 1) : -L;
  const int phi = L - 1;
  const int n1 = d1.n;
  const int n2 = d2.n;
  const R2* __restrict__ pha = reinterpret_cast<const R2*>(p.ph_adj);
  for (int j = threadIdx.x; j < n1; j += blockDim.x) {
    const int pp = j <= phi ? j : j - n1;  // the bin p in [plo, phi] with p = j (mod n1)
    const int k = (pp + n2) % n2;
    tmp[j] = pp < plo ? czero<R2>() : cmul(dft_get<Real>(s2, d2, p.tb, false, k), pha[k]);
  }
  __syncthreads();
  dft_run<Real>(s1, d1, p.tb, true, [&](int j) { return tmp[j]; });  // unnormalised inverse DFT over n1
  const int par = ((m + p.spin) % 2 + 2) % 2;
  const Real sgn = par ? Real(-1) : Real(1);
  // transpose of the forward's pole correction: the pole ring gains sum_k conj(c_k) y_k
  R2 gpole = czero<R2>();
  if (p.mw && par && p.pole) {
    const R2* __restrict__ pole = reinterpret_cast<const R2*>(p.pole);
    R2 acc = czero<R2>();
    for (int t = threadIdx.x; t < nout; t += blockDim.x) acc = cadd(acc, cmul(cconj(pole[t]), load2(t)));
    for (int sh = 16; sh > 0; sh >>= 1) {
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, sh);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, sh);
    }
    __shared__ R2 wsum[32];  // one partial sum per warp (blockDim.x <= 1024, a multiple of 32)
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
    __syncthreads();
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) gpole = cadd(gpole, wsum[w]);
  }
  for (int t = threadIdx.x; t < p.nin; t += blockDim.x) {
    R2 x = dft_get<Real>(s1, d1, p.tb, true, t);
    if (t == L - 1) x = cadd(x, gpole);
    if (p.mw) {
      if (t <= L - 2) x = cadd(x, cscale(dft_get<Real>(s1, d1, p.tb, true, 2 * L - 2 - t), sgn));
    } else {
      if (t >= 1 && t <= L - 1)
        x = cadd(x, cscale(dft_get<Real>(s1, d1, p.tb, true, 2 * L - t), sgn));
    }
    out[(size_t)t * ncol_out] = x;
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// Threads of a transform CTA: two 8-element groups per thread in every fused pass (M / 16
// threads) measured 3.7 % faster on the L=1024 step than one group per thread (M / 8)
// and 7 % faster than four (M / 32): the second independent group hides shared-memory
// latency and halves the warps that meet at each barrier.
static int fft_threads(int M) {
  int t = M / 16;
  if (t > 512) t = 512;
  if (t < 32) t = 32;
  return t;
}

// Register engine for one working length 2^LOGM: 10 <= LOGM <= 13 (1024 .. 8192 points; in
// double up to 4096, where 16 points of a thread still fit the register file).
template <typename Real>
static int reg_logm(int M) {
  const int top = sizeof(Real) == 4 ? 13 : 12;
  for (int lg = 8; lg <= top; ++lg)
    if (M == (1 << lg)) return lg;
  return 0;
}
static constexpr int kRegBufs = 1;  // exchange buffers of the register engine

// carveout: the percentage of the unified L1 / shared memory given to shared memory. The
// shared-memory passes want all of it (occupancy); the register engine takes what its
// CTAs per SM need (reg_carveout) and leaves the rest to L1.
template <typename Real, typename Kernel, typename Params>
static cudaError_t launch_fft_kernel(Kernel k, dim3 grid, int threads, size_t smem,
                                     const Params& p, cudaStream_t s, int carveout = 100) {
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
  if (e != cudaSuccess) return e;
  return launch_chained(k, grid, dim3(threads), smem, s, p);
}

template <typename Real, int LOGM>
static size_t reg_smem(int extra) {
  return ((size_t)RegFFT<LOGM, kRegBufs>::SMEM_ELEMS + extra) * sizeof(typename C2<Real>::t);
}

// shared-memory share of the unified L1 (percent) for the register engine: room for the
// CTAs per SM of its launch bounds, the rest stays L1 for its twiddle, chirp and filter
// tables
template <typename Real, int LOGM>
static int reg_carveout(int extra) {
  const size_t need = (size_t)reg_min_blocks<Real>(LOGM) * (reg_smem<Real, LOGM>(extra) + 1024);
  const int pct = (int)((100 * need + 228 * 1024 - 1) / (228 * 1024)) + 1;
  return pct < 100 ? pct : 100;
}

// the rows use the register engine when every ring has the same working length (no per-ring
// descriptors: equiangular samplings) and no ring phase
template <typename Real>
static int rows_reg_logm(const RowsParams<Real>& p, int maxM) {
  return (p.ring_desc == nullptr && p.phi0 == nullptr) ? reg_logm<Real>(maxM) : 0;
}

template <typename Real>
cudaError_t launch_inv_rows(const RowsParams<Real>& p, int nrings, int batch, int maxM,
                            cudaStream_t s) {
  using R2 = typename C2<Real>::t;
  const dim3 grid(nrings, batch);
  switch (rows_reg_logm(p, maxM)) {
    case 8: return launch_fft_kernel<Real>(inv_rows_kernel<Real, 8, kRegBufs>, grid, 16, reg_smem<Real, 8>(0), p, s, reg_carveout<Real, 8>(0));
    case 9: return launch_fft_kernel<Real>(inv_rows_kernel<Real, 9, kRegBufs>, grid, 32, reg_smem<Real, 9>(0), p, s, reg_carveout<Real, 9>(0));
    case 10: return launch_fft_kernel<Real>(inv_rows_kernel<Real, 10, kRegBufs>, grid, 64, reg_smem<Real, 10>(0), p, s, reg_carveout<Real, 10>(0));
    case 11: return launch_fft_kernel<Real>(inv_rows_kernel<Real, 11, kRegBufs>, grid, 128, reg_smem<Real, 11>(0), p, s, reg_carveout<Real, 11>(0));
    case 12: return launch_fft_kernel<Real>(inv_rows_kernel<Real, 12, kRegBufs>, grid, 256, reg_smem<Real, 12>(0), p, s, reg_carveout<Real, 12>(0));
    case 13: return launch_fft_kernel<Real>(inv_rows_kernel<Real, 13, kRegBufs>, grid, 512, reg_smem<Real, 13>(0), p, s, reg_carveout<Real, 13>(0));
    default: break;
  }
  // shared-memory passes, plus (when it fits) the buffer of the aliased sums
  RowsParams<Real> q = p;
  const int nt = fft_threads(maxM);
  size_t smem = (size_t)padded_len(maxM) * sizeof(R2);
  const size_t extra = (size_t)(nt > maxM ? nt : maxM) * sizeof(R2);
  q.alias_off = 0;
  if (smem + extra <= (size_t)227 * 1024) {
    q.alias_off = padded_len(maxM);
    smem += extra;
  }
  return launch_fft_kernel<Real>(inv_rows_kernel<Real, 0, 1>, grid, nt, smem, q, s);
}

template <typename Real>
cudaError_t launch_fwd_rows(const RowsParams<Real>& p, int nrings, int batch, int maxM,
                            cudaStream_t s) {
  using R2 = typename C2<Real>::t;
  const dim3 grid(nrings, batch);
  switch (rows_reg_logm(p, maxM)) {
    case 8: return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 8, kRegBufs>, grid, 16, reg_smem<Real, 8>(0), p, s, reg_carveout<Real, 8>(0));
    case 9: return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 9, kRegBufs>, grid, 32, reg_smem<Real, 9>(0), p, s, reg_carveout<Real, 9>(0));
    case 10: return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 10, kRegBufs>, grid, 64, reg_smem<Real, 10>(0), p, s, reg_carveout<Real, 10>(0));
    case 11: return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 11, kRegBufs>, grid, 128, reg_smem<Real, 11>(0), p, s, reg_carveout<Real, 11>(0));
    case 12: return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 12, kRegBufs>, grid, 256, reg_smem<Real, 12>(0), p, s, reg_carveout<Real, 12>(0));
    case 13: return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 13, kRegBufs>, grid, 512, reg_smem<Real, 13>(0), p, s, reg_carveout<Real, 13>(0));
    default: break;
  }
  const size_t smem = (size_t)padded_len(maxM) * sizeof(R2);
  return launch_fft_kernel<Real>(fwd_rows_kernel<Real, 0, 1>, grid, fft_threads(maxM), smem, p, s);
}

template <typename Real>
cudaError_t launch_mw_cols(const ColsParams<Real>& p, int ncm, int batch, int M1, int M2,
                           cudaStream_t s) {
  using R2 = typename C2<Real>::t;
  const dim3 grid(ncm, batch);
  // register engine: one working length for both transforms, the second a plain power of two
  const int lg = (M1 == M2 && p.d2_pow2) ? reg_logm<Real>(M1) : 0;
  const int extra = 2 * p.L;
  if (p.imp) {
    // columns m, m+1 per CTA: L CTAs per map cover m = -(L-1) .. L-1
    const dim3 gp(p.L, batch);
    switch (lg) {
      case 8: return launch_fft_kernel<Real>(mw_cols_pair_kernel<Real, 8, kRegBufs>, gp, 16, reg_smem<Real, 8>(extra), p, s, reg_carveout<Real, 8>(extra));
      case 9: return launch_fft_kernel<Real>(mw_cols_pair_kernel<Real, 9, kRegBufs>, gp, 32, reg_smem<Real, 9>(extra), p, s, reg_carveout<Real, 9>(extra));
      case 10: return launch_fft_kernel<Real>(mw_cols_pair_kernel<Real, 10, kRegBufs>, gp, 64, reg_smem<Real, 10>(extra), p, s, reg_carveout<Real, 10>(extra));
      case 11: return launch_fft_kernel<Real>(mw_cols_pair_kernel<Real, 11, kRegBufs>, gp, 128, reg_smem<Real, 11>(extra), p, s, reg_carveout<Real, 11>(extra));
      case 12: return launch_fft_kernel<Real>(mw_cols_pair_kernel<Real, 12, kRegBufs>, gp, 256, reg_smem<Real, 12>(extra), p, s, reg_carveout<Real, 12>(extra));
      case 13: return launch_fft_kernel<Real>(mw_cols_pair_kernel<Real, 13, kRegBufs>, gp, 512, reg_smem<Real, 13>(extra), p, s, reg_carveout<Real, 13>(extra));
      default: break;
    }
  }
  switch (lg) {
    case 8: return launch_fft_kernel<Real>(mw_cols_kernel<Real, 8, kRegBufs>, grid, 16, reg_smem<Real, 8>(extra), p, s, reg_carveout<Real, 8>(extra));
    case 9: return launch_fft_kernel<Real>(mw_cols_kernel<Real, 9, kRegBufs>, grid, 32, reg_smem<Real, 9>(extra), p, s, reg_carveout<Real, 9>(extra));
    case 10: return launch_fft_kernel<Real>(mw_cols_kernel<Real, 10, kRegBufs>, grid, 64, reg_smem<Real, 10>(extra), p, s, reg_carveout<Real, 10>(extra));
    case 11: return launch_fft_kernel<Real>(mw_cols_kernel<Real, 11, kRegBufs>, grid, 128, reg_smem<Real, 11>(extra), p, s, reg_carveout<Real, 11>(extra));
    case 12: return launch_fft_kernel<Real>(mw_cols_kernel<Real, 12, kRegBufs>, grid, 256, reg_smem<Real, 12>(extra), p, s, reg_carveout<Real, 12>(extra));
    case 13: return launch_fft_kernel<Real>(mw_cols_kernel<Real, 13, kRegBufs>, grid, 512, reg_smem<Real, 13>(extra), p, s, reg_carveout<Real, 13>(extra));
    default: break;
  }
  // one DFT buffer plus the 2L bins carried between the two transforms
  const size_t smem = (size_t)(padded_len(M1 > M2 ? M1 : M2) + 2 * p.L) * sizeof(R2);
  return launch_fft_kernel<Real>(mw_cols_kernel<Real, 0, 1>, grid, fft_threads(M1 > M2 ? M1 : M2),
                                 smem, p, s);
}

template <typename Real>
cudaError_t launch_mw_cols_adj(const ColsParams<Real>& p, int ncm, int batch, int M1, int M2,
                               int ncol_out, int mo_out, cudaStream_t s) {
  using R2 = typename C2<Real>::t;
  // one DFT buffer plus the n1 = 2L-1 or 2L inputs of the second transform
  const size_t smem = (size_t)(padded_len(M1 > M2 ? M1 : M2) + 2 * p.L) * sizeof(R2);
  cudaError_t e = cudaFuncSetAttribute(mw_cols_adj_kernel<Real>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(mw_cols_adj_kernel<Real>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  mw_cols_adj_kernel<Real><<<dim3(ncm, batch), fft_threads(M1 > M2 ? M1 : M2), smem, s>>>(
      p, ncol_out, mo_out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Ring-pair fold (equator-symmetric forward): one thread per (map, half, row, pair, component).
// Idx is the flat index type (32-bit whenever the arrays fit: 64-bit division by a
// runtime divisor would dominate these element-wise kernels).
// ---------------------------------------------------------------------------
template <typename Real, typename Idx>
__global__ void fold_pairs_kernel(FoldParams p) {
  using R2 = typename C2<Real>::t;
  const int per = p.dual ? 2 : 1;  // Real2 entries of one spectrum (dual: +m and -m)
  const int halves = p.dual ? 1 : p.nhalf;
  const Idx total = (Idx)p.batch * halves * p.TR * p.Gs2 * per;
  const R2* G = reinterpret_cast<const R2*>(p.G);
  R2* G2 = reinterpret_cast<R2*>(p.G2);
  for (Idx i = blockIdx.x * (Idx)blockDim.x + threadIdx.x; i < total;
       i += (Idx)gridDim.x * blockDim.x) {
    const int c = p.dual ? (int)(i & 1) : 0;
    const Idx iq = p.dual ? i >> 1 : i;
    const Idx rw = iq / (Idx)p.Gs2;
    const int q = (int)(iq - rw * (Idx)p.Gs2);
    const size_t row = rw;  // (b, half, m row)
    const int mrow = (int)(rw % (Idx)p.TR);
    R2 e = czero<R2>(), o = czero<R2>();
    if (q < p.npair && mrow >= kPadLo && mrow < p.L + kPadLo) {
      const int qm = p.nrows - 1 - q;  // mirror ring
      const R2 a = G[(row * p.Gs + q) * per + c];
      e = a;
      if (qm != q) {
        const R2 z = G[(row * p.Gs + qm) * per + c];
        e = cadd(a, z);
        o = csub(a, z);
      }
    }
    G2[((row * p.Gs2 + q) * 2 + 0) * per + c] = e;
    G2[((row * p.Gs2 + q) * 2 + 1) * per + c] = o;
  }
}

// cross mode: one thread per (map, half, row, pair)
template <typename Real, typename Idx>
__global__ void fold_cross_kernel(FoldParams p) {
  using R2 = typename C2<Real>::t;
  const Idx total = (Idx)p.batch * 2 * p.TR * p.Gs2;
  const R2* G = reinterpret_cast<const R2*>(p.G);
  R2* G2 = reinterpret_cast<R2*>(p.G2);
  for (Idx i = blockIdx.x * (Idx)blockDim.x + threadIdx.x; i < total;
       i += (Idx)gridDim.x * blockDim.x) {
    const Idx rw = i / (Idx)p.Gs2;
    const int q = (int)(i - rw * (Idx)p.Gs2);
    const long row = (long)rw;  // (b, half, m row)
    const Idx bh = rw / (Idx)p.TR;
    const int mrow = (int)(rw - bh * (Idx)p.TR);
    const int half = (int)(bh & 1);
    const long orow = row + (half ? -1L : 1L) * p.TR;  // the other half, same map and m
    R2 a = czero<R2>(), z = czero<R2>();
    if (q < p.npair && mrow >= kPadLo && mrow < p.L + kPadLo) {
      const int qm = p.nrows - 1 - q;
      a = G[row * p.Gs + q];
      if (qm != q) z = G[orow * p.Gs + qm];
    }
    R2* e = G2 + (row * p.Gs2 + q) * 4;  // two Real4 = four Real2
    e[0] = a;
    e[1] = z;
    e[2] = a;
    e[3] = cscale(z, Real(-1));
  }
}

cudaError_t launch_fold_pairs(bool fp64, const FoldParams& p, cudaStream_t s) {
  if (p.cross) {
    const long total = (long)p.batch * 2 * p.TR * p.Gs2;
    long blocks = (total + 255) / 256;
    if (blocks > 65535L * 8) blocks = 65535L * 8;
    if (blocks < 1) blocks = 1;
    const bool i32 = total + 65535L * 8 * 256 < (1L << 32);
    if (fp64 && i32)
      fold_cross_kernel<double, uint32_t><<<(unsigned)blocks, 256, 0, s>>>(p);
    else if (fp64)
      fold_cross_kernel<double, uint64_t><<<(unsigned)blocks, 256, 0, s>>>(p);
    else if (i32)
      fold_cross_kernel<float, uint32_t><<<(unsigned)blocks, 256, 0, s>>>(p);
    else
      fold_cross_kernel<float, uint64_t><<<(unsigned)blocks, 256, 0, s>>>(p);
    return cudaGetLastError();
  }
  const long total = (long)p.batch * (p.dual ? 1 : p.nhalf) * p.TR * p.Gs2 * (p.dual ? 2 : 1);
  long blocks = (total + 255) / 256;
  if (blocks > 65535L * 8) blocks = 65535L * 8;
  if (blocks < 1) blocks = 1;
  const bool i32 = total + 65535L * 8 * 256 < (1L << 32);
  if (fp64 && i32)
    fold_pairs_kernel<double, uint32_t><<<(unsigned)blocks, 256, 0, s>>>(p);
  else if (fp64)
    fold_pairs_kernel<double, uint64_t><<<(unsigned)blocks, 256, 0, s>>>(p);
  else if (i32)
    fold_pairs_kernel<float, uint32_t><<<(unsigned)blocks, 256, 0, s>>>(p);
  else
    fold_pairs_kernel<float, uint64_t><<<(unsigned)blocks, 256, 0, s>>>(p);
  return cudaGetLastError();
}

template cudaError_t launch_mw_cols_adj<float>(const ColsParams<float>&, int, int, int, int, int,
                                               int, cudaStream_t);
template cudaError_t launch_mw_cols_adj<double>(const ColsParams<double>&, int, int, int, int, int,
                                                int, cudaStream_t);
template cudaError_t launch_inv_rows<float>(const RowsParams<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_inv_rows<double>(const RowsParams<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_fwd_rows<float>(const RowsParams<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_fwd_rows<double>(const RowsParams<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_mw_cols<float>(const ColsParams<float>&, int, int, int, int, cudaStream_t);
template cudaError_t launch_mw_cols<double>(const ColsParams<double>&, int, int, int, int, cudaStream_t);

}  // namespace s2b
