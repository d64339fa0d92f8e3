// Block-level FFT building blocks shared by the ring-FFT and Fourier-Wigner kernels:
// complex helpers, the padded shared-memory layout, fused radix-2 passes and the
// any-length DFT (power of two, or Bluestein) of one CTA.
#pragma once

#include <cuda_runtime.h>

#include "s2b_fft.h"

namespace s2b {

template <typename Real>
struct C2;
template <>
struct C2<float> {
  using t = float2;
};
template <>
struct C2<double> {
  using t = double2;
};

template <typename R2>
__device__ __forceinline__ R2 cmul(R2 a, R2 b) {
  R2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename R2>
__device__ __forceinline__ R2 cadd(R2 a, R2 b) {
  R2 r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename R2>
__device__ __forceinline__ R2 csub(R2 a, R2 b) {
  R2 r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
template <typename R2>
__device__ __forceinline__ R2 cconj(R2 a) {
  a.y = -a.y;
  return a;
}
template <typename R2, typename Real>
__device__ __forceinline__ R2 cscale(R2 a, Real s) {
  a.x *= s;
  a.y *= s;
  return a;
}
template <typename R2>
__device__ __forceinline__ R2 czero() {
  R2 r;
  r.x = 0;
  r.y = 0;
  return r;
}

// Shared-memory layout of a transform buffer: one padding slot per 8 elements,
// so that the contiguous 8-element groups of the last DIF / first DIT pass fall
// into distinct banks. A buffer for length M holds M + M/8 elements.
__device__ __forceinline__ int pidx(int e) { return e + (e >> 3); }
__host__ __device__ inline int padded_len(int M) { return M + (M >> 3); }

// Radix-2 butterflies fused NS <= 3 stages per pass: a thread loads the 2^NS
// elements base + a q that NS consecutive stages combine, runs the stages in
// registers and writes them back in place (same data order as plain radix-2),
// so a length-4096 transform takes 4 passes and 4 barriers instead of 12.
// tw[k] = exp(-2 pi i k / M), k < M/2.
//
// DIF stage of span hs: (x, x + hs) -> (x + y, (x - y) w), w = tw[(x mod hs) M / (2 hs)],
// spans decreasing (h, h/2, ...); DIT stage: (x, x + hs) -> (x + y w, x - y w), spans
// increasing (q, 2q, ...). In both, the pass covers elements base + a q, a < 2^NS.
// Every twiddle of a pass derives from one table entry b = tw[r M / (2h)]
// (h = largest span of the pass, r = position of the group): the stage whose
// pairs are sj q apart uses b^(2^(NS-1)/sj) * exp(-i pi k / sj), k = a mod sj,
// i.e. powers of b times constant roots of unity of order <= 8.
template <int S, typename R2>
__device__ __forceinline__ R2 root_rot(R2 w, int k, bool inv) {
  // w * exp(-i pi k / S) (conjugate rotation when inv), k < S, S in {1, 2, 4}
  using Real = decltype(w.x);
  if (S == 1 || k == 0) return w;
  const Real c = Real(0.70710678118654752440);
  R2 o;
  if (S == 2 || k == 2) {  // -i (or +i)
    o.x = inv ? -w.y : w.y;
    o.y = inv ? w.x : -w.x;
    return o;
  }
  if (k == 1) {  // (1 - i)/sqrt2  (inv: (1 + i)/sqrt2)
    o.x = inv ? (w.x - w.y) * c : (w.x + w.y) * c;
    o.y = inv ? (w.x + w.y) * c : (w.y - w.x) * c;
    return o;
  }
  // k == 3: (-1 - i)/sqrt2  (inv: (-1 + i)/sqrt2)
  o.x = inv ? (-w.x - w.y) * c : (w.y - w.x) * c;
  o.y = inv ? (w.x - w.y) * c : (-w.x - w.y) * c;
  return o;
}

template <int NS, bool DIF, typename R2>
__device__ __forceinline__ void fft_pass(R2* s, int M, int lq, const R2* __restrict__ tw, bool inv,
                                         const R2* __restrict__ post) {
  constexpr int NA = 1 << NS;
  const int q = 1 << lq;  // q = 2^lq: group position and index by shifts and masks
  const int ls0 = __ffs(M) - 1 - lq - NS;  // log2(M / (2 h)), h = q 2^(NS-1) the largest span
  for (int g = threadIdx.x; g < (M >> NS); g += blockDim.x) {
    const int r = g & (q - 1);
    const int base = ((g >> lq) << (lq + NS)) + r;
    R2 x[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) x[a] = s[pidx(base + a * q)];
    R2 bp[3];  // b, b^2, b^4
    bp[0] = tw[r << ls0];
    if (inv) bp[0].y = -bp[0].y;
    bp[1] = cmul(bp[0], bp[0]);
    bp[2] = cmul(bp[1], bp[1]);
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const int sj = DIF ? (1 << (NS - 1 - j)) : (1 << j);  // pair distance in units of q
      const int pw = DIF ? j : NS - 1 - j;                  // power index: b^(2^pw)
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        if (a & sj) continue;
        R2 w;
        if (sj == 4)
          w = root_rot<4>(bp[pw], a & 3, inv);
        else if (sj == 2)
          w = root_rot<2>(bp[pw], a & 1, inv);
        else
          w = bp[pw];
        if (DIF) {
          const R2 u = x[a], v = x[a + sj];
          x[a] = cadd(u, v);
          x[a + sj] = cmul(csub(u, v), w);
        } else {
          const R2 u = x[a];
          const R2 v = cmul(x[a + sj], w);
          x[a] = cadd(u, v);
          x[a + sj] = csub(u, v);
        }
      }
    }
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      const int e = base + a * q;
      s[pidx(e)] = post ? cmul(x[a], post[e]) : x[a];
    }
  }
}

// DIF: natural order in, bit-reversed out; if post != nullptr the output element
// e (bit-reversed position) is multiplied by post[e] in the last pass.
template <typename R2>
__device__ void fft_dif(R2* s, int M, int logM, const R2* __restrict__ tw, bool inv,
                        const R2* __restrict__ post = nullptr) {
  for (int done = 0; done < logM;) {
    const int ns = logM - done < 3 ? logM - done : 3;
    const int lq = logM - done - ns;  // log2 of the span of the last fused stage
    const R2* pp = done + ns == logM ? post : nullptr;
    __syncthreads();
    if (ns == 3)
      fft_pass<3, true>(s, M, lq, tw, inv, pp);
    else if (ns == 2)
      fft_pass<2, true>(s, M, lq, tw, inv, pp);
    else
      fft_pass<1, true>(s, M, lq, tw, inv, pp);
    done += ns;
  }
  __syncthreads();
}

// DIT: bit-reversed order in, natural out.
template <typename R2>
__device__ void fft_dit(R2* s, int M, int logM, const R2* __restrict__ tw, bool inv) {
  for (int done = 0; done < logM;) {
    const int ns = logM - done < 3 ? logM - done : 3;
    const int lq = done;  // log2 of the span of the first fused stage
    __syncthreads();
    if (ns == 3)
      fft_pass<3, false>(s, M, lq, tw, inv, (const R2*)nullptr);
    else if (ns == 2)
      fft_pass<2, false>(s, M, lq, tw, inv, (const R2*)nullptr);
    else
      fft_pass<1, false>(s, M, lq, tw, inv, (const R2*)nullptr);
    done += ns;
  }
  __syncthreads();
}

__device__ __forceinline__ int bitrev(int x, int logM) { return __brev(x) >> (32 - logM); }

// DFT of length d.n of the sequence produced by load(k) (k < n); after the call
// get(j) returns X_j (j < n). inv selects exp(+2 pi i jk / n).
// The buffer s must hold d.M complex values.
template <typename Real, typename Load>
__device__ void dft_run(typename C2<Real>::t* s, const FFTDesc& d, const FFTTables<Real>& tb,
                        bool inv, Load load) {
  using R2 = typename C2<Real>::t;
  const R2* tw = tb.tw + d.tw_off;
  if (d.bluestein) {
    const R2* ch = tb.chirp + d.chirp_off;
    const R2* bf = tb.bfilt + d.bf_off;
    for (int k = threadIdx.x; k < d.M; k += blockDim.x) {
      R2 x = czero<R2>();
      if (k < d.n) {
        x = load(k);
        if (inv) x = cconj(x);
        x = cmul(x, ch[k]);
      }
      s[pidx(k)] = x;
    }
    fft_dif(s, d.M, d.logM, tw, false, bf);
    fft_dit(s, d.M, d.logM, tw, true);
  } else {
    for (int k = threadIdx.x; k < d.M; k += blockDim.x) {
      R2 x = load(k);
      if (inv) x = cconj(x);
      s[pidx(k)] = x;
    }
    fft_dif(s, d.M, d.logM, tw, false);
  }
}

template <typename Real>
__device__ __forceinline__ typename C2<Real>::t dft_get(const typename C2<Real>::t* s,
                                                        const FFTDesc& d,
                                                        const FFTTables<Real>& tb, bool inv,
                                                        int j) {
  using R2 = typename C2<Real>::t;
  R2 x;
  if (d.bluestein)
    x = cmul(s[pidx(j)], tb.chirp[d.chirp_off + j]);
  else
    x = s[pidx(bitrev(j, d.logM))];
  return inv ? cconj(x) : x;
}

__device__ __forceinline__ int pmod(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

}  // namespace s2b
