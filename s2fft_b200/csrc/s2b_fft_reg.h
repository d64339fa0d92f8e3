// Register-resident power-of-two FFT of one CTA: M = 2^LOGM points, T = M / 16 threads,
// 16 points per thread.
//
// The transform is the same sequence of radix-2 decimation-in-frequency (DIF) and
// decimation-in-time (DIT) stages as the shared-memory passes of s2b_fft_dev.h, with the
// same twiddle derivation and the same bit-reversed intermediate order, so the Bluestein
// filter tables serve both. What changes is where the data lives between stages:
//   * the first DIF pass takes its points straight from the caller (thread j holds points
//     j + T a, a < 16: coalesced in memory order), and the last DIT pass leaves them in
//     the same places, so inputs and outputs need not pass through shared memory;
//   * each pass fuses up to four stages on 16 points held in registers; only between
//     passes do the points cross shared memory;
//   * in a Bluestein transform the last DIF pass, the product with the filter and the
//     first DIT pass run on the same registers.
// A 4096-point Bluestein transform thus makes 4 shared-memory exchanges instead of the 8
// read-write passes plus the load and store passes of the shared-memory version.
//
// Stage grouping for LOGM = 4 k + r: DIF passes of r (or 4), then 4, 4, ... stages, spans
// decreasing; DIT mirrors it. A radix-16 pass with smallest span q = 2^lq gives thread j
// the group based at ((j >> lq) << (lq + 4)) + (j & (q - 1)) with points base + q a; the
// first DIF / last DIT pass (spans M/2 .. M/2^r) uses the points j + T a, which form
// 2^(4-r) groups of 2^r points (a = a_lo + 2^(4-r) a_hi, a_hi the position in the group).
#pragma once

#include <cuda_runtime.h>

#include "s2b_fft_dev.h"

namespace s2b {

// w * exp(-i pi k / 8) (conjugate rotation when inv), k < 8 (compile-time constants)
template <typename R2>
__device__ __forceinline__ R2 rot16(R2 w, int k, bool inv) {
  using Real = decltype(w.x);
  if (k == 0) return w;
  if (k == 4) {  // -i (+i)
    R2 o;
    o.x = inv ? -w.y : w.y;
    o.y = inv ? w.x : -w.x;
    return o;
  }
  // cos and sin of pi k / 8
  const Real C[8] = {Real(1), Real(0.92387953251128675613), Real(0.70710678118654752440),
                     Real(0.38268343236508977173), Real(0), Real(-0.38268343236508977173),
                     Real(-0.70710678118654752440), Real(-0.92387953251128675613)};
  const Real S[8] = {Real(0), Real(0.38268343236508977173), Real(0.70710678118654752440),
                     Real(0.92387953251128675613), Real(1), Real(0.92387953251128675613),
                     Real(0.70710678118654752440), Real(0.38268343236508977173)};
  const Real c = C[k], s = inv ? S[k] : -S[k];  // exp(-+ i pi k / 8) = c + i s
  R2 o;
  o.x = w.x * c - w.y * s;
  o.y = w.x * s + w.y * c;
  return o;
}

// Stage J of NS fused radix-2 stages on the 2^NS points x[ST * a] of one group (see
// reg_stages); template recursion keeps every index a compile-time constant, so the points
// stay in registers.
template <int NS, bool DIF, int ST, int J, typename R2>
__device__ __forceinline__ void reg_stage(R2* x, const R2 (&bp)[NS], bool inv) {
  if constexpr (J < NS) {
    constexpr int NA = 1 << NS;
    constexpr int SJ = DIF ? (1 << (NS - 1 - J)) : (1 << J);  // pair distance (units of q)
    constexpr int PW = DIF ? J : NS - 1 - J;                  // power index: b^(2^PW)
    R2 w[SJ];
#pragma unroll
    for (int k = 0; k < SJ; ++k) w[k] = rot16(bp[PW], k * (8 / SJ), inv);
#pragma unroll
    for (int blk = 0; blk < NA; blk += 2 * SJ) {
#pragma unroll
      for (int k = 0; k < SJ; ++k) {
        const int a = blk + k;
        if constexpr (DIF) {
          const R2 u = x[a * ST], v = x[(a + SJ) * ST];
          x[a * ST] = cadd(u, v);
          x[(a + SJ) * ST] = cmul(csub(u, v), w[k]);
        } else {
          const R2 u = x[a * ST];
          const R2 v = cmul(x[(a + SJ) * ST], w[k]);
          x[a * ST] = cadd(u, v);
          x[(a + SJ) * ST] = csub(u, v);
        }
      }
    }
    reg_stage<NS, DIF, ST, J + 1>(x, bp, inv);
  }
}

// NS fused radix-2 stages on the 2^NS points x[ST * a] (a < 2^NS) of one group whose base
// point is r modulo its smallest span q. tws[k * stride] = b^(2^k), k < NS, with
// b = exp(-2 pi i r 2^sh / M), sh = log2(M / (2^NS q)) (conjugated when inv): the twiddles
// of the group, read from the register-engine table (FFTDesc::rtw_off), where consecutive
// threads read consecutive entries. DIF: spans decreasing; DIT: increasing. The stage of
// span s q pairs points s apart and multiplies by b^(2^NS / (2 s)) exp(-i pi k / s), k the
// position within the pair block (the derivation of fft_pass in s2b_fft_dev.h).
// the twiddles b^(2^k) = tws[k * stride], k < NS, of one group (conjugated when inv)
template <int NS, typename R2>
__device__ __forceinline__ void reg_twiddles(R2 (&bp)[NS], const R2* __restrict__ tws, int stride,
                                             bool inv) {
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    bp[k] = tws[k * stride];
    if (inv) bp[k].y = -bp[k].y;
  }
}

// NS fused radix-2 stages on the 2^NS points x[ST * a] (a < 2^NS) of one group whose base
// point is r modulo its smallest span q. tws[k * stride] = b^(2^k), k < NS, with
// b = exp(-2 pi i r 2^sh / M), sh = log2(M / (2^NS q)) (conjugated when inv): the twiddles
// of the group, read from the register-engine table (FFTDesc::rtw_off), where consecutive
// threads read consecutive entries. DIF: spans decreasing; DIT: increasing. The stage of
// span s q pairs points s apart and multiplies by b^(2^NS / (2 s)) exp(-i pi k / s), k the
// position within the pair block (the derivation of fft_pass in s2b_fft_dev.h).
template <int NS, bool DIF, int ST, typename R2>
__device__ __forceinline__ void reg_stages(R2* x, const R2* __restrict__ tws, int stride,
                                           bool inv) {
  R2 bp[NS];
  reg_twiddles(bp, tws, stride, inv);
  reg_stage<NS, DIF, ST, 0>(x, bp, inv);
}

// shared-memory slot of point e: one pad slot per 16 points keeps the passes' accesses
// free of bank conflicts (the last DIF pass reads points 16 j + a: stride 17 slots)
__device__ __forceinline__ int ridx(int e) { return e + (e >> 4); }

template <int LOGM, int NBUF>
struct RegFFT {
  static constexpr int M = 1 << LOGM;
  static constexpr int T = M >> 4;
  static constexpr int NS0 = (LOGM & 3) ? (LOGM & 3) : 4;
  static constexpr int NMID = (LOGM - NS0) / 4;  // radix-16 passes after the first
  static_assert(LOGM >= 8 && NMID >= 1, "register FFT needs M >= 256");
  // shared memory: NBUF exchange buffers (2: ping-pong, one barrier per exchange; 1: two
  // barriers per exchange, half the space)
  static constexpr int BUF = M + (M >> 4);
  static constexpr int SMEM_ELEMS = NBUF * BUF;

  // point held in x[a] by thread j in the radix-16 pass whose smallest span is 2^lq, or in
  // the first DIF / last DIT pass (lq < 0)
  __device__ __forceinline__ static int point(int j, int a, int lq) {
    if (lq < 0) return j + T * a;
    const int q = 1 << lq;
    return ((j >> lq) << (lq + 4)) + (j & (q - 1)) + q * a;
  }

  // the points move from the layout of pass lq_from to that of pass lq_to
  template <typename R2>
  __device__ __forceinline__ static void exchange(R2 (&x)[16], R2* buf, int& ping, int lq_from,
                                                  int lq_to) {
    const int j = threadIdx.x;
    R2* s = buf + (NBUF == 2 ? ping * BUF : 0);
    if (NBUF == 1) __syncthreads();  // readers of the previous exchange are done
#pragma unroll
    for (int a = 0; a < 16; ++a) s[ridx(point(j, a, lq_from))] = x[a];
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 16; ++a) x[a] = s[ridx(point(j, a, lq_to))];
    ping ^= 1;
  }

  // the twiddle table (FFTDesc::rtw_off): the first pass's rows (q0 entries each), then the
  // radix-16 passes in DIF order (lq decreasing), 4 rows of 2^lq entries each
  static constexpr int Q0 = M >> NS0;
  __host__ __device__ static constexpr int mid_off(int lq) {
    int off = NS0 * Q0;
    for (int l = 4 * (NMID - 1); l > lq; l -= 4) off += 4 << l;
    return off;
  }

  // twiddles of the first DIF / last DIT pass for this thread's G groups
  template <typename R2>
  __device__ __forceinline__ static void first_tw(R2 (&bp)[1 << (4 - NS0)][NS0], const R2* rtw,
                                                  bool inv) {
    constexpr int G = 1 << (4 - NS0);
#pragma unroll
    for (int g = 0; g < G; ++g) reg_twiddles(bp[g], rtw + threadIdx.x + T * g, Q0, inv);
  }
  // twiddles of the radix-16 pass with smallest span 2^lq
  template <typename R2>
  __device__ __forceinline__ static void mid_tw(R2 (&bp)[4], int lq, const R2* rtw, bool inv) {
    reg_twiddles(bp, rtw + mid_off(lq) + (threadIdx.x & ((1 << lq) - 1)), 1 << lq, inv);
  }

  // DIF: x holds points j + T a in natural order; on return x[a] holds the bit-reversed
  // position point(j, a, 0) (the layout of the last pass, smallest span 1). The radix-16
  // passes share one loop body (a compact instruction footprint), and each pass's
  // twiddles are loaded before the barrier that precedes it.
  template <typename R2>
  __device__ __forceinline__ static void dif(R2 (&x)[16], R2* buf, const R2* tw, bool inv,
                                             int& ping) {
    constexpr int G = 1 << (4 - NS0);
    R2 b0[G][NS0], bp[4];
    first_tw(b0, tw, inv);
    mid_tw(bp, 4 * (NMID - 1), tw, inv);
#pragma unroll
    for (int g = 0; g < G; ++g) reg_stage<NS0, true, G, 0>(x + g, b0[g], inv);
#pragma unroll 1
    for (int p = 0; p < NMID; ++p) {
      const int lq = 4 * (NMID - 1 - p);
      exchange(x, buf, ping, p == 0 ? -1 : lq + 4, lq);
      R2 cur[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) cur[k] = bp[k];
      if (p + 1 < NMID) mid_tw(bp, lq - 4, tw, inv);
      reg_stage<4, true, 1, 0>(x, cur, inv);
    }
  }
  // DIT: x holds bit-reversed positions in dif's output layout; on return, natural order
  // with thread j holding points j + T a.
  template <typename R2>
  __device__ __forceinline__ static void dit(R2 (&x)[16], R2* buf, const R2* tw, bool inv,
                                             int& ping) {
    constexpr int G = 1 << (4 - NS0);
    R2 bp[4];
    mid_tw(bp, 0, tw, inv);
#pragma unroll 1
    for (int p = 0; p < NMID; ++p) {
      if (p > 0) exchange(x, buf, ping, 4 * (p - 1), 4 * p);
      R2 cur[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) cur[k] = bp[k];
      if (p + 1 < NMID) mid_tw(bp, 4 * (p + 1), tw, inv);
      reg_stage<4, false, 1, 0>(x, cur, inv);
    }
    R2 b0[G][NS0];
    first_tw(b0, tw, inv);
    exchange(x, buf, ping, 4 * (NMID - 1), -1);
#pragma unroll
    for (int g = 0; g < G; ++g) reg_stage<NS0, false, G, 0>(x + g, b0[g], inv);
  }
};

}  // namespace s2b
