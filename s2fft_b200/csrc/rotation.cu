// Rotation of spherical-harmonic coefficients by Euler angles (alpha, beta, gamma):
//   flm'[l, m] = exp(-i m alpha) sum_n d^l_{m,n}(beta) exp(-i n gamma) flm[l, n]
// (upstream s2fft/utils/rotation.py:9-64, rotate_flms; the planes of generate_rotate_dls,
// rotation.py:75-96).
//
// Upstream builds the Wigner-d planes degree by degree with Risbo's recursion
// (s2fft/recursions/risbo.py:4-120), so every degree waits for the whole previous plane.
// Here every entry (m, n) follows its own three-term recurrence in the degree
// (Varshalovich, Moskalev & Khersonskii, Quantum Theory of Angular Momentum, sec. 4.8;
// Kostelec & Rockmore, J. Fourier Anal. Appl. 14 (2008) 145-179):
//   d^{l+1}_{mn} = U_l(m) R_l(n) [ (cos beta - m n q_l) d^l_{mn} - V_l(m) P_l(n) d^{l-1}_{mn} ],
//   R_l(k) = 1/sqrt((l+1)^2 - k^2), P_l(k) = sqrt(l^2 - k^2), q_l = 1/(l(l+1)),
//   U_l(m) = (l+1)(2l+1) R_l(m), V_l(m) = P_l(m) / (l(2l+1)),
// started at l0 = max(|m|, |n|) from E[l0][a] = d^{l0}_{l0,a} = (-1)^{l0-a}
// sqrt(binom(2 l0, l0+a)) c^{l0+a} s^{l0-a} (c = cos(beta/2), s = sin(beta/2)) through
// d_{m,n} = (-1)^{m-n} d_{n,m} = d_{-n,-m}. Orders m < 0 follow from
// d_{-m,-n} = (-1)^{m-n} d_{m,n}, so only m >= 0 is recurred. In double precision the
// recurrence matches Risbo's planes to rounding (against a long-double run at L = 256:
// 1e-15..8e-14 here, 1e-13..2e-13 for Risbo).
//
// Start values below 2^-960 are carried as a mantissa times 2^k (an int k < 0 per
// entry), renormalised in steps of 2^64 as they grow, and weighted by 2^k where they
// contribute. The start table is the exponent-tracked product W = E^2,
//   W_l = W_{l-1} 2l(2l-1) / ((l+a)(l-a)) (cs)^2,  W_{|a|} = c^{4a} (a >= 0), s^{4|a|} (a < 0),
// formed in segments of 32 degrees with a carry pass, so no log-gamma enters.
//
// Schedule: a cluster of CTAs owns MT orders m0..m0+MT-1 (with their negatives) and all
// n; lanes run along n in zigzag order (0, -1, 1, -2, ...) dealt to the cluster's CTAs
// and warps in turn, so short and long n are shared alike. Each lane carries MT x S
// recurrences in registers and walks l from m0 to L-1; its operands (T[l][|n|],
// flm[l][+-n]) arrive through a cp.async ring in shared memory a few degrees ahead. Per
// degree a warp reduces its 4 MT sums (+-m, re / im) by halving shuffles into shared
// memory. Every kRotChunk degrees a CTA sums its warps and publishes the result with a
// cluster arrive; after the matching wait, at the end of the next chunk, each CTA sums its
// share of the outputs over the cluster's CTAs through distributed shared memory in rank
// order (deterministic, no atomics) and writes them with exp(-i m alpha). With 8 orders
// per tile and one n per lane (rotate_mma_kernel; clusters of up to 16 CTAs up to
// L = 2048) the sum over a warp's 32 n runs on the FP64 tensor cores instead of shuffles.
// The planes path writes every entry of [L][2L-1][2L-1] once, zeros included. All
// arithmetic is double.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "s2b.h"
#include "s2b_dev.h"
#include "s2b_internal.h"
#include "s2b_rotation.h"

namespace cg = cooperative_groups;

namespace s2b {
namespace {

constexpr int kRotSeg = 32;    // degrees per segment of the start-table product
constexpr int kRotChunk = 16;  // degrees between cluster reductions

template <typename R2>
struct RotIO;
template <>
struct RotIO<float2> {
  static __device__ double2 get(const void* p, size_t i) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p) + i);
    return make_double2(v.x, v.y);
  }
  static __device__ void put(void* p, size_t i, double2 v) {
    reinterpret_cast<float2*>(p)[i] = make_float2((float)v.x, (float)v.y);
  }
};
template <>
struct RotIO<double2> {
  static __device__ double2 get(const void* p, size_t i) {
    return __ldg(reinterpret_cast<const double2*>(p) + i);
  }
  static __device__ void put(void* p, size_t i, double2 v) {
    reinterpret_cast<double2*>(p)[i] = v;
  }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------------

// exp(-i m alpha), exp(-i n gamma), m, n in [-(L-1), L-1]
__global__ void rotate_phase_kernel(RotParams p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * p.L - 1;
       i += gridDim.x * blockDim.x) {
    const double k = (double)(i - (p.L - 1));
    double s, c;
    sincos(-k * p.alpha, &s, &c);
    p.ea[i] = make_double2(c, s);
    sincos(-k * p.gamma, &s, &c);
    p.eg[i] = make_double2(c, s);
  }
}

// recurrence coefficients T and UVQ (beta-independent)
__global__ void rotate_coef_kernel(RotParams p) {
  const int L = p.L;
  const long total = (long)L * L;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const int l = (int)(e / L), k = (int)(e % L);
    double2 t = make_double2(0.0, 0.0);
    double4 uv = make_double4(0.0, 0.0, 0.0, 0.0);
    if (k <= l) {
      const double dl = (double)l, dk = (double)k;
      const double R = 1.0 / sqrt((dl + 1.0) * (dl + 1.0) - dk * dk);
      const double P = sqrt(dl * dl - dk * dk);
      t = make_double2(R, P);
      if (l > 0)
        uv = make_double4((dl + 1.0) * (2.0 * dl + 1.0) * R, P / (dl * (2.0 * dl + 1.0)),
                          -dk / (dl * (dl + 1.0)), 0.0);
      else
        uv = make_double4(R, 0.0, 0.0, 0.0);
    }
    p.T[e] = t;
    p.UVQ[e] = uv;
  }
}

__device__ __forceinline__ RotXD xd_make(double x) {
  RotXD r;
  r.m = frexp(x, &r.e);
  r.pad = 0;
  if (r.m == 0.0) r.e = 0;
  return r;
}
__device__ __forceinline__ RotXD xd_mul(RotXD a, RotXD b) {
  int d;
  RotXD r;
  r.m = frexp(a.m * b.m, &d);
  r.e = r.m == 0.0 ? 0 : a.e + b.e + d;
  r.pad = 0;
  return r;
}
__device__ RotXD xd_pow(double x, int n) {  // x^n, n >= 0
  RotXD r = xd_make(1.0), b = xd_make(x);
  while (n) {
    if (n & 1) r = xd_mul(r, b);
    b = xd_mul(b, b);
    n >>= 1;
  }
  return r;
}

// start table, pass 1: W_l / W_{segment start} inside each segment of kRotSeg degrees
// (the segment holding l = |a| starts from W_{|a|}); the segment product goes to carry
__global__ void rotate_start_seg_kernel(RotParams p) {
  const int L = p.L, NN = 2 * L - 1;
  const int ai = blockIdx.x * blockDim.x + threadIdx.x, g = blockIdx.y;
  if (ai >= NN) return;
  const int a = ai - (L - 1), aa = a < 0 ? -a : a;
  const int lb = max(g * kRotSeg, aa), le = min(g * kRotSeg + kRotSeg, L);
  RotXD w = xd_make(1.0);
  if (lb < le) {
    if (lb == aa) w = a >= 0 ? xd_pow(p.c2, 2 * a) : xd_pow(p.s2, 2 * aa);
#pragma unroll 1
    for (int l = lb; l < le; ++l) {
      if (l > aa) {
        const double f = (2.0 * l) * (2.0 * l - 1.0) / ((double)(l + a) * (double)(l - a));
        w = xd_mul(w, xd_make(f * p.cs2));
      }
      p.start[(size_t)l * NN + ai] = w;
    }
  }
  p.carry[(size_t)g * NN + ai] = w;
}

// pass 2: exclusive products of the segment products, per a
__global__ void rotate_start_carry_kernel(RotParams p) {
  const int L = p.L, NN = 2 * L - 1, G = (L + kRotSeg - 1) / kRotSeg;
  const int ai = blockIdx.x * blockDim.x + threadIdx.x;
  if (ai >= NN) return;
  RotXD c = xd_make(1.0);
#pragma unroll 1
  for (int g0 = 0; g0 < G; g0 += 8) {  // eight segment products in flight at a time
    RotXD t[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (g0 + u < G) t[u] = p.carry[(size_t)(g0 + u) * NN + ai];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (g0 + u < G) {
        p.carry[(size_t)(g0 + u) * NN + ai] = c;
        c = xd_mul(c, t[u]);
      }
  }
}

// pass 3: E = sign sqrt(W) as the start value (v, k) of the recurrence
__global__ void rotate_start_final_kernel(RotParams p) {
  const int L = p.L, NN = 2 * L - 1;
  const int ai = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y;
  if (ai >= NN) return;
  const int a = ai - (L - 1);
  if (a < -l || a > l) return;
  const size_t e = (size_t)l * NN + ai;
  const RotXD w = xd_mul(p.start[e], p.carry[(size_t)(l / kRotSeg) * NN + ai]);
  double m = w.m;
  int x = w.e;
  if (x & 1) {
    m *= 2.0;
    x -= 1;
  }
  RotXD r;
  r.pad = 0;
  r.m = sqrt(m);
  r.e = x / 2;
  if (m == 0.0) {
    r.e = 0;
  } else if (r.e >= -960) {
    r.m = ldexp(r.m, r.e);
    r.e = 0;
  }
  const int neg = ((l - a) & 1) ^ (p.c_neg & ((l + a) & 1)) ^ (p.s_neg & ((l - a) & 1));
  if (neg) r.m = -r.m;
  p.start[e] = r;
}

// ---------------------------------------------------------------------------------
// recurrence kernel
// ---------------------------------------------------------------------------------

// 2^k for -1022 <= k <= 0, 0 below (a term of at most 2^(64+k) is then far below rounding)
__device__ __forceinline__ double pow2k(int k) {
  return k < -1022 ? 0.0 : __hiloint2double((k + 1023) << 20, 0);
}

// x[0..V-1] summed over the warp when slot s of lane holds value s ^ mask(lane),
// mask = (lane >> (5 - log2 V)) & (V - 1): the halving exchanges need no selects, and
// every lane ends with the total of value mask(lane)
template <int V>
__device__ __forceinline__ double reduce_perm(double* x) {
#pragma unroll
  for (int n = V, o = 16; n > 1; n >>= 1, o >>= 1) {
#pragma unroll
    for (int i = 0; i < n / 2; ++i) x[i] += __shfl_xor_sync(0xffffffffu, x[i + n / 2], o);
  }
  double r = x[0];
#pragma unroll
  for (int o = 16 / V; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  return r;
}

// split cluster barrier: arrive publishes this thread's earlier shared-memory writes to
// the cluster, wait returns once every thread of the cluster has arrived
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// the cluster's sums of one chunk (cpart slot cp of every CTA, in rank order) phased and
// written to out[b][l_first .. l_first + lc]; CTA `rank` takes every nr-th output
template <typename R2, int MT>
__device__ __forceinline__ void rotate_flush(const RotParams& p, const double* cp, int b,
                                             int l_first, int lc, int m0, int rank) {
  const int L = p.L, NN = 2 * L - 1, nr = p.nr, nt = blockDim.x;
  cg::cluster_group cl = cg::this_cluster();
  const int nout = (lc + 1) * 2 * MT;
  for (int o = rank + nr * (int)threadIdx.x; o < nout; o += nr * nt) {
    const int lco = o / (2 * MT), ci = o % (2 * MT), i = ci >> 1, sg = ci & 1;
    const int m = m0 + i;
    if (m >= L || (m == 0 && sg)) continue;
    const int off = lco * 4 * MT + 4 * i + 2 * sg;
    double re = 0.0, im = 0.0;
#pragma unroll 1
    for (int q0 = 0; q0 < nr; q0 += 4) {  // four remote loads in flight
      double2 t[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        t[q] = q0 + q < nr ? *reinterpret_cast<const double2*>(
                                 cl.map_shared_rank(const_cast<double*>(cp), q0 + q) + off)
                           : make_double2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        re += t[q].x;
        im += t[q].y;
      }
    }
    if (sg && (m & 1)) {  // (-1)^m of the order -m
      re = -re;
      im = -im;
    }
    const int mo = sg ? -m : m;
    const double2 a = p.ea[L - 1 + mo];
    RotIO<R2>::put(p.out, ((size_t)b * L + l_first + lco) * NN + L - 1 + mo,
                   make_double2(re * a.x - im * a.y, re * a.y + im * a.x));
  }
}

// coefficients UVQ[l][m0 + i] of kRotChunk degrees from l0 into uvq[lc][i] (cp.async)
template <int MT>
__device__ __forceinline__ void rotate_stage(const RotParams& p, double4* uvq, int l0, int m0) {
  for (int e = threadIdx.x; e < 2 * kRotChunk * MT; e += blockDim.x) {
    const int h = e & 1, lc = (e >> 1) / MT, i = (e >> 1) % MT, l = l0 + lc;
    const double4* src = p.UVQ + (size_t)min(l, p.L - 1) * p.L + min(m0 + i, p.L - 1);
    cp_async<16>((unsigned)__cvta_generic_to_shared(uvq + lc * MT + i) + 16 * h,
                 reinterpret_cast<const char*>(src) + 16 * h, l < p.L);
  }
}

template <int S>
constexpr int rot_depth() {  // degrees of the per-lane copy pipeline
  return S == 1 ? 4 : S == 2 ? 3 : 2;
}

// One cluster of p.nr CTAs (rank blockIdx.x) owns the orders m0 = MT blockIdx.y ..
// m0 + MT - 1. Dynamic shared memory:
//   ring  [D][S][3][blockDim] 16-byte slots: T[l][|n|], flm[l][n], flm[l][-n] of each lane,
//         copied D - 1 degrees ahead
//   uvq   [2][kRotChunk][MT] double4 coefficients, staged a chunk ahead
//   (contraction) sbuf [kRotChunk][nw][4 MT] per-warp sums, cpart [3][kRotChunk][4 MT]
//         per-CTA sums read by the cluster
// Chunk k's CTA sums are published by a cluster arrive at its end and read after the
// matching wait at the end of chunk k + 1, so CTAs run up to a chunk apart; three cpart
// slots keep a slot unwritten until every CTA has read it.
template <typename R2, int MT, int S, bool PL>
__global__ void __launch_bounds__(kRotThreads, 2) rotate_lrec_kernel(RotParams p) {
  extern __shared__ double4 smem4[];
  constexpr int MG = MT < 4 ? MT : 4;  // orders per reduction group
  constexpr int V = 4 * MG;            // sums per group: +m re, +m im, -m re, -m im per order
  constexpr int LV = V == 8 ? 3 : 4;   // log2 V
  constexpr int D = rot_depth<S>();
  constexpr bool contract = !PL;       // PL: planes only (generate_rotate_dls)
  static_assert(MT % 2 == 0, "tiles start at even orders");
  const int L = p.L, NN = 2 * L - 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nt = blockDim.x;
  const int nw = p.nw, nr = p.nr, rank = blockIdx.x;
  const int m0 = blockIdx.y * MT;
  double* const dl = p.dl_out;
  double2* const ring = reinterpret_cast<double2*>(smem4);
  double4* const uvq = smem4 + (D * S * 3 * nt) / 2;
  double* const sbuf = reinterpret_cast<double*>(uvq + 2 * kRotChunk * MT);
  double* const cpart = sbuf + kRotChunk * nw * 4 * MT;

  // lane permutation of the reduction: slot s of a group holds sum s ^ mask, i.e. state
  // slot is holds order is ^ pm within the group and sum slot c holds component c ^ cm
  const int mask = contract ? (lane >> (5 - LV)) & (V - 1) : 0;
  const int pm = mask >> 2, cm = mask & 3;

  // this lane's n, one per S: the contraction deals n in zigzag order (j -> 0, -1, 1, -2,
  // 2, ...) so that every warp slot holds short and long n alike; the planes take n in
  // natural order (j -> j - (L-1)), so that a warp's stores cover 32 consecutive columns
  int nv[S], an[S], wmin[S], wmax[S];
  double nd[S];
  double2 eph[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int gw = (s * nw + warp) * nr + rank;  // warp slot in the cluster's n order
    const int j = gw * 32 + lane;
    const int n = PL ? j - (L - 1) : (j & 1) ? -((j + 1) >> 1) : (j >> 1);
    const bool ok = j < NN;
    nv[s] = ok ? n : 0;
    nd[s] = (double)nv[s];
    an[s] = ok ? abs(n) : L;  // L: never starts
    if constexpr (PL) {  // least and largest |n| of the warp slot's (valid) n
      const int lo = gw * 32 - (L - 1), hi = min(lo + 31, L - 1);
      wmin[s] = (lo <= 0 && hi >= 0) ? 0 : min(abs(lo), abs(hi));
      wmax[s] = max(abs(lo), abs(hi));
    } else {
      wmin[s] = 16 * gw;
      wmax[s] = 16 * gw + 16;
    }
    eph[s] = ok && contract ? p.eg[L - 1 + n] : make_double2(0.0, 0.0);
  }
  // degrees at which some entry of the warp slot starts: max(m, |n|) over its orders and lanes
  int wlo[S], whi[S], wany = wmin[0];  // wany: least |n| of the warp
#pragma unroll
  for (int s = 0; s < S; ++s) {
    wlo[s] = max(m0, wmin[s]);
    whi[s] = min(L - 1, max(m0 + MT - 1, wmax[s]));
    wany = min(wany, wmin[s]);
  }

  const int nmaps = contract ? p.batch : 1;
  int ck = 0;                          // chunks completed (all maps)
  int pb = 0, plf = 0, plc = 0;        // the pending chunk: map, first degree, last index
#pragma unroll 1
  for (int b = 0; b < nmaps; ++b) {
    // degrees below m0: the tile's rows are zero there
    if constexpr (contract) {
      const int tot = m0 * 2 * MT;
#pragma unroll 1
      for (int e = rank * nt + tid; e < tot; e += nr * nt) {
        const int l = e / (2 * MT), ci = e % (2 * MT), m = m0 + (ci >> 1);
        if (m >= L || (m == 0 && (ci & 1))) continue;
        RotIO<R2>::put(p.out, ((size_t)b * L + l) * NN + L - 1 + ((ci & 1) ? -m : m),
                       make_double2(0.0, 0.0));
      }
    } else {
#pragma unroll 1
      for (int l = 0; l < m0; ++l)
#pragma unroll
        for (int s = 0; s < S; ++s) {
          if (an[s] >= L) continue;
#pragma unroll
          for (int i = 0; i < MT; ++i) {
            const int m = m0 + i;
            if (m >= L) continue;
            dl[((size_t)l * NN + L - 1 + m) * NN + L - 1 + nv[s]] = 0.0;
            if (m > 0) dl[((size_t)l * NN + L - 1 - m) * NN + L - 1 - nv[s]] = 0.0;
          }
        }
    }
    const R2* const fb =
        contract ? reinterpret_cast<const R2*>(p.flm) + (size_t)b * L * NN + L - 1 : nullptr;
    // copies of consecutive degrees ll = m0, m0 + 1, ... into ring stage st (zero where
    // nothing has started); with one n per lane the source pointers advance by one row
    // per call, with more they are recomputed (fewer live registers)
    const unsigned rbase = (unsigned)__cvta_generic_to_shared(ring + tid);
    const double2* tq = p.T + (size_t)m0 * L + min(an[0], L - 1);
    const R2* fq = contract ? fb + (size_t)m0 * NN + nv[0] : nullptr;
    int ll = m0;
    auto issue = [&](int st) {
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const bool vt = ll < L && ll >= wmin[s];
        const unsigned r = rbase + (unsigned)(((st * S + s) * 3) * nt) * 16u;
        const int lt = min(ll, L - 1);
        const double2* ts = S == 1 ? tq : p.T + (size_t)lt * L + min(an[s], L - 1);
        const R2* fs = S == 1 ? fq : fb + (size_t)lt * NN + nv[s];
        cp_async<16>(r, ts, vt);
        if constexpr (contract) {
          const bool vf = vt && an[s] <= ll;
          cp_async<sizeof(R2)>(r + 16u * nt, fs, vf);
          cp_async<sizeof(R2)>(r + 32u * nt, fs - 2 * nv[s], vf);
        }
      }
      if (S == 1 && ll + 1 < L) {
        tq += L;
        if constexpr (contract) fq += NN;
      }
      ++ll;
    };
    rotate_stage<MT>(p, uvq, m0, m0);
    cp_async_commit();
#pragma unroll
    for (int k = 0; k < D - 1; ++k) {
      issue(k);
      cp_async_commit();
    }
    cp_async_wait<D - 1>();  // the coefficients of the first chunk
    __syncthreads();

    double v[MT][S], vp[MT][S];
    int kx[MT][S];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int s = 0; s < S; ++s) {
        v[i][s] = 0.0;
        vp[i][s] = 0.0;
        kx[i][s] = 0;
      }
    // some lane of the warp carries a start value below 2^-960 (kx < 0): warp-uniform
    bool scaled = false;
    int lc = 0, ub = 0, rs = 0;  // degree in chunk, coefficient buffer, ring stage
#pragma unroll 1
    for (int l = m0; l < L; ++l) {
      const bool step = l + 1 < L;
      // copies D - 1 degrees ahead, and the next chunk's coefficients at a chunk start
      issue(rs == 0 ? D - 1 : rs - 1);  // degree l + D - 1
      if (lc == 0 && l + kRotChunk < L)
        rotate_stage<MT>(p, uvq + (ub ^ 1) * kRotChunk * MT, l + kRotChunk, m0);
      cp_async_commit();
      cp_async_wait<D - 1>();  // this degree's copies (this thread's own)
      double2 tn[S], xa[S], xb[S];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const double2* r = ring + ((rs * S + s) * 3) * nt + tid;
        tn[s] = r[0];
        if constexpr (contract) {
          if constexpr (sizeof(R2) == 16) {
            xa[s] = r[nt];
            xb[s] = r[2 * nt];
          } else {
            const float2 fa = *reinterpret_cast<const float2*>(r + nt);
            const float2 fc = *reinterpret_cast<const float2*>(r + 2 * nt);
            xa[s] = make_double2(fa.x, fa.y);
            xb[s] = make_double2(fc.x, fc.y);
          }
        }
      }
      rs = rs == D - 1 ? 0 : rs + 1;
      const double4* const uvl = uvq + (ub * kRotChunk + lc) * MT;

      // entries starting at this degree (only inside the warp slot's start window)
#pragma unroll
      for (int s = 0; s < S; ++s) {
        if (l < wlo[s] || l > whi[s]) continue;
        bool neg = false;
#pragma unroll
        for (int st = 0; st < MT; ++st) {
          const int m = m0 + (st & ~(MG - 1)) + ((st & (MG - 1)) ^ pm);
          if (l == max(m, an[s])) {  // E[l][col] (symmetries of d)
            int col;
            bool flip = false;
            if (m >= an[s]) {
              col = nv[s];
            } else if (nv[s] > 0) {
              col = m;
              flip = ((m - nv[s]) & 1) != 0;
            } else {
              col = -m;
            }
            const RotXD e0 = p.start[(size_t)l * NN + L - 1 + col];
            v[st][s] = flip ? -e0.m : e0.m;
            kx[st][s] = e0.e;
            vp[st][s] = 0.0;
          }
          neg |= kx[st][s] < 0;
        }
        scaled = __any_sync(0xffffffffu, neg) || scaled;
      }
      if constexpr (PL) {  // warp slots not started yet: their entries of the planes are 0
#pragma unroll
        for (int s = 0; s < S; ++s) {
          if (l >= wmin[s] || an[s] >= L) continue;
#pragma unroll
          for (int i = 0; i < MT; ++i) {
            const int m = m0 + i;
            if (m >= L) continue;
            dl[((size_t)l * NN + L - 1 + m) * NN + L - 1 + nv[s]] = 0.0;
            if (m > 0) dl[((size_t)l * NN + L - 1 - m) * NN + L - 1 - nv[s]] = 0.0;
          }
        }
      }

      // the four weights of a lane's n in its sum-slot order:
      // e^{-in gamma} flm[n] (order +m) and (-1)^n e^{in gamma} flm[-n] (order -m, times
      // (-1)^m at the flush)
      double Y[S][4];
      if constexpr (contract) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const double2 g = eph[s], x = xa[s], y = xb[s];
          const double sg = (nv[s] & 1) ? -1.0 : 1.0;
          const double p0 = x.x * g.x - x.y * g.y, p1 = x.x * g.y + x.y * g.x;
          const double q0 = sg * (y.x * g.x + y.y * g.y), q1 = sg * (y.y * g.x - y.x * g.y);
          const double a0 = (cm & 2) ? q0 : p0, a1 = (cm & 2) ? q1 : p1;
          const double b0 = (cm & 2) ? p0 : q0, b1 = (cm & 2) ? p1 : q1;
          Y[s][0] = (cm & 1) ? a1 : a0;
          Y[s][1] = (cm & 1) ? a0 : a1;
          Y[s][2] = (cm & 1) ? b1 : b0;
          Y[s][3] = (cm & 1) ? b0 : b1;
        }
      }

      // one degree of every started entry, branch-free so that the MT x S recurrences
      // interleave; SC: with the 2^kx weights and the renormalisation
      auto advance = [&](auto sc_tag) {
        constexpr bool SC = decltype(sc_tag)::value;
#pragma unroll
        for (int g = 0; g < MT / MG; ++g) {
          double x[V];
#pragma unroll
          for (int u = 0; u < V; ++u) x[u] = 0.0;
#pragma unroll
          for (int is = 0; is < MG; ++is) {
            const int st = g * MG + is;        // state slot
            const int i = g * MG + (is ^ pm);  // order of the slot on this lane
            const double4 uv = uvl[i];
#pragma unroll
            for (int s = 0; s < S; ++s) {
              if (S > 1 && l < wmin[s]) continue;  // warp-uniform
              double dv = v[st][s];
              if constexpr (SC) dv *= pow2k(kx[st][s]);
              if constexpr (contract) {
#pragma unroll
                for (int c = 0; c < 4; ++c) x[4 * is + c] = fma(dv, Y[s][c], x[4 * is + c]);
              } else {
                const int m = m0 + i;
                if (an[s] < L && m < L) {
                  dl[((size_t)l * NN + L - 1 + m) * NN + L - 1 + nv[s]] = dv;
                  if (m > 0)
                    dl[((size_t)l * NN + L - 1 - m) * NN + L - 1 - nv[s]] =
                        ((m - nv[s]) & 1) ? -dv : dv;
                }
              }
              if (step) {
                const double t = fma(uv.z, nd[s], p.cb);
                double vn = (uv.x * tn[s].x) * fma(t, v[st][s], -(uv.y * tn[s].y) * vp[st][s]);
                double vc = v[st][s];
                if constexpr (SC) {  // renormalise by up to 2^64 once |vn| >= 2^65
                  const bool big =
                      kx[st][s] < 0 && (__double2hiint(vn) & 0x7ff00000) > ((1023 + 64) << 20);
                  const int sh = big ? min(64, -kx[st][s]) : 0;
                  const double f = __hiloint2double((1023 - sh) << 20, 0);
                  vn *= f;
                  vc *= f;
                  kx[st][s] += sh;
                }
                vp[st][s] = vc;
                v[st][s] = vn;
              }
            }
          }
          if constexpr (contract) {
            const double r = reduce_perm<V>(x);
            if ((lane & (32 / V - 1)) == 0) sbuf[(lc * nw + warp) * (4 * MT) + g * V + mask] = r;
          }
        }
        if constexpr (SC) {
          bool neg = false;
#pragma unroll
          for (int st = 0; st < MT; ++st)
#pragma unroll
            for (int s = 0; s < S; ++s) neg |= kx[st][s] < 0;
          scaled = __any_sync(0xffffffffu, neg);
        }
      };
      if (l >= wany) {  // some entry of the warp has started (warp-uniform)
        if (scaled)
          advance(std::true_type{});
        else
          advance(std::false_type{});
      } else if constexpr (contract) {
#pragma unroll
        for (int g = 0; g < MT / MG; ++g)
          if ((lane & (32 / V - 1)) == 0) sbuf[(lc * nw + warp) * (4 * MT) + g * V + mask] = 0.0;
      }

      if (lc == kRotChunk - 1 || l == L - 1) {
        __syncthreads();  // sums of the chunk and the next chunk's coefficients in place
        if constexpr (contract) {
          // this CTA's warps summed into cpart slot ck % 3
          double* const cp = cpart + (ck % 3) * kRotChunk * 4 * MT;
          const int nv4 = (lc + 1) * 4 * MT;
          for (int e = tid; e < nv4; e += nt) {
            const double* src = sbuf + (size_t)(e / (4 * MT)) * nw * 4 * MT + e % (4 * MT);
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < kRotThreads / 32; ++w)
              if (w < nw) t += src[w * 4 * MT];
            cp[e] = t;
          }
          __syncthreads();  // sbuf free for the next chunk
          if (ck > 0) {     // the previous chunk: every CTA has published it
            cluster_wait();
            rotate_flush<R2, MT>(p, cpart + ((ck - 1) % 3) * kRotChunk * 4 * MT, pb, plf, plc,
                                 m0, rank);
          }
          cluster_arrive();
          pb = b;
          plf = l - lc;
          plc = lc;
          ++ck;
        }
        ub ^= 1;
        lc = 0;
      } else {
        ++lc;
      }
    }
    cp_async_wait<0>();  // the pipeline's trailing (empty) copies
  }
  if constexpr (contract) {
    if (ck > 0) {
      cluster_wait();
      rotate_flush<R2, MT>(p, cpart + ((ck - 1) % 3) * kRotChunk * 4 * MT, pb, plf, plc, m0, rank);
      cluster_arrive();  // no CTA leaves while others read its sums
      cluster_wait();
    }
  }
}

// FP64 tensor-core step: D (8 x 8) += A (8 x 4) B (4 x 8), lane t holding A[t/4][t%4],
// B[t%4][t/4] and D[t/4][2 (t%4) + {0, 1}] (mma.m8n8k4 .f64 fragments)
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// The contraction on the FP64 tensor cores (one n per fetching lane, 8 orders per tile).
// A warp owns a warp slot of 32 n (fetched as in rotate_lrec_kernel, one per lane) and the
// tile's 8 orders; for the arithmetic lane t takes order m0 + t/4 and the 8 n of positions
// 4j + t%4, j = 0..7, so its 8 recurrences are exactly its A fragments of 8 MMA steps. The
// B fragments are the weights of those n: lane t supplies component t/4 (+m re, +m im,
// -m re, -m im; zero for t/4 >= 4), read from a per-warp table that each lane fills for
// its own n. D[order][component] is the warp's sum over its 32 n, so no shuffle reduction
// runs; lanes with t%4 < 2 park their two components in the same per-warp slots as
// rotate_lrec_kernel, and the cluster reduction is the same.
// Dynamic shared memory: ring [D][3][nt] double2 | uvq [2][kRotChunk][8] double4 |
// ybuf [nw][32][4] double | sbuf [kRotChunk][nw][32] | cpart [3][kRotChunk][32].
template <typename R2>
__global__ void __launch_bounds__(kRotThreads, 2) rotate_mma_kernel(RotParams p) {
  extern __shared__ double4 smem4[];
  constexpr int MT = 8, D = 4;
  const int L = p.L, NN = 2 * L - 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nt = blockDim.x;
  const int nw = p.nw, nr = p.nr, rank = blockIdx.x;
  const int m0 = blockIdx.y * MT;
  double2* const ring = reinterpret_cast<double2*>(smem4);
  double4* const uvq = smem4 + (D * 3 * nt) / 2;
  double* const ybuf = reinterpret_cast<double*>(uvq + 2 * kRotChunk * MT);
  double* const sbuf = ybuf + nw * 32 * 4;
  double* const cpart = sbuf + kRotChunk * nw * 4 * MT;
  double* const yw = ybuf + warp * 32 * 4;

  // the fetching lane's n (zigzag order, as rotate_lrec_kernel)
  const int gw = warp * nr + rank;
  const int wmin = 16 * gw;  // least |n| of the warp slot
  const int jf = gw * 32 + lane;
  const int nf = (jf & 1) ? -((jf + 1) >> 1) : (jf >> 1);
  const bool okf = jf < NN;
  const int nvf = okf ? nf : 0, anf = okf ? abs(nf) : L;
  const double2 eph = okf ? p.eg[L - 1 + nf] : make_double2(0.0, 0.0);
  // the arithmetic lane's order and n
  const int row = lane >> 2, q = lane & 3;
  const int m = m0 + row;
  int nv[8], an[8];
  double nd[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int jj = gw * 32 + 4 * j + q;
    const int n = (jj & 1) ? -((jj + 1) >> 1) : (jj >> 1);
    const bool ok = jj < NN;
    nv[j] = ok ? n : 0;
    an[j] = ok ? abs(n) : L;
    nd[j] = (double)nv[j];
  }
  const int wlo = max(m0, wmin), whi = min(L - 1, max(m0 + MT - 1, wmin + 16));

  int ck = 0, pb = 0, plf = 0, plc = 0;
#pragma unroll 1
  for (int b = 0; b < p.batch; ++b) {
    {  // degrees below m0: the tile's rows are zero there
      const int tot = m0 * 2 * MT;
#pragma unroll 1
      for (int e = rank * nt + tid; e < tot; e += nr * nt) {
        const int l = e / (2 * MT), ci = e % (2 * MT), mm = m0 + (ci >> 1);
        if (mm >= L || (mm == 0 && (ci & 1))) continue;
        RotIO<R2>::put(p.out, ((size_t)b * L + l) * NN + L - 1 + ((ci & 1) ? -mm : mm),
                       make_double2(0.0, 0.0));
      }
    }
    const R2* const fb = reinterpret_cast<const R2*>(p.flm) + (size_t)b * L * NN + L - 1;
    const unsigned rbase = (unsigned)__cvta_generic_to_shared(ring + tid);
    const double2* tq = p.T + (size_t)m0 * L + min(anf, L - 1);
    const R2* fq = fb + (size_t)m0 * NN + nvf;
    int ll = m0;
    auto issue = [&](int st) {  // the fetching lane's operands of degree ll into stage st
      const bool vt = ll < L && ll >= wmin;
      const unsigned r = rbase + (unsigned)(st * 3 * nt) * 16u;
      cp_async<16>(r, tq, vt);
      const bool vf = vt && anf <= ll;
      cp_async<sizeof(R2)>(r + 16u * nt, fq, vf);
      cp_async<sizeof(R2)>(r + 32u * nt, fq - 2 * nvf, vf);
      if (ll + 1 < L) {
        tq += L;
        fq += NN;
      }
      ++ll;
    };
    rotate_stage<MT>(p, uvq, m0, m0);
    cp_async_commit();
#pragma unroll
    for (int k = 0; k < D - 1; ++k) {
      issue(k);
      cp_async_commit();
    }
    cp_async_wait<D - 1>();
    __syncthreads();

    double v[8], vp[8];
    int kx[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      v[j] = 0.0;
      vp[j] = 0.0;
      kx[j] = 0;
    }
    bool scaled = false;  // some lane of the warp carries a start value below 2^-960
    int lc = 0, ub = 0, rs = 0;
#pragma unroll 1
    for (int l = m0; l < L; ++l) {
      const bool step = l + 1 < L;
      __syncwarp();  // every lane is done with the stage the next copies overwrite
      issue(rs == 0 ? D - 1 : rs - 1);  // degree l + D - 1
      if (lc == 0 && l + kRotChunk < L)
        rotate_stage<MT>(p, uvq + (ub ^ 1) * kRotChunk * MT, l + kRotChunk, m0);
      cp_async_commit();
      cp_async_wait<D - 1>();
      __syncwarp();  // the warp's copies of this degree are visible to all its lanes
      const double2* const rg = ring + rs * 3 * nt + warp * 32;  // T of the warp's n
      const int rso = rs;
      rs = rs == D - 1 ? 0 : rs + 1;
      double* const slot = sbuf + (lc * nw + warp) * (4 * MT);
      if (l >= wmin) {  // some entry of the warp has started (warp-uniform)
        {  // the weights of the fetching lane's n: e^{-in gamma} flm[n], (-1)^n e^{in gamma} flm[-n]
          double2 xa, xb;
          const double2* r = ring + rso * 3 * nt + tid;
          if constexpr (sizeof(R2) == 16) {
            xa = r[nt];
            xb = r[2 * nt];
          } else {
            const float2 fa = *reinterpret_cast<const float2*>(r + nt);
            const float2 fc = *reinterpret_cast<const float2*>(r + 2 * nt);
            xa = make_double2(fa.x, fa.y);
            xb = make_double2(fc.x, fc.y);
          }
          const double sg = (nvf & 1) ? -1.0 : 1.0;
          double4 y;
          y.x = xa.x * eph.x - xa.y * eph.y;
          y.y = xa.x * eph.y + xa.y * eph.x;
          y.z = sg * (xb.x * eph.x + xb.y * eph.y);
          y.w = sg * (xb.y * eph.x - xb.x * eph.y);
          reinterpret_cast<double4*>(yw)[lane] = y;
        }
        // entries starting at this degree (only inside the warp slot's start window)
        if (l >= wlo && l <= whi) {
          bool neg = false;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (l == max(m, an[j])) {  // E[l][col] (symmetries of d)
              int col;
              bool flip = false;
              if (m >= an[j]) {
                col = nv[j];
              } else if (nv[j] > 0) {
                col = m;
                flip = ((m - nv[j]) & 1) != 0;
              } else {
                col = -m;
              }
              const RotXD e0 = p.start[(size_t)l * NN + L - 1 + col];
              v[j] = flip ? -e0.m : e0.m;
              kx[j] = e0.e;
              vp[j] = 0.0;
            }
            neg |= kx[j] < 0;
          }
          scaled = __any_sync(0xffffffffu, neg) || scaled;
        }
        __syncwarp();  // the weight table is written
        const double4 uv = uvq[(ub * kRotChunk + lc) * MT + row];
        auto advance = [&](auto sc_tag) {
          constexpr bool SC = decltype(sc_tag)::value;
          double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;  // two accumulators: even, odd j
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int k = 4 * j + q;
            const double2 tk = rg[k];
            const double y = row < 4 ? yw[k * 4 + row] : 0.0;
            double dv = v[j];
            if constexpr (SC) dv *= pow2k(kx[j]);
            if (j & 1)
              dmma_884(e0, e1, dv, y);
            else
              dmma_884(d0, d1, dv, y);
            if (step) {
              const double t = fma(uv.z, nd[j], p.cb);
              double vn = (uv.x * tk.x) * fma(t, v[j], -(uv.y * tk.y) * vp[j]);
              double vc = v[j];
              if constexpr (SC) {  // renormalise by up to 2^64 once |vn| >= 2^65
                const bool big =
                    kx[j] < 0 && (__double2hiint(vn) & 0x7ff00000) > ((1023 + 64) << 20);
                const int sh = big ? min(64, -kx[j]) : 0;
                const double f = __hiloint2double((1023 - sh) << 20, 0);
                vn *= f;
                vc *= f;
                kx[j] += sh;
              }
              vp[j] = vc;
              v[j] = vn;
            }
          }
          if (q < 2)
            reinterpret_cast<double2*>(slot)[2 * row + q] = make_double2(d0 + e0, d1 + e1);
          if constexpr (SC) {
            bool neg = false;
#pragma unroll
            for (int j = 0; j < 8; ++j) neg |= kx[j] < 0;
            scaled = __any_sync(0xffffffffu, neg);
          }
        };
        if (scaled)
          advance(std::true_type{});
        else
          advance(std::false_type{});
      } else if (q < 2) {
        reinterpret_cast<double2*>(slot)[2 * row + q] = make_double2(0.0, 0.0);
      }

      if (lc == kRotChunk - 1 || l == L - 1) {
        __syncthreads();  // sums of the chunk and the next chunk's coefficients in place
        double* const cp = cpart + (ck % 3) * kRotChunk * 4 * MT;
        const int nv4 = (lc + 1) * 4 * MT;
        for (int e = tid; e < nv4; e += nt) {
          const double* src = sbuf + (size_t)(e / (4 * MT)) * nw * 4 * MT + e % (4 * MT);
          double t = 0.0;
#pragma unroll
          for (int w = 0; w < kRotThreads / 32; ++w)
            if (w < nw) t += src[w * 4 * MT];
          cp[e] = t;
        }
        __syncthreads();  // sbuf free for the next chunk
        if (ck > 0) {     // the previous chunk: every CTA has published it
          cluster_wait();
          rotate_flush<R2, MT>(p, cpart + ((ck - 1) % 3) * kRotChunk * 4 * MT, pb, plf, plc, m0,
                               rank);
        }
        cluster_arrive();
        pb = b;
        plf = l - lc;
        plc = lc;
        ++ck;
        ub ^= 1;
        lc = 0;
      } else {
        ++lc;
      }
    }
    cp_async_wait<0>();
  }
  if (ck > 0) {
    cluster_wait();
    rotate_flush<R2, MT>(p, cpart + ((ck - 1) % 3) * kRotChunk * 4 * MT, pb, plf, plc, m0, rank);
    cluster_arrive();  // no CTA leaves while others read its sums
    cluster_wait();
  }
}

// rotation with caller-supplied planes dl[l][L-1+m][L-1+n]: one warp per (map, l, m)
template <typename R2>
__global__ void rotate_planes_kernel(RotParams p) {
  const int L = p.L, W = 2 * L - 1, lane = threadIdx.x & 31;
  const long rows = (long)p.batch * L * W;
  const long nwarps = (long)gridDim.x * blockDim.x / 32;
  for (long e = (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32; e < rows; e += nwarps) {
    const int col = (int)(e % W), l = (int)((e / W) % L), b = (int)(e / ((long)W * L));
    const int m = col - (L - 1);
    const size_t row = ((size_t)b * L + l) * W;
    if (m < -l || m > l) {
      if (lane == 0) RotIO<R2>::put(p.out, row + col, make_double2(0.0, 0.0));
      continue;
    }
    const double* P = p.dl_in + ((size_t)l * W + col) * W;  // row m of degree l
    double re = 0.0, im = 0.0;
    for (int n = -l + lane; n <= l; n += 32) {
      const double2 x = RotIO<R2>::get(p.flm, row + L - 1 + n);
      const double2 g = p.eg[L - 1 + n];
      const double d = __ldg(P + L - 1 + n);
      re += d * (x.x * g.x - x.y * g.y);
      im += d * (x.x * g.y + x.y * g.x);
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if (lane == 0) {
      const double2 a = p.ea[L - 1 + m];
      RotIO<R2>::put(p.out, row + col, make_double2(re * a.x - im * a.y, re * a.y + im * a.x));
    }
  }
}

struct RotShape {
  int mt, s, nw, nr;
};

// S n per lane so that a cluster of at most kRotMaxCluster CTAs of 8 warps covers all
// 2L-1 n; MT (orders per cluster) as large as keeps two CTAs per SM busy, with MT x S
// = 8 recurrences per lane at most (16 for L > 4096)
RotShape rotate_shape(int L, int sms) {
  const int NN = 2 * L - 1, slots = (NN + 31) / 32, wmax = kRotThreads / 32;
  RotShape r;
  r.s = 1;
  while ((slots + r.s - 1) / r.s > kRotMaxCluster * wmax) r.s *= 2;
  const int ws = (slots + r.s - 1) / r.s;
  r.nw = ws < wmax ? ws : wmax;
  r.nr = (ws + r.nw - 1) / r.nw;
  if (r.s == 1) {
    r.mt = 8;
    while (r.mt > 2 && (long)r.nr * ((L + r.mt - 1) / r.mt) < 2L * sms) r.mt >>= 1;
    // four orders per tile: CTAs of 4 warps in twice the clusters (L = 512: 0.60 -> 0.55 ms)
    if (r.mt == 4 && r.nw == wmax && 2 * r.nr <= kRotMaxCluster) {
      r.nw /= 2;
      r.nr *= 2;
    }
  } else {
    r.mt = r.s == 2 ? 4 : 2;
  }
  return r;
}

template <typename R2, int MT, int S, bool PL>
cudaError_t launch_lrec(const RotParams& p, cudaStream_t s) {
  // ring, uvq, and with the contraction sbuf and cpart (rotate_lrec_kernel)
  const size_t nt = 32 * (size_t)p.nw;
  const size_t smem = (size_t)rot_depth<S>() * S * 3 * nt * 16 + 2 * kRotChunk * MT * 32 +
                      (!PL ? ((size_t)kRotChunk * p.nw * 4 * MT + 3 * kRotChunk * 4 * MT) * 8 : 0);
  void (*kern)(RotParams) = rotate_lrec_kernel<R2, MT, S, PL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)p.nr, (unsigned)((p.L + MT - 1) / MT), 1);
  cfg.blockDim = dim3((unsigned)(32 * p.nw), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)p.nr;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, p);
}

template <typename R2>
cudaError_t launch_mma(const RotParams& p, cudaStream_t s) {
  constexpr int MT = 8;
  // ring, uvq, ybuf, sbuf and cpart (rotate_mma_kernel)
  const size_t nt = 32 * (size_t)p.nw;
  const size_t smem = (size_t)4 * 3 * nt * 16 + 2 * kRotChunk * MT * 32 +
                      ((size_t)p.nw * 32 * 4 + (size_t)kRotChunk * p.nw * 4 * MT +
                       3 * kRotChunk * 4 * MT) * 8;
  void (*kern)(RotParams) = rotate_mma_kernel<R2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)p.nr, (unsigned)((p.L + MT - 1) / MT), 1);
  cfg.blockDim = dim3((unsigned)(32 * p.nw), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)p.nr;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (p.nr > kRotMaxCluster) {  // non-portable cluster size: launch only where one fits
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    int nclusters = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg);
    if (e != cudaSuccess || nclusters < 1) {
      (void)cudaGetLastError();
      return cudaErrorNotSupported;
    }
  }
  return cudaLaunchKernelEx(&cfg, kern, p);
}

template <typename R2, bool PL>
cudaError_t launch_shape(const RotParams& p, const RotShape& sh, cudaStream_t s) {
  switch (sh.s * 16 + sh.mt) {
    case 16 + 8: return launch_lrec<R2, 8, 1, PL>(p, s);
    case 16 + 4: return launch_lrec<R2, 4, 1, PL>(p, s);
    case 16 + 2: return launch_lrec<R2, 2, 1, PL>(p, s);
    case 32 + 4: return launch_lrec<R2, 4, 2, PL>(p, s);
    case 64 + 2: return launch_lrec<R2, 2, 4, PL>(p, s);
    case 128 + 2: return launch_lrec<R2, 2, 8, PL>(p, s);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R2>
cudaError_t rotate_launch(RotParams p, cudaStream_t s) {
  const int L = p.L, NN = 2 * L - 1;
  const double c = std::cos(0.5 * p.beta), sn = std::sin(0.5 * p.beta);
  p.cb = std::cos(p.beta);
  p.c2 = c * c;
  p.s2 = sn * sn;
  p.cs2 = (c * sn) * (c * sn);
  p.c_neg = c < 0.0;
  p.s_neg = sn < 0.0;
  rotate_phase_kernel<<<(NN + 255) / 256, 256, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (p.dl_in) {
    const long warps = (long)p.batch * L * NN;
    long blocks = (warps + 7) / 8;
    if (blocks > 65535L * 16) blocks = 65535L * 16;
    rotate_planes_kernel<R2><<<(unsigned)blocks, 256, 0, s>>>(p);
    return cudaGetLastError();
  }
  int dev = 0, sms = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const RotShape sh = rotate_shape(L, sms);
  p.nw = sh.nw;
  p.nr = sh.nr;
  const long nco = ((long)L * L + 255) / 256;
  rotate_coef_kernel<<<(unsigned)(nco < 8192 ? nco : 8192), 256, 0, s>>>(p);
  const int G = (L + kRotSeg - 1) / kRotSeg, nb = (NN + 127) / 128;
  rotate_start_seg_kernel<<<dim3(nb, G), 128, 0, s>>>(p);
  rotate_start_carry_kernel<<<nb, 128, 0, s>>>(p);
  rotate_start_final_kernel<<<dim3(nb, L), 128, 0, s>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (p.flm) {
    const int slots = (NN + 31) / 32, wmax = kRotThreads / 32;
    if (sh.s == 2 && slots <= 2 * kRotMaxCluster * wmax) {
      // up to 4096 n (L <= 2048): the tensor-core kernel with one n per lane in clusters of
      // up to 16 CTAs, where the device has them; else two n per lane below
      RotParams q = p;
      q.nw = wmax;
      q.nr = (slots + wmax - 1) / wmax;
      e = launch_mma<R2>(q, s);
      if (e != cudaErrorNotSupported) return e;
    }
    if (sh.s == 1 && sh.mt == 8) return launch_mma<R2>(p, s);
  }
  return p.flm ? launch_shape<R2, false>(p, sh, s) : launch_shape<double2, true>(p, sh, s);
}

}  // namespace

static size_t rot_align(size_t b) { return (b + 255) & ~(size_t)255; }

size_t rotate_workspace_bytes(int L) {
  const size_t NN = 2 * (size_t)L - 1, G = ((size_t)L + kRotSeg - 1) / kRotSeg;
  return rot_align((size_t)L * L * sizeof(double2)) + rot_align((size_t)L * L * sizeof(double4)) +
         rot_align((size_t)L * NN * sizeof(RotXD)) + rot_align(G * NN * sizeof(RotXD)) +
         2 * rot_align(NN * sizeof(double2));
}

void rotate_bind_workspace(RotParams& p, void* ws) {
  char* c = static_cast<char*>(ws);
  const size_t L = (size_t)p.L, NN = 2 * L - 1, G = (L + kRotSeg - 1) / kRotSeg;
  p.T = reinterpret_cast<double2*>(c);
  c += rot_align(L * L * sizeof(double2));
  p.UVQ = reinterpret_cast<double4*>(c);
  c += rot_align(L * L * sizeof(double4));
  p.start = reinterpret_cast<RotXD*>(c);
  c += rot_align(L * NN * sizeof(RotXD));
  p.carry = reinterpret_cast<RotXD*>(c);
  c += rot_align(G * NN * sizeof(RotXD));
  p.ea = reinterpret_cast<double2*>(c);
  c += rot_align(NN * sizeof(double2));
  p.eg = reinterpret_cast<double2*>(c);
}

cudaError_t launch_rotate(bool fp64, RotParams p, cudaStream_t s) {
  return fp64 ? rotate_launch<double2>(p, s) : rotate_launch<float2>(p, s);
}

}  // namespace s2b

// ----------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------
extern "C" {

size_t s2b_rotate_workspace_size(int L) { return L >= 1 ? s2b::rotate_workspace_bytes(L) : 0; }

int s2b_rotate_flms(int L, int batch, int precision, double alpha, double beta, double gamma,
                    const void* flm, void* out, const double* dl, void* ws, size_t ws_bytes,
                    void* stream) {
  if (L < 1 || batch < 1 || !flm || !out || !ws)
    return s2b::set_last_error(S2B_ERR_INVALID, "rotate: L >= 1, batch >= 1 and non-NULL buffers");
  if (!dl && L > s2b::kRotMaxL)
    return s2b::set_last_error(S2B_ERR_INVALID, "rotate: L <= 8192 unless the planes are given");
  if (flm == out)
    return s2b::set_last_error(S2B_ERR_INVALID, "rotate: out must not alias flm");
  if (precision != S2B_F64 && precision != S2B_F32)
    return s2b::set_last_error(S2B_ERR_INVALID, "rotate: precision must be S2B_F64 or S2B_F32");
  if (ws_bytes < s2b::rotate_workspace_bytes(L))
    return s2b::set_last_error(S2B_ERR_WORKSPACE, "rotate: workspace too small");
  s2b::RotParams p{};
  p.L = L;
  p.batch = batch;
  p.alpha = alpha;
  p.beta = beta;
  p.gamma = gamma;
  p.flm = flm;
  p.out = out;
  p.dl_in = dl;
  s2b::rotate_bind_workspace(p, ws);
  const cudaError_t e =
      s2b::launch_rotate(precision == S2B_F64, p, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return s2b::set_last_error(S2B_ERR_CUDA, cudaGetErrorString(e));
  return S2B_OK;
}

int s2b_rotate_dls(int L, double beta, double* dl, void* ws, size_t ws_bytes, void* stream) {
  if (L < 1 || !dl || !ws)
    return s2b::set_last_error(S2B_ERR_INVALID, "rotate_dls: L >= 1 and non-NULL buffers");
  if (L > s2b::kRotMaxL)
    return s2b::set_last_error(S2B_ERR_INVALID, "rotate_dls: L <= 8192");
  if (ws_bytes < s2b::rotate_workspace_bytes(L))
    return s2b::set_last_error(S2B_ERR_WORKSPACE, "rotate_dls: workspace too small");
  s2b::RotParams p{};
  p.L = L;
  p.batch = 0;
  p.beta = beta;
  p.dl_out = dl;
  s2b::rotate_bind_workspace(p, ws);
  const cudaError_t e = s2b::launch_rotate(true, p, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return s2b::set_last_error(S2B_ERR_CUDA, cudaGetErrorString(e));
  return S2B_OK;
}

}  // extern "C"
