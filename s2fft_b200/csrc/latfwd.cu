// Forward latitudinal step (projection of weighted ring spectra onto flm),
// restart formulation of the Price-McEwen m-recursion.
//
// Same recursion and projection as upstream s2fft
// (s2fft/transforms/otf_recursions.py:432-588, forward_latitudinal_step;
// coefficients s2fft/recursions/price_mcewen.py:118-255): for every (theta, l)
// the values d^l_{m,n}(theta), n = -spin, are generated from m = l towards
// m = 0 and flm[l, m] accumulates d * G(theta, m) over the rings.
//
// B200 formulation (own design):
//  * A state (theta, l) is only started where d first becomes significant
//    (|d| >= 2^floor going down from m = l). The start values are computed
//    once per plan in double (fwd_start_kernel); the transform itself then runs
//    the monic recursion dt_{m-1} = lambda_m h_{l,m} dt_m - dt_{m+1} in the plan
//    precision with no exponent bookkeeping, no gating multiply and no
//    renormalisation: once significant, |dt| stays within [2^-110, 2^10].
//  * Starts are taken per (ring, block of 32 consecutive l) at the largest first
//    significant m of the block, rounded up to a group start (m = -1 mod R), so a
//    whole warp starts a ring together. Degrees of the block below that start
//    begin with the exact continuation of the recursion above m = l
//    (h_{l,m} = 0 for m > l gives dt_{l+2j} = (-1)^j dt_l, dt_{l+2j+1} = 0).
//  * CTA tile: W warps x T rings (rings shared by the lanes of a warp, so the
//    spectra and lambda loads are shared-memory broadcasts) x two l blocks
//    (lane = l within the block, blocks p and NB-1-p for balance). The sum over
//    the T rings of a thread stays in registers; warps' partial sums meet in
//    shared memory every R steps and are added to flm with vector atomics.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "s2b_dev.h"
#include "s2b_latfwd.h"

namespace s2b {

// ---------------------------------------------------------------------------
// Start table. One warp per (half, block, ring); lane = degree within the block.
// Double arithmetic with a running power-of-two exponent (value = v * 2^E).
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void fwd_start_kernel(const FwdStartParams p) {
  using R2 = typename Vec<Real>::t2;
  const int lane = threadIdx.x & 31;
  const long wid = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const long nw = (long)p.nhalf * p.NB * p.nrings;
  if (wid >= nw) return;  // uniform per warp
  const int r = (int)(wid % p.nrings);
  const int blk = (int)((wid / p.nrings) % p.NB);
  const int half = (int)(wid / ((long)p.nrings * p.NB));
  const int n = half == 0 ? -p.spin : p.spin;
  const int an = n < 0 ? -n : n;
  const int L = p.L;
  const int l = blk * kFwdBlock + lane;
  const bool valid = l < L && l >= p.L0 && l >= an;
  const RingInfo ri = p.rings[r];
  const int fl = (int)p.floor_log2;

  double lg = 0.0;
  if (valid) lg = p.lbin[l] + (double)(l + n) * ri.lc + (double)(l - n) * ri.ls;
  const double sgn = ((l - n) & 1) ? -1.0 : 1.0;

  // one step of the monic recursion at m: (v, w) = (dt_m, dt_{m+1}) -> (dt_{m-1}, dt_m)
  auto step = [&](double& v, double& w, int& E, int m) {
    const double lam = fma(-(double)m, ri.B, (double)n * ri.A);
    double h = 1.0;
    if (m < l) {
      const double f = sqrt((double)(l + m + 1) * (double)(l - m));
      h = p.g[(size_t)m * L + l] / (f * p.g[(size_t)(m + 1) * L + l]);
    }
    const double nv = lam * h * v - w;
    w = v;
    v = nv;
    if (fabs(v) > 0x1p200) {
      v *= 0x1p-200;
      w *= 0x1p-200;
      E += 200;
    }
  };

  // pass 1: first m (going down from l) with |d_m| = |dt_m| g_{l,m} >= 2^fl
  int ms = -1;
  if (valid) {
    int E = (int)floor(lg);
    double v = sgn * exp2(lg - (double)E), w = 0.0;
    for (int m = l; m >= 0; --m) {
      if (fabs(v) * p.g[(size_t)m * L + l] >= ldexp(1.0, fl - E)) {
        ms = m;
        break;
      }
      if (m == 0) break;
      step(v, w, E, m);
    }
  }
  // pass 2: common start of the block on this ring, aligned to a group start
  int M = __reduce_max_sync(0xffffffffu, ms);
  if (M >= 0) M |= p.group - 1;

  // pass 3: (dt_X, dt_{X+1}) of this degree at the start X = M and, for the inverse kernel's
  // m-split, at the restarts X = b - 1 of the boundaries b <= M; the points are requested in
  // decreasing order, so one walk down from m = l serves them all (starts at or above l
  // take the exact continuation above m = l)
  int E3 = 0, mc = l;
  double v3 = 0.0, w3 = 0.0;
  if (valid) {
    E3 = (int)floor(lg);
    v3 = sgn * exp2(lg - (double)E3);
  }
  auto start_pair = [&](int X, double& cur, double& prv) {
    cur = 0.0;
    prv = 0.0;
    if (!valid || X < 0) return;
    if (X >= l) {
      const double dl = sgn * exp2(lg);
      const int dlt = X - l;
      if ((dlt & 1) == 0)
        cur = ((dlt >> 1) & 1) ? -dl : dl;
      else
        prv = (((dlt + 1) >> 1) & 1) ? -dl : dl;
      return;
    }
    while (mc > X) {
      step(v3, w3, E3, mc);
      --mc;
    }
    cur = ldexp(v3, E3);
    prv = ldexp(w3, E3);
  };
  double cur = 0.0, prv = 0.0;
  start_pair(M, cur, prv);
  R2 o;
  o.x = (Real)cur;
  o.y = (Real)prv;
  reinterpret_cast<R2*>(p.Vst)[wid * kFwdBlock + lane] = o;
  if (lane == 0) p.Mst[wid] = M;
  if (p.Mst1) {
    // restart tables of the m-split, one per inner boundary (boundaries decrease with k)
    const int q = blk < p.NB - 1 - blk ? blk : p.NB - 1 - blk;
    const size_t nst = (size_t)p.nhalf * p.NB * p.nrings;
    for (int k = 1; k < kInvSegMax; ++k) {
      const int bk = inv_mbound(L, p.NB, q, k);
      int Mk = M;
      double ck = cur, pk = prv;
      if (M >= bk) {
        Mk = bk > 0 ? bk - 1 : -1;
        start_pair(Mk, ck, pk);
      }
      R2 ok;
      ok.x = (Real)ck;
      ok.y = (Real)pk;
      reinterpret_cast<R2*>(p.Vst1)[((k - 1) * nst + wid) * kFwdBlock + lane] = ok;
      if (lane == 0) p.Mst1[(k - 1) * nst + wid] = Mk;
    }
  }
}

size_t fwd_start_bytes(bool fp64, int L, int nhalf, int nrings) {
  return (size_t)nhalf * fwd_nblocks(L) * nrings * kFwdBlock * 2 * (fp64 ? 8 : 4);
}

cudaError_t launch_fwd_start(bool fp64, const FwdStartParams& p, cudaStream_t s) {
  const long warps = (long)p.nhalf * p.NB * p.nrings;
  const int threads = 128;
  const long blocks = (warps * 32 + threads - 1) / threads;
  if (blocks > 0x7fffffffL) return cudaErrorInvalidValue;
  if (fp64)
    fwd_start_kernel<double><<<(unsigned)blocks, threads, 0, s>>>(p);
  else
    fwd_start_kernel<float><<<(unsigned)blocks, threads, 0, s>>>(p);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Main kernel
// ---------------------------------------------------------------------------
// SYM: 0 one recursion per ring; 1 spin-0 ring pairs; 2 spin != 0 ring pairs (cross: the
// partial sums carry this half's projection and the other half's mirrored one)
template <typename Real, bool DUAL, int T, int W, int R, int SYM>
struct Fwd2Layout {
  using Acc = std::conditional_t<DUAL || SYM == 2, typename Vec<Real>::t4, typename Vec<Real>::t2>;
  static constexpr int NRT = W * T;  // rings per CTA
  static constexpr int NT = W * 32;
  // stage: h rows [2 blocks][R][32] | spectra rows [R][NRT] | lambda rows [R][NRT]
  static constexpr size_t h_bytes = 2 * R * kFwdBlock * sizeof(Real);
  static constexpr int GM = SYM ? 2 : 1;  // spectra per ring: G, or (E, O) of a ring pair
  static constexpr size_t g_bytes = (size_t)R * NRT * GM * sizeof(Acc);
  static constexpr size_t l_bytes = (size_t)R * NRT * sizeof(Real);
  static constexpr size_t stage_bytes = h_bytes + g_bytes + l_bytes;
  // partial sums [R][W][2][32], twice: a group's reduction and the next group's steps use
  // different halves, so one barrier per group separates them
  // (once when two copies would leave room for fewer than 3 CTAs per SM: then a second
  // barrier per group)
  static constexpr int buf_elems = R * W * 2 * kFwdBlock;
  static constexpr size_t act_bytes = (size_t)W * 2 * T * sizeof(int);
  static constexpr size_t fixed_bytes = 2 * stage_bytes + act_bytes + 16 + 16;
  static constexpr int NBUF =
      3 * (fixed_bytes + 2 * buf_elems * sizeof(Acc) + 1024) <= 228 * 1024 ? 2 : 1;
  static constexpr size_t buf_bytes = (size_t)NBUF * buf_elems * sizeof(Acc);
  static constexpr size_t total = fixed_bytes + buf_bytes;
  static_assert(stage_bytes % 16 == 0 && buf_bytes % 16 == 0 && act_bytes % 16 == 0, "align");
  static_assert((2 * T) % 32 == 0 || 2 * T < 32, "act entries are spread over the lanes");
};

// One recursion step over the T rings of one slot: cur = dt_m, prv = dt_{m+1} -> dt_{m-1};
// a += dt_m G(theta_i, m) over the rings (float: measured faster than the paired form
// below, which trades shared-memory loads for registers).
template <typename Real, typename Acc, int T, int GS>
__device__ __forceinline__ void fwd_slot_step(Real (&cur)[T], Real (&prv)[T], Real h,
                                              const Real* __restrict__ lrow,
                                              const Acc* __restrict__ grow, Acc& a) {
#pragma unroll
  for (int i = 0; i < T; ++i) {
    const Real x = cur[i];
    acc_fma(a, x, grow[GS * i]);
    prv[i] = fma(lrow[i] * h, x, -prv[i]);
  }
}

// One recursion step over the T rings for both slots (K0 / K1: the slot is active;
// double: 6 % faster than two slot steps at L = 1024):
// cur = dt_m, prv = dt_{m+1} -> dt_{m-1}; a_k += dt_m G(theta_i, m) over the rings. The
// spectrum and lambda of a ring are loaded once for both slots (they do not depend on the
// degree), lambda as 16-byte vectors.
template <typename Real, typename Acc, int T, int GS, bool K0, bool K1>
__device__ __forceinline__ void fwd_pair_step(Real (&c0)[T], Real (&p0)[T], Real (&c1)[T],
                                              Real (&p1)[T], Real h0, Real h1,
                                              const Real* __restrict__ lrow,
                                              const Acc* __restrict__ grow, Acc& a0, Acc& a1) {
  constexpr int VL = 16 / (int)sizeof(Real);  // lambdas per vector load
  static_assert(T % VL == 0, "rings per warp must fill whole lambda vectors");
  using LV = std::conditional_t<sizeof(Real) == 4, float4, double2>;
#pragma unroll
  for (int i0 = 0; i0 < T; i0 += VL) {
    const LV lv = *reinterpret_cast<const LV*>(lrow + i0);
    Real lam[VL];
    if constexpr (VL == 4) {
      lam[0] = lv.x;
      lam[1] = lv.y;
      lam[2] = lv.z;
      lam[3] = lv.w;
    } else {
      lam[0] = lv.x;
      lam[1] = lv.y;
    }
#pragma unroll
    for (int j = 0; j < VL; ++j) {
      const int i = i0 + j;
      const Acc g = grow[GS * i];
      if constexpr (K0) {
        const Real x = c0[i];
        acc_fma(a0, x, g);
        p0[i] = fma(lam[j] * h0, x, -p0[i]);
      }
      if constexpr (K1) {
        const Real x = c1[i];
        acc_fma(a1, x, g);
        p1[i] = fma(lam[j] * h1, x, -p1[i]);
      }
    }
  }
}

// 3 CTAs per SM: the shared-memory footprint (two stages + partial sums) allows no more
// One tile of the forward kernel: ring tile bx, block pair and segment by, (half, map) bz.
// Returns false when a bounded wait ran out (the plan's status word is set). live: the
// CTA's mbarriers were initialised by an earlier tile (persistent launches) and are
// invalidated before they are set up again.
template <typename Real, bool DUAL, int T, int W, int R, int SYM>
__device__ __forceinline__ bool lat_fwd2_tile(const Fwd2Params& p, int bx, int by, int bz,
                                              unsigned char* smem_raw, bool& live) {
  using Lay = Fwd2Layout<Real, DUAL, T, W, R, SYM>;
  constexpr int GM = Lay::GM;
  using Acc = typename Lay::Acc;
  using R2 = typename Vec<Real>::t2;
  constexpr int NRT = Lay::NRT;
  constexpr int NT = Lay::NT;
  static_assert(R == 4 || R == 8, "the group body below is written for R = 4 or 8");
  constexpr int U = (2 * T + 31) / 32;  // act entries per lane: entry e = lane + 32 u -> (k, i) = (e / T, e % T)
  unsigned char* stage_base = smem_raw;
  Acc* const bufs = reinterpret_cast<Acc*>(smem_raw + 2 * Lay::stage_bytes);
  int* act = reinterpret_cast<int*>(smem_raw + 2 * Lay::stage_bytes + Lay::buf_bytes);
  int* mk = act + W * 2 * T;  // CTA-wide first m per slot (2 ints)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(mk) + 16);

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wp = tid >> 5;
  const int L = p.L;
  const int NB = p.NB;
  const int TR = tab_rows(L);
  const int Lp = NB * kFwdBlock;
  // ring tiles from the equator outwards: the largest tiles are scheduled first
  const int ntiles = (p.nrings + NRT - 1) / NRT;
  const int mid = ntiles >> 1;
  const int t = bx;
  // (symmetric mode: the rings run from the pole to the equator, so the largest tiles last)
  const int tile = SYM ? ntiles - 1 - t : ((t & 1) ? mid - 1 - (t >> 1) : mid + (t >> 1));
  const int RS = p.tab_stride ? p.tab_stride : p.nrings;  // ring stride of the start tables
  const int r0 = tile * NRT;
  // by = block pair + NB/2 * segment along m (boundaries of inv_mbound)
  const int npair = NB / 2;
  const int q = by % npair, seg = by / npair;
  const int kb0 = q, kb1 = NB - 1 - q;
  const int nseg = p.Mst1 ? p.nseg : 1;
  const int gstep = kInvSegMax / nseg, g0 = seg * gstep;
  const int half = (int)(bz % p.nhalf);
  const int b = (int)(bz / p.nhalf);

  const size_t nst = (size_t)p.nhalf * NB * RS;  // entries of one start table
  const int* __restrict__ Mtab = g0 ? p.Mst1 + (size_t)(g0 - 1) * nst : p.Mst;

  // start m of every (slot, ring) of this warp: lane < 2T holds (k, i) = (lane / T, lane % T)
  int a_m[U];
  int mt0 = -1, mt1 = -1;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int e = lane + 32 * u;
    a_m[u] = -1;
    if (e < 2 * T) {
      const int k = e / T, i = e % T;
      const int r = r0 + wp * T + i;
      if (r < p.nrings) a_m[u] = Mtab[((size_t)half * NB + (k ? kb1 : kb0)) * RS + r];
      act[(wp * 2 + k) * T + i] = a_m[u];
    }
    mt0 = max(mt0, __reduce_max_sync(0xffffffffu, (e < T) ? a_m[u] : -1));
    mt1 = max(mt1, __reduce_max_sync(0xffffffffu, (e >= T && e < 2 * T) ? a_m[u] : -1));
  }
  if (tid == 0) {
    mk[0] = -1;
    mk[1] = -1;
  }
  // zero both stages once: columns beyond a copy's extent then read as zeros
  for (size_t x = tid * 16; x < 2 * Lay::stage_bytes; x += (size_t)NT * 16)
    *reinterpret_cast<uint4*>(stage_base + x) = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (lane == 0) {
    atomicMax(&mk[0], mt0);
    atomicMax(&mk[1], mt1);
  }
  if (tid == 0) {
    if (live) {
      mbar_inval(&mbar[0]);
      mbar_inval(&mbar[1]);
    }
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  live = true;
  __syncthreads();
  const int mc0 = mk[0], mc1 = mk[1];
  const int mtop = mc0 > mc1 ? mc0 : mc1;
  const int mbot = inv_mbound(L, NB, q, g0 + gstep);  // lowest m of the segment
  if (mtop < mbot) return true;  // nothing significant in this tile and segment (uniform)
  const int ngroups = (mtop + 1 - mbot) / R;  // mtop = -1 mod 8, mbot = 0 mod 8

  const Real* __restrict__ Hb = reinterpret_cast<const Real*>(p.Hb);
  const Acc* __restrict__ Gin =
      reinterpret_cast<const Acc*>(p.G) + ((size_t)b * p.nhalf + half) * TR * p.Gs * GM;
  const Real* __restrict__ lamh = reinterpret_cast<const Real*>(p.lam) + (size_t)half * TR * p.Ls;
  const R2* __restrict__ Vst =
      g0 ? reinterpret_cast<const R2*>(p.Vst1) + (size_t)(g0 - 1) * nst * kFwdBlock
         : reinterpret_cast<const R2*>(p.Vst);
  Acc* __restrict__ out = reinterpret_cast<Acc*>(p.acc) + ((size_t)b * p.nhalf + half) * L * Lp;
  int ncopy = p.Gs - r0;
  if (ncopy > NRT) ncopy = NRT;
  int nlam = p.Ls - r0;
  if (nlam > NRT) nlam = NRT;

  auto issue = [&](int g) {
    unsigned char* st = stage_base + (size_t)(g & 1) * Lay::stage_bytes;
    const int row0 = mtop - g * R - R + 1 + kPadLo;
    constexpr unsigned hb = R * kFwdBlock * sizeof(Real);
    const unsigned bytes = 2 * hb + (unsigned)(R * ncopy * GM * sizeof(Acc)) +
                           (unsigned)(R * nlam * sizeof(Real));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&mbar[g & 1], bytes);
    bulk_g2s(st, Hb + ((size_t)kb0 * TR + row0) * kFwdBlock, hb, &mbar[g & 1]);
    bulk_g2s(st + hb, Hb + ((size_t)kb1 * TR + row0) * kFwdBlock, hb, &mbar[g & 1]);
    unsigned char* gdst = st + Lay::h_bytes;
#pragma unroll
    for (int s = 0; s < R; ++s)
      bulk_g2s(gdst + (size_t)s * NRT * GM * sizeof(Acc),
               Gin + ((size_t)(row0 + s) * p.Gs + r0) * GM, (unsigned)(ncopy * GM * sizeof(Acc)),
               &mbar[g & 1]);
    unsigned char* ldst = st + Lay::h_bytes + Lay::g_bytes;
#pragma unroll
    for (int s = 0; s < R; ++s)
      bulk_g2s(ldst + (size_t)s * NRT * sizeof(Real), lamh + (size_t)(row0 + s) * p.Ls + r0,
               (unsigned)(nlam * sizeof(Real)), &mbar[g & 1]);
  };
  if (tid == 0) {
    issue(0);
    if (ngroups > 1) issue(1);
  }

  Real v[2][T], w[2][T];
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int i = 0; i < T; ++i) {
      v[k][i] = Real(0);
      w[k][i] = Real(0);
    }
  int next_act = mt0 > mt1 ? mt0 : mt1;  // warp-uniform
  const int kb[2] = {kb0, kb1};
  const int mtw[2] = {mt0, mt1};

  for (int grp = 0; grp < ngroups; ++grp) {
    const int mgrp = mtop - grp * R;
    const bool ok = mbar_wait(&mbar[grp & 1], (grp >> 1) & 1);
    // start the (slot, ring) states whose first m is this group's first m
    if (mgrp == next_act) {
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < T; ++i)
          if (act[(wp * 2 + k) * T + i] == mgrp) {
            const R2 sv = Vst[(((size_t)half * NB + kb[k]) * RS + r0 + wp * T + i) *
                                  kFwdBlock + lane];
            v[k][i] = sv.x;
            w[k][i] = sv.y;
          }
      int na = -1;
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (lane + 32 * u < 2 * T && a_m[u] < mgrp && a_m[u] > na) na = a_m[u];
      next_act = __reduce_max_sync(0xffffffffu, na);
    }
    // the next group starts states: their start values into L1 while this group runs
    if (next_act >= 0 && next_act == mgrp - R) {
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < T; ++i)
          if (act[(wp * 2 + k) * T + i] == next_act)
            prefetch_l1(&Vst[(((size_t)half * NB + kb[k]) * RS + r0 + wp * T + i) * kFwdBlock +
                             lane]);
    }
    const unsigned char* st = stage_base + (size_t)(grp & 1) * Lay::stage_bytes;
    Acc* const buf = bufs + (Lay::NBUF == 2 ? (grp & 1) * Lay::buf_elems : 0);
    const Real* hS = reinterpret_cast<const Real*>(st);
    const Acc* gS = reinterpret_cast<const Acc*>(st + Lay::h_bytes) + wp * T * GM;
    const Real* lS = reinterpret_cast<const Real*>(st + Lay::h_bytes + Lay::g_bytes) + wp * T;

#define S2B_FWD2_STEP(CUR, PRV, S)                                                        \
  {                                                                                       \
    const int srow = R - 1 - (S);                                                         \
    const int m = mgrp - (S);                                                             \
    const bool k0 = m <= mtw[0], k1 = m <= mtw[1];                                        \
    const Real* lr = lS + srow * NRT;                                                     \
    /* symmetric mode: E where l + m is even, O where odd (l = 32 block + lane) */        \
    const Acc* gr = gS + srow * NRT * GM + (SYM ? ((lane + m) & 1) : 0);                  \
    Acc a0 = zero_acc<Acc>(), a1 = zero_acc<Acc>();                                       \
    if constexpr (sizeof(Real) == 8) {                                                    \
      const Real h0 = k0 ? hS[(0 * R + srow) * kFwdBlock + lane] : Real(0);               \
      const Real h1 = k1 ? hS[(1 * R + srow) * kFwdBlock + lane] : Real(0);               \
      /* an inactive slot's states are still zero, so both-slot steps serve k0 alone */   \
      if (k0)                                                                             \
        fwd_pair_step<Real, Acc, T, GM, true, true>(CUR[0], PRV[0], CUR[1], PRV[1], h0, h1,   \
                                                lr, gr, a0, a1);                          \
      else if (k1)                                                                        \
        fwd_pair_step<Real, Acc, T, GM, false, true>(CUR[0], PRV[0], CUR[1], PRV[1], h0, h1,  \
                                                 lr, gr, a0, a1);                         \
    } else {                                                                              \
      if (k0)                                                                             \
        fwd_slot_step<Real, Acc, T, GM>(CUR[0], PRV[0], hS[(0 * R + srow) * kFwdBlock + lane], \
                                    lr, gr, a0);                                          \
      if (k1)                                                                             \
        fwd_slot_step<Real, Acc, T, GM>(CUR[1], PRV[1], hS[(1 * R + srow) * kFwdBlock + lane], \
                                    lr, gr, a1);                                          \
    }                                                                                     \
    /* the flush reads a slot's rows only where the slot is active somewhere in the CTA */ \
    if (m <= mc0) buf[(((S) * W + wp) * 2 + 0) * kFwdBlock + lane] = a0;                  \
    if (m <= mc1) buf[(((S) * W + wp) * 2 + 1) * kFwdBlock + lane] = a1;                  \
  }
    // two steps per iteration keep the roles of v and w static; the loop is not unrolled
    // further so the group body stays small in the instruction cache
#pragma unroll 1
    for (int S = 0; S < R; S += 2) {
      S2B_FWD2_STEP(v, w, S)
      S2B_FWD2_STEP(w, v, S + 1)
    }
#undef S2B_FWD2_STEP

    if (!__syncthreads_and(ok)) {
      if (tid == 0) {
        atomicExch(p.status, 1);
        mbar_wait(&mbar[(grp + 1) & 1], ((grp + 1) >> 1) & 1);
      }
      return false;
    }
    // every warp is past this group's stage: refill it for group grp + 2
    if (tid == 0 && grp + 2 < ngroups) issue(grp + 2);
    // warps' partial sums -> flm accumulator
    for (int it = tid; it < R * 2 * kFwdBlock; it += NT) {
      const int S = it / (2 * kFwdBlock);
      const int k = (it / kFwdBlock) & 1;
      const int ln = it % kFwdBlock;
      const int m = mgrp - S;
      const int l = (k ? kb1 : kb0) * kFwdBlock + ln;
      if (m < p.mlo || m > (k ? mc1 : mc0) || l >= L || l < m) continue;
      Acc s = buf[((S * W + 0) * 2 + k) * kFwdBlock + ln];
#pragma unroll
      for (int x = 1; x < W; ++x) acc_add(s, buf[((S * W + x) * 2 + k) * kFwdBlock + ln]);
      if constexpr (SYM == 2) {
        // this half's projection and the other half's mirrored one
        using R2o = typename Vec<Real>::t2;
        R2o own, oth;
        own.x = s.x;
        own.y = s.y;
        oth.x = s.z;
        oth.y = s.w;
        R2o* o2 = reinterpret_cast<R2o*>(p.acc);
        red_add(o2 + (((size_t)b * p.nhalf + half) * L + m) * Lp + l, own);
        red_add(o2 + (((size_t)b * p.nhalf + (1 - half)) * L + m) * Lp + l, oth);
      } else {
        red_add(out + (size_t)m * Lp + l, s);
      }
    }
    if constexpr (Lay::NBUF == 1) __syncthreads();  // buf is rewritten by the next group
  }
  return true;
}

template <typename Real, bool DUAL, int T, int W, int R, int SYM>
__global__ void __launch_bounds__(W * 32, 3) lat_fwd2_kernel(const Fwd2Params p) {
  chain_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bool live = false;
  lat_fwd2_tile<Real, DUAL, T, W, R, SYM>(p, (int)blockIdx.x, (int)blockIdx.y,
                                          (int)blockIdx.z, smem_raw, live);
}

// Persistent form over the plans of a batch (as lat_inv2_persistent).
template <typename Real, bool DUAL, int T, int W, int R, int SYM>
__global__ void __launch_bounds__(W * 32, 3) lat_fwd2_persistent(const Fwd2Batch w) {
  using Lay = Fwd2Layout<Real, DUAL, T, W, R, SYM>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int item;
  bool live = false;
  for (;;) {
    __syncthreads();  // the previous tile is done with shared memory and item
    if (threadIdx.x == 0) item = atomicAdd(w.counter, 1);
    __syncthreads();
    const int it = item;
    if (it >= w.start[w.nplans]) return;
    int pl = 0;
    while (w.start[pl + 1] <= it) ++pl;
    const Fwd2Params& p = w.p[pl];
    const int gx = (p.nrings + Lay::NRT - 1) / Lay::NRT;
    const int gy = (p.NB / 2) * (p.Mst1 ? p.nseg : 1);
    const int loc = it - w.start[pl];
    if (!lat_fwd2_tile<Real, DUAL, T, W, R, SYM>(p, loc % gx, (loc / gx) % gy, loc / (gx * gy),
                                                 smem_raw, live))
      return;
  }
}

template <typename Real, bool DUAL, int T, int W, int R, int SYM>
static cudaError_t launch_fwd2_cfg(const Fwd2Params& p, cudaStream_t s) {
  using Lay = Fwd2Layout<Real, DUAL, T, W, R, SYM>;
  auto kern = lat_fwd2_kernel<Real, DUAL, T, W, R, SYM>;
  cudaError_t err =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::total);
  if (err != cudaSuccess) return err;
  const int ntiles = (p.nrings + Lay::NRT - 1) / Lay::NRT;
  dim3 grid(ntiles, (p.NB / 2) * (p.Mst1 ? p.nseg : 1), p.nhalf * p.batch);
  return launch_chained(kern, grid, dim3(Lay::NT), Lay::total, s, p);
}

template <typename Real, int T, int R, int SYM>
static cudaError_t launch_fwd2_dual(bool dual, const Fwd2Params& p, cudaStream_t s) {
  if constexpr (SYM == 2) {  // spin != 0: never the dual layout
    if (dual) return cudaErrorInvalidValue;
    return launch_fwd2_cfg<Real, false, T, 4, R, 2>(p, s);
  } else {
    return dual ? launch_fwd2_cfg<Real, true, T, 4, R, SYM>(p, s)
                : launch_fwd2_cfg<Real, false, T, 4, R, SYM>(p, s);
  }
}

int fwd_group(bool fp64) {
  (void)fp64;
  return 8;  // start tables serve 8-step groups (and 4-step ones: 7 = 3 mod 4)
}

// float: 16 rings x 4 warps (measured at L=1024: 0.46 ms; 2 warps 0.52 ms, 15 rings
// 0.52 ms), tile 1: 8 rings; double: 8 rings, tile 1: 4 rings
template <int SYM>
static cudaError_t launch_fwd2_prec(bool fp64, bool dual, const Fwd2Params& p, cudaStream_t s) {
  if (!fp64)
    return p.tile == 1 ? launch_fwd2_dual<float, 8, 8, SYM>(dual, p, s)
                       : launch_fwd2_dual<float, 16, 8, SYM>(dual, p, s);
  return p.tile == 1 ? launch_fwd2_dual<double, 4, 4, SYM>(dual, p, s)
                     : launch_fwd2_dual<double, 8, 4, SYM>(dual, p, s);
}

template <typename Kernel>
static cudaError_t persistent_grid(Kernel k, int threads, size_t smem, int items, int per_sm_cap,
                                   int* grid) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm_cap > 0 && per_sm > per_sm_cap) per_sm = per_sm_cap;
  const long cap = (long)sms * (per_sm > 0 ? per_sm : 1);
  *grid = (int)(items < cap ? items : cap);
  return cudaSuccess;
}

template <typename Real, bool DUAL, int T, int R, int SYM>
static cudaError_t launch_fwd2_batch_cfg(const Fwd2Params* ps, int n, int* counter, int per_sm,
                                         cudaStream_t s) {
  using Lay = Fwd2Layout<Real, DUAL, T, 4, R, SYM>;
  auto kern = lat_fwd2_persistent<Real, DUAL, T, 4, R, SYM>;
  cudaError_t err =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::total);
  if (err != cudaSuccess) return err;
  Fwd2Batch w{};
  w.nplans = n;
  w.counter = counter;
  w.start[0] = 0;
  for (int i = 0; i < n; ++i) {
    w.p[i] = ps[i];
    const long gx = (ps[i].nrings + Lay::NRT - 1) / Lay::NRT;
    const long gy = (long)(ps[i].NB / 2) * (ps[i].Mst1 ? ps[i].nseg : 1);
    const long gz = (long)ps[i].nhalf * ps[i].batch;
    const long tot = w.start[i] + (ps[i].nrings > 0 ? gx * gy * gz : 0);
    if (tot > (1L << 30)) return cudaErrorInvalidValue;
    w.start[i + 1] = (int)tot;
  }
  if (w.start[n] == 0) return cudaSuccess;
  int grid = 0;
  if ((err = persistent_grid(kern, Lay::NT, Lay::total, w.start[n], per_sm, &grid))) return err;
  if ((err = cudaMemsetAsync(counter, 0, sizeof(int), s))) return err;
  kern<<<grid, Lay::NT, Lay::total, s>>>(w);
  return cudaGetLastError();
}

template <int SYM>
static cudaError_t launch_fwd2_batch_prec(bool fp64, bool dual, const Fwd2Params* ps, int n,
                                          int* counter, int per_sm, cudaStream_t s) {
  const bool half = ps[0].tile == 1;
  if constexpr (SYM == 2) {
    if (dual) return cudaErrorInvalidValue;
    if (!fp64)
      return half ? launch_fwd2_batch_cfg<float, false, 8, 8, 2>(ps, n, counter, per_sm, s)
                  : launch_fwd2_batch_cfg<float, false, 16, 8, 2>(ps, n, counter, per_sm, s);
    return half ? launch_fwd2_batch_cfg<double, false, 4, 4, 2>(ps, n, counter, per_sm, s)
                : launch_fwd2_batch_cfg<double, false, 8, 4, 2>(ps, n, counter, per_sm, s);
  } else {
#define S2B_FWD2B(REAL, TT, RR)                                                       \
  return dual ? launch_fwd2_batch_cfg<REAL, true, TT, RR, SYM>(ps, n, counter, per_sm, s) \
              : launch_fwd2_batch_cfg<REAL, false, TT, RR, SYM>(ps, n, counter, per_sm, s)
    if (!fp64) {
      if (half) S2B_FWD2B(float, 8, 8);
      S2B_FWD2B(float, 16, 8);
    }
    if (half) S2B_FWD2B(double, 4, 4);
    S2B_FWD2B(double, 8, 4);
#undef S2B_FWD2B
  }
}

cudaError_t launch_fwd2_batch(bool fp64, bool dual, const Fwd2Params* ps, int nplans,
                              int* counter, int per_sm, cudaStream_t s) {
  if (nplans <= 0) return cudaSuccess;
  if (nplans > kBatchPlans) return cudaErrorInvalidValue;
  for (int i = 0; i < nplans; ++i) {
    if (ps[i].Mst1 && !(ps[i].nseg == 1 || ps[i].nseg == 2 || ps[i].nseg == 4 || ps[i].nseg == 8))
      return cudaErrorInvalidValue;
    if (ps[i].sym != ps[0].sym || ps[i].cross != ps[0].cross || ps[i].tile != ps[0].tile)
      return cudaErrorInvalidValue;
  }
  if (ps[0].sym && ps[0].cross) return launch_fwd2_batch_prec<2>(fp64, dual, ps, nplans, counter, per_sm, s);
  return ps[0].sym ? launch_fwd2_batch_prec<1>(fp64, dual, ps, nplans, counter, per_sm, s)
                   : launch_fwd2_batch_prec<0>(fp64, dual, ps, nplans, counter, per_sm, s);
}

cudaError_t launch_fwd2(bool fp64, bool dual, const Fwd2Params& p, cudaStream_t s) {
  if (p.nrings <= 0) return cudaSuccess;
  if (p.Mst1 && !(p.nseg == 1 || p.nseg == 2 || p.nseg == 4 || p.nseg == 8)) return cudaErrorInvalidValue;
  if (p.sym && p.cross) return launch_fwd2_prec<2>(fp64, dual, p, s);
  return p.sym ? launch_fwd2_prec<1>(fp64, dual, p, s) : launch_fwd2_prec<0>(fp64, dual, p, s);
}

}  // namespace s2b
