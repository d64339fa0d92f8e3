// Inverse latitudinal step (synthesis of ring spectra from flm), blocked tiling.
//
// Same recursion and projection as upstream s2fft
// (s2fft/transforms/otf_recursions.py:15-171, inverse_latitudinal_step;
// coefficients s2fft/recursions/price_mcewen.py:118-255):
// ftm[theta, m] = sum_l d^l_{m,n}(theta) flm'[l, m], n = -spin, with d generated
// by the m-recursion from the seeds d^l_{l,n}(theta).
//
// B200 formulation (own design):
//  * lanes run along theta (T rings per lane), and every lane of a warp holds the
//    same K = 16 degrees (8 consecutive ones from each of the CTA's two 32-degree
//    blocks p and NB-1-p, so all warps stay busy), so the coefficient loads h_{l,m} and
//    flm'[l, m] are shared-memory broadcasts and the sum over l stays in
//    registers over 16 terms before warps' partial sums meet in shared memory;
//  * restart at first significance, as in the forward kernel: per (ring, 32-degree
//    block) the recursion starts at the block's first significant group start M with
//    the double-precision start values (d~_M, d~_{M+1}) of every degree (degrees below
//    M begin with the exact continuation above m = l); the loop runs the plain monic
//    recursion with no exponent, no gating multiply and no renormalisation, and a
//    block's degrees are skipped until the recursion reaches the block on any ring of
//    the CTA. A lane starts its (ring, block) states when the group start equals M.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "s2b_dev.h"
#include "s2b_latfwd.h"

namespace s2b {

// n consecutive values from 16-byte aligned shared memory by 16-byte loads
template <typename V, int N>
__device__ __forceinline__ void ld_vec16(V (&o)[N], const V* src) {
  static_assert((N * sizeof(V)) % 16 == 0, "whole 16-byte vectors");
  constexpr int NV = N * (int)sizeof(V) / 16;
  uint4 t[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) t[i] = reinterpret_cast<const uint4*>(src)[i];
  __builtin_memcpy(o, t, sizeof(t));
}

template <typename Real, bool DUAL, int T, int W, int R, bool VST, bool SYM>
struct Inv2Layout {
  using Acc = std::conditional_t<DUAL, typename Vec<Real>::t4, typename Vec<Real>::t2>;
  static constexpr int K = 16;       // degrees per warp
  static constexpr int NRT = 32 * T; // rings per CTA
  static constexpr int NT = W * 32;
  // stage: h rows [2 blocks][R][32] | coefficient rows [2 blocks][R][32] | lambda [R][NRT]
  static constexpr size_t h_bytes = 2 * R * kFwdBlock * sizeof(Real);
  static constexpr size_t f_bytes = 2 * R * kFwdBlock * sizeof(Acc);
  static constexpr size_t l_bytes = (size_t)R * NRT * sizeof(Real);
  static constexpr size_t stage_bytes = h_bytes + f_bytes + l_bytes;
  static constexpr int NE = SYM ? 2 : 1;  // partial sums per lane slot: (E, O) of a ring pair
  // warps' partial sums of one group, twice: a group's reduction and the next group's steps
  // use different halves, so one barrier per group separates them
  // (once when two copies would leave room for fewer than 3 CTAs per SM: then a second
  // barrier per group)
  static constexpr int buf_elems = R * W * NRT * NE;
  // start values of the CTA's states: [2 blocks][NRT rings][32] (d~_M, d~_{M+1})
  // (VST: staged by bulk copy; otherwise each lane reads its own from global memory, which
  // leaves room for one more CTA per SM)
  static constexpr size_t v_bytes = VST ? (size_t)2 * NRT * kFwdBlock * 2 * sizeof(Real) : 0;
  static constexpr size_t fixed_bytes = 2 * stage_bytes + v_bytes + 32;
  static constexpr int NBUF =
      3 * (fixed_bytes + 2 * buf_elems * sizeof(Acc) + 1024) <= 228 * 1024 ? 2 : 1;
  static constexpr size_t buf_bytes = (size_t)NBUF * buf_elems * sizeof(Acc);
  static constexpr size_t total = fixed_bytes + buf_bytes;
  static_assert(W == 4, "two warps per 32-degree block, two blocks per CTA");
  static_assert(stage_bytes % 16 == 0 && buf_bytes % 16 == 0, "align");
};

// Adds a ring's partial spectrum for order m to its ftm row: column L-1+m+mo (half 0), and
// L-1-m+mo for the second half or, in the dual layout, the -m components.
template <bool DUAL, typename R2, typename Acc>
__device__ __forceinline__ void inv2_store(R2* ftm, const Acc& s, int L, int m, int mo,
                                           int half) {
  R2 ap;
  ap.x = s.x;
  ap.y = s.y;
  if constexpr (DUAL) {
    R2 an;
    an.x = s.z;
    an.y = s.w;
    red_add(ftm + (L - 1 + m + mo), ap);
    if (m > 0) red_add(ftm + (L - 1 - m + mo), an);
  } else {
    if (half == 0)
      red_add(ftm + (L - 1 + m + mo), ap);
    else if (m > 0)
      red_add(ftm + (L - 1 - m + mo), ap);
  }
}

// One tile of the inverse kernel: ring tile bx, block pair and segment by, (half, map) bz.
// Returns false when a bounded wait ran out (the plan's status word is set). live: the
// CTA's mbarriers were initialised by an earlier tile (persistent launches) and are
// invalidated before they are set up again.
template <typename Real, bool DUAL, int T, int W, int R, bool VST, bool SYM>
__device__ __forceinline__ bool lat_inv2_tile(const Inv2Params& p, int bx, int by, int bz,
                                              unsigned char* smem_raw, bool& live) {
  using Lay = Inv2Layout<Real, DUAL, T, W, R, VST, SYM>;
  constexpr int NE = Lay::NE;
  using Acc = typename Lay::Acc;
  using R2 = typename Vec<Real>::t2;
  constexpr int K = Lay::K;
  constexpr int NRT = Lay::NRT;
  constexpr int NT = Lay::NT;
  static_assert(R == 4 || R == 8, "the group body below is written for R = 4 or 8");
  unsigned char* stage_base = smem_raw;
  Acc* const bufs = reinterpret_cast<Acc*>(smem_raw + 2 * Lay::stage_bytes);
  const typename Vec<Real>::t2* vS = reinterpret_cast<const typename Vec<Real>::t2*>(
      smem_raw + 2 * Lay::stage_bytes + Lay::buf_bytes);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + 2 * Lay::stage_bytes + Lay::buf_bytes +
                                               Lay::v_bytes);  // [0], [1] stages, [2] start values

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wp = tid >> 5;
  const int L = p.L;
  const int NB = p.NB;
  const int TR = tab_rows(L);
  const int r0 = bx * NRT;
  // by = block pair + NB/2 * segment; segment seg of nseg spans the boundaries
  // g = seg * kInvSegMax / nseg and g + kInvSegMax / nseg (inv_mbound)
  const int npair = NB / 2;
  const int q = by % npair, seg = by / npair;
  const int kb0 = q, kb1 = NB - 1 - q;
  const int nseg = p.Mst1 ? p.nseg : 1;
  const int gstep = kInvSegMax / nseg, g0 = seg * gstep;
  const int RS = p.tab_stride ? p.tab_stride : p.nrings;  // table stride = rings of the set
  const size_t nst = (size_t)p.nhalf * NB * RS;
  const int* __restrict__ Mtab = g0 ? p.Mst1 + (size_t)(g0 - 1) * nst : p.Mst;
  const int mbot = inv_mbound(L, NB, q, g0 + gstep);  // lowest m of the segment
  const int half = (int)(bz % p.nhalf);
  const int b = (int)(bz / p.nhalf);

  // degrees of this warp: slot k < 8 -> l = 32 kb0 + 8 wp + k, slot k >= 8 -> 32 kb1 + 8 wp + k - 8,
  // so every warp works on both blocks of the CTA
  const int col0 = wp * (K / 2);
  // first group start of every (ring, block) state of this lane, and per block the
  // earliest one over the CTA (all warps hold the same rings)
  int Ms[2][T];
  int Mb[2];
#pragma unroll
  for (int x = 0; x < 2; ++x) {
    int mx = -1;
#pragma unroll
    for (int i = 0; i < T; ++i) {
      const int r = r0 + lane * T + i;
      Ms[x][i] = r < p.nrings ? Mtab[((size_t)half * NB + (x ? kb1 : kb0)) * RS + r] : -1;
      mx = Ms[x][i] > mx ? Ms[x][i] : mx;
    }
    Mb[x] = __reduce_max_sync(0xffffffffu, mx);
  }
  const int mtop = Mb[0] > Mb[1] ? Mb[0] : Mb[1];
  if (mtop < mbot) return true;  // nothing significant in this tile and segment (uniform)
  const int ngroups = (mtop + 1 - mbot) / R;  // mtop = -1 mod 8, mbot = 0 mod 8
  const R2* __restrict__ Vst =
      g0 ? reinterpret_cast<const R2*>(p.Vst1) + (size_t)(g0 - 1) * nst * kFwdBlock
         : reinterpret_cast<const R2*>(p.Vst);

  Real v[K][T], w[K][T];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int i = 0; i < T; ++i) {
      v[k][i] = Real(0);
      w[k][i] = Real(0);
    }

  const Real* __restrict__ Hb = reinterpret_cast<const Real*>(p.Hb);
  const Acc* __restrict__ Fin =
      reinterpret_cast<const Acc*>(p.F) + ((size_t)b * p.nhalf + half) * NB * TR * kFwdBlock;
  const Real* __restrict__ lamh = reinterpret_cast<const Real*>(p.lam) + (size_t)half * TR * p.Ls;
  int nlam = p.Ls - r0;
  if (nlam > NRT) nlam = NRT;

  auto issue = [&](int g) {
    unsigned char* st = stage_base + (size_t)(g & 1) * Lay::stage_bytes;
    const int row0 = mtop - g * R - R + 1 + kPadLo;
    constexpr unsigned hb = R * kFwdBlock * sizeof(Real);
    constexpr unsigned fb = R * kFwdBlock * sizeof(Acc);
    const unsigned bytes = 2 * hb + 2 * fb + (unsigned)(R * nlam * sizeof(Real));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&mbar[g & 1], bytes);
    bulk_g2s(st, Hb + ((size_t)kb0 * TR + row0) * kFwdBlock, hb, &mbar[g & 1]);
    bulk_g2s(st + hb, Hb + ((size_t)kb1 * TR + row0) * kFwdBlock, hb, &mbar[g & 1]);
    bulk_g2s(st + Lay::h_bytes, Fin + ((size_t)kb0 * TR + row0) * kFwdBlock, fb, &mbar[g & 1]);
    bulk_g2s(st + Lay::h_bytes + fb, Fin + ((size_t)kb1 * TR + row0) * kFwdBlock, fb,
             &mbar[g & 1]);
    unsigned char* ldst = st + Lay::h_bytes + Lay::f_bytes;
#pragma unroll
    for (int s = 0; s < R; ++s)
      bulk_g2s(ldst + (size_t)s * NRT * sizeof(Real), lamh + (size_t)(row0 + s) * p.Ls + r0,
               (unsigned)(nlam * sizeof(Real)), &mbar[g & 1]);
  };
  for (size_t x = tid * 16; x < 2 * Lay::stage_bytes; x += (size_t)NT * 16)
    *reinterpret_cast<uint4*>(stage_base + x) = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (tid == 0) {
    if (live) {
      mbar_inval(&mbar[0]);
      mbar_inval(&mbar[1]);
      mbar_inval(&mbar[2]);
    }
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init(&mbar[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  live = true;
  __syncthreads();
  if (tid == 0) {
    if constexpr (VST) {
      // the start values of both blocks for this CTA's rings, once
      int nr = p.nrings - r0;
      if (nr > NRT) nr = NRT;
      const unsigned vb = (unsigned)(nr * kFwdBlock * sizeof(R2));
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&mbar[2], 2 * vb);
#pragma unroll
      for (int x = 0; x < 2; ++x)
        bulk_g2s(const_cast<R2*>(vS) + (size_t)x * NRT * kFwdBlock,
                 Vst + (((size_t)half * NB + (x ? kb1 : kb0)) * RS + r0) * kFwdBlock, vb,
                 &mbar[2]);
    }
    issue(0);
    if (ngroups > 1) issue(1);
  }
  bool vok = true;
  if constexpr (VST) vok = mbar_wait(&mbar[2], 0);
  // highest degree of the CTA: partial sums above it are zero
  int lmax = -1;
  if (kb0 * kFwdBlock < L) lmax = kb0 * kFwdBlock + kFwdBlock - 1;
  if (kb1 * kFwdBlock < L && kb1 * kFwdBlock + kFwdBlock - 1 > lmax)
    lmax = kb1 * kFwdBlock + kFwdBlock - 1;
  if (lmax > L - 1) lmax = L - 1;

  // the reduction gives every thread one ring of the tile (NT is a multiple of NRT): its
  // ftm rows (and, symmetric, its mirror's), looked up once
  static_assert(NT % NRT == 0, "one reduction ring per thread");
  const int rr_red = tid % NRT;
  const int r_red = r0 + rr_red;
  const bool ring_live = r_red < p.nrings;
  R2* ftm_r = nullptr;
  R2* ftm_rm = nullptr;  // symmetric: the mirror ring (none for the equator)
  if (ring_live) {
    ftm_r = reinterpret_cast<R2*>(p.ftm) + ((size_t)b * p.nrows + p.ring_row[r_red]) * p.ncol;
    if (SYM && RS - 1 - r_red != r_red)
      ftm_rm = reinterpret_cast<R2*>(p.ftm) +
               ((size_t)b * p.nrows + p.ring_row[RS - 1 - r_red]) * p.ncol;
  }
  // start values read from global memory: each lane's line is prefetched into L1 one group
  // before the group that starts the state (a group is thousands of cycles of FMAs)
  auto vst_line = [&](int x, int i) {
    return Vst + (((size_t)half * NB + (x ? kb1 : kb0)) * RS + r0 + lane * T + i) * kFwdBlock +
           col0;
  };
  if constexpr (!VST) {
#pragma unroll
    for (int x = 0; x < 2; ++x)
#pragma unroll
      for (int i = 0; i < T; ++i)
        if (Ms[x][i] >= 0 && Ms[x][i] == mtop) prefetch_l1(vst_line(x, i));
  }
  for (int grp = 0; grp < ngroups; ++grp) {
    const int mgrp = mtop - grp * R;
    if constexpr (!VST) {
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int i = 0; i < T; ++i)
          if (Ms[x][i] >= 0 && Ms[x][i] == mgrp - R) prefetch_l1(vst_line(x, i));
    }
    const bool ok = mbar_wait(&mbar[grp & 1], (grp >> 1) & 1);
    // start the (ring, block) states whose first group start is this group's
#pragma unroll
    for (int x = 0; x < 2; ++x)
#pragma unroll
      for (int i = 0; i < T; ++i)
        if (Ms[x][i] == mgrp) {
          const R2* src = VST ? vS + ((size_t)x * NRT + lane * T + i) * kFwdBlock + col0
                              : vst_line(x, i);
#pragma unroll
          for (int kk = 0; kk < K / 2; ++kk) {
            const R2 sv = src[kk];
            v[x * (K / 2) + kk][i] = sv.x;
            w[x * (K / 2) + kk][i] = sv.y;
          }
        }
    const unsigned char* st = stage_base + (size_t)(grp & 1) * Lay::stage_bytes;
    Acc* const buf = bufs + (Lay::NBUF == 2 ? (grp & 1) * Lay::buf_elems : 0);
    const Real* hS = reinterpret_cast<const Real*>(st) + col0;
    const Acc* fS = reinterpret_cast<const Acc*>(st + Lay::h_bytes) + col0;
    const Real* lS = reinterpret_cast<const Real*>(st + Lay::h_bytes + Lay::f_bytes) + lane * T;

#define S2B_INV2_STEP(CUR, PRV, S)                                                      \
  {                                                                                     \
    constexpr int srow = R - 1 - (S);                                                   \
    const int m = mgrp - (S);                                                           \
    Real lam[T];                                                                        \
    _Pragma("unroll") for (int i = 0; i < T; ++i) lam[i] = lS[srow * NRT + i];          \
    /* two independent FMA chains: one per block, or (symmetric) one per degree parity */ \
    Acc a[2][T];                                                                        \
    _Pragma("unroll") for (int i = 0; i < T; ++i) {                                     \
      a[0][i] = zero_acc<Acc>();                                                        \
      a[1][i] = zero_acc<Acc>();                                                        \
    }                                                                                   \
    _Pragma("unroll") for (int x = 1; x >= 0; --x) {                                    \
      if (m <= Mb[x]) {                                                                 \
        /* the warp's 8 h values of the row: 16-byte broadcast loads */                  \
        Real hv[K / 2];                                                                 \
        ld_vec16(hv, hS + (x * R + srow) * kFwdBlock);                                  \
        /* and its 8 coefficients: 16-byte loads (each a one-wavefront broadcast) */    \
        Acc fv[K / 2];                                                                  \
        ld_vec16(fv, fS + (x * R + srow) * kFwdBlock);                                  \
        _Pragma("unroll") for (int kk = 0; kk < K / 2; ++kk) {                          \
          const int k = x * (K / 2) + kk;                                               \
          const Real h = hv[kk];                                                        \
          const Acc f = fv[kk];                                                         \
          _Pragma("unroll") for (int i = 0; i < T; ++i) {                               \
            acc_fma(a[SYM ? (kk & 1) : x][i], CUR[k][i], f);                            \
            PRV[k][i] = fma(lam[i] * h, CUR[k][i], -PRV[k][i]);                         \
          }                                                                             \
        }                                                                               \
      }                                                                                 \
    }                                                                                   \
    _Pragma("unroll") for (int i = 0; i < T; ++i) {                                     \
      if constexpr (SYM) {                                                              \
        /* l = 32 block + 8 warp + kk: l + m even for kk = m mod 2 */                   \
        const int pe = m & 1;                                                           \
        Acc* e = buf + (((S) * W + wp) * NRT + lane * T + i) * 2;                       \
        e[0] = pe ? a[1][i] : a[0][i];                                                  \
        e[1] = pe ? a[0][i] : a[1][i];                                                  \
      } else {                                                                          \
        acc_add(a[0][i], a[1][i]);                                                      \
        buf[((S) * W + wp) * NRT + lane * T + i] = a[0][i];                             \
      }                                                                                 \
    }                                                                                   \
  }
    S2B_INV2_STEP(v, w, 0)
    S2B_INV2_STEP(w, v, 1)
    S2B_INV2_STEP(v, w, 2)
    S2B_INV2_STEP(w, v, 3)
    if constexpr (R == 8) {
      S2B_INV2_STEP(v, w, 4)
      S2B_INV2_STEP(w, v, 5)
      S2B_INV2_STEP(v, w, 6)
      S2B_INV2_STEP(w, v, 7)
    }
#undef S2B_INV2_STEP

    if (!__syncthreads_and(ok && vok)) {
      if (tid == 0) {
        atomicExch(p.status, 1);
        mbar_wait(&mbar[(grp + 1) & 1], ((grp + 1) >> 1) & 1);
      }
      return false;
    }
    // every warp is past this group's stage: refill it for group grp + 2
    if (tid == 0 && grp + 2 < ngroups) issue(grp + 2);
    // warps' partial sums -> ring spectra (NT is a multiple of NRT: one ring per thread)
    for (int it = tid; it < R * NRT; it += NT) {
      const int S = it / NRT;
      const int m = mgrp - S;
      if (m < p.mlo || m > lmax || !ring_live) continue;
      const int rr = rr_red;
      Acc s = buf[((S * W + 0) * NRT + rr) * NE];
#pragma unroll
      for (int x = 1; x < W; ++x) acc_add(s, buf[((S * W + x) * NRT + rr) * NE]);
      if constexpr (SYM) {
        // ring r gets E + O, its mirror E - O (the equator, its own mirror, E + O once)
        Acc o = buf[((S * W + 0) * NRT + rr) * NE + 1];
#pragma unroll
        for (int x = 1; x < W; ++x) acc_add(o, buf[((S * W + x) * NRT + rr) * NE + 1]);
        if (ftm_rm) {
          Acc d = s;
          acc_fma(d, Real(-1), o);
          inv2_store<DUAL>(ftm_rm, d, L, m, p.mo, half);
        }
        acc_add(s, o);
      }
      inv2_store<DUAL>(ftm_r, s, L, m, p.mo, half);
    }
    if constexpr (Lay::NBUF == 1) __syncthreads();  // buf is rewritten by the next group
  }
  return true;
}

template <typename Real, bool DUAL, int T, int W, int R, bool VST, bool SYM>
__global__ void __launch_bounds__(W * 32, 3) lat_inv2_kernel(const Inv2Params p) {
  chain_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bool live = false;
  lat_inv2_tile<Real, DUAL, T, W, R, VST, SYM>(p, (int)blockIdx.x, (int)blockIdx.y,
                                               (int)blockIdx.z, smem_raw, live);
}

// Persistent form over the plans of a batch: every CTA takes (plan, tile) items from the
// work counter until none are left; the items of the first plans (the batch orders its plans
// by work, largest first) go first. Stops after a bounded wait ran out.
template <typename Real, bool DUAL, int T, int W, int R, bool VST, bool SYM>
__global__ void __launch_bounds__(W * 32, 3) lat_inv2_persistent(const Inv2Batch w) {
  using Lay = Inv2Layout<Real, DUAL, T, W, R, VST, SYM>;
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
    const Inv2Params& p = w.p[pl];
    const int gx = (p.nrings + Lay::NRT - 1) / Lay::NRT;
    const int gy = (p.NB / 2) * (p.Mst1 ? p.nseg : 1);
    const int loc = it - w.start[pl];
    if (!lat_inv2_tile<Real, DUAL, T, W, R, VST, SYM>(p, loc % gx, (loc / gx) % gy,
                                                      loc / (gx * gy), smem_raw, live))
      return;
  }
}

template <typename Real, bool DUAL, int T, int R, bool VST, bool SYM>
static cudaError_t launch_inv2_cfg(const Inv2Params& p, cudaStream_t s) {
  using Lay = Inv2Layout<Real, DUAL, T, 4, R, VST, SYM>;
  auto kern = lat_inv2_kernel<Real, DUAL, T, 4, R, VST, SYM>;
  cudaError_t err =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::total);
  if (err != cudaSuccess) return err;
  dim3 grid((p.nrings + Lay::NRT - 1) / Lay::NRT, (p.NB / 2) * (p.Mst1 ? p.nseg : 1),
            p.nhalf * p.batch);
  return launch_chained(kern, grid, dim3(Lay::NT), Lay::total, s, p);
}

template <typename Real, int T, bool VST, bool SYM>
static cudaError_t launch_inv2_dual(bool dual, const Inv2Params& p, cudaStream_t s) {
  return dual ? launch_inv2_cfg<Real, true, T, 8, VST, SYM>(p, s)
              : launch_inv2_cfg<Real, false, T, 8, VST, SYM>(p, s);
}

// tile bit 0: one ring per lane (float; double always has one); bit 1: start values read
// from global memory instead of staged in shared memory. 8-step groups (the start tables'
// alignment).
template <bool SYM>
static cudaError_t launch_inv2_prec(bool fp64, bool dual, const Inv2Params& p, cudaStream_t s) {
  const bool vst = (p.tile & 2) == 0;
  if (!fp64) {
    if (p.tile & 1)
      return vst ? launch_inv2_dual<float, 1, true, SYM>(dual, p, s)
                 : launch_inv2_dual<float, 1, false, SYM>(dual, p, s);
    return vst ? launch_inv2_dual<float, 2, true, SYM>(dual, p, s)
               : launch_inv2_dual<float, 2, false, SYM>(dual, p, s);
  }
  return vst ? launch_inv2_dual<double, 1, true, SYM>(dual, p, s)
             : launch_inv2_dual<double, 1, false, SYM>(dual, p, s);
}

// CTAs of a persistent launch: what fits on the device at once, at most one per item
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

template <typename Real, bool DUAL, int T, int R, bool VST, bool SYM>
static cudaError_t launch_inv2_batch_cfg(const Inv2Params* ps, int n, int* counter, int per_sm,
                                         cudaStream_t s) {
  using Lay = Inv2Layout<Real, DUAL, T, 4, R, VST, SYM>;
  auto kern = lat_inv2_persistent<Real, DUAL, T, 4, R, VST, SYM>;
  cudaError_t err =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::total);
  if (err != cudaSuccess) return err;
  Inv2Batch w{};
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

template <bool SYM>
static cudaError_t launch_inv2_batch_prec(bool fp64, bool dual, const Inv2Params* ps, int n,
                                          int* counter, int per_sm, cudaStream_t s) {
  // the launch shape of the first plan (the batch groups plans by it)
  const bool vst = (ps[0].tile & 2) == 0;
  const bool one = (ps[0].tile & 1) != 0;
#define S2B_INV2B(REAL, TT, VV)                                                          \
  return dual ? launch_inv2_batch_cfg<REAL, true, TT, 8, VV, SYM>(ps, n, counter, per_sm, s) \
              : launch_inv2_batch_cfg<REAL, false, TT, 8, VV, SYM>(ps, n, counter, per_sm, s)
  if (!fp64) {
    if (one) {
      if (vst) S2B_INV2B(float, 1, true);
      S2B_INV2B(float, 1, false);
    }
    if (vst) S2B_INV2B(float, 2, true);
    S2B_INV2B(float, 2, false);
  }
  if (vst) S2B_INV2B(double, 1, true);
  S2B_INV2B(double, 1, false);
#undef S2B_INV2B
}

cudaError_t launch_inv2_batch(bool fp64, bool dual, const Inv2Params* ps, int nplans,
                              int* counter, int per_sm, cudaStream_t s) {
  if (nplans <= 0) return cudaSuccess;
  if (nplans > kBatchPlans) return cudaErrorInvalidValue;
  for (int i = 0; i < nplans; ++i) {
    if (ps[i].Mst1 && !(ps[i].nseg == 1 || ps[i].nseg == 2 || ps[i].nseg == 4 || ps[i].nseg == 8))
      return cudaErrorInvalidValue;
    if (ps[i].sym != ps[0].sym || ps[i].tile != ps[0].tile) return cudaErrorInvalidValue;
  }
  return ps[0].sym ? launch_inv2_batch_prec<true>(fp64, dual, ps, nplans, counter, per_sm, s)
                   : launch_inv2_batch_prec<false>(fp64, dual, ps, nplans, counter, per_sm, s);
}

cudaError_t launch_inv2(bool fp64, bool dual, const Inv2Params& p, cudaStream_t s) {
  if (p.nrings <= 0) return cudaSuccess;
  if (p.Mst1 && !(p.nseg == 1 || p.nseg == 2 || p.nseg == 4 || p.nseg == 8)) return cudaErrorInvalidValue;
  return p.sym ? launch_inv2_prec<true>(fp64, dual, p, s)
               : launch_inv2_prec<false>(fp64, dual, p, s);
}

}  // namespace s2b
