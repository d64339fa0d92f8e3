// Fused Wigner-d recursion + projection (the latitudinal step of the spin SHT).
//
// Follows the Price-McEwen recursion of upstream s2fft
// (s2fft/transforms/otf_recursions.py:15-171 inverse, 432-588 forward;
// coefficients s2fft/recursions/price_mcewen.py:118-255): for fixed (theta, l)
// the values d^l_{m,n}(theta), n = -spin, are generated from the edge m = l
// towards m = 0 with a three-term recursion in m, so every (theta, l) pair is
// an independent state. The projection onto ftm (inverse) or flm (forward)
// happens in the same step, so the O(L^3) d-table never exists in memory.
//
// B200 formulation (own design, not the upstream loop):
//  * monic form: d_m = g_{l,m} dt_m with dt_{m-1} = (lambda_m h_{l,m}) dt_m - dt_{m+1},
//    lambda_m = 2 (n - m cos theta) / sin theta; g is folded into the inputs
//    (inverse) or outputs (forward), so a step costs one MUL and one FMA;
//  * lambda_m is evaluated once per (theta, m) as a single double FMA and then
//    rounded (a float cot(theta) would shift theta systematically);
//  * instead of renormalising every step in log space, each state carries a
//    mantissa and an integer exponent (units of 2^kScale) that is updated every
//    R steps, and only states above the significance floor are projected;
//  * negative m comes from the symmetry d^l_{-m,n} = (-1)^(m-n) d^l_{m,-n}: a
//    second recursion with n -> -n ("half" 1); for spin 0 both halves share one
//    recursion and every state feeds two projections ("dual");
//  * CTA tile = (QT*T rings) x (QA*K l's of one residue class l = j mod C), the
//    l's of a thread strided by QA*C so that the triangular l >= m work stays
//    balanced across lanes; states live in registers; per-step partial sums go
//    to shared memory and are reduced every R steps, then accumulated into the
//    output with vector atomics (reduction over l classes / ring tiles).
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "s2b_dev.h"
#include "s2b_internal.h"

namespace s2b {


// ---------------------------------------------------------------------------
// Seeds d^l_{l,n}(theta) = (-1)^(l-n) sqrt(binom(2l, l+n)) cos^(l+n)(t/2) sin^(l-n)(t/2)
// stored as mantissa * 2^(kScale * e) (price_mcewen.py:212-243 keeps the same
// quantity as a float64 logarithm). Layout [half][class j][q][ring], l = j + C q.
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void seed_kernel(int L, int L0, int spin, int nhalf, int C, int Q,
                            const RingInfo* __restrict__ rings, int nrings,
                            const double* __restrict__ lbin, SeedT<Real>* __restrict__ out) {
  const long total = (long)nhalf * C * Q * nrings;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % nrings);
    long rest = idx / nrings;
    const int q = (int)(rest % Q);
    rest /= Q;
    const int j = (int)(rest % C);
    const int half = (int)(rest / C);
    const int l = j + C * q;
    const int n = half == 0 ? -spin : spin;
    SeedT<Real> s{Real(0), 0};
    if (l < L && l >= L0 && l >= (n < 0 ? -n : n)) {
      const RingInfo ri = rings[r];
      const double lg = lbin[l] + (double)(l + n) * ri.lc + (double)(l - n) * ri.ls;
      int e = 0;
      if (lg < Scaling<Real>::kSignif)
        e = -(int)ceil((Scaling<Real>::kSignif - lg) / Scaling<Real>::kScale);
      const double mant = exp2(lg - Scaling<Real>::kScale * (double)e);
      s.v = (Real)((((l - n) & 1) ? -1.0 : 1.0) * mant);
      s.e = e;
    }
    out[idx] = s;
  }
}

// lambda(theta_r, m) = 2 (n - m cos theta) / sin theta = n A_r - m B_r, evaluated in
// double and rounded once; layout [half][m + kPadLo][Ls], zero outside 0 <= m < L.
template <typename Real>
__global__ void lambda_kernel(int L, int spin, int nhalf, const RingInfo* __restrict__ rings,
                              int nrings, int Ls, Real* __restrict__ out) {
  const int TR = tab_rows(L);
  const long total = (long)nhalf * TR * Ls;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % Ls);
    const int mr = (int)((idx / Ls) % TR);
    const int half = (int)(idx / ((long)Ls * TR));
    const int m = mr - kPadLo;
    const int n = half == 0 ? -spin : spin;
    double v = 0.0;
    if (r < nrings && m >= 0 && m < L) v = fma(-(double)m, rings[r].B, (double)n * rings[r].A);
    out[idx] = (Real)v;
  }
}

// ---------------------------------------------------------------------------
// main kernel
// ---------------------------------------------------------------------------
template <typename Real, bool FWD, bool DUAL, int T, int K, int QA, int QT, int R>
struct LatCfg {
  using R2 = typename Vec<Real>::t2;
  using R4 = typename Vec<Real>::t4;
  using Acc = std::conditional_t<DUAL, R4, R2>;
  static constexpr int NT = QA * QT;
  // shared buffer: inverse [R][T][QT][QA+1] Acc ; forward [R][K][QT][QA] Acc
  static constexpr int kSmemInv = R * T * QT * (QA + 1);
  static constexpr int kSmemFwd = R * K * QT * QA;
  static constexpr int kSmemElems = FWD ? kSmemFwd : kSmemInv;
  static constexpr size_t kSmemBytes = sizeof(Acc) * kSmemElems;
};

// Shared-memory carve-up of the latitudinal kernel (bytes, all 16-aligned):
//   [reduction buffer][stage 0: H rows | data rows][stage 1: ...][2 mbarriers]
template <typename Real, typename Acc, bool FWD, int T, int K, int QA, int QT, int R>
struct LatSmem {
  static constexpr int NRT = QT * T;
  static constexpr size_t red_elems = FWD ? (size_t)R * K * QT * QA : (size_t)R * T * QT * (QA + 1);
  __host__ __device__ static size_t red_bytes() { return (red_elems * sizeof(Acc) + 15) & ~(size_t)15; }
  __host__ __device__ static size_t h_bytes(int Qp) { return (size_t)R * Qp * sizeof(Real); }
  __host__ __device__ static size_t d_bytes(int Qp) {
    return (size_t)R * (FWD ? NRT : Qp) * sizeof(Acc);
  }
  __host__ __device__ static size_t l_bytes() { return (size_t)R * NRT * sizeof(Real); }
  __host__ __device__ static size_t stage_bytes(int Qp) { return h_bytes(Qp) + d_bytes(Qp) + l_bytes(); }
  __host__ __device__ static size_t seed_area() {
    return ((size_t)QA * QT * T * 2 * sizeof(Real) + 15) & ~(size_t)15;
  }
  __host__ __device__ static size_t total(int Qp) {
    return red_bytes() + 2 * stage_bytes(Qp) + seed_area() + 16;
  }
};

template <typename Real, bool FWD, bool DUAL, int T, int K, int QA, int QT, int R>
__global__ void __launch_bounds__(QA* QT, sizeof(Real) == 4 ? 4 : 3)
    lat_kernel(const LatParams p) {
  using Cfg = LatCfg<Real, FWD, DUAL, T, K, QA, QT, R>;
  using Acc = typename Cfg::Acc;
  using SM = LatSmem<Real, Acc, FWD, T, K, QA, QT, R>;
  constexpr int NRT = SM::NRT;
  static_assert(R % 2 == 0, "R must be even");
  static_assert(QA % 2 == 0, "QA must be even");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Qp = p.Qp;
  Acc* buf = reinterpret_cast<Acc*>(smem_raw);
  unsigned char* stage_base = smem_raw + SM::red_bytes();
  SeedT<Real>* seed_sm = reinterpret_cast<SeedT<Real>*>(stage_base + 2 * SM::stage_bytes(Qp));
  uint64_t* mbar =
      reinterpret_cast<uint64_t*>(stage_base + 2 * SM::stage_bytes(Qp) + SM::seed_area());

  const int tid = threadIdx.x;
  const int ql = tid % QA;
  const int qt = tid / QA;
  const int L = p.L;
  const int C = p.nclass;
  const int j = blockIdx.y;
  const int half = (int)(blockIdx.z % p.nhalf);
  const int b = (int)(blockIdx.z / p.nhalf);
  const int n = half == 0 ? -p.spin : p.spin;
  const int r0 = blockIdx.x * NRT;
  const int rbase = r0 + qt * T;
  if (j >= L) return;
  const int lmax = j + C * ((L - 1 - j) / C);
  const int TR = tab_rows(L);

  (void)n;

  Real v[K][T], w[K][T], sc[K][T];
  // exponents, two 16-bit values per register (only read on the renormalisation path)
  constexpr int TE = (T + 1) / 2;
  int ex2[K][TE];
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int i = 0; i < T; ++i) {
      v[k][i] = Real(0);
      w[k][i] = Real(0);
      sc[k][i] = Real(0);
    }
#pragma unroll
    for (int i = 0; i < TE; ++i) ex2[k][i] = 0;
  }
  auto ex_get = [&](int k, int i) -> int {
    return (int)(short)((ex2[k][i >> 1] >> ((i & 1) * 16)) & 0xffff);
  };
  auto ex_set = [&](int k, int i, int e) {
    const int sh = (i & 1) * 16;
    ex2[k][i >> 1] = (ex2[k][i >> 1] & ~(0xffff << sh)) | ((e & 0xffff) << sh);
  };

  const Real* __restrict__ Hc = reinterpret_cast<const Real*>(p.H) + (size_t)j * TR * Qp;
  const SeedT<Real>* __restrict__ seeds =
      reinterpret_cast<const SeedT<Real>*>(p.seeds) + ((size_t)half * C + j) * Qp * p.nrings;
  // inverse input F [b][half][j][row][Qp]; forward input G [b][half][row][Gs]
  const Acc* __restrict__ Din;
  if constexpr (!FWD)
    Din = reinterpret_cast<const Acc*>(p.in) + (((size_t)b * p.nhalf + half) * C + j) * TR * Qp;
  else
    Din = reinterpret_cast<const Acc*>(p.in) + ((size_t)b * p.nhalf + half) * TR * p.Gs;
  int ncopy = NRT;
  if constexpr (FWD) {
    ncopy = p.Gs - r0;
    if (ncopy > NRT) ncopy = NRT;
  }
  const Real* __restrict__ lamh = reinterpret_cast<const Real*>(p.lam) + (size_t)half * TR * p.Ls;
  int nlam = p.Ls - r0;
  if (nlam > NRT) nlam = NRT;

  // even-aligned chunk boundaries: chunk k covers m in [clo(k), clo(k+1)-1]
  // chunk boundaries aligned to the group length R (a power of two)
  auto clo = [&](int k) -> int {
    const int x = j + C * QA * k;
    return k == 0 ? 0 : (x & ~(R - 1));
  };
  const int mtop = lmax | (R - 1);  // == R-1 (mod R), >= lmax
  int ktop = (lmax - j) / (C * QA);
  if (ktop > K - 1) ktop = K - 1;
  const int ngroups = (mtop + 1) / R;

  // group g covers steps m = mtop - g R ... mtop - g R - R + 1 (table rows ascending)
  auto issue = [&](int g) {
    unsigned char* st = stage_base + (size_t)(g & 1) * SM::stage_bytes(Qp);
    const int row0 = mtop - g * R - R + 1 + kPadLo;
    unsigned bytes = (unsigned)SM::h_bytes(Qp) + (unsigned)(R * nlam * sizeof(Real));
    if constexpr (!FWD)
      bytes += (unsigned)SM::d_bytes(Qp);
    else
      bytes += (unsigned)(R * ncopy * sizeof(Acc));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&mbar[g & 1], bytes);
    bulk_g2s(st, Hc + (size_t)row0 * Qp, (unsigned)SM::h_bytes(Qp), &mbar[g & 1]);
    unsigned char* dst = st + SM::h_bytes(Qp);
    if constexpr (!FWD) {
      bulk_g2s(dst, Din + (size_t)row0 * Qp, (unsigned)SM::d_bytes(Qp), &mbar[g & 1]);
    } else {
#pragma unroll
      for (int s = 0; s < R; ++s)
        bulk_g2s(dst + (size_t)s * NRT * sizeof(Acc), Din + (size_t)(row0 + s) * p.Gs + r0,
                 (unsigned)(ncopy * sizeof(Acc)), &mbar[g & 1]);
    }
    unsigned char* ldst = st + SM::h_bytes(Qp) + SM::d_bytes(Qp);
#pragma unroll
    for (int s = 0; s < R; ++s)
      bulk_g2s(ldst + (size_t)s * NRT * sizeof(Real), lamh + (size_t)(row0 + s) * p.Ls + r0,
               (unsigned)(nlam * sizeof(Real)), &mbar[g & 1]);
  };
  // zero both stages once: columns beyond a copy's extent then read as zeros
  for (size_t x = tid * 16; x < 2 * SM::stage_bytes(Qp); x += (size_t)Cfg::NT * 16)
    *reinterpret_cast<uint4*>(stage_base + x) = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    issue(0);
    if (ngroups > 1) issue(1);
  }

  int grp = 0;      // current group
  int mgrp = mtop;  // m of the first step of the current group
  const Real* Hs = nullptr;
  const Acc* Ds = nullptr;
  const Real* Ls_ = nullptr;

  // reduction + renormalisation, every R steps (and at the end)
  auto flush = [&](int nsteps) {
    __syncthreads();
    if constexpr (!FWD) {
      // buf [s][i][qt][ql] (row stride QA+1) -> sum over ql
      const int items = R * T * QT;
      for (int o = tid; o < items; o += Cfg::NT) {
        const int s = o / (T * QT);
        const int rem = o % (T * QT);
        const int i = rem / QT;
        const int qq = rem % QT;
        if (s >= nsteps) continue;
        const int m = mgrp - s;
        const int r = r0 + qq * T + i;
        if (m < 0 || m >= L || r >= p.nrings) continue;
        const Acc* row = buf + ((s * T + i) * QT + qq) * (QA + 1);
        Acc a = zero_acc<Acc>();
#pragma unroll 4
        for (int x = 0; x < QA; ++x) acc_add(a, row[x]);
        using R2 = typename Cfg::R2;
        R2* ftm = reinterpret_cast<R2*>(p.out) + ((size_t)b * p.nrows + p.ring_row[r]) * p.ncol;
        const int mo = p.mo;
        if constexpr (DUAL) {
          R2 ap, an;
          ap.x = a.x;
          ap.y = a.y;
          an.x = a.z;
          an.y = a.w;
          red_add(ftm + (L - 1 + m + mo), ap);
          if (m > 0) red_add(ftm + (L - 1 - m + mo), an);
        } else {
          R2 ap;
          ap.x = a.x;
          ap.y = a.y;
          if (half == 0)
            red_add(ftm + (L - 1 + m + mo), ap);
          else if (m > 0)
            red_add(ftm + (L - 1 - m + mo), ap);
        }
      }
    } else {
      // buf [s][k][qt][ql] -> sum over qt; out acc [b][half][j][m][Qp]
      const int items = R * K * QA;
      for (int o = tid; o < items; o += Cfg::NT) {
        const int s = o / (K * QA);
        const int rem = o % (K * QA);
        const int k = rem / QA;
        const int x = rem % QA;
        if (s >= nsteps) continue;
        const int m = mgrp - s;
        const int q = x + QA * k;
        const int l = j + C * q;
        if (m < 0 || m >= L || l >= L || l < m) continue;
        Acc a = zero_acc<Acc>();
#pragma unroll 4
        for (int y = 0; y < QT; ++y) acc_add(a, buf[((s * K + k) * QT + y) * QA + x]);
        Acc* out = reinterpret_cast<Acc*>(p.out) +
                   ((((size_t)b * p.nhalf + half) * C + j) * L + m) * Qp + q;
        red_add(out, a);
      }
    }
    __syncthreads();
    // renormalise states whose mantissa grew past the trigger
    Real mx = Real(0);
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int i = 0; i < T; ++i) mx = fmax(mx, fabs(v[k][i]));
    const Real trig = Scaling<Real>::kTrig;
    if (mx > trig) {
      const Real down = Scaling<Real>::kDown;
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int i = 0; i < T; ++i)
          if (fabs(v[k][i]) > trig) {
            v[k][i] *= down;
            w[k][i] *= down;
            const int e = ex_get(k, i) + 1;
            ex_set(k, i, e);
            sc[k][i] = e >= 0 ? Real(1) : Real(0);
          }
    }
  };

  // one recursion step at m (S = step index inside the group, compile-time);
  // CUR holds dt_m, PRV holds dt_{m+1} and receives dt_{m-1}
#define S2B_STEP(CUR, PRV, KC, S)                                                      \
  {                                                                                    \
    constexpr int srow = R - 1 - (S);                                                  \
    const Real* Hrow = Hs + srow * Qp;                                                 \
    Real lam[T];                                                                       \
    _Pragma("unroll") for (int i = 0; i < T; ++i) lam[i] = Ls_[srow * NRT + qt * T + i]; \
    Acc accT[T];                                                                       \
    Acc gin[T];                                                                        \
    if constexpr (FWD) {                                                               \
      const Acc* Grow = Ds + srow * NRT + qt * T;                                      \
      _Pragma("unroll") for (int i = 0; i < T; ++i) gin[i] = Grow[i];                  \
    } else {                                                                           \
      _Pragma("unroll") for (int i = 0; i < T; ++i) accT[i] = zero_acc<Acc>();         \
    }                                                                                  \
    if (rem == 0) {                                                                    \
      /* CTA-uniform: some lane's slot KC reaches l == m on this step */              \
      if (lkc == m) {                                                                  \
        _Pragma("unroll") for (int i = 0; i < T; ++i) {                                \
          const SeedT<Real> sd = seed_sm[tid * T + i];                                 \
          CUR[KC][i] = sd.v;                                                           \
          PRV[KC][i] = Real(0);                                                        \
          ex_set(KC, i, sd.e);                                                         \
          sc[KC][i] = sd.e >= 0 ? Real(1) : Real(0);                                   \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
    _Pragma("unroll") for (int k = KC; k < K; ++k) {                                   \
      const int q = ql + QA * k;                                                       \
      const Real h = Hrow[q];                                                          \
      Acc fk;                                                                          \
      if constexpr (!FWD) fk = Ds[srow * Qp + q];                                      \
      Acc accK = zero_acc<Acc>();                                                      \
      _Pragma("unroll") for (int i = 0; i < T; ++i) {                                  \
        const Real x = CUR[k][i] * sc[k][i];                                           \
        if constexpr (!FWD)                                                            \
          acc_fma(accT[i], x, fk);                                                     \
        else                                                                           \
          acc_fma(accK, x, gin[i]);                                                    \
        PRV[k][i] = fma(lam[i] * h, CUR[k][i], -PRV[k][i]);                            \
      }                                                                                \
      if constexpr (FWD) buf[((srow_b(S) * K + k) * QT + qt) * QA + ql] = accK;        \
    }                                                                                  \
    if constexpr (!FWD) {                                                              \
      _Pragma("unroll") for (int i = 0; i < T; ++i)                                    \
          buf[((srow_b(S) * T + i) * QT + qt) * (QA + 1) + ql] = accT[i];              \
    }                                                                                  \
    --m;                                                                               \
    rem = rem == 0 ? C - 1 : rem - 1;                                                  \
  }
#define srow_b(S) (S)

  int m = mtop;
  int rem = (mtop - j) % C;  // (m - j) mod C; activation possible only when 0
#pragma unroll
  for (int kc = K - 1; kc >= 0; --kc) {
    if (kc > ktop) continue;
    // seeds of slot kc for this thread (activated when m reaches l)
    const int qkc = ql + QA * kc;
    const int lkc = j + C * qkc;
#pragma unroll
    for (int i = 0; i < T; ++i) {
      SeedT<Real> sd{Real(0), 0};
      if (lkc < L && rbase + i < p.nrings) sd = seeds[(size_t)qkc * p.nrings + rbase + i];
      seed_sm[tid * T + i] = sd;  // thread-private slot
    }
    const int lo = clo(kc);
    while (m >= lo) {
      // one reduction group of R steps per iteration
      const bool ok = mbar_wait(&mbar[grp & 1], (grp >> 1) & 1);
      if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicExch(p.status, 1);
        return;
      }
      {
        unsigned char* st = stage_base + (size_t)(grp & 1) * SM::stage_bytes(Qp);
        Hs = reinterpret_cast<const Real*>(st);
        Ds = reinterpret_cast<const Acc*>(st + SM::h_bytes(Qp));
        Ls_ = reinterpret_cast<const Real*>(st + SM::h_bytes(Qp) + SM::d_bytes(Qp));
      }
      static_assert(R == 4, "the group body below is written for R = 4");
      S2B_STEP(v, w, kc, 0)
      S2B_STEP(w, v, kc, 1)
      S2B_STEP(v, w, kc, 2)
      S2B_STEP(w, v, kc, 3)
      flush(R);
      mgrp = m;
      ++grp;
      if (tid == 0 && grp + 1 < ngroups) issue(grp + 1);
    }
  }
#undef srow_b
#undef S2B_STEP
}

// ---------------------------------------------------------------------------
// launch configuration
// ---------------------------------------------------------------------------
constexpr int kQA = 16, kQT = 8, kK = 4, kR = 4;

int lat_nclass(bool fp64, int L) {
  (void)fp64;
  const int per = kQA * kK;
  return (L + per - 1) / per;
}

int lat_qp(bool fp64, int L) {
  (void)fp64;
  (void)L;
  return kQA * kK;  // fixed row width: every slot load of the kernel stays inside the row
}

template <typename Real, bool FWD, bool DUAL, int T, int K, int QA, int QT, int R>
static cudaError_t launch_cfg(const LatParams& p0, cudaStream_t s) {
  using Cfg = LatCfg<Real, FWD, DUAL, T, K, QA, QT, R>;
  using SM = LatSmem<Real, typename Cfg::Acc, FWD, T, K, QA, QT, R>;
  LatParams p = p0;
  p.nclass = lat_nclass(sizeof(Real) == 8, p.L);
  p.Qp = lat_qp(sizeof(Real) == 8, p.L);
  const size_t smem = SM::total(p.Qp);
  auto kern = lat_kernel<Real, FWD, DUAL, T, K, QA, QT, R>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  dim3 grid((p.nrings + QT * T - 1) / (QT * T), p.nclass, p.nhalf * p.batch);
  kern<<<grid, Cfg::NT, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_latitudinal(bool fp64, bool forward, bool dual, const LatParams& p,
                               cudaStream_t s) {
  if (!fp64) {
    if (!forward)
      return dual ? launch_cfg<float, false, true, 4, kK, kQA, kQT, kR>(p, s)
                  : launch_cfg<float, false, false, 4, kK, kQA, kQT, kR>(p, s);
    return dual ? launch_cfg<float, true, true, 4, kK, kQA, kQT, kR>(p, s)
                : launch_cfg<float, true, false, 4, kK, kQA, kQT, kR>(p, s);
  }
  if (!forward)
    return dual ? launch_cfg<double, false, true, 2, kK, kQA, kQT, kR>(p, s)
                : launch_cfg<double, false, false, 2, kK, kQA, kQT, kR>(p, s);
  return dual ? launch_cfg<double, true, true, 2, kK, kQA, kQT, kR>(p, s)
              : launch_cfg<double, true, false, 2, kK, kQA, kQT, kR>(p, s);
}

cudaError_t launch_seeds(bool fp64, int L, int L0, int spin, int nhalf, const RingInfo* rings,
                         int nrings, const double* lbin, void* seeds, cudaStream_t s) {
  const int C = lat_nclass(fp64, L);
  const int Qp = lat_qp(fp64, L);
  const long total = (long)nhalf * C * Qp * nrings;
  const int threads = 256;
  long blocks = (total + threads - 1) / threads;
  if (blocks > 4096) blocks = 4096;
  if (blocks < 1) blocks = 1;
  if (fp64)
    seed_kernel<double><<<(int)blocks, threads, 0, s>>>(L, L0, spin, nhalf, C, Qp, rings, nrings,
                                                        lbin, reinterpret_cast<SeedT<double>*>(seeds));
  else
    seed_kernel<float><<<(int)blocks, threads, 0, s>>>(L, L0, spin, nhalf, C, Qp, rings, nrings,
                                                       lbin, reinterpret_cast<SeedT<float>*>(seeds));
  return cudaGetLastError();
}

cudaError_t launch_lambda(bool fp64, int L, int spin, int nhalf, const RingInfo* rings, int nrings,
                          int Ls, void* lam, cudaStream_t s) {
  const long total = (long)nhalf * tab_rows(L) * Ls;
  long blocks = (total + 255) / 256;
  if (blocks > 8192) blocks = 8192;
  if (fp64)
    lambda_kernel<double><<<(int)blocks, 256, 0, s>>>(L, spin, nhalf, rings, nrings, Ls, (double*)lam);
  else
    lambda_kernel<float><<<(int)blocks, 256, 0, s>>>(L, spin, nhalf, rings, nrings, Ls, (float*)lam);
  return cudaGetLastError();
}

size_t seed_bytes(bool fp64, int L, int nhalf, int nrings) {
  const int C = lat_nclass(fp64, L);
  const int Qp = lat_qp(fp64, L);
  return (size_t)nhalf * C * Qp * nrings * (fp64 ? sizeof(SeedT<double>) : sizeof(SeedT<float>));
}

}  // namespace s2b
