// Precompute-kernel path: build the Wigner-d kernel table on the device and
// contract it against ring spectra.
//
// Table (the upstream layout, s2fft/precompute_transforms/construct.py:16-161):
//   K[t][l][mi] = d^l_{m,-s}(theta_t) sqrt((2l+1)/4pi) [x w_t if forward]
//                 [x exp(-+i m phi0_t) for HEALPix], m = m0 + mi,
// m0 = 0 when reality (spin 0) else -(L-1). Real for equiangular samplings,
// complex (interleaved) for HEALPix.
//
// Construction: one thread per (ring, l) runs the three-term recursion in m in
// double (from the edge m = +-l inwards, both halves, spin n = -s and the
// d^l_{-m,n} = (-1)^(m-n) d^l_{m,-n} symmetry), with a scaled exponent so the
// polar seeds do not underflow; rows of K are written contiguously in m.
// Pole rings use the closed forms d^l_{m,n}(0) = delta_{m,n},
// d^l_{m,n}(pi) = (-1)^(l-n) delta_{m,-n}.
//
// Contractions (s2fft/precompute_transforms/spherical.py:87-149, 314-380):
//   inverse: ftm[b][t][m] = (-1)^s sum_l K[t][l][m] flm[b][l][m]
//   forward: flm[b][l][m] = (-1)^s sum_t K[t][l][m] ftm[b][t][m]
// streamed so that every K element is read from HBM once per group of maps.
#include <cuda_runtime.h>

#include <type_traits>

#include "s2b_degree.h"
#include "s2b_precompute.h"

namespace s2b {

template <typename Real>
using P2 = std::conditional_t<sizeof(Real) == 4, float2, double2>;

static int pgrid(long n, int threads) {
  long b = (n + threads - 1) / threads;
  if (b > 1048576) b = 1048576;
  return b < 1 ? 1 : (int)b;
}

// ---------------------------------------------------------------------------
// table construction
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void kernel_table_kernel(KernelTableParams p) {
  const long total = (long)p.nth * p.L;
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int t = (int)(idx / p.L);
  const int l = (int)(idx % p.L);
  const int L = p.L;
  const int s = p.spin;
  const int as = s < 0 ? -s : s;
  const double th = p.theta[t];
  const double nl = sqrt((2.0 * l + 1.0) / (4.0 * 3.141592653589793));
  const double w = p.weights ? p.weights[t] : 1.0;
  const int m0 = p.reality ? 0 : -(L - 1);
  const int M = L - m0;
  Real* rowr = nullptr;
  P2<Real>* rowc = nullptr;
  if (p.complex_out)
    rowc = reinterpret_cast<P2<Real>*>(p.out) + ((size_t)t * L + l) * M;
  else
    rowr = reinterpret_cast<Real*>(p.out) + ((size_t)t * L + l) * M;
  auto store = [&](int m, double d) {
    const int mi = m - m0;
    if (mi < 0 || mi >= M) return;
    const double v = d * nl * w;
    if (p.complex_out) {
      double sn = 0.0, cs = 1.0;
      if (p.phi0) sincos((p.forward ? -1.0 : 1.0) * (double)m * p.phi0[t], &sn, &cs);
      P2<Real> o;
      o.x = (Real)(v * cs);
      o.y = (Real)(v * sn);
      rowc[mi] = o;
    } else {
      rowr[mi] = (Real)v;
    }
  };
  // zero the row first (entries with |m| > l, l < |s| stay zero)
  for (int mi = 0; mi < M; ++mi) {
    if (p.complex_out) {
      P2<Real> z;
      z.x = 0;
      z.y = 0;
      rowc[mi] = z;
    } else {
      rowr[mi] = Real(0);
    }
  }
  if (l < as) return;
  const bool north = th < 1e-12, south = th > 3.141592653589793 - 1e-12;
  if (north) {  // d^l_{m,-s}(0) = delta_{m,-s}
    store(-s, 1.0);
    return;
  }
  if (south) {  // d^l_{m,-s}(pi) = (-1)^(l+s) delta_{m,s}
    store(s, ((l + s) & 1) ? -1.0 : 1.0);
    return;
  }
  const double c = cos(th), sn = sin(th);
  const double lc = log2(cos(th / 2.0)), ls = log2(sin(th / 2.0));
  const double lb = p.lbin[l];
  constexpr double kS = 800.0, kTh = 0x1p400, kDn = 0x1p-800, kSig = -200.0;
  for (int half = 0; half < 2; ++half) {
    if (p.reality && half == 1) break;
    const int n = half == 0 ? -s : s;  // recursion for d^l_{m,n}, m from l down
    // seed d^l_{l,n}
    const double lg = lb + (double)(l + n) * lc + (double)(l - n) * ls;
    int e = 0;
    if (lg < kSig) e = -(int)ceil((kSig - lg) / kS);
    double v = ((((l - n) & 1) ? -1.0 : 1.0)) * exp2(lg - kS * (double)e);
    double wv = 0.0;  // d_{m+1}
    const int mlast = half == 0 ? 0 : 1;
    for (int m = l; m >= mlast; --m) {
      const double val = e == 0 ? v : 0.0;
      if (half == 0)
        store(m, val);
      else  // d^l_{-m,-s} = (-1)^(m+s) d^l_{m,s}
        store(-m, (((m + s) % 2 + 2) % 2 ? -1.0 : 1.0) * val);
      if (m == mlast) break;
      // d_{m-1} = (lambda d_m - f_{m+1} d_{m+1}) / f_m
      const double lam = 2.0 * ((double)n - (double)m * c) / sn;
      const double fm = sqrt((double)(l + m) * (double)(l - m + 1));
      const double fp = sqrt((double)(l + m + 1) * (double)(l - m));
      const double nv = (lam * v - fp * wv) / fm;
      wv = v;
      v = nv;
      if (fabs(v) > kTh && e < 0) {
        v *= kDn;
        wv *= kDn;
        e += 1;
      }
    }
  }
}

// Orders |m| < |s| of the table by the degree recursion (s2b_degree.h): the m-recursion
// above runs, on rings with n cos(theta) > 0, through a range below m = n cos(theta) where
// d^l_{m,n} decays as m decreases and loses digits there; that range lies inside |m| < |s|.
// One thread per (ring, half, order) overwrites those entries for every l (poles keep
// their closed forms).
template <typename Real>
__global__ void kernel_table_lowm_kernel(KernelTableParams p) {
  const int as = p.spin < 0 ? -p.spin : p.spin;
  const long total = (long)p.nth * 2 * as;
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int t = (int)(idx / (2 * as));
  const int half = (int)((idx / as) % 2);
  const int m = (int)(idx % as);
  if (half == 1 && (m == 0 || p.reality)) return;  // order 0 and m >= 0 tables: half 0 only
  const int L = p.L, s = p.spin;
  const double th = p.theta[t];
  if (th < 1e-12 || th > 3.141592653589793 - 1e-12) return;
  const int n = half == 0 ? -s : s;
  const int col = half == 0 ? m : -m;  // d^l_{-m,-s} = (-1)^(m+s) d^l_{m,s}
  const double sgn = (half == 1 && ((m + s) % 2 + 2) % 2) ? -1.0 : 1.0;
  const double w = p.weights ? p.weights[t] : 1.0;
  const int m0 = p.reality ? 0 : -(L - 1);
  const int M = L - m0;
  const int mi = col - m0;
  if (mi < 0 || mi >= M) return;
  double ph_c = 1.0, ph_s = 0.0;
  if (p.complex_out && p.phi0) sincos((p.forward ? -1.0 : 1.0) * (double)col * p.phi0[t], &ph_s, &ph_c);
  const double ct = cos(th);
  double cur, prv = 0.0;
  int E;
  degree_seed(log2(cos(th / 2.0)), log2(sin(th / 2.0)), m, n, cur, E);
  double sc = ldexp(1.0, E);
  for (int l = as; l < L; ++l) {
    const double v = sgn * cur * sc * sqrt((2.0 * l + 1.0) / (4.0 * 3.141592653589793)) * w;
    const size_t at = ((size_t)t * L + l) * M + mi;
    if (p.complex_out) {
      P2<Real> o;
      o.x = (Real)(v * ph_c);
      o.y = (Real)(v * ph_s);
      reinterpret_cast<P2<Real>*>(p.out)[at] = o;
    } else {
      reinterpret_cast<Real*>(p.out)[at] = (Real)v;
    }
    if (l + 1 < L) {
      const DegreeCoef k = degree_coef(l, m, n);
      degree_step(k.a, k.c, k.b, ct, cur, prv, E, sc);
    }
  }
}

// ---------------------------------------------------------------------------
// streaming contractions; threads run along mi (contiguous in K and in the data).
// Register tiles: each thread owns RT rows of the output (t for the inverse, l
// for the forward) for BB maps, so every data element loaded is reused RT times
// and every K element BB times. Accumulation in the plan precision.
// ---------------------------------------------------------------------------
// Register tile: RT output rows (t for the inverse, l for the forward) x BB maps per thread.
template <typename Real>
struct PreTile {
  static constexpr int RT = sizeof(Real) == 4 ? 8 : 4;
  static constexpr int BB = sizeof(Real) == 4 ? 8 : 4;
  static constexpr int LANES = 64;  // columns mi per CTA
};

// Row tiles run along blockIdx.x and map tiles along blockIdx.y, so the CTAs resident at
// one time cover every row and map tile of one or two column blocks (blockIdx.z): the K
// columns and data columns of the block stay in L2 and come from DRAM about once. The
// loads of two summation indices are issued ahead of their arithmetic.
//
// FWD = false (inverse): out[b][t][mo + mi] = sgn * sum_l K[t][l][mi] in[b][l][mshift + mi]
// FWD = true (forward):  out[b][l][mshift + mi] = sgn * sum_t K[t][l][mi] in[b][t][mi]
template <typename Real, bool CPLX, bool FWD>
__global__ void pre_contract_kernel(PreContractParams p) {
  using C = P2<Real>;
  constexpr int RT = PreTile<Real>::RT, BB = PreTile<Real>::BB;
  const int M = p.M;
  const int mi = blockIdx.z * blockDim.x + threadIdx.x;
  const int r0 = blockIdx.x * RT;
  const int b0 = blockIdx.y * BB;
  if (mi >= M) return;
  const int L = p.L;
  const int nrow = FWD ? L : p.nth;   // output rows
  const int nsum = FWD ? p.nth : L;   // summation length
  Real ar[RT][BB], ai[RT][BB];
#pragma unroll
  for (int r = 0; r < RT; ++r)
#pragma unroll
    for (int x = 0; x < BB; ++x) ar[r][x] = ai[r][x] = Real(0);
  const C* in = reinterpret_cast<const C*>(p.in);
  // data element (map x, summation index q) and kernel element (row r, index q)
  auto dat = [&](int x, int q) -> C {
    const int b = min(b0 + x, p.batch - 1);
    return FWD ? in[((size_t)b * p.nth + q) * M + mi]
               : in[((size_t)b * L + q) * (2 * L - 1) + p.mshift + mi];
  };
  auto ker = [&](int r, int q) -> C {
    const int row = min(r0 + r, nrow - 1);
    const size_t o = FWD ? ((size_t)q * L + row) * M + mi : ((size_t)row * L + q) * M + mi;
    C k;
    if (CPLX) {
      k = reinterpret_cast<const C*>(p.K)[o];
      if (p.conj) k.y = -k.y;
    } else {
      k.x = reinterpret_cast<const Real*>(p.K)[o];
      k.y = Real(0);
    }
    return k;
  };
  int q = 0;
  for (; q + 1 < nsum; q += 2) {
    C f[2][BB], k[2][RT];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
#pragma unroll
      for (int x = 0; x < BB; ++x) f[u][x] = dat(x, q + u);
#pragma unroll
      for (int r = 0; r < RT; ++r) k[u][r] = ker(r, q + u);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int r = 0; r < RT; ++r)
#pragma unroll
        for (int x = 0; x < BB; ++x) {
          ar[r][x] = fma(k[u][r].x, f[u][x].x, ar[r][x]);
          ai[r][x] = fma(k[u][r].x, f[u][x].y, ai[r][x]);
          if (CPLX) {
            ar[r][x] = fma(-k[u][r].y, f[u][x].y, ar[r][x]);
            ai[r][x] = fma(k[u][r].y, f[u][x].x, ai[r][x]);
          }
        }
  }
  for (; q < nsum; ++q) {
#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const C k = ker(r, q);
#pragma unroll
      for (int x = 0; x < BB; ++x) {
        const C f = dat(x, q);
        ar[r][x] = fma(k.x, f.x, ar[r][x]);
        ai[r][x] = fma(k.x, f.y, ai[r][x]);
        if (CPLX) {
          ar[r][x] = fma(-k.y, f.y, ar[r][x]);
          ai[r][x] = fma(k.y, f.x, ai[r][x]);
        }
      }
    }
  }
  C* out = reinterpret_cast<C*>(p.out);
#pragma unroll
  for (int r = 0; r < RT; ++r) {
    const int row = r0 + r;
    if (row >= nrow) break;
#pragma unroll
    for (int x = 0; x < BB; ++x) {
      if (b0 + x >= p.batch) break;
      C o;
      o.x = (Real)(p.sign * ar[r][x]);
      o.y = (Real)(p.sign * ai[r][x]);
      if (FWD)
        out[((size_t)(b0 + x) * L + row) * (2 * L - 1) + p.mshift + mi] = o;
      else
        out[((size_t)(b0 + x) * p.nth + row) * p.ncol + p.mo + mi] = o;
    }
  }
}

// Batched contraction (batch >= kGemmMinBatch): for every column mi an independent GEMM
// (rows x maps, summed over q), computed by CTAs that own 8 consecutive columns, a tile of
// 32 rows and a tile of 32 (float) or 16 (double) maps. Chunks of Q summation
// indices of K and of the data are staged in shared memory with coalesced loads (the 8
// columns of a row are one 32-byte sector of K) and prefetched into registers while the
// previous chunk is consumed. Thread (column c, row group rg, map group bg) keeps 4 rows x
// BT maps of complex sums and reads them from shared memory with 16-byte loads.
constexpr int kGemmMinBatch = 16;
constexpr int kGemmMI = 8;      // columns per CTA
constexpr int kGemmRows = 32;   // rows per CTA (8 row groups x 4)

template <typename Real>
struct GemmTile {
  static constexpr int BT = sizeof(Real) == 4 ? 8 : 4;  // maps per thread
  static constexpr int MAPS = 4 * BT;                    // maps per CTA (4 map groups)
};

// n consecutive Real from 16-byte aligned shared memory by 16-byte loads
template <int N, typename Real>
__device__ __forceinline__ void lds_vec(Real (&dst)[N], const Real* src) {
  if constexpr (sizeof(Real) == 4) {
    static_assert(N % 4 == 0, "float vectors of 4");
#pragma unroll
    for (int i = 0; i < N / 4; ++i) {
      const float4 v = reinterpret_cast<const float4*>(src)[i];
      dst[4 * i] = v.x;
      dst[4 * i + 1] = v.y;
      dst[4 * i + 2] = v.z;
      dst[4 * i + 3] = v.w;
    }
  } else {
    static_assert(N % 2 == 0, "double vectors of 2");
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const double2 v = reinterpret_cast<const double2*>(src)[i];
      dst[2 * i] = v.x;
      dst[2 * i + 1] = v.y;
    }
  }
}

template <typename Real, bool CPLX, bool FWD>
__global__ void __launch_bounds__(256, sizeof(Real) == 8 ? 2 : 1) pre_gemm_kernel(PreContractParams p) {
  using C = P2<Real>;
  using KT = std::conditional_t<CPLX, C, Real>;
  constexpr int BT = GemmTile<Real>::BT, MAPS = GemmTile<Real>::MAPS;
  constexpr int kGemmQ = sizeof(Real) == 8 ? 4 : 8;  // summation indices per chunk (<= 48 KB)
  constexpr int KW = CPLX ? 2 : 1;                    // Real per K entry
  constexpr int PAD = 16 / (int)sizeof(Real);         // 16 bytes: rows of a warp phase
  constexpr int KS = kGemmRows * KW + PAD;            //   start on distinct bank groups
  constexpr int DS = MAPS * 2 + PAD;
  constexpr int NK = kGemmQ * kGemmRows * kGemmMI;    // K entries per chunk
  constexpr int ND = kGemmQ * MAPS * kGemmMI;         // data entries per chunk
  constexpr int KPT = NK / 256, DPT = ND / 256;       // per thread
  // [q][column][rows] and [q][column][maps (re, im)]: a thread reads its 4 rows and BT maps
  // of one column with 16-byte loads
  __shared__ __align__(16) Real Ks[kGemmQ][kGemmMI][KS];
  __shared__ __align__(16) Real Ds[kGemmQ][kGemmMI][DS];
  const int tid = threadIdx.x;
  const int c = tid & 7, rg = (tid >> 3) & 7, bg = tid >> 6;
  const int L = p.L, M = p.M;
  const int nrow = FWD ? L : p.nth;
  const int nsum = FWD ? p.nth : L;
  const int row0 = blockIdx.x * kGemmRows;
  const int b0 = blockIdx.y * MAPS;
  const int mi0 = blockIdx.z * kGemmMI;

  // chunk loaders: element e of the chunk -> (q, row or map, column), column fastest
  auto kload = [&](int q0, int e) -> KT {
    const int cc = e & 7, rr = (e >> 3) % kGemmRows, qq = e / (8 * kGemmRows);
    const int q = q0 + qq, row = row0 + rr, mi = mi0 + cc;
    KT v{};
    if (q < nsum && row < nrow && mi < M) {
      const size_t o = FWD ? ((size_t)q * L + row) * M + mi : ((size_t)row * L + q) * M + mi;
      v = reinterpret_cast<const KT*>(p.K)[o];
      if constexpr (CPLX) {
        if (p.conj) v.y = -v.y;
      }
    }
    return v;
  };
  auto dload = [&](int q0, int e) -> C {
    const int cc = e & 7, bb = (e >> 3) % MAPS, qq = e / (8 * MAPS);
    const int q = q0 + qq, b = b0 + bb, mi = mi0 + cc;
    C v;
    v.x = v.y = Real(0);
    if (q < nsum && b < p.batch && mi < M) {
      const C* in = reinterpret_cast<const C*>(p.in);
      v = FWD ? in[((size_t)b * p.nth + q) * M + mi]
              : in[((size_t)b * L + q) * (2 * L - 1) + p.mshift + mi];
    }
    return v;
  };

  Real ar[4][BT], ai[4][BT];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int x = 0; x < BT; ++x) ar[r][x] = ai[r][x] = Real(0);

  KT kreg[KPT];
  C dreg[DPT];
#pragma unroll
  for (int i = 0; i < KPT; ++i) kreg[i] = kload(0, tid + i * 256);
#pragma unroll
  for (int i = 0; i < DPT; ++i) dreg[i] = dload(0, tid + i * 256);

  for (int q0 = 0; q0 < nsum; q0 += kGemmQ) {
    __syncthreads();  // the previous chunk is consumed
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const int e = tid + i * 256;
      Real* dst = &Ks[e / (8 * kGemmRows)][e & 7][((e >> 3) % kGemmRows) * KW];
      if constexpr (CPLX) {
        dst[0] = kreg[i].x;
        dst[1] = kreg[i].y;
      } else {
        dst[0] = kreg[i];
      }
    }
#pragma unroll
    for (int i = 0; i < DPT; ++i) {
      const int e = tid + i * 256;
      Real* dst = &Ds[e / (8 * MAPS)][e & 7][((e >> 3) % MAPS) * 2];
      dst[0] = dreg[i].x;
      dst[1] = dreg[i].y;
    }
    __syncthreads();
    if (q0 + kGemmQ < nsum) {  // prefetch the next chunk
#pragma unroll
      for (int i = 0; i < KPT; ++i) kreg[i] = kload(q0 + kGemmQ, tid + i * 256);
#pragma unroll
      for (int i = 0; i < DPT; ++i) dreg[i] = dload(q0 + kGemmQ, tid + i * 256);
    }
#pragma unroll 2
    for (int qq = 0; qq < kGemmQ; ++qq) {
      Real k[4 * KW], d[2 * BT];
      lds_vec(k, &Ks[qq][c][rg * 4 * KW]);
      lds_vec(d, &Ds[qq][c][bg * BT * 2]);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int x = 0; x < BT; ++x) {
          const Real kr = k[r * KW];
          ar[r][x] = fma(kr, d[2 * x], ar[r][x]);
          ai[r][x] = fma(kr, d[2 * x + 1], ai[r][x]);
          if constexpr (CPLX) {
            const Real ki = k[r * KW + 1];
            ar[r][x] = fma(-ki, d[2 * x + 1], ar[r][x]);
            ai[r][x] = fma(ki, d[2 * x], ai[r][x]);
          }
        }
    }
  }

  const int mi = mi0 + c;
  if (mi >= M) return;
  C* out = reinterpret_cast<C*>(p.out);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int row = row0 + rg * 4 + r;
    if (row >= nrow) break;
#pragma unroll
    for (int x = 0; x < BT; ++x) {
      const int b = b0 + bg * BT + x;
      if (b >= p.batch) break;
      C o;
      o.x = (Real)(p.sign * ar[r][x]);
      o.y = (Real)(p.sign * ai[r][x]);
      if (FWD)
        out[((size_t)b * L + row) * (2 * L - 1) + p.mshift + mi] = o;
      else
        out[((size_t)b * p.nth + row) * p.ncol + p.mo + mi] = o;
    }
  }
}

// reality mirror flm[b][l][L-1-m] = (-1)^m conj(flm[b][l][L-1+m]), m >= 1
template <typename Real>
__global__ void reality_mirror_kernel(void* flm, int B, int L) {
  using C = P2<Real>;
  const long total = (long)B * L * (L - 1);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int m = 1 + (int)(i % (L - 1));
    const long bl = i / (L - 1);
    C* row = reinterpret_cast<C*>(flm) + bl * (2 * L - 1);
    C v = row[L - 1 + m];
    const Real sg = (m & 1) ? Real(-1) : Real(1);
    C o;
    o.x = sg * v.x;
    o.y = -sg * v.y;
    row[L - 1 - m] = o;
  }
}

cudaError_t launch_kernel_table(bool fp64, const KernelTableParams& p, cudaStream_t s) {
  const long total = (long)p.nth * p.L;
  if (fp64)
    kernel_table_kernel<double><<<pgrid(total, 128), 128, 0, s>>>(p);
  else
    kernel_table_kernel<float><<<pgrid(total, 128), 128, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || p.spin == 0) return e;
  const long low = (long)p.nth * 2 * (p.spin < 0 ? -p.spin : p.spin);
  if (fp64)
    kernel_table_lowm_kernel<double><<<pgrid(low, 128), 128, 0, s>>>(p);
  else
    kernel_table_lowm_kernel<float><<<pgrid(low, 128), 128, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_pre_contract(bool fp64, bool forward, bool cplx, const PreContractParams& p,
                                cudaStream_t s) {
  const int nrow = forward ? p.L : p.nth;
  if (p.batch >= kGemmMinBatch) {
    const int maps = fp64 ? GemmTile<double>::MAPS : GemmTile<float>::MAPS;
    dim3 g((nrow + kGemmRows - 1) / kGemmRows, (p.batch + maps - 1) / maps,
           (p.M + kGemmMI - 1) / kGemmMI);
    if (g.y > 65535 || g.z > 65535) return cudaErrorInvalidConfiguration;
#define S2B_GEMM(R, C)                                                     \
  if (forward)                                                             \
    pre_gemm_kernel<R, C, true><<<g, 256, 0, s>>>(p);                      \
  else                                                                     \
    pre_gemm_kernel<R, C, false><<<g, 256, 0, s>>>(p);
    if (fp64) {
      if (cplx) {
        S2B_GEMM(double, true)
      } else {
        S2B_GEMM(double, false)
      }
    } else {
      if (cplx) {
        S2B_GEMM(float, true)
      } else {
        S2B_GEMM(float, false)
      }
    }
#undef S2B_GEMM
    return cudaGetLastError();
  }
  const int threads = fp64 ? PreTile<double>::LANES : PreTile<float>::LANES;
  const int RT = fp64 ? PreTile<double>::RT : PreTile<float>::RT;
  const int BB = fp64 ? PreTile<double>::BB : PreTile<float>::BB;
  dim3 grid((nrow + RT - 1) / RT, (p.batch + BB - 1) / BB, (p.M + threads - 1) / threads);
  if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidConfiguration;
#define S2B_LAUNCH(R, C)                                                   \
  if (forward)                                                             \
    pre_contract_kernel<R, C, true><<<grid, threads, 0, s>>>(p);           \
  else                                                                     \
    pre_contract_kernel<R, C, false><<<grid, threads, 0, s>>>(p);
  if (fp64) {
    if (cplx) {
      S2B_LAUNCH(double, true)
    } else {
      S2B_LAUNCH(double, false)
    }
  } else {
    if (cplx) {
      S2B_LAUNCH(float, true)
    } else {
      S2B_LAUNCH(float, false)
    }
  }
#undef S2B_LAUNCH
  return cudaGetLastError();
}

cudaError_t launch_reality_mirror(bool fp64, void* flm, int B, int L, cudaStream_t s) {
  if (L < 2) return cudaSuccess;
  const long total = (long)B * L * (L - 1);
  if (fp64)
    reality_mirror_kernel<double><<<pgrid(total, 256) > 65535 ? 65535 : pgrid(total, 256), 256, 0, s>>>(flm, B, L);
  else
    reality_mirror_kernel<float><<<pgrid(total, 256) > 65535 ? 65535 : pgrid(total, 256), 256, 0, s>>>(flm, B, L);
  return cudaGetLastError();
}

}  // namespace s2b
