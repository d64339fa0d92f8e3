// Host side of the C ABI: plan construction and execution order.
//
// A plan holds every table a transform needs, computed once in double on the
// host and uploaded (the role of upstream's precomps / generate_precomputes_jax,
// s2fft/recursions/price_mcewen.py:118-255, and of the cuFFT plan cache,
// lib/src/plan_cache.cc:12-50): ring colatitudes and quadrature weights
// (s2fft/sampling/s2_samples.py:203-308, s2fft/utils/quadrature.py:7-320),
// monic recursion coefficients, log-binomial seed prefactors, HEALPix ring
// geometry and phase offsets (healpix_ffts.py:429-452), FFT twiddles, chirps
// and pre-transformed Bluestein filters. Plans are owned by the caller
// (create / destroy); execution is stream-ordered and allocation-free.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/s2b.h"
#include "s2b_fft.h"
#include "s2b_internal.h"
#include "s2b_stages.h"
#include "s2b_wigner.h"
#include "s2b_precompute.h"
#include "s2b_tc.h"
#include "s2b_latfwd.h"
#include "s2b_lowm.h"

using namespace s2b;
using cd = std::complex<double>;

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// Lets other translation units of the library report through s2b_last_error().
int s2b::set_last_error(int code, const char* msg) { return fail(code, msg); }

// Every device allocation of the library goes through here and is counted, so that a
// caller (or a test) can check that a call allocated nothing.
static std::atomic<long long> g_dev_allocs{0};
cudaError_t s2b::dev_malloc_void(void** ptr, size_t bytes) {
  g_dev_allocs.fetch_add(1, std::memory_order_relaxed);
  return cudaMalloc(ptr, bytes);
}

#define S2B_CK(call)                                                                    \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess)                                                              \
      return fail(S2B_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));    \
  } while (0)

static const double kPi = 3.14159265358979323846;

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// ----------------------------------------------------------------------------
// sampling geometry and quadrature (double)
// ----------------------------------------------------------------------------
static int ntheta(int L, int sampling, int nside) {
  switch (sampling) {
    case S2B_MW:
    case S2B_GL:
      return L;
    case S2B_MWSS:
      return L + 1;
    case S2B_DH:
      return 2 * L;
    default:
      return 4 * nside - 1;
  }
}

static int nphi_equiang(int L, int sampling) { return sampling == S2B_MWSS ? 2 * L : 2 * L - 1; }

static void gauss_legendre(int L, std::vector<double>& nodes, std::vector<double>& weights) {
  // Newton iteration on P_L (quadrature.py:125-161); nodes ascending in x.
  nodes.assign(L, 0.0);
  weights.assign(L, 0.0);
  const int m = (L + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(kPi * (i - 0.25) / (L + 0.5)), z1 = 2.0, pp = 0.0;
    for (int it = 0; it < 100 && std::fabs(z - z1) > 1e-15; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= L; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = L * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    }
    {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= L; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = L * (z * p1 - p2) / (z * z - 1.0);
    }
    const double w = 2.0 / ((1.0 - z * z) * pp * pp);
    nodes[L - i] = z;  // descending cos -> ascending theta after arccos
    nodes[i - 1] = -z;
    weights[i - 1] = w;
    weights[L - i] = w;
  }
}

static std::vector<double> thetas(int L, int sampling, int nside) {
  const int nt = ntheta(L, sampling, nside);
  std::vector<double> th(nt);
  if (sampling == S2B_GL) {
    std::vector<double> x, w;
    gauss_legendre(L, x, w);
    // thetas = flip(arccos(nodes ascending)) -> ascending theta
    for (int t = 0; t < L; ++t) th[t] = std::acos(x[L - 1 - t]);
    return th;
  }
  for (int t = 0; t < nt; ++t) {
    switch (sampling) {
      case S2B_MW:
        th[t] = (2.0 * t + 1.0) * kPi / (2.0 * L - 1.0);
        break;
      case S2B_MWSS:
        th[t] = 2.0 * t * kPi / (2.0 * L);
        break;
      case S2B_DH:
        th[t] = (2.0 * t + 1.0) * kPi / (4.0 * L);
        break;
      default: {
        double z;
        if (t < nside - 1)
          z = 1.0 - (t + 1.0) * (t + 1.0) / (3.0 * nside * nside);
        else if (t <= 3 * nside - 1)
          z = 4.0 / 3.0 - 2.0 * (t + 1.0) / (3.0 * nside);
        else
          z = (4.0 * nside - 1.0 - t) * (4.0 * nside - 1.0 - t) / (3.0 * nside * nside) - 1.0;
        th[t] = std::acos(z);
      }
    }
  }
  return th;
}

// exact DFT helper on the host (used only at plan time for small tables)

static cd mw_weight(int m) {
  if (m == 1) return cd(0, kPi / 2);
  if (m == -1) return cd(0, -kPi / 2);
  if (m % 2 == 0) return cd(2.0 / (1.0 - (double)m * m), 0);
  return 0;
}

static std::vector<cd> dft_host(std::vector<cd> x);

// transform weights (quadrature.py:7-50); MW/MWSS use the MWSS grid at 2L
static std::vector<double> transform_weights(int L, int sampling, int nside) {
  std::vector<double> q;
  if (sampling == S2B_MW || sampling == S2B_MWSS) {
    const int Lp = 2 * L;  // quad_weights_mwss_theta_only(2L)
    std::vector<cd> w(2 * Lp, 0.0);
    for (int i = -(Lp - 1) + 1; i < Lp + 1; ++i) w[i + Lp - 1] = mw_weight(i - 1);
    // ifftshift: index k of shifted = (k + n/2) mod n of the original
    const int n = 2 * Lp;
    std::vector<cd> ws(n);
    for (int k = 0; k < n; ++k) ws[k] = w[(k + n / 2) % n];
    std::vector<cd> W = dft_host(ws);
    std::vector<double> wr(n);
    for (int k = 0; k < n; ++k) wr[k] = W[k].real() / n;
    q.assign(wr.begin(), wr.begin() + Lp + 1);
    for (int i = 1; i < Lp; ++i) q[i] += wr[n - i];  // (-1)^0 * wr[-1:L:-1]
    for (auto& v : q) v *= 2.0 * kPi / (2.0 * L);
  } else if (sampling == S2B_DH) {
    std::vector<double> th = thetas(L, S2B_DH, 0);
    q.resize(th.size());
    for (size_t t = 0; t < th.size(); ++t) {
      double s = 0.0;
      for (int k = 0; k < L; ++k) s += std::sin((2.0 * k + 1.0) * th[t]) / (2.0 * k + 1.0);
      q[t] = s * 2.0 / L * std::sin(th[t]) * 2.0 * kPi / (2.0 * L - 1.0);
    }
  } else if (sampling == S2B_GL) {
    std::vector<double> x, w;
    gauss_legendre(L, x, w);
    q.resize(L);
    for (int t = 0; t < L; ++t) q[t] = w[t] * 2.0 * kPi / (2.0 * L - 1.0);
  } else {
    q.assign(4 * nside - 1, 4.0 * kPi / (12.0 * nside * nside));
  }
  return q;
}

static int hp_nphi(int t, int nside) {
  if (t < nside - 1) return 4 * (t + 1);
  if (t <= 3 * nside - 1) return 4 * nside;
  return 4 * (4 * nside - t - 1);
}

static double hp_phi0(int t, int nside) {
  if (t + 1 >= nside && t + 1 <= 3 * nside) return 0.5 * ((t - nside + 2) % 2) * kPi / (2.0 * nside);
  if (t + 1 > 3 * nside) return 0.5 * kPi / (2.0 * (4 * nside - t - 1));
  return 0.5 * kPi / (2.0 * (t + 1));
}

// ----------------------------------------------------------------------------
// FFT tables
// ----------------------------------------------------------------------------
static void fft_pow2_host(std::vector<cd>& a) {
  const int n = (int)a.size();
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; ++k) {
        const double ang = -2.0 * kPi * k / len;
        const cd w(std::cos(ang), std::sin(ang));
        const cd u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

// DFT X_j = sum_k x_k exp(-2 pi i jk / n) of any length in O(n log n): the power-of-two FFT
// directly, other lengths by Bluestein's chirp-z convolution (chirp angles reduced modulo
// 2n, so the error stays at the level of the FFTs).
static std::vector<cd> dft_host(std::vector<cd> x) {
  const int n = (int)x.size();
  if (n <= 1) return x;
  if ((n & (n - 1)) == 0) {
    fft_pow2_host(x);
    return x;
  }
  int M = 1;
  while (M < 2 * n - 1) M <<= 1;
  std::vector<cd> c(n), a(M, 0.0), bf(M, 0.0);
  for (int k = 0; k < n; ++k) {
    const long kk = ((long)k * k) % (2L * n);
    c[k] = cd(std::cos(kPi * kk / n), -std::sin(kPi * kk / n));  // exp(-i pi k^2 / n)
    a[k] = x[k] * c[k];
    bf[k] = std::conj(c[k]);
    if (k > 0) bf[M - k] = std::conj(c[k]);
  }
  fft_pow2_host(a);
  fft_pow2_host(bf);
  for (int k = 0; k < M; ++k) a[k] = std::conj(a[k] * bf[k]);  // inverse FFT by conjugation
  fft_pow2_host(a);
  std::vector<cd> X(n);
  for (int k = 0; k < n; ++k) X[k] = c[k] * std::conj(a[k]) / (double)M;
  return X;
}

static int ilog2(int x) {
  int r = 0;
  while ((1 << r) < x) ++r;
  return r;
}

// Twiddle table of the register engine for M = 2^logM (the layout s2b_fft_reg.h reads):
// the first DIF pass (NS0 stages, groups based at r < q0 = M / 2^NS0), rows k < NS0 of
// tw[r 2^k]; then each radix-16 pass with smallest span q = 2^lq, lq = 4 (NMID - 1) down to 0,
// rows k < 4 of tw[r 2^(logM - 4 - lq + k)] for r < q. tw[k] = exp(-2 pi i k / M).
static std::vector<cd> reg_twiddles(int logM) {
  const int M = 1 << logM;
  const int ns0 = (logM & 3) ? (logM & 3) : 4;
  const int nmid = (logM - ns0) / 4;
  auto w = [&](long k) { return std::polar(1.0, -2.0 * kPi * (double)k / M); };
  std::vector<cd> t;
  const int q0 = M >> ns0;
  for (int k = 0; k < ns0; ++k)
    for (int r = 0; r < q0; ++r) t.push_back(w((long)r << k));
  for (int p = 0; p < nmid; ++p) {
    const int lq = 4 * (nmid - 1 - p);
    const int sh = logM - 4 - lq;
    for (int k = 0; k < 4; ++k)
      for (int r = 0; r < (1 << lq); ++r) t.push_back(w(((long)r << sh) << k));
  }
  return t;
}

struct FFTBuild {
  std::vector<FFTDesc> descs;
  std::vector<cd> tw, chirp, bf, rtw, rbf;
  std::map<int, int> by_n;       // n -> desc index
  std::map<int, long> tw_by_M;   // M -> tw offset
  std::map<int, long> rtw_by_M;  // M -> register-engine twiddle offset
  int maxM = 1;

  int add(int n) {
    auto it = by_n.find(n);
    if (it != by_n.end()) return it->second;
    FFTDesc d{};
    d.n = n;
    const bool pow2 = (n & (n - 1)) == 0;
    d.bluestein = pow2 ? 0 : 1;
    d.M = pow2 ? n : (1 << ilog2(2 * n - 1));
    if (d.M < 2) d.M = 2;
    d.logM = ilog2(d.M);
    auto tt = tw_by_M.find(d.M);
    if (tt == tw_by_M.end()) {
      const long off = (long)tw.size();
      for (int k = 0; k < d.M / 2; ++k) {
        const double ang = -2.0 * kPi * k / d.M;
        tw.emplace_back(std::cos(ang), std::sin(ang));
      }
      tw_by_M[d.M] = off;
      d.tw_off = off;
    } else {
      d.tw_off = tt->second;
    }
    d.rtw_off = -1;
    d.rbf_off = -1;
    const bool reg = d.logM >= 8 && d.logM <= 13;
    if (reg) {
      auto rt = rtw_by_M.find(d.M);
      if (rt == rtw_by_M.end()) {
        d.rtw_off = (long)rtw.size();
        const std::vector<cd> t = reg_twiddles(d.logM);
        rtw.insert(rtw.end(), t.begin(), t.end());
        rtw_by_M[d.M] = d.rtw_off;
      } else {
        d.rtw_off = rt->second;
      }
    }
    if (d.bluestein) {
      d.chirp_off = (long)chirp.size();
      std::vector<cd> w(n);
      for (int k = 0; k < n; ++k) {
        const long r = ((long)k * k) % (2L * n);  // exact k^2 mod 2n
        const double ang = -kPi * (double)r / n;
        w[k] = cd(std::cos(ang), std::sin(ang));
        chirp.push_back(w[k]);
      }
      std::vector<cd> b(d.M, 0.0);
      b[0] = std::conj(w[0]);
      for (int k = 1; k < n; ++k) {
        b[k] = std::conj(w[k]);
        b[d.M - k] = std::conj(w[k]);
      }
      fft_pow2_host(b);
      d.bf_off = (long)bf.size();
      std::vector<cd> br(d.M);
      for (int k = 0; k < d.M; ++k) {
        int rv = 0;
        for (int bit = 0; bit < d.logM; ++bit)
          if (k & (1 << bit)) rv |= 1 << (d.logM - 1 - bit);
        br[rv] = b[k] / (double)d.M;
      }
      bf.insert(bf.end(), br.begin(), br.end());
      if (reg) {  // position 16 j + a at [a T + j]
        const int T = d.M / 16;
        d.rbf_off = (long)rbf.size();
        std::vector<cd> rb(d.M);
        for (int j = 0; j < T; ++j)
          for (int a = 0; a < 16; ++a) rb[(size_t)a * T + j] = br[16 * j + a];
        rbf.insert(rbf.end(), rb.begin(), rb.end());
      }
    }
    maxM = std::max(maxM, d.M);
    const int idx = (int)descs.size();
    descs.push_back(d);
    by_n[n] = idx;
    return idx;
  }
};

// ----------------------------------------------------------------------------
// plan
// ----------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
};

struct s2b_plan {
  s2b_desc d;
  int device = -1;  // CUDA device the plan was created on (its tables live there)
  bool fp64;
  bool tc;      // S2B_BF16X3: tensor-core precompute contractions
  size_t rsz;   // sizeof(Real)
  int nth;      // rings of the sampling
  int nphi;     // equiangular ring length
  long npix;    // pixels per map
  int nclass, Q, TR, Gs;
  int dual;     // spin 0 complex: both m signs from one recursion
  int nhalf;
  // inverse geometry
  int inv_nrings, inv_ncol, inv_mo, inv_pole_s, inv_pole_n;
  // forward geometry
  int fwd_nrows, fwd_nrings, fwd_pole_s, fwd_pole_n;
  int fwd_mode;  // 0 direct rows, 1 mw chain, 2 mwss chain
  // device tables
  std::vector<void*> allocs;
  RingInfo* inv_rings = nullptr;
  int* inv_ring_row = nullptr;
  RingInfo* fwd_rings = nullptr;
  int* fwd_ring_row = nullptr;
  void* inv_lam = nullptr;
  void* fwd_lam = nullptr;
  int inv_Ls = 4, fwd_Ls = 4;
  double* lbin = nullptr;
  double* gtab = nullptr;
  void* htab = nullptr;
  // forward recursion, restart formulation: h by 32-degree block, start tables
  int fwd_NB = 0;
  void* fwd_Hb = nullptr;   // [NB][tab_rows][32]
  int* fwd_Mst = nullptr;   // [nhalf][NB][fwd rings]
  void* fwd_Vst = nullptr;  // [nhalf][NB][fwd rings][32] (dt_M, dt_{M+1})
  double* fwd_weights = nullptr;   // per MWSS(2L) ring (mw/mwss) or per ring
  int* status = nullptr;           // device status word (timed-out waits)
  double* hp_phi0 = nullptr;
  long* ring_off = nullptr;        // pixel offsets of the sampling rings
  int* ring_desc = nullptr;        // per ring FFT desc (healpix)
  FFTDesc* descs = nullptr;
  void* tw = nullptr;
  void* chirp = nullptr;
  void* bf = nullptr;
  void* rtw = nullptr;  // register-engine twiddles and filters
  void* rbf = nullptr;
  int row_desc = 0, col_d1 = 0, col_d2 = 0, maxM = 2, M1 = 2, M2 = 2;
  void* col_ph = nullptr;  // column chain: chirp * half-sample phase / n1 per 4L-bin
  // start tables of the inverse rings (inverse and its adjoint), ring -> column map of the
  // adjoint spectra (recursed rings first, then north / south pole), adjoint chain table
  int* inv_Mst = nullptr;
  void* inv_Vst = nullptr;
  int* inv_Mst1 = nullptr;  // restart tables of the inverse kernel's m-split
  void* inv_Vst1 = nullptr;
  int inv_nseg = 1;         // segments along m of the inverse kernel (1, 2, 4, 8)
  // equator-symmetric inverse (spin 0, rings symmetric about the equator): ring pairs
  int inv_sym = 0, inv_npair = 0;
  int* adj_col = nullptr;
  int adj_Gs = 4, adj_pole_s = -1, adj_pole_n = -1;
  void* col_ph_adj = nullptr;
  // MW column chain: correction for the south-pole ring's odd (m + s) content (see
  // mw_pole_correction); MWSS real maps: theta-Nyquist bin split between -L and +L
  void* col_pole = nullptr;
  void* col_imp = nullptr;  // impulse responses of the chain (col_impulse)
  int col_nyq_split = 0;
  size_t ws_adj_G = 0, ws_adj_y = 0;
  // precompute path: ring colatitudes of the kernel tables, table width
  double* kth_inv = nullptr;
  double* kth_fwd = nullptr;
  int knth_inv = 0, knth_fwd = 0, kM = 0;
  size_t ws_pre_fwd = 0, ws_pre_inv = 0;
  // Wigner: one spin transform plan per n, gamma-DFT buffers
  std::vector<s2b_plan*> subs;
  size_t ws_w_fban = 0, ws_w_tmp = 0, ws_w_sub = 0;
  // Wigner: the spin transforms of different n run concurrently on internal streams, forked
  // from and joined back to the caller's stream with events; one workspace slice per stream
  // spin != 0: a second stream on which the low orders (lowm.cu) run beside the latitudinal
  // kernel of a single-plan call
  cudaStream_t aux = nullptr;
  cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
  // makes each event record + wait pair of a fork atomic, so that calls from several host
  // threads on one plan do not fork from each other's streams
  std::mutex fork_mu;
  static constexpr int kMaxWStreams = 8;
  int nwstream = 0;
  cudaStream_t wstream[kMaxWStreams] = {};
  cudaEvent_t wfork = nullptr, wjoin[kMaxWStreams] = {};
  // optional events recorded around the latitudinal launch ([0] inverse, [1] forward)
  int tile_fwd = 0, tile_inv = 0;  // latitudinal tile variants (s2b_plan_set_tuning)
  cudaEvent_t ev_begin[2] = {nullptr, nullptr};
  cudaEvent_t ev_end[2] = {nullptr, nullptr};
  // workspace layout (bytes)
  size_t ws_inv_F, ws_inv_ftm, ws_fwd_cols, ws_fwd_G, ws_fwd_acc, ws_iter_f, ws_iter_flm;
  // equator-symmetric forward (spin 0, MW/MWSS): ring-pair spectra (E, O), Gs2 pairs per row
  int fwd_sym = 0, Gs2 = 0, sym_npair = 0;
  int fwd_cross = 0;  // spin != 0: ring pairs serve both halves (fold of G into G2)
  size_t ws_fwd_G2 = 0;
  // start and restart tables of the symmetric forward (the L northern rings and the equator)
  int* sym_Mst = nullptr;
  void* sym_Vst = nullptr;
  int* sym_Mst1 = nullptr;
  void* sym_Vst1 = nullptr;
  int fwd_nseg = 1;  // segments along m of the forward kernel (1, 2, 4, 8)
};

template <typename T>
static int upload(s2b_plan* p, T** dst, const std::vector<T>& src) {
  if (src.empty()) {
    *dst = nullptr;
    return S2B_OK;
  }
  void* ptr = nullptr;
  S2B_CK(dev_malloc(&ptr, src.size() * sizeof(T)));
  p->allocs.push_back(ptr);
  S2B_CK(cudaMemcpy(ptr, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  *dst = reinterpret_cast<T*>(ptr);
  return S2B_OK;
}

static int upload_complex(s2b_plan* p, void** dst, const std::vector<cd>& src) {
  if (src.empty()) {
    *dst = nullptr;
    return S2B_OK;
  }
  if (p->fp64) {
    std::vector<double2> v(src.size());
    for (size_t i = 0; i < src.size(); ++i) v[i] = make_double2(src[i].real(), src[i].imag());
    double2* d = nullptr;
    int rc = upload(p, &d, v);
    *dst = d;
    return rc;
  }
  std::vector<float2> v(src.size());
  for (size_t i = 0; i < src.size(); ++i)
    v[i] = make_float2((float)src[i].real(), (float)src[i].imag());
  float2* d = nullptr;
  int rc = upload(p, &d, v);
  *dst = d;
  return rc;
}

static RingInfo ring_info(double th) {
  RingInfo r;
  r.B = 2.0 * std::cos(th) / std::sin(th);
  r.A = 2.0 / std::sin(th);
  r.lc = std::log2(std::cos(th / 2.0));
  r.ls = std::log2(std::sin(th / 2.0));
  return r;
}

// Upstream resamples MW maps through MWSS at L (s2fft/utils/resampling.py:284-355) and
// then rebuilds the full theta circle from those L+1 rings by the spin symmetry before the
// x2 upsampling (resampling.py:64-160). For a band-limited map that detour is exact and the
// device's direct chain (DFT over the 2L-1 extended samples, half-sample phase, zero-pad to
// 4L, inverse DFT) gives the same values. The one difference is the MW ring at theta = pi:
// it is its own mirror, so for phi-frequencies with odd m + s a map that is not band-limited
// has a part there that the rebuilt circle turns into its antisymmetric image. That part is
// one sample per column, so upstream's chain equals the direct chain plus x_pole * c, with
// c = (upstream chain - direct chain)(unit impulse at the pole), here for k = 0..2L on the
// MWSS(2L) rings, in the units of the device's inverse-DFT output (before the phi factor
// and the weights). For real maps upstream takes the real part after the upsampling, which
// turns c into Re(c) (the impulse is real and the direct chain's image of it is real).
// Unnormalised inverse DFT y_k = sum_j x_j exp(+2 pi i jk / n), any length, O(n log n).
static std::vector<cd> idft_host(std::vector<cd> x) {
  for (cd& v : x) v = std::conj(v);
  x = dft_host(std::move(x));
  for (cd& v : x) v = std::conj(v);
  return x;
}

// The chain's sums over theta bins, each a DFT over bins p at index p mod n (O(L log L)).
static std::vector<cd> mw_pole_correction(int L) {
  const int n1 = 2 * L - 1, n2 = 2 * L, n4 = 4 * L;
  // theta bins p = -(L-1)..L-1 of the impulse at t = L-1 after the half-sample phase:
  // exp(-2 pi i p (L-1) / n1) exp(-i pi p / n1) / n1 = (-1)^p / n1
  auto G = [&](int p) { return ((p & 1) ? -1.0 : 1.0) / (double)n1; };
  auto bins = [&](int n) {
    std::vector<cd> a(n, cd(0.0, 0.0));
    for (int p = -(L - 1); p <= L - 1; ++p) a[((p % n) + n) % n] = G(p);
    return a;
  };
  // upstream: unnormalised inverse DFT over 2L (MWSS rings j = 0..L), the circle rebuilt
  // with the odd-column sign -1, DFT over 2L divided by 2L, zero-pad (bin -L kept at -L),
  // unnormalised inverse DFT over 4L
  const std::vector<cd> g = idft_host(bins(n2));  // g[j], j = 0..L used
  std::vector<cd> ext(n2);
  for (int j = 0; j < n2; ++j) ext[j] = j <= L ? g[j] : -g[n2 - j];
  const std::vector<cd> E = dft_host(ext);  // E[q mod n2] = 2L H[q]
  std::vector<cd> B(n4, cd(0.0, 0.0));
  for (int q = -L; q < L; ++q) B[((q % n4) + n4) % n4] = E[((q % n2) + n2) % n2] / (double)n2;
  const std::vector<cd> u = idft_host(B);
  const std::vector<cd> direct = idft_host(bins(n4));
  std::vector<cd> c(2 * L + 1);
  for (int k = 0; k <= 2 * L; ++k) c[k] = u[k] - direct[k];
  return c;
}

// Response of the forward column chain (to the MWSS(2L) rings t = 0..2L, in the units of
// the device's inverse-DFT output, before the overall factor and the weights) to a unit
// impulse on the samples that are their own mirror in the theta extension of a column with
// odd m + s: MW the pole ring (the direct chain's image of it plus the pole correction
// `pole`), MWSS the poles t = 0 and t = L ([2][2L+1], with the Nyquist split for real
// maps). The paired-column kernel keeps these samples out of the transform it shares
// between two columns and adds them through this table.
static std::vector<cd> col_impulse(int L, bool mw, const std::vector<cd>& pole, bool nyq_split) {
  const int n4 = 4 * L, nout = 2 * L + 1;
  // sum over theta bins p of b(p) exp(2 pi i p k / 4L), k = 0..2L: an inverse DFT over 4L
  auto chain = [&](int plo, auto b) {
    std::vector<cd> a(n4, cd(0.0, 0.0));
    for (int p = plo; p <= L - 1; ++p) a[((p % n4) + n4) % n4] = b(p);
    return idft_host(a);
  };
  if (mw) {
    // bins after the half-sample phase and 1/n1: (-1)^p / n1 (see mw_pole_correction)
    const double n1 = 2.0 * L - 1.0;
    const std::vector<cd> d = chain(-(L - 1), [&](int p) { return cd(((p & 1) ? -1.0 : 1.0) / n1, 0.0); });
    std::vector<cd> imp(nout);
    for (int k = 0; k < nout; ++k) imp[k] = d[k] + pole[k];
    return imp;
  }
  // MWSS: bins 1 / n1 (t = 0) and (-1)^p / n1 (t = L), p = -L..L-1
  const double n1 = 2.0 * L;
  std::vector<cd> imp(2 * nout);
  for (int which = 0; which < 2; ++which) {
    const std::vector<cd> d = chain(-L, [&](int p) {
      return cd(((which && (p & 1)) ? -1.0 : 1.0) / n1, 0.0);
    });
    for (int k = 0; k < nout; ++k) {
      cd v = d[k];
      if (nyq_split && (k & 1)) {  // i N sin(pi k / 2), N = bin -L
        const double N = ((which && (L & 1)) ? -1.0 : 1.0) / n1;
        v += cd(0.0, ((k & 2) ? -1.0 : 1.0) * N);
      }
      imp[which * nout + k] = v;
    }
  }
  return imp;
}

// The column chain's correction tables (pole correction, impulse responses, Nyquist split)
// for complex maps or, real_map, as upstream treats real maps.
static int set_col_tables(s2b_plan* p, bool real_map) {
  const int L = p->d.L;
  int rc;
  std::vector<cd> c;
  if (p->fwd_mode == 1) {
    c = mw_pole_correction(L);
    if (real_map)
      for (cd& v : c) v = cd(v.real(), 0.0);
    if ((rc = upload_complex(p, &p->col_pole, c))) return rc;
  }
  p->col_nyq_split = (p->fwd_mode == 2 && real_map) ? 1 : 0;
  if ((rc = upload_complex(p, &p->col_imp,
                           col_impulse(L, p->fwd_mode == 1, c, p->col_nyq_split != 0))))
    return rc;
  return S2B_OK;
}

static int build_plan(s2b_plan* p) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  p->fp64 = d.precision == S2B_F64;
  p->tc = d.precision == S2B_BF16X3;
  p->rsz = p->fp64 ? 8 : 4;
  p->nth = ntheta(L, d.sampling, d.nside);
  p->nphi = d.sampling == S2B_HEALPIX ? 0 : nphi_equiang(L, d.sampling);
  p->npix = d.sampling == S2B_HEALPIX ? 12L * d.nside * d.nside : (long)p->nth * p->nphi;
  p->dual = (d.spin == 0 && !d.reality) ? 1 : 0;
  p->nhalf = (d.spin == 0) ? 1 : 2;
  // degree classes of the coefficient tables: l = j + nclass q with q < Q = 64 slots
  p->Q = 64;
  p->nclass = (L + p->Q - 1) / p->Q;
  p->TR = tab_rows(L);

  // ---- recursion tables: g[m][l], h[j][m][q], lbin[l]
  std::vector<double> g((size_t)L * L, 0.0), h((size_t)L * L, 0.0);
  for (int l = 0; l < L; ++l) {
    auto f = [&](int m) { return std::sqrt((double)(l + m) * (double)(l - m + 1)); };
    std::vector<double> gl(l + 2, 0.0);
    gl[l] = 1.0;
    if (l >= 1) gl[l - 1] = 1.0 / f(l);
    for (int m = l - 1; m >= 1; --m) gl[m - 1] = f(m + 1) * gl[m + 1] / f(m);
    for (int m = 0; m <= l; ++m) g[(size_t)m * L + l] = gl[m];
    h[(size_t)l * L + l] = 1.0;
    for (int m = l - 1; m >= 0; --m) h[(size_t)m * L + l] = gl[m] / (f(m + 1) * gl[m + 1]);
  }
  int rc = upload(p, &p->gtab, g);
  if (rc) return rc;
  {
    const int C = p->nclass, Q = p->Q, TR = p->TR;
    if (p->fp64) {
      std::vector<double> hc((size_t)C * TR * Q, 0.0);
      for (int j = 0; j < C; ++j)
        for (int m = 0; m < L; ++m)
          for (int q = 0; q < Q; ++q) {
            const int l = j + C * q;
            if (l < L) hc[((size_t)j * TR + m + kPadLo) * Q + q] = h[(size_t)m * L + l];
          }
      double* dp = nullptr;
      rc = upload(p, &dp, hc);
      p->htab = dp;
    } else {
      std::vector<float> hc((size_t)C * TR * Q, 0.0f);
      for (int j = 0; j < C; ++j)
        for (int m = 0; m < L; ++m)
          for (int q = 0; q < Q; ++q) {
            const int l = j + C * q;
            if (l < L) hc[((size_t)j * TR + m + kPadLo) * Q + q] = (float)h[(size_t)m * L + l];
          }
      float* fp = nullptr;
      rc = upload(p, &fp, hc);
      p->htab = fp;
    }
    if (rc) return rc;
  }
  {
    const int as = std::abs(d.spin);
    std::vector<double> lb(L, 0.0);
    for (int l = 0; l < L; ++l) {
      if (l < as) continue;
      lb[l] = 0.5 * (std::lgamma(2.0 * l + 1.0) - std::lgamma(l + as + 1.0) -
                     std::lgamma(l - as + 1.0)) / std::log(2.0);
    }
    rc = upload(p, &p->lbin, lb);
    if (rc) return rc;
  }
  {
    // h_{l,m} by 32-degree block (zero for m > l and for l >= L)
    const int NB = fwd_nblocks(L), TR = p->TR;
    p->fwd_NB = NB;
    const size_t n = (size_t)NB * TR * kFwdBlock;
    if (p->fp64) {
      std::vector<double> hb(n, 0.0);
      for (int l = 0; l < L; ++l)
        for (int m = 0; m <= l; ++m)
          hb[((size_t)(l / kFwdBlock) * TR + m + kPadLo) * kFwdBlock + l % kFwdBlock] =
              h[(size_t)m * L + l];
      double* dp = nullptr;
      rc = upload(p, &dp, hb);
      p->fwd_Hb = dp;
    } else {
      std::vector<float> hb(n, 0.0f);
      for (int l = 0; l < L; ++l)
        for (int m = 0; m <= l; ++m)
          hb[((size_t)(l / kFwdBlock) * TR + m + kPadLo) * kFwdBlock + l % kFwdBlock] =
              (float)h[(size_t)m * L + l];
      float* fp = nullptr;
      rc = upload(p, &fp, hb);
      p->fwd_Hb = fp;
    }
    if (rc) return rc;
  }

  // ---- inverse geometry: rings of the sampling, poles in closed form
  std::vector<double> th = thetas(L, d.sampling, d.nside);
  {
    std::vector<RingInfo> ri;
    std::vector<int> rr;
    p->inv_pole_s = -1;
    p->inv_pole_n = -1;
    for (int t = 0; t < p->nth; ++t) {
      if (d.sampling == S2B_MW && t == p->nth - 1) {
        p->inv_pole_s = t;
        continue;
      }
      if (d.sampling == S2B_MWSS && (t == 0 || t == p->nth - 1)) {
        if (t == 0)
          p->inv_pole_n = t;
        else
          p->inv_pole_s = t;
        continue;
      }
      ri.push_back(ring_info(th[t]));
      rr.push_back(t);
    }
    p->inv_nrings = (int)ri.size();
    // spin 0 on a recursed ring set symmetric about the equator (MWSS inner rings, GL, DH,
    // HEALPix; not MW): ring r and inv_nrings - 1 - r share one recursion
    {
      bool symmetric = d.spin == 0 && p->inv_nrings >= 2;
      for (int r = 0; symmetric && r < p->inv_nrings; ++r)
        symmetric = std::fabs(th[rr[r]] + th[rr[p->inv_nrings - 1 - r]] - kPi) < 1e-12;
      p->inv_sym = symmetric ? 1 : 0;
      p->inv_npair = (p->inv_nrings + 1) / 2;
    }
    p->inv_ncol = (d.sampling == S2B_MWSS || d.sampling == S2B_HEALPIX) ? 2 * L : 2 * L - 1;
    p->inv_mo = (d.sampling == S2B_MWSS || d.sampling == S2B_HEALPIX) ? 1 : 0;
    if ((rc = upload(p, &p->inv_rings, ri))) return rc;
    if ((rc = upload(p, &p->inv_ring_row, rr))) return rc;
    std::vector<int> col(p->nth, 0);
    for (int r = 0; r < (int)rr.size(); ++r) col[rr[r]] = r;
    int next = p->inv_nrings;
    if (p->inv_pole_n >= 0) {
      p->adj_pole_n = next;
      col[p->inv_pole_n] = next++;
    }
    if (p->inv_pole_s >= 0) {
      p->adj_pole_s = next;
      col[p->inv_pole_s] = next++;
    }
    p->adj_Gs = round4(p->nth);
    if ((rc = upload(p, &p->adj_col, col))) return rc;
  }
  // ---- forward geometry
  {
    std::vector<RingInfo> ri;
    std::vector<int> rr;
    std::vector<double> w = transform_weights(L, d.sampling, d.nside);
    if (d.sampling == S2B_MW || d.sampling == S2B_MWSS) {
      p->fwd_mode = d.sampling == S2B_MW ? 1 : 2;
      // the MWSS(2L) rings t and 2L - t mirror each other: spin 0 projects ring pairs
      p->fwd_sym = 1;
      p->fwd_cross = d.spin != 0 ? 1 : 0;
      p->sym_npair = L;
      p->Gs2 = round4(L);
      std::vector<double> th2 = thetas(2 * L, S2B_MWSS, 0);
      p->fwd_nrows = 2 * L + 1;
      p->fwd_pole_n = 2 * L - 1;  // rows 0..2L-2: rings t = 1..2L-1; then the two poles
      p->fwd_pole_s = 2 * L;
      for (int t = 1; t < 2 * L; ++t) {
        ri.push_back(ring_info(th2[t]));
        rr.push_back(t - 1);
      }
    } else {
      p->fwd_mode = 0;
      p->fwd_nrows = p->nth;
      p->fwd_pole_n = -1;
      p->fwd_pole_s = -1;
      for (int t = 0; t < p->nth; ++t) {
        ri.push_back(ring_info(th[t]));
        rr.push_back(t);
      }
      // spin 0 on a ring set symmetric about the equator (GL, DH, HEALPix): ring pairs
      bool symmetric = p->nth >= 2;
      for (int t = 0; symmetric && t < p->nth; ++t)
        symmetric = std::fabs(th[t] + th[p->nth - 1 - t] - kPi) < 1e-12;
      if (symmetric) {
        p->fwd_sym = 1;
        p->fwd_cross = d.spin != 0 ? 1 : 0;
        p->sym_npair = (p->nth + 1) / 2;
        p->Gs2 = round4(p->sym_npair);
      }
    }
    p->fwd_nrings = (int)ri.size();
    p->Gs = round4(p->fwd_nrows);
    if ((rc = upload(p, &p->fwd_rings, ri))) return rc;
    if ((rc = upload(p, &p->fwd_ring_row, rr))) return rc;
    if ((rc = upload(p, &p->fwd_weights, w))) return rc;
  }

  S2B_CK(dev_malloc(&p->status, sizeof(int)));
  p->allocs.push_back(p->status);
  S2B_CK(cudaMemset(p->status, 0, sizeof(int)));

  // ---- forward start tables (device kernel, double arithmetic)
  if (p->fwd_nrings > 0) {
    const size_t nst = (size_t)p->nhalf * p->fwd_NB * p->fwd_nrings;
    S2B_CK(dev_malloc(&p->fwd_Mst, nst * sizeof(int)));
    p->allocs.push_back(p->fwd_Mst);
    S2B_CK(dev_malloc(&p->fwd_Vst, fwd_start_bytes(p->fp64, L, p->nhalf, p->fwd_nrings)));
    p->allocs.push_back(p->fwd_Vst);
    FwdStartParams fp{};
    fp.L = L;
    fp.L0 = d.L_lower;
    fp.spin = d.spin;
    fp.nhalf = p->nhalf;
    fp.nrings = p->fwd_nrings;
    fp.NB = p->fwd_NB;
    // contributions below 2^-32 (float) / 2^-70 (double) of |d| <= 1 are dropped
    fp.floor_log2 = p->fp64 ? -70.0 : -32.0;
    fp.group = fwd_group(p->fp64);
    fp.rings = p->fwd_rings;
    fp.lbin = p->lbin;
    fp.g = p->gtab;
    fp.Mst = p->fwd_Mst;
    fp.Vst = p->fwd_Vst;
    S2B_CK(launch_fwd_start(p->fp64, fp, 0));
  }
  // ---- start and restart tables of the symmetric forward: the northern rings and the equator
  if (p->fwd_sym) {
    const size_t nst = (size_t)p->nhalf * p->fwd_NB * p->sym_npair;
    const size_t vb = fwd_start_bytes(p->fp64, L, p->nhalf, p->sym_npair);
    S2B_CK(dev_malloc(&p->sym_Mst, kInvSegMax * nst * sizeof(int)));
    p->allocs.push_back(p->sym_Mst);
    S2B_CK(dev_malloc(&p->sym_Vst, kInvSegMax * vb));
    p->allocs.push_back(p->sym_Vst);
    p->sym_Mst1 = p->sym_Mst + nst;
    p->sym_Vst1 = static_cast<char*>(p->sym_Vst) + vb;
    FwdStartParams fp{};
    fp.L = L;
    fp.L0 = d.L_lower;
    fp.spin = d.spin;
    fp.nhalf = p->nhalf;
    fp.nrings = p->sym_npair;
    fp.NB = p->fwd_NB;
    fp.floor_log2 = p->fp64 ? -70.0 : -32.0;
    fp.group = fwd_group(p->fp64);
    fp.rings = p->fwd_rings;
    fp.lbin = p->lbin;
    fp.g = p->gtab;
    fp.Mst = p->sym_Mst;
    fp.Vst = p->sym_Vst;
    fp.Mst1 = p->sym_Mst1;
    fp.Vst1 = p->sym_Vst1;
    S2B_CK(launch_fwd_start(p->fp64, fp, 0));
    // launch shape measured at L = 256 ... 1024 (MW, HEALPix; float): eight segments along
    // m (against four: 8-12 % faster up to L = 512, 2 % at 1024); spin-0 float takes 8 ring
    // pairs per warp up to L = 256, 16 above (spin != 0: 16 throughout)
    p->fwd_nseg = kInvSegMax;
    p->tile_fwd = (!p->fp64 && L <= 256 && !p->fwd_cross) ? 1 : 0;
  }
  // ---- start tables of the inverse rings (inverse kernel and adjoint of the inverse)
  if (p->inv_nrings > 0) {
    const size_t nst = (size_t)p->nhalf * p->fwd_NB * p->inv_nrings;
    S2B_CK(dev_malloc(&p->inv_Mst, nst * sizeof(int)));
    p->allocs.push_back(p->inv_Mst);
    S2B_CK(dev_malloc(&p->inv_Vst, fwd_start_bytes(p->fp64, L, p->nhalf, p->inv_nrings)));
    p->allocs.push_back(p->inv_Vst);
    S2B_CK(dev_malloc(&p->inv_Mst1, (kInvSegMax - 1) * nst * sizeof(int)));
    p->allocs.push_back(p->inv_Mst1);
    S2B_CK(dev_malloc(&p->inv_Vst1, (kInvSegMax - 1) *
                                        fwd_start_bytes(p->fp64, L, p->nhalf, p->inv_nrings)));
    p->allocs.push_back(p->inv_Vst1);
    // launch shape of the inverse kernel, measured at L = 256 ... 1024 (MW, HEALPix; float):
    // eight segments along m (against four: 10-11 % faster at L = 256 and 512 with the
    // tiles below, 1 % at 1024), start values read from global memory (shared memory for 3
    // CTAs per SM), two rings per lane in float from L = 512 and one below
    p->inv_nseg = kInvSegMax;
    p->tile_inv = (!p->fp64 && L >= 512) ? 2 : 3;
    // symmetric inverse: one ring pair per lane (two would double the partial sums in
    // shared memory and drop to 2 CTAs per SM; measured slower at L = 256 ... 2048)
    if (p->inv_sym) p->tile_inv = 3;
    FwdStartParams fp{};
    fp.L = L;
    fp.L0 = d.L_lower;
    fp.spin = d.spin;
    fp.nhalf = p->nhalf;
    fp.nrings = p->inv_nrings;
    fp.NB = p->fwd_NB;
    fp.floor_log2 = p->fp64 ? -70.0 : -32.0;
    fp.group = fwd_group(p->fp64);
    fp.rings = p->inv_rings;
    fp.lbin = p->lbin;
    fp.g = p->gtab;
    fp.Mst = p->inv_Mst;
    fp.Vst = p->inv_Vst;
    fp.Mst1 = p->inv_Mst1;
    fp.Vst1 = p->inv_Vst1;
    S2B_CK(launch_fwd_start(p->fp64, fp, 0));
  }

  // ---- lambda(theta, m) tables (double, rounded once to the plan precision)
  {
    p->inv_Ls = round4(std::max(p->inv_nrings, 1));
    p->fwd_Ls = round4(p->fwd_nrings);
    const size_t bi = (size_t)p->nhalf * p->TR * p->inv_Ls * p->rsz;
    const size_t bf = (size_t)p->nhalf * p->TR * p->fwd_Ls * p->rsz;
    S2B_CK(dev_malloc(&p->inv_lam, bi));
    p->allocs.push_back(p->inv_lam);
    S2B_CK(dev_malloc(&p->fwd_lam, bf));
    p->allocs.push_back(p->fwd_lam);
    if (p->inv_nrings > 0)
      S2B_CK(launch_lambda(p->fp64, L, d.spin, p->nhalf, p->inv_rings, p->inv_nrings, p->inv_Ls,
                           p->inv_lam, 0));
    else
      S2B_CK(cudaMemset(p->inv_lam, 0, bi));
    S2B_CK(launch_lambda(p->fp64, L, d.spin, p->nhalf, p->fwd_rings, p->fwd_nrings, p->fwd_Ls,
                         p->fwd_lam, 0));
  }

  // ---- FFT tables and ring layout
  FFTBuild fb;
  std::vector<long> roff(p->nth);
  std::vector<int> rdesc;
  if (d.sampling == S2B_HEALPIX) {
    std::vector<double> phi0(p->nth);
    rdesc.resize(p->nth);
    long off = 0;
    for (int t = 0; t < p->nth; ++t) {
      const int n = hp_nphi(t, d.nside);
      roff[t] = off;
      off += n;
      rdesc[t] = fb.add(n);
      phi0[t] = hp_phi0(t, d.nside);
    }
    if ((rc = upload(p, &p->hp_phi0, phi0))) return rc;
    if ((rc = upload(p, &p->ring_desc, rdesc))) return rc;
  } else {
    for (int t = 0; t < p->nth; ++t) roff[t] = (long)t * p->nphi;
    p->row_desc = fb.add(p->nphi);
  }
  if ((rc = upload(p, &p->ring_off, roff))) return rc;
  if (p->fwd_mode != 0) {
    p->col_d1 = fb.add(p->fwd_mode == 1 ? 2 * L - 1 : 2 * L);
    p->col_d2 = fb.add(4 * L);
    p->M1 = fb.descs[p->col_d1].M;
    p->M2 = fb.descs[p->col_d2].M;
  }
  p->maxM = 2;
  if (d.sampling == S2B_HEALPIX) {
    for (int t = 0; t < p->nth; ++t) p->maxM = std::max(p->maxM, fb.descs[rdesc[t]].M);
  } else {
    p->maxM = fb.descs[p->row_desc].M;
  }
  if ((rc = upload(p, &p->descs, fb.descs))) return rc;
  if ((rc = upload_complex(p, &p->tw, fb.tw))) return rc;
  if ((rc = upload_complex(p, &p->chirp, fb.chirp))) return rc;
  if ((rc = upload_complex(p, &p->bf, fb.bf))) return rc;
  if (!fb.rtw.empty() && (rc = upload_complex(p, &p->rtw, fb.rtw))) return rc;
  if (!fb.rbf.empty() && (rc = upload_complex(p, &p->rbf, fb.rbf))) return rc;
  if (p->fwd_mode != 0) {
    // factor applied to theta-DFT bin pp (stored at k = pp mod 4L) before the
    // inverse 4L DFT: Bluestein output chirp, MW half-sample shift exp(-i pp pi/(2L-1)),
    // and 1/n1
    const FFTDesc& d1 = fb.descs[p->col_d1];
    const int n1 = d1.n, n2 = 4 * L;
    const int plo = p->fwd_mode == 1 ? -(L - 1) : -L, phi = L - 1;
    std::vector<cd> ph(n2, cd(0.0, 0.0));
    for (int pp = plo; pp <= phi; ++pp) {
      const int j = ((pp % n1) + n1) % n1;
      cd f(1.0 / n1, 0.0);
      if (d1.bluestein) f *= fb.chirp[d1.chirp_off + j];
      if (p->fwd_mode == 1) f *= std::polar(1.0, -kPi * (double)pp / (2.0 * L - 1.0));
      ph[(pp + n2) % n2] = f;
    }
    if ((rc = upload_complex(p, &p->col_ph, ph))) return rc;
    std::vector<cd> pa(n2, cd(0.0, 0.0));
    for (int pp = plo; pp <= phi; ++pp) {
      cd f(1.0 / n1, 0.0);
      if (p->fwd_mode == 1) f *= std::polar(1.0, kPi * (double)pp / (2.0 * L - 1.0));
      pa[(pp + n2) % n2] = f;
    }
    if ((rc = upload_complex(p, &p->col_ph_adj, pa))) return rc;
    if ((rc = set_col_tables(p, d.reality != 0))) return rc;
  }
  const size_t maxsmem = (size_t)227 * 1024;
  auto padded = [](int M) { return (size_t)M + (size_t)(M >> 3); };  // ring FFT buffer layout
  if (padded(p->maxM) * 2 * p->rsz > maxsmem || (padded(p->M1) + padded(p->M2)) * 2 * p->rsz > maxsmem)
    return fail(S2B_ERR_INVALID, "band-limit too large for the shared-memory ring FFT");

  // ---- precompute-kernel geometry (tables include the pole rings)
  {
    std::vector<double> thk = thetas(L, d.sampling, d.nside);
    p->knth_inv = (int)thk.size();
    if ((rc = upload(p, &p->kth_inv, thk))) return rc;
    std::vector<double> thf = (d.sampling == S2B_MW || d.sampling == S2B_MWSS)
                                  ? thetas(2 * L, S2B_MWSS, 0)
                                  : thk;
    p->knth_fwd = (int)thf.size();
    if ((rc = upload(p, &p->kth_fwd, thf))) return rc;
    p->kM = d.reality ? L : 2 * L - 1;
  }

  // ---- workspace layout
  const size_t c2 = 2 * p->rsz;
  const size_t acc = p->dual ? 2 * c2 : c2;
  const size_t B = (size_t)d.batch;
  p->ws_inv_F = B * p->nhalf * p->nclass * (size_t)p->TR * p->Q * acc;
  p->ws_inv_ftm = B * (size_t)p->nth * p->inv_ncol * c2;
  const int ncm = p->fwd_mode == 1 ? 2 * L - 1 : 2 * L;
  p->ws_fwd_cols = p->fwd_mode ? B * (size_t)ncm * p->nth * c2 : 0;
  p->ws_fwd_G = B * p->nhalf * (size_t)p->TR * p->Gs * acc;
  p->ws_fwd_acc = B * p->nhalf * (size_t)L * ((size_t)p->fwd_NB * kFwdBlock) * acc;
  // (E, O) per pair: Real4 in the dual and the cross layouts, Real2 otherwise
  p->ws_fwd_G2 = p->fwd_sym ? B * p->nhalf * (size_t)p->TR * p->Gs2 * 2 *
                                  (p->fwd_cross ? 2 * c2 : acc)
                            : 0;
  const size_t fel = d.reality ? p->rsz : c2;
  p->ws_iter_f = d.iter > 0 ? B * (size_t)p->npix * fel : 0;
  p->ws_iter_flm = d.iter > 0 ? B * (size_t)L * (2 * L - 1) * c2 : 0;
  p->ws_adj_G = B * p->nhalf * (size_t)p->TR * p->adj_Gs * acc;
  p->ws_adj_y = p->fwd_mode ? B * (size_t)(2 * L + 1) * (2 * L - 1) * c2 : 0;
  p->ws_pre_fwd = B * (size_t)p->knth_fwd * p->kM * c2;
  const int hpc = d.sampling == S2B_HEALPIX;  // complex kernel tables
  if (p->tc)
    p->ws_pre_fwd = align256(p->ws_pre_fwd) + tc_packed_b_bytes(p->knth_fwd, d.batch, p->kM, hpc);
  p->ws_pre_inv = p->tc ? tc_packed_b_bytes(L, d.batch, p->kM, hpc) : 0;
  if (d.spin != 0) {  // orders m < |s| (lowm.cu) run beside the latitudinal kernels
    S2B_CK(cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking));
    S2B_CK(cudaEventCreateWithFlags(&p->aux_fork, cudaEventDisableTiming));
    S2B_CK(cudaEventCreateWithFlags(&p->aux_join, cudaEventDisableTiming));
  }
  S2B_CK(cudaDeviceSynchronize());
  return S2B_OK;
}


static size_t inv_ws(const s2b_plan* p) {
  // spin inverse: F and ftm; precompute inverse: ftm and (tensor cores) the packed flm
  return std::max(align256(p->ws_inv_F) + align256(p->ws_inv_ftm),
                  align256(p->ws_inv_ftm) + align256(p->ws_pre_inv));
}
static size_t inv_adj_ws(const s2b_plan* p) {
  return align256(p->ws_adj_G) + align256(p->ws_fwd_acc);
}
static size_t fwd_adj_ws(const s2b_plan* p) {
  return p->fwd_mode ? align256(p->ws_inv_F) + align256(p->ws_adj_y) + align256(p->ws_inv_ftm)
                     : inv_ws(p);
}
static size_t pre_fwd_ws(const s2b_plan* p) {
  return align256(p->ws_fwd_cols) + align256(p->ws_pre_fwd);
}
static size_t fwd_once_ws(const s2b_plan* p) {
  return align256(p->ws_fwd_cols) + align256(p->ws_fwd_G) + align256(p->ws_fwd_acc) +
         align256(p->ws_fwd_G2);
}
static size_t fwd_ws(const s2b_plan* p) {
  size_t once = fwd_once_ws(p);
  if (p->d.iter > 0)
    once = std::max(once, inv_ws(p)) + align256(p->ws_iter_f) + align256(p->ws_iter_flm);
  return once;
}

// ----------------------------------------------------------------------------
// execution
// ----------------------------------------------------------------------------
template <typename Real>
static FFTTables<Real> tables(const s2b_plan* p) {
  FFTTables<Real> t;
  t.tw = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->tw);
  t.chirp = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->chirp);
  t.bfilt = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->bf);
  t.rtw = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->rtw);
  t.rbf = reinterpret_cast<const typename FFTTables<Real>::R2*>(p->rbf);
  return t;
}

// Execute calls launch on the current device; the plan's tables live on the device it was
// created on, so the two must agree (a plan used from another device would hand one GPU's
// pointers to another's kernels).
static int check_device(const s2b_plan* p) {
  int dev = -1;
  S2B_CK(cudaGetDevice(&dev));
  if (dev != p->device)
    return fail(S2B_ERR_INVALID, "the current device (" + std::to_string(dev) +
                                     ") is not the plan's device (" + std::to_string(p->device) +
                                     "): make the plan's device current before the call");
  return S2B_OK;
}

int s2b::check_plan_device(const s2b_plan* p) { return check_device(p); }

static int check_ptr(const void* ptr, const char* what) {
  if (!ptr) return fail(S2B_ERR_ALIGN, std::string(what) + " is NULL");
  if (reinterpret_cast<uintptr_t>(ptr) % 16 != 0)
    return fail(S2B_ERR_ALIGN, std::string(what) + " is not 16-byte aligned");
  return S2B_OK;
}

// Orders m < |spin| are left out of the latitudinal kernels and added by the degree
// recursion (lowm.cu): the m-recursion is unstable below m = n cos(theta) on rings where
// n cos(theta) > 0, a range that lies inside m < |spin|.
static int lowm_orders(const s2b_plan* p) { return p->d.spin < 0 ? -p->d.spin : p->d.spin; }

static int run_lowm_synth(const s2b_plan* p, const Inv2Params& lp, const RingInfo* rings,
                          cudaStream_t s) {
  if (lp.mlo <= 0 || lp.nrings <= 0) return S2B_OK;
  LowmParams q{};
  q.L = lp.L;
  q.spin = p->d.spin;
  q.nhalf = lp.nhalf;
  q.batch = lp.batch;
  q.nrings = lp.nrings;
  q.NB = lp.NB;
  q.mlo = lp.mlo;
  q.rings = rings;
  q.g = p->gtab;
  q.F = lp.F;
  q.ftm = lp.ftm;
  q.ring_row = lp.ring_row;
  q.nrows = lp.nrows;
  q.ncol = lp.ncol;
  q.mo = lp.mo;
  S2B_CK(launch_lowm_synth(p->fp64, q, s));
  return S2B_OK;
}

static int run_lowm_project(const s2b_plan* p, const Fwd2Params& lp, const RingInfo* rings,
                            cudaStream_t s) {
  if (lp.mlo <= 0 || lp.nrings <= 0) return S2B_OK;
  LowmParams q{};
  q.L = lp.L;
  q.spin = p->d.spin;
  q.nhalf = lp.nhalf;
  q.batch = lp.batch;
  q.nrings = lp.nrings;
  q.NB = lp.NB;
  q.mlo = lp.mlo;
  q.rings = rings;
  q.g = p->gtab;
  q.G = lp.G;
  q.Gs = lp.Gs;
  q.acc = lp.acc;
  S2B_CK(launch_lowm_project(p->fp64, q, s));
  return S2B_OK;
}

// The inverse in three stages: before the latitudinal kernel (coefficient table, pole rows;
// fills the kernel's parameters, nrings = 0 when there is nothing to recurse), the kernel,
// and after it (low orders, ring FFTs). A batch runs each stage over all its plans, with
// the kernels of all plans in persistent launches.
template <typename Real>
static int inv_stage_pre(s2b_plan* p, const void* flm, char* ws, cudaStream_t s,
                         Inv2Params* out) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  void* F = ws;
  void* ftm = ws + align256(p->ws_inv_F);
  StageParams sp{};
  sp.ftm_zero_bytes = p->ws_inv_ftm;
  sp.L = L;
  sp.L0 = d.L_lower;
  sp.spin = d.spin;
  sp.batch = d.batch;
  sp.nclass = p->nclass;
  sp.Q = p->Q;
  sp.TR = p->TR;
  sp.Gs = p->Gs;
  sp.nhalf = p->nhalf;
  sp.dual = p->dual;
  sp.nrows = p->nth;
  sp.ncol = p->inv_ncol;
  sp.mo = p->inv_mo;
  sp.pole_south = p->inv_pole_s;
  sp.pole_north = p->inv_pole_n;
  sp.g = p->gtab;
  sp.flm = flm;
  sp.F = F;
  sp.ftm = ftm;
  // blocked coefficient table for the latitudinal kernel: [NB][row][32], l = 32 block + column
  sp.nclass = p->fwd_NB;
  sp.Q = kFwdBlock;
  sp.Lp = p->fwd_NB * kFwdBlock;
  S2B_CK(launch_prologue(p->fp64, sp, s));
  out->nrings = 0;
  if (p->inv_nrings > 0) {
    Inv2Params lp{};
    lp.L = L;
    lp.nrings = p->inv_nrings;
    lp.nhalf = p->nhalf;
    lp.batch = d.batch;
    lp.NB = p->fwd_NB;
    lp.Mst = p->inv_Mst;
    lp.Vst = p->inv_Vst;
    lp.Mst1 = p->inv_Mst1;
    lp.Vst1 = p->inv_Vst1;
    lp.nseg = p->inv_nseg;
    if (p->inv_sym) {
      lp.sym = 1;
      lp.nrings = p->inv_npair;
      lp.tab_stride = p->inv_nrings;
    }
    lp.Hb = p->fwd_Hb;
    lp.lam = p->inv_lam;
    lp.Ls = p->inv_Ls;
    lp.F = F;
    lp.ftm = ftm;
    lp.ring_row = p->inv_ring_row;
    lp.nrows = p->nth;
    lp.ncol = p->inv_ncol;
    lp.mo = p->inv_mo;
    lp.status = p->status;
    lp.tile = p->tile_inv;
    lp.mlo = lowm_orders(p);
    *out = lp;
  }
  return S2B_OK;
}

template <typename Real>
static int inv_stage_post(s2b_plan* p, const Inv2Params& lp, void* f, char* ws, cudaStream_t s,
                          const double* ring_w, bool lowm_done = false) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  void* ftm = ws + align256(p->ws_inv_F);
  if (lp.nrings > 0 && !lowm_done)
    if (int rc_ = run_lowm_synth(p, lp, p->inv_rings, s)) return rc_;
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.ncol = p->inv_ncol;
  rp.mo = p->inv_mo;
  rp.reality = d.reality;
  rp.real_out = d.reality;
  rp.scale = 1.0;
  rp.desc = p->descs + p->row_desc;
  rp.ring_desc = d.sampling == S2B_HEALPIX ? p->ring_desc : nullptr;
  if (d.sampling == S2B_HEALPIX) rp.desc = p->descs;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.phi0 = d.sampling == S2B_HEALPIX ? p->hp_phi0 : nullptr;
  rp.tb = tables<Real>(p);
  rp.weights = ring_w;
  rp.in = ftm;
  rp.out = f;
  S2B_CK(launch_inv_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  return S2B_OK;
}

// Fork of the plan's auxiliary stream from s (atomic per plan) and its join back to s.
static int aux_fork(s2b_plan* p, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(p->fork_mu);
  S2B_CK(cudaEventRecord(p->aux_fork, s));
  S2B_CK(cudaStreamWaitEvent(p->aux, p->aux_fork, 0));
  return S2B_OK;
}

static int aux_join(s2b_plan* p, cudaStream_t s) {
  S2B_CK(cudaEventRecord(p->aux_join, p->aux));
  S2B_CK(cudaStreamWaitEvent(s, p->aux_join, 0));
  return S2B_OK;
}

// The latitudinal kernel of a single-plan call, between the plan's timing events.
static int launch_lat_inv(s2b_plan* p, const Inv2Params& lp, cudaStream_t s) {
  if (p->ev_begin[0]) S2B_CK(cudaEventRecord(p->ev_begin[0], s));
  S2B_CK(launch_inv2(p->fp64, p->dual, lp, s));
  if (p->ev_end[0]) S2B_CK(cudaEventRecord(p->ev_end[0], s));
  return S2B_OK;
}

static int launch_lat_fwd(s2b_plan* p, const Fwd2Params& lp, cudaStream_t s) {
  if (p->ev_begin[1]) S2B_CK(cudaEventRecord(p->ev_begin[1], s));
  S2B_CK(launch_fwd2(p->fp64, p->dual, lp, s));
  if (p->ev_end[1]) S2B_CK(cudaEventRecord(p->ev_end[1], s));
  return S2B_OK;
}

template <typename Real>
static int run_inverse(s2b_plan* p, const void* flm, void* f, char* ws, cudaStream_t s,
                       const double* ring_w = nullptr) {
  Inv2Params lp{};
  int rc;
  if ((rc = inv_stage_pre<Real>(p, flm, ws, s, &lp))) return rc;
  bool lowm_done = false;
  if (lp.nrings > 0) {
    // the low orders (columns m < |s|, disjoint from the kernel's) beside the kernel: a few
    // CTAs of long sequential loops that would otherwise run alone after it
    if (lp.mlo > 0 && p->aux) {
      if ((rc = aux_fork(p, s))) return rc;
      if ((rc = run_lowm_synth(p, lp, p->inv_rings, p->aux))) {
        aux_join(p, s);
        return rc;
      }
      lowm_done = true;
    }
    rc = launch_lat_inv(p, lp, s);
    if (lowm_done) {
      const int jr = aux_join(p, s);  // after a failed launch too: nothing outlives the call
      if (!rc) rc = jr;
    }
    if (rc) return rc;
  }
  return inv_stage_post<Real>(p, lp, f, ws, s, ring_w, lowm_done);
}

// HEALPix ring FFTs alone (s2fft/utils/healpix_ffts.py:187-423): per ring FFT, fftshift and
// periodic extension to 2L columns (column c holds m = c - L), and the inverse with spectral
// folding; no ring phases, no normalisation in either direction.
template <typename Real>
static int run_healpix_fft(s2b_plan* p, const void* f, void* ftm, cudaStream_t s) {
  const s2b_desc& d = p->d;
  RowsParams<Real> rp{};
  rp.L = d.L;
  rp.nrows = p->nth;
  rp.real_in = d.reality;
  rp.reality = d.reality;
  rp.mode = FWD_TO_RAW;
  rp.M = 2 * d.L;
  rp.m0 = -d.L;
  rp.scale = 1.0;
  rp.desc = p->descs;
  rp.ring_desc = p->ring_desc;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.in = f;
  rp.out = ftm;
  S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  return S2B_OK;
}

template <typename Real>
static int run_healpix_ifft(s2b_plan* p, const void* ftm, void* f, cudaStream_t s) {
  const s2b_desc& d = p->d;
  RowsParams<Real> rp{};
  rp.L = d.L;
  rp.nrows = p->nth;
  rp.ncol = 2 * d.L;
  rp.mo = 1;
  rp.reality = d.reality;
  rp.rings_real_2L = 1;
  rp.real_out = d.reality;
  rp.scale = 1.0;
  rp.desc = p->descs;
  rp.ring_desc = p->ring_desc;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.in = ftm;
  rp.out = f;
  S2B_CK(launch_inv_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  return S2B_OK;
}

// Adjoint (conjugate transpose) of the inverse: unweighted ring DFTs of g_f, the forward
// projection over the inverse rings, and the pole rings in closed form.
template <typename Real>
static int run_inverse_adjoint(s2b_plan* p, const void* gf, void* gflm, char* ws,
                               cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  char* G = ws;
  char* acc = G + align256(p->ws_adj_G);
  S2B_CK(cudaMemsetAsync(acc, 0, p->ws_fwd_acc, s));
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.dual = p->dual;
  rp.nhalf = p->nhalf;
  rp.TR = p->TR;
  rp.Gs = p->adj_Gs;
  rp.scale = 1.0;
  rp.desc = p->descs + p->row_desc;
  if (d.sampling == S2B_HEALPIX) {
    rp.desc = p->descs;
    rp.ring_desc = p->ring_desc;
    rp.phi0 = p->hp_phi0;
  }
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.mode = FWD_TO_SPECTRA;
  rp.col_of_ring = p->adj_col;
  rp.in = gf;
  rp.out = G;
  S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  if (p->inv_nrings > 0) {
    Fwd2Params lp{};
    lp.L = L;
    lp.nrings = p->inv_nrings;
    lp.nhalf = p->nhalf;
    lp.batch = d.batch;
    lp.NB = p->fwd_NB;
    lp.Mst = p->inv_Mst;
    lp.Vst = p->inv_Vst;
    lp.Hb = p->fwd_Hb;
    lp.lam = p->inv_lam;
    lp.Ls = p->inv_Ls;
    lp.G = G;
    lp.Gs = p->adj_Gs;
    lp.acc = acc;
    lp.status = p->status;
    lp.mlo = lowm_orders(p);
    S2B_CK(launch_fwd2(p->fp64, p->dual, lp, s));
    if (int rc_ = run_lowm_project(p, lp, p->inv_rings, s)) return rc_;
  }
  StageParams sp{};
  sp.L = L;
  sp.L0 = d.L_lower;
  sp.spin = d.spin;
  sp.batch = d.batch;
  sp.nclass = p->nclass;
  sp.Q = p->Q;
  sp.TR = p->TR;
  sp.Gs = p->adj_Gs;
  sp.nhalf = p->nhalf;
  sp.dual = p->dual;
  sp.nrows = p->nth;
  sp.pole_south = p->adj_pole_s;
  sp.pole_north = p->adj_pole_n;
  sp.g = p->gtab;
  sp.G = G;
  sp.acc = acc;
  sp.Lp = p->fwd_NB * kFwdBlock;
  sp.flm_out = gflm;
  S2B_CK(launch_epilogue(p->fp64, sp, s));
  return S2B_OK;
}

// Adjoint of the (single-pass) forward. Direct samplings: the inverse followed by the ring
// quadrature weights. MW / MWSS: the inverse projection onto the MWSS(2L) rings, the adjoint
// of the column resampling chain, then unnormalised inverse ring DFTs.
template <typename Real>
static int run_forward_adjoint(s2b_plan* p, const void* gflm, void* gf, char* ws,
                               cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  if (p->fwd_mode == 0) return run_inverse<Real>(p, gflm, gf, ws, s, p->fwd_weights);
  char* F = ws;
  char* y = F + align256(p->ws_inv_F);
  char* ftm2 = y + align256(p->ws_adj_y);
  StageParams sp{};
  sp.ftm_zero_bytes = p->ws_adj_y;
  sp.L = L;
  sp.L0 = d.L_lower;
  sp.spin = d.spin;
  sp.batch = d.batch;
  sp.nclass = p->fwd_NB;
  sp.Q = kFwdBlock;
  sp.Lp = p->fwd_NB * kFwdBlock;
  sp.TR = p->TR;
  sp.nhalf = p->nhalf;
  sp.dual = p->dual;
  sp.nrows = 2 * L + 1;
  sp.ncol = 2 * L - 1;
  sp.mo = 0;
  sp.pole_south = p->fwd_pole_s;
  sp.pole_north = p->fwd_pole_n;
  sp.g = p->gtab;
  sp.flm = gflm;
  sp.F = F;
  sp.ftm = y;
  S2B_CK(launch_prologue(p->fp64, sp, s));
  Inv2Params lp{};
  lp.L = L;
  lp.nrings = p->fwd_nrings;
  lp.nhalf = p->nhalf;
  lp.batch = d.batch;
  lp.NB = p->fwd_NB;
  lp.Mst = p->fwd_Mst;
  lp.Vst = p->fwd_Vst;
  lp.Hb = p->fwd_Hb;
  lp.lam = p->fwd_lam;
  lp.Ls = p->fwd_Ls;
  lp.F = F;
  lp.ftm = y;
  lp.ring_row = p->fwd_ring_row;
  lp.nrows = 2 * L + 1;
  lp.ncol = 2 * L - 1;
  lp.mo = 0;
  lp.status = p->status;
  lp.mlo = lowm_orders(p);
  S2B_CK(launch_inv2(p->fp64, p->dual, lp, s));
  if (int rc_ = run_lowm_synth(p, lp, p->fwd_rings, s)) return rc_;
  ColsParams<Real> cp{};
  cp.L = L;
  cp.spin = d.spin;
  cp.mw = p->fwd_mode == 1;
  cp.nin = p->nth;
  cp.dual = p->dual;
  cp.nhalf = p->nhalf;
  cp.TR = p->TR;
  cp.scale = p->fwd_mode == 1 ? (2.0 * L) / (2.0 * L - 1.0) : 1.0;
  cp.d1 = p->descs + p->col_d1;
  cp.d2 = p->descs + p->col_d2;
  cp.weights = p->fwd_weights;
  cp.ph_adj = p->col_ph_adj;
  cp.pole = p->col_pole;
  cp.tb = tables<Real>(p);
  cp.in = y;
  cp.out = ftm2;
  const int ncm = p->fwd_mode == 1 ? 2 * L - 1 : 2 * L;
  S2B_CK(launch_mw_cols_adj<Real>(cp, ncm, d.batch, p->M1, p->M2, p->inv_ncol, p->inv_mo, s));
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.ncol = p->inv_ncol;
  rp.mo = p->inv_mo;
  rp.scale = 1.0;
  rp.desc = p->descs + p->row_desc;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.in = ftm2;
  rp.out = gf;
  S2B_CK(launch_inv_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  return S2B_OK;
}

// The forward in the same three stages as the inverse: ring FFTs (and the column chain)
// filling the latitudinal kernel's parameters (`lp`, and `lp_all` with every ring for the
// low orders), the kernel, and the low orders with the epilogue.
template <typename Real>
static int fwd_stage_pre(s2b_plan* p, const void* f, char* ws, cudaStream_t s, Fwd2Params* lp_out,
                         Fwd2Params* lp_all_out) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  char* cols = ws;
  char* G = cols + align256(p->ws_fwd_cols);
  char* acc = G + align256(p->ws_fwd_G);
  char* G2 = acc + align256(p->ws_fwd_acc);
  RowsParams<Real> rp{};
  // the ring transforms clear the accumulators (a whole number of 16-byte units)
  if (p->ws_fwd_acc % 16 == 0) {
    rp.zero = acc;
    rp.zero16 = (long)(p->ws_fwd_acc / 16);
  } else {
    S2B_CK(cudaMemsetAsync(acc, 0, p->ws_fwd_acc, s));
  }
  rp.L = L;
  rp.nrows = p->fwd_mode ? p->nth : p->fwd_nrows;
  rp.mo = p->fwd_mode == 2 ? 1 : 0;
  rp.real_in = d.reality;
  rp.dual = p->dual;
  rp.nhalf = p->nhalf;
  rp.TR = p->TR;
  rp.Gs = p->Gs;
  rp.scale = 1.0;
  rp.desc = p->descs + p->row_desc;
  rp.ring_desc = nullptr;
  if (d.sampling == S2B_HEALPIX) {
    rp.desc = p->descs;
    rp.ring_desc = p->ring_desc;
    rp.phi0 = p->hp_phi0;
  }
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.in = f;
  if (p->fwd_mode == 0) {
    rp.mode = FWD_TO_SPECTRA;
    rp.weights = p->fwd_weights;
    rp.out = G;
    S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
    if (p->fwd_sym) {
      FoldParams fo{};
      fo.L = L;
      fo.nhalf = p->nhalf;
      fo.dual = p->dual;
      fo.TR = p->TR;
      fo.Gs = p->Gs;
      fo.Gs2 = p->Gs2;
      fo.nrows = p->nth;
      fo.npair = p->sym_npair;
      fo.batch = d.batch;
      fo.cross = p->fwd_cross;
      fo.G = G;
      fo.G2 = G2;
      S2B_CK(launch_fold_pairs(p->fp64, fo, s));
    }
  } else {
    rp.mode = FWD_TO_COLS;
    rp.out = cols;
    S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
    ColsParams<Real> cp{};
    cp.L = L;
    cp.spin = d.spin;
    cp.mw = p->fwd_mode == 1;
    cp.nin = p->nth;
    cp.dual = p->dual;
    cp.nhalf = p->nhalf;
    cp.TR = p->TR;
    cp.Gs = p->Gs;
    cp.scale = p->fwd_mode == 1 ? (2.0 * L) / (2.0 * L - 1.0) : 1.0;
    cp.d1 = p->descs + p->col_d1;
    cp.d2 = p->descs + p->col_d2;
    cp.d2_pow2 = p->M2 == 4 * L;
    cp.ph = p->col_ph;
    cp.pole = p->col_pole;
    cp.imp = p->col_imp;
    cp.nyq_split = p->col_nyq_split;
    cp.weights = p->fwd_weights;
    cp.tb = tables<Real>(p);
    cp.in = cols;
    cp.out = G;
    cp.out2 = (p->fwd_sym && !p->fwd_cross) ? G2 : nullptr;
    cp.Gs2 = p->Gs2;
    const int ncm = p->fwd_mode == 1 ? 2 * L - 1 : 2 * L;
    S2B_CK(launch_mw_cols<Real>(cp, ncm, d.batch, p->M1, p->M2, s));
    if (p->fwd_cross) {
      FoldParams fo{};
      fo.L = L;
      fo.nhalf = p->nhalf;
      fo.TR = p->TR;
      fo.Gs = p->Gs;
      fo.Gs2 = p->Gs2;
      fo.nrows = p->fwd_nrings;  // rows 0..2L-2: the recursed MWSS(2L) rings in theta order
      fo.npair = p->sym_npair;
      fo.batch = d.batch;
      fo.cross = 1;
      fo.G = G;
      fo.G2 = G2;
      S2B_CK(launch_fold_pairs(p->fp64, fo, s));
    }
  }
  Fwd2Params lp{};
  lp.L = L;
  lp.nrings = p->fwd_nrings;
  lp.nhalf = p->nhalf;
  lp.batch = d.batch;
  lp.NB = p->fwd_NB;
  lp.Mst = p->fwd_Mst;
  lp.Vst = p->fwd_Vst;
  lp.Hb = p->fwd_Hb;
  lp.lam = p->fwd_lam;
  lp.Ls = p->fwd_Ls;
  lp.G = G;
  lp.Gs = p->Gs;
  lp.acc = acc;
  lp.status = p->status;
  lp.tile = p->tile_fwd;
  lp.mlo = lowm_orders(p);
  *lp_all_out = lp;  // every ring and G: the low orders (lowm.cu) run on these
  if (p->fwd_sym) {
    // ring pairs: the northern forward rings (and the equator) with their mirrors folded in
    lp.sym = 1;
    lp.cross = p->fwd_cross;
    lp.nrings = p->sym_npair;
    lp.Mst = p->sym_Mst;
    lp.Vst = p->sym_Vst;
    lp.Mst1 = p->sym_Mst1;
    lp.Vst1 = p->sym_Vst1;
    lp.nseg = p->fwd_nseg;
    lp.G = G2;
    lp.Gs = p->Gs2;
  }
  *lp_out = lp;
  return S2B_OK;
}

template <typename Real>
static int fwd_stage_post(s2b_plan* p, const Fwd2Params& lp_all, void* flm, char* ws,
                          cudaStream_t s, bool lowm_done = false) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  char* G = ws + align256(p->ws_fwd_cols);
  char* acc = G + align256(p->ws_fwd_G);
  if (!lowm_done)
    if (int rc_ = run_lowm_project(p, lp_all, p->fwd_rings, s)) return rc_;
  StageParams sp{};
  sp.L = L;
  sp.L0 = d.L_lower;
  sp.spin = d.spin;
  sp.batch = d.batch;
  sp.nclass = p->nclass;
  sp.Q = p->Q;
  sp.TR = p->TR;
  sp.Gs = p->Gs;
  sp.nhalf = p->nhalf;
  sp.dual = p->dual;
  sp.nrows = p->fwd_nrows;
  sp.pole_south = p->fwd_pole_s;
  sp.pole_north = p->fwd_pole_n;
  sp.g = p->gtab;
  sp.G = G;
  sp.acc = acc;
  sp.Lp = p->fwd_NB * kFwdBlock;
  sp.flm_out = flm;
  S2B_CK(launch_epilogue(p->fp64, sp, s));
  return S2B_OK;
}

template <typename Real>
static int run_forward_once(s2b_plan* p, const void* f, void* flm, char* ws, cudaStream_t s) {
  Fwd2Params lp{}, lp_all{};
  int rc;
  if ((rc = fwd_stage_pre<Real>(p, f, ws, s, &lp, &lp_all))) return rc;
  // the low orders (rows m < |s| of the accumulator, disjoint from the kernel's) beside it
  const bool lowm_aux = lp_all.mlo > 0 && lp_all.nrings > 0 && p->aux;
  if (lowm_aux) {
    if ((rc = aux_fork(p, s))) return rc;
    if ((rc = run_lowm_project(p, lp_all, p->fwd_rings, p->aux))) {
      aux_join(p, s);
      return rc;
    }
  }
  rc = launch_lat_fwd(p, lp, s);
  if (lowm_aux) {
    const int jr = aux_join(p, s);  // after a failed launch too: nothing outlives the call
    if (!rc) rc = jr;
  }
  if (rc) return rc;
  return fwd_stage_post<Real>(p, lp_all, flm, ws, s, lowm_aux);
}

template <typename Real>
static int run_forward(s2b_plan* p, const void* f, void* flm, char* ws, cudaStream_t s) {
  const s2b_desc& d = p->d;
  int rc = run_forward_once<Real>(p, f, flm, ws, s);
  if (rc || d.iter <= 0) return rc;
  // Jacobi refinement: flm += F(f - I(flm))   (iterative_refinement.py:9-46)
  const size_t scratch = std::max(fwd_once_ws(p), inv_ws(p));
  char* fr = ws + scratch;
  char* dflm = fr + align256(p->ws_iter_f);
  const long nf = (long)d.batch * p->npix * (d.reality ? 1 : 2);
  const long nflm = (long)d.batch * d.L * (2 * d.L - 1);
  for (int it = 0; it < d.iter; ++it) {
    if ((rc = run_inverse<Real>(p, flm, fr, ws, s))) return rc;
    S2B_CK(launch_sub(p->fp64, nf, f, fr, fr, s));
    if ((rc = run_forward_once<Real>(p, fr, dflm, ws, s))) return rc;
    S2B_CK(launch_axpy(p->fp64, nflm, 1.0, dflm, flm, s));
  }
  return S2B_OK;
}

// ----------------------------------------------------------------------------
// Precompute-kernel transforms (s2fft/precompute_transforms/spherical.py)
// ----------------------------------------------------------------------------
static size_t kernel_bytes(const s2b_plan* p, bool forward) {
  const int nth = forward ? p->knth_fwd : p->knth_inv;
  const int hpc = p->d.sampling == S2B_HEALPIX;
  if (p->tc) return forward ? tc_packed_a_bytes(nth, p->d.L, p->kM, hpc)
                            : tc_packed_a_bytes(p->d.L, nth, p->kM, hpc);
  const size_t el = (p->d.sampling == S2B_HEALPIX ? 2 : 1) * p->rsz;
  return (size_t)nth * p->d.L * p->kM * el;
}

static int build_kernel(s2b_plan* p, bool forward, void* K, cudaStream_t s) {
  const s2b_desc& d = p->d;
  KernelTableParams kp{};
  kp.L = d.L;
  kp.spin = d.spin;
  kp.reality = d.reality;
  kp.forward = forward;
  kp.complex_out = d.sampling == S2B_HEALPIX;
  kp.nth = forward ? p->knth_fwd : p->knth_inv;
  kp.theta = forward ? p->kth_fwd : p->kth_inv;
  kp.weights = forward ? p->fwd_weights : nullptr;
  kp.phi0 = d.sampling == S2B_HEALPIX ? p->hp_phi0 : nullptr;
  kp.lbin = p->lbin;
  kp.out = K;
  if (p->tc) {
    // float table in a temporary buffer, then split into bf16 hi/lo and packed for the MMA
    // (rows l and k = theta for the forward, rows theta and k = l for the inverse)
    const size_t tb = (size_t)kp.nth * d.L * p->kM * sizeof(float) * (kp.complex_out ? 2 : 1);
    void* tmp = nullptr;
    S2B_CK(dev_malloc(&tmp, tb));
    kp.out = tmp;
    cudaError_t e = launch_kernel_table(false, kp, s);
    if (e == cudaSuccess)
      e = launch_tc_pack_a((const float*)tmp, kp.nth, d.L, p->kM, forward ? 0 : 1,
                           kp.complex_out ? 1 : 0, K, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(tmp);
    S2B_CK(e);
    return S2B_OK;
  }
  S2B_CK(launch_kernel_table(p->fp64, kp, s));
  return S2B_OK;
}

template <typename Real>
static int run_pre_inverse(s2b_plan* p, const void* K, const void* flm, void* f, char* ws,
                           cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  void* ftm = ws;
  const size_t ftm_bytes = (size_t)d.batch * p->nth * p->inv_ncol * 2 * p->rsz;
  S2B_CK(cudaMemsetAsync(ftm, 0, ftm_bytes, s));
  PreContractParams cp{};
  cp.L = L;
  cp.nth = p->nth;
  cp.M = p->kM;
  cp.batch = d.batch;
  cp.mshift = d.reality ? L - 1 : 0;
  cp.mo = p->inv_mo + cp.mshift;
  cp.ncol = p->inv_ncol;
  cp.sign = (d.spin & 1) ? -1.0 : 1.0;
  cp.K = K;
  cp.in = flm;
  cp.out = ftm;
  if (p->tc) {
    // per column: ftm[b][t] = sum_l K[t][l] flm[b][l] on the tensor cores (bf16 x3)
    char* bp = ws + align256(ftm_bytes);
    const int hpc = d.sampling == S2B_HEALPIX;
    S2B_CK(launch_tc_pack_b(flm, d.batch, L, p->kM, (long)L * (2 * L - 1), 2 * L - 1,
                            cp.mshift, hpc, bp, s));
    TcParams tp{};
    tp.L = L;
    tp.nth = p->nth;
    tp.M = p->kM;
    tp.B = d.batch;
    tp.rows = p->nth;
    tp.kdim = L;
    tp.cplx = hpc;
    tp.sign = (float)cp.sign;
    tp.Ap = reinterpret_cast<const __nv_bfloat16*>(K);
    tp.Bp = reinterpret_cast<const __nv_bfloat16*>(bp);
    tp.out = reinterpret_cast<float2*>(ftm);
    tp.out_map = (long)p->nth * p->inv_ncol;
    tp.out_row = p->inv_ncol;
    tp.out_col0 = cp.mo;
    tp.status = p->status;
    if (p->ev_begin[0]) S2B_CK(cudaEventRecord(p->ev_begin[0], s));
    S2B_CK(launch_tc_forward(tp, s));
    if (p->ev_end[0]) S2B_CK(cudaEventRecord(p->ev_end[0], s));
  } else {
    S2B_CK(launch_pre_contract(p->fp64, false, d.sampling == S2B_HEALPIX, cp, s));
  }
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.ncol = p->inv_ncol;
  rp.mo = p->inv_mo;
  rp.reality = d.reality;
  rp.real_out = d.reality;
  rp.scale = 1.0;
  rp.desc = d.sampling == S2B_HEALPIX ? p->descs : p->descs + p->row_desc;
  rp.ring_desc = d.sampling == S2B_HEALPIX ? p->ring_desc : nullptr;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.phi0 = nullptr;  // the HEALPix phases are folded into the kernel table
  rp.tb = tables<Real>(p);
  rp.in = ftm;
  rp.out = f;
  S2B_CK(launch_inv_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  return S2B_OK;
}

template <typename Real>
static int run_pre_forward(s2b_plan* p, const void* K, const void* f, void* flm, char* ws,
                           cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  char* cols = ws;
  char* raw = cols + align256(p->ws_fwd_cols);
  const int m0 = d.reality ? 0 : -(L - 1);
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.mo = p->fwd_mode == 2 ? 1 : 0;
  rp.real_in = d.reality;
  rp.scale = 1.0;
  rp.desc = d.sampling == S2B_HEALPIX ? p->descs : p->descs + p->row_desc;
  rp.ring_desc = d.sampling == S2B_HEALPIX ? p->ring_desc : nullptr;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.in = f;
  rp.M = p->kM;
  rp.m0 = m0;
  if (p->fwd_mode == 0) {
    rp.mode = FWD_TO_RAW;
    rp.out = raw;
    S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  } else {
    rp.mode = FWD_TO_COLS;
    rp.out = cols;
    S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
    ColsParams<Real> cp{};
    cp.L = L;
    cp.spin = d.spin;
    cp.mw = p->fwd_mode == 1;
    cp.nin = p->nth;
    cp.raw = 1;
    cp.M = p->kM;
    cp.m0 = m0;
    cp.scale = p->fwd_mode == 1 ? (2.0 * L) / (2.0 * L - 1.0) : 1.0;
    cp.d1 = p->descs + p->col_d1;
    cp.d2 = p->descs + p->col_d2;
    cp.d2_pow2 = p->M2 == 4 * L;
    cp.ph = p->col_ph;
    cp.pole = p->col_pole;
    cp.imp = p->col_imp;
    cp.nyq_split = p->col_nyq_split;
    cp.weights = p->fwd_weights;
    cp.tb = tables<Real>(p);
    cp.in = cols;
    cp.out = raw;
    const int ncm = p->fwd_mode == 1 ? 2 * L - 1 : 2 * L;
    S2B_CK(launch_mw_cols<Real>(cp, ncm, d.batch, p->M1, p->M2, s));
  }
  S2B_CK(cudaMemsetAsync(flm, 0, (size_t)d.batch * L * (2 * L - 1) * 2 * p->rsz, s));
  if (p->tc) {
    char* bp = raw + align256((size_t)d.batch * p->knth_fwd * p->kM * 2 * p->rsz);
    const int hpc = d.sampling == S2B_HEALPIX;
    S2B_CK(launch_tc_pack_b(raw, d.batch, p->knth_fwd, p->kM, (long)p->knth_fwd * p->kM, p->kM,
                            0, hpc, bp, s));
    TcParams tp{};
    tp.L = L;
    tp.nth = p->knth_fwd;
    tp.M = p->kM;
    tp.B = d.batch;
    tp.rows = L;
    tp.kdim = p->knth_fwd;
    tp.cplx = hpc;
    tp.out_map = (long)L * (2 * L - 1);
    tp.out_row = 2 * L - 1;
    tp.out_col0 = L - 1 + m0;
    tp.sign = (d.spin & 1) ? -1.f : 1.f;
    tp.Ap = reinterpret_cast<const __nv_bfloat16*>(K);
    tp.Bp = reinterpret_cast<const __nv_bfloat16*>(bp);
    tp.out = reinterpret_cast<float2*>(flm);
    tp.status = p->status;
    if (p->ev_begin[1]) S2B_CK(cudaEventRecord(p->ev_begin[1], s));
    S2B_CK(launch_tc_forward(tp, s));
    if (p->ev_end[1]) S2B_CK(cudaEventRecord(p->ev_end[1], s));
    if (d.reality) S2B_CK(launch_reality_mirror(false, flm, d.batch, L, s));
    return S2B_OK;
  }
  PreContractParams cp{};
  cp.L = L;
  cp.nth = p->knth_fwd;
  cp.M = p->kM;
  cp.batch = d.batch;
  cp.mshift = L - 1 + m0;
  cp.sign = (d.spin & 1) ? -1.0 : 1.0;
  cp.K = K;
  cp.in = raw;
  cp.out = flm;
  S2B_CK(launch_pre_contract(p->fp64, true, d.sampling == S2B_HEALPIX, cp, s));
  if (d.reality) S2B_CK(launch_reality_mirror(p->fp64, flm, d.batch, L, s));
  return S2B_OK;
}

// Adjoints of the precompute transforms (complex plans, float or double tables): the
// conjugate-transposed contraction with the same kernel table, composed with the adjoints
// of the ring stages (unnormalised ring DFTs for the inverse; for the forward, inverse
// ring DFTs and, on mw / mwss, the adjoint of the resampling chain in its raw form).
template <typename Real>
static int run_pre_inverse_adjoint(s2b_plan* p, const void* K, const void* gf, void* gflm,
                                   char* ws, cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  char* raw = ws;  // [B][nth][M] spectra of g_f, m = -(L-1) .. L-1
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.scale = 1.0;
  rp.desc = d.sampling == S2B_HEALPIX ? p->descs : p->descs + p->row_desc;
  rp.ring_desc = d.sampling == S2B_HEALPIX ? p->ring_desc : nullptr;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.in = gf;
  rp.out = raw;
  rp.mode = FWD_TO_RAW;
  rp.M = p->kM;
  rp.m0 = -(L - 1);
  S2B_CK(launch_fwd_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  PreContractParams cp{};
  cp.L = L;
  cp.nth = p->nth;  // the inverse table has the sampling's rings (as s2b_precompute_inverse)
  cp.M = p->kM;
  cp.batch = d.batch;
  cp.mshift = 0;
  cp.sign = (d.spin & 1) ? -1.0 : 1.0;
  cp.conj = 1;
  cp.K = K;
  cp.in = raw;
  cp.out = gflm;
  S2B_CK(launch_pre_contract(p->fp64, true, d.sampling == S2B_HEALPIX, cp, s));
  return S2B_OK;
}

template <typename Real>
static int run_pre_forward_adjoint(s2b_plan* p, const void* K, const void* gflm, void* gf,
                                   char* ws, cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int L = d.L;
  char* cols = ws;
  char* raw = cols + align256(p->ws_fwd_cols);  // [B][knth_fwd][M]
  PreContractParams cp{};
  cp.L = L;
  cp.nth = p->knth_fwd;
  cp.M = p->kM;
  cp.batch = d.batch;
  cp.mshift = 0;
  cp.mo = 0;
  cp.ncol = p->kM;
  cp.sign = (d.spin & 1) ? -1.0 : 1.0;
  cp.conj = 1;
  cp.K = K;
  cp.in = gflm;
  cp.out = raw;
  S2B_CK(launch_pre_contract(p->fp64, false, d.sampling == S2B_HEALPIX, cp, s));
  RowsParams<Real> rp{};
  rp.L = L;
  rp.nrows = p->nth;
  rp.scale = 1.0;
  rp.desc = d.sampling == S2B_HEALPIX ? p->descs : p->descs + p->row_desc;
  rp.ring_desc = d.sampling == S2B_HEALPIX ? p->ring_desc : nullptr;
  rp.ring_off = p->ring_off;
  rp.out_batch_stride = p->npix;
  rp.tb = tables<Real>(p);
  rp.out = gf;
  if (p->fwd_mode == 0) {
    rp.ncol = p->kM;
    rp.mo = 0;
    rp.in = raw;
  } else {
    ColsParams<Real> cc{};
    cc.L = L;
    cc.spin = d.spin;
    cc.mw = p->fwd_mode == 1;
    cc.nin = p->nth;
    cc.raw = 1;
    cc.scale = p->fwd_mode == 1 ? (2.0 * L) / (2.0 * L - 1.0) : 1.0;
    cc.d1 = p->descs + p->col_d1;
    cc.d2 = p->descs + p->col_d2;
    cc.ph_adj = p->col_ph_adj;
    cc.pole = p->col_pole;
    cc.tb = tables<Real>(p);
    cc.in = raw;
    cc.out = cols;
    const int ncm = p->fwd_mode == 1 ? 2 * L - 1 : 2 * L;
    S2B_CK(launch_mw_cols_adj<Real>(cc, ncm, d.batch, p->M1, p->M2, p->inv_ncol, p->inv_mo, s));
    rp.ncol = p->inv_ncol;
    rp.mo = p->inv_mo;
    rp.in = cols;
  }
  S2B_CK(launch_inv_rows<Real>(rp, p->nth, d.batch, p->maxM, s));
  return S2B_OK;
}

// ----------------------------------------------------------------------------
// Wigner (SO(3)) transforms: 2N-1 spin transforms + gamma DFT
// (s2fft/transforms/wigner.py:110-196, 442-533)
// ----------------------------------------------------------------------------
// Workspace of a call of the given kind (0 inverse, 1 forward, 2 inverse adjoint,
// 3 forward adjoint) on a spin plan.
static size_t ws_of(const s2b_plan* p, int kind) {
  switch (kind) {
    case 0: return inv_ws(p);
    case 1: return std::max(fwd_ws(p), pre_fwd_ws(p));
    case 2: return inv_adj_ws(p);
    default: return fwd_adj_ws(p);
  }
}

// One spin-transform call of the given kind in the plan's precision.
static int exec_call(s2b_plan* p, int kind, const void* in, void* out, char* ws, cudaStream_t s) {
  switch (kind) {
    case 0:
      return p->fp64 ? run_inverse<double>(p, in, out, ws, s) : run_inverse<float>(p, in, out, ws, s);
    case 1:
      return p->fp64 ? run_forward<double>(p, in, out, ws, s) : run_forward<float>(p, in, out, ws, s);
    case 2:
      return p->fp64 ? run_inverse_adjoint<double>(p, in, out, ws, s)
                     : run_inverse_adjoint<float>(p, in, out, ws, s);
    default:
      return p->fp64 ? run_forward_adjoint<double>(p, in, out, ws, s)
                     : run_forward_adjoint<float>(p, in, out, ws, s);
  }
}

// ----------------------------------------------------------------------------
// Batches of plans (an uneven batch: maps of different L, spin and sampling)
// ----------------------------------------------------------------------------
// Every stage before and after the latitudinal kernels runs per plan, spread over a few
// streams; the latitudinal kernels of all plans run as persistent launches (latinv.cu,
// latfwd.cu), one per kernel variant, whose CTAs pull (plan, tile) items from a device
// counter until the batch's work is done.
struct s2b_batch {
  int device = -1;
  bool fp64 = false;
  std::vector<s2b_plan*> plans;
  int* counters = nullptr;  // one work counter per launch slot (stream-ordered reuse)
  int ncounters = 0;
  static constexpr int kMaxStreams = 4;
  static constexpr int kMaxWaves = 4;
  int nstreams = 0;
  cudaStream_t stream[kMaxStreams] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kMaxStreams] = {};
  cudaEvent_t wave_done[kMaxWaves] = {};
  int waves = 1;   // s2b_batch_set_option key 0
  int per_sm = 0;  // key 1: CTAs per SM of the persistent launches (0: as many as fit)
};

// The lanes wait for everything issued so far on s (ev: an event of the batch).
static int batch_fork(s2b_batch* b, cudaStream_t s, cudaEvent_t ev = nullptr) {
  if (b->nstreams < 2) return S2B_OK;
  if (!ev) {
    ev = b->fork;
    S2B_CK(cudaEventRecord(ev, s));
  }
  for (int k = 0; k < b->nstreams; ++k) S2B_CK(cudaStreamWaitEvent(b->stream[k], ev, 0));
  return S2B_OK;
}

static int batch_join(s2b_batch* b, cudaStream_t s) {
  if (b->nstreams < 2) return S2B_OK;
  for (int k = 0; k < b->nstreams; ++k) {
    S2B_CK(cudaEventRecord(b->join[k], b->stream[k]));
    S2B_CK(cudaStreamWaitEvent(s, b->join[k], 0));
  }
  return S2B_OK;
}

static cudaStream_t batch_lane(const s2b_batch* b, int k, cudaStream_t s) {
  return b->nstreams < 2 ? s : b->stream[k % b->nstreams];
}

// Entries of wave w when n entries are dealt round-robin into nw waves.
static std::vector<int> wave_members(int n, int nw, int w) {
  std::vector<int> m;
  for (int k = w; k < n; k += nw) m.push_back(k);
  return m;
}

// The latitudinal kernels of the entries `sel`: one persistent launch per kernel variant
// (Key: the fields a launch must share) and per kBatchPlans entries.
template <typename P, typename Key>
static int batch_launch_lat(s2b_batch* b, const std::vector<int>& idx, const std::vector<P>& lp,
                            const std::vector<int>& sel, Key key, int* slot, cudaStream_t s,
                            cudaError_t (*launch)(bool, bool, const P*, int, int*, int,
                                                  cudaStream_t)) {
  std::vector<char> done(sel.size(), 0);
  std::vector<P> grp;
  for (size_t a = 0; a < sel.size(); ++a) {
    const int k = sel[a];
    if (done[a] || lp[k].nrings <= 0) continue;
    const bool dual = b->plans[idx[k]]->dual;
    grp.clear();
    for (size_t c = a; c < sel.size() && (int)grp.size() < kBatchPlans; ++c) {
      const int j = sel[c];
      if (done[c] || lp[j].nrings <= 0 || b->plans[idx[j]]->dual != dual || !key(lp[j], lp[k]))
        continue;
      grp.push_back(lp[j]);
      done[c] = 1;
    }
    S2B_CK(launch(b->fp64, dual, grp.data(), (int)grp.size(),
                  b->counters + ((*slot)++ % b->ncounters), b->per_sm, s));
  }
  return S2B_OK;
}

// Stage-wise execution of entries idx[0..n): every entry's pre-stage on the lanes, the
// latitudinal kernels of each wave as persistent launches on s, and each wave's post-stages
// on the lanes once its launches are done. With several waves, the lanes' work of one wave
// (the ring FFTs are memory-bound) can overlap the latitudinal launches (FP32-bound) of the
// next. pre(k, lane, &lp[k]) and post(k, lane, lp[k]) run the stages of entry k.
template <typename P, typename Pre, typename Key, typename Post>
static int batch_staged_body(s2b_batch* b, const std::vector<int>& idx, cudaStream_t s, Pre pre,
                             Key key, Post post,
                             cudaError_t (*launch)(bool, bool, const P*, int, int*, int,
                                                   cudaStream_t)) {
  const int n = (int)idx.size();
  const int nw = std::max(1, std::min(std::min(b->waves, n), (int)s2b_batch::kMaxWaves));
  std::vector<P> lp(n);
  int rc, slot = 0;
  if ((rc = batch_fork(b, s))) return rc;
  for (int w = 0; w < nw; ++w) {
    const std::vector<int> mem = wave_members(n, nw, w);
    for (int k : mem)
      if ((rc = pre(k, batch_lane(b, k, s), &lp[k]))) return rc;
    if ((rc = batch_join(b, s))) return rc;
    if ((rc = batch_launch_lat<P>(b, idx, lp, mem, key, &slot, s, launch))) return rc;
    if (nw > 1) S2B_CK(cudaEventRecord(b->wave_done[w], s));
    if (w > 0) {  // the previous wave's post-stages, behind this wave's pre-stages
      if ((rc = batch_fork(b, s, b->wave_done[w - 1]))) return rc;
      for (int k : wave_members(n, nw, w - 1))
        if ((rc = post(k, batch_lane(b, k, s), lp[k]))) return rc;
    }
  }
  if ((rc = batch_fork(b, s, nw > 1 ? b->wave_done[nw - 1] : nullptr))) return rc;
  for (int k : wave_members(n, nw, nw - 1))
    if ((rc = post(k, batch_lane(b, k, s), lp[k]))) return rc;
  return batch_join(b, s);
}

// The staged execution; after a failure the batch's streams are still joined back to s, so
// that no work queued on them outlives the call and a capture of s stays complete.
template <typename P, typename Pre, typename Key, typename Post>
static int batch_staged(s2b_batch* b, const std::vector<int>& idx, cudaStream_t s, Pre pre,
                        Key key, Post post,
                        cudaError_t (*launch)(bool, bool, const P*, int, int*, int, cudaStream_t)) {
  const int rc = batch_staged_body<P>(b, idx, s, pre, key, post, launch);
  if (rc && b->nstreams > 1) {
    const std::string msg = g_last_error;
    batch_join(b, s);
    g_last_error = msg;  // report the first failure
  }
  return rc;
}

// The entries idx[0..n) of the batch: inputs in[k], outputs out[k], workspaces ws[k].
template <typename Real>
static int batch_run_inverse(s2b_batch* b, const std::vector<int>& idx, const void* const* in,
                             void* const* out, char* const* ws, cudaStream_t s) {
  return batch_staged<Inv2Params>(
      b, idx, s,
      [&](int k, cudaStream_t ls, Inv2Params* lp) {
        return inv_stage_pre<Real>(b->plans[idx[k]], in[k], ws[k], ls, lp);
      },
      [](const Inv2Params& x, const Inv2Params& y) { return x.sym == y.sym && x.tile == y.tile; },
      [&](int k, cudaStream_t ls, const Inv2Params& lp) {
        return inv_stage_post<Real>(b->plans[idx[k]], lp, out[k], ws[k], ls, nullptr);
      },
      launch_inv2_batch);
}

template <typename Real>
static int batch_run_forward_once(s2b_batch* b, const std::vector<int>& idx, const void* const* in,
                                  void* const* out, char* const* ws, cudaStream_t s) {
  std::vector<Fwd2Params> all(idx.size());
  return batch_staged<Fwd2Params>(
      b, idx, s,
      [&](int k, cudaStream_t ls, Fwd2Params* lp) {
        return fwd_stage_pre<Real>(b->plans[idx[k]], in[k], ws[k], ls, lp, &all[k]);
      },
      [](const Fwd2Params& x, const Fwd2Params& y) {
        return x.sym == y.sym && x.cross == y.cross && x.tile == y.tile;
      },
      [&](int k, cudaStream_t ls, const Fwd2Params&) {
        return fwd_stage_post<Real>(b->plans[idx[k]], all[k], out[k], ws[k], ls);
      },
      launch_fwd2_batch);
}

// Forward of every entry, with each plan's Jacobi refinement iterations run batch-wide
// (the entries with iter > it take part in iteration it), as run_forward does per plan.
template <typename Real>
static int batch_run_forward(s2b_batch* b, const void* const* f, void* const* flm,
                             char* const* ws, cudaStream_t s) {
  const int n = (int)b->plans.size();
  std::vector<int> idx(n);
  int maxit = 0;
  for (int k = 0; k < n; ++k) {
    idx[k] = k;
    maxit = std::max(maxit, b->plans[k]->d.iter);
  }
  int rc = batch_run_forward_once<Real>(b, idx, f, flm, ws, s);
  for (int it = 0; !rc && it < maxit; ++it) {
    std::vector<int> sub;
    std::vector<const void*> in_f, in_flm;
    std::vector<void*> fr, dflm, acc_flm;
    std::vector<char*> wsub;
    for (int k = 0; k < n; ++k) {
      const s2b_plan* p = b->plans[k];
      if (p->d.iter <= it) continue;
      char* r = ws[k] + std::max(fwd_once_ws(p), inv_ws(p));
      sub.push_back(k);
      in_f.push_back(f[k]);
      in_flm.push_back(flm[k]);
      acc_flm.push_back(flm[k]);
      fr.push_back(r);
      dflm.push_back(r + align256(p->ws_iter_f));
      wsub.push_back(ws[k]);
    }
    if ((rc = batch_run_inverse<Real>(b, sub, in_flm.data(), fr.data(), wsub.data(), s))) break;
    for (size_t k = 0; k < sub.size(); ++k) {
      const s2b_plan* p = b->plans[sub[k]];
      const long nf = (long)p->d.batch * p->npix * (p->d.reality ? 1 : 2);
      S2B_CK(launch_sub(p->fp64, nf, in_f[k], fr[k], fr[k], s));
    }
    std::vector<const void*> fr_in(fr.begin(), fr.end());
    if ((rc = batch_run_forward_once<Real>(b, sub, fr_in.data(), dflm.data(), wsub.data(), s)))
      break;
    for (size_t k = 0; k < sub.size(); ++k) {
      const s2b_plan* p = b->plans[sub[k]];
      const long nflm = (long)p->d.batch * p->d.L * (2 * p->d.L - 1);
      S2B_CK(launch_axpy(p->fp64, nflm, 1.0, dflm[k], acc_flm[k], s));
    }
  }
  return rc;
}

// Column chain of a complex plan that transforms real maps (forward direction only):
// Re(c) for the MW pole correction and the split theta-Nyquist bin for MWSS, as a reality
// plan has them.
static int use_real_map_chain(s2b_plan* p) {
  return p->fwd_mode != 0 ? set_col_tables(p, true) : S2B_OK;
}

static int build_wigner(s2b_plan* p) {
  const s2b_desc& d = p->d;
  p->fp64 = d.precision == S2B_F64;
  p->rsz = p->fp64 ? 8 : 4;
  p->nth = ntheta(d.L, d.sampling, d.nside);
  p->nphi = d.sampling == S2B_HEALPIX ? 0 : nphi_equiang(d.L, d.sampling);
  p->npix = d.sampling == S2B_HEALPIX ? 12L * d.nside * d.nside : (long)p->nth * p->nphi;
  const int n0 = d.reality ? 0 : -(d.N - 1);
  for (int n = n0; n < d.N; ++n) {
    s2b_desc sd = d;
    sd.spin = -n;
    sd.reality = 0;
    sd.N = 0;
    sd.iter = 0;
    s2b_plan* sub = nullptr;
    int rc = s2b_plan_create(&sd, &sub);
    if (rc) return rc;
    p->subs.push_back(sub);
    // the slice n = 0 of a real signal is a real map: upstream transforms it as one
    // (wigner.py:521-530), so its MW / MWSS column chain takes the real-map corrections
    if (d.reality && n == 0 && (rc = use_real_map_chain(sub))) return rc;
    p->ws_w_sub = std::max(p->ws_w_sub, std::max(ws_of(sub, 0), ws_of(sub, 1)));
  }
  const size_t c2 = 2 * p->rsz;
  p->ws_w_fban = (size_t)(2 * d.N - 1) * d.batch * p->npix * c2;
  p->ws_w_tmp = (size_t)d.batch * d.L * (2 * d.L - 1) * c2;
  p->nwstream = std::min<int>(s2b_plan::kMaxWStreams, (int)p->subs.size());
  if (p->nwstream > 1) {
    S2B_CK(cudaEventCreateWithFlags(&p->wfork, cudaEventDisableTiming));
    for (int k = 0; k < p->nwstream; ++k) {
      S2B_CK(cudaStreamCreateWithFlags(&p->wstream[k], cudaStreamNonBlocking));
      S2B_CK(cudaEventCreateWithFlags(&p->wjoin[k], cudaEventDisableTiming));
    }
  }
  return S2B_OK;
}

// fban | per stream: (tmp | sub-transform workspace)
static size_t wigner_slot(const s2b_plan* p) { return align256(p->ws_w_tmp) + align256(p->ws_w_sub); }
static size_t wigner_ws(const s2b_plan* p) {
  return align256(p->ws_w_fban) + (size_t)std::max(1, p->nwstream) * wigner_slot(p);
}

static int run_wigner(s2b_plan* p, bool forward, const void* in, void* out, char* ws,
                      cudaStream_t s) {
  const s2b_desc& d = p->d;
  const int n0 = d.reality ? 0 : -(d.N - 1);
  const int K = p->nwstream > 1 ? p->nwstream : 1;
  char* fban = ws;
  const size_t slice = (size_t)d.batch * p->npix * 2 * p->rsz;
  int rc;
  if (forward) S2B_CK(launch_gamma_forward(p->fp64, in, fban, d.batch, d.N, p->npix, d.reality, s));
  if (K > 1) {
    std::lock_guard<std::mutex> lk(p->fork_mu);
    S2B_CK(cudaEventRecord(p->wfork, s));
    for (int k = 0; k < K; ++k) S2B_CK(cudaStreamWaitEvent(p->wstream[k], p->wfork, 0));
  }
  rc = S2B_OK;
  for (int n = n0; n < d.N && !rc; ++n) {
    const int k = (n - n0) % K;
    cudaStream_t sk = K > 1 ? p->wstream[k] : s;
    char* tmp = fban + align256(p->ws_w_fban) + (size_t)k * wigner_slot(p);
    char* subws = tmp + align256(p->ws_w_tmp);
    s2b_plan* sub = p->subs[n - n0];
    char* band = fban + (size_t)(d.N - 1 + n) * slice;
    cudaError_t e = cudaSuccess;
    if (!forward) {
      e = launch_gather_n(p->fp64, in, tmp, d.batch, d.N, d.L, n, d.reality && n == 0, sk);
      if (e == cudaSuccess) rc = exec_call(sub, 0, tmp, band, subws, sk);
    } else {
      rc = exec_call(sub, 1, band, tmp, subws, sk);
      if (!rc) e = launch_scatter_n(p->fp64, tmp, out, d.batch, d.N, d.L, n, d.L_lower, sk);
    }
    if (e != cudaSuccess) rc = fail(S2B_ERR_CUDA, std::string("Wigner gather/scatter: ") + cudaGetErrorString(e));
  }
  if (K > 1) {
    // join every forked stream back to the caller's stream, after an error too, so that no
    // work queued on them outlives the call (it uses the caller's workspace) and a stream
    // capture of the caller's stream stays complete
    for (int k = 0; k < K; ++k) {
      cudaError_t e = cudaEventRecord(p->wjoin[k], p->wstream[k]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, p->wjoin[k], 0);
      if (e != cudaSuccess && !rc) rc = fail(S2B_ERR_CUDA, std::string("Wigner join: ") + cudaGetErrorString(e));
    }
  }
  if (rc) return rc;
  if (!forward) {
    S2B_CK(launch_gamma_inverse(p->fp64, fban, out, d.batch, d.N, p->npix, d.reality, s));
  } else if (d.reality) {
    S2B_CK(launch_wigner_mirror(p->fp64, out, d.batch, d.N, d.L, s));
  }
  return S2B_OK;
}

// FFT descriptors and tables for a list of lengths, in device memory owned by *allocs
// (used by the Fourier-Wigner plans, which have no spin plan around them).
template <typename T>
static int upload_to(std::vector<void*>* allocs, T** dst, const std::vector<T>& src) {
  *dst = nullptr;
  if (src.empty()) return S2B_OK;
  void* ptr = nullptr;
  S2B_CK(dev_malloc(&ptr, src.size() * sizeof(T)));
  allocs->push_back(ptr);
  S2B_CK(cudaMemcpy(ptr, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  *dst = reinterpret_cast<T*>(ptr);
  return S2B_OK;
}

static int upload_complex_to(std::vector<void*>* allocs, bool fp64, void** dst,
                             const std::vector<cd>& src) {
  if (fp64) {
    std::vector<double2> v(src.size());
    for (size_t i = 0; i < src.size(); ++i) v[i] = make_double2(src[i].real(), src[i].imag());
    double2* d = nullptr;
    const int rc = upload_to(allocs, &d, v);
    *dst = d;
    return rc;
  }
  std::vector<float2> v(src.size());
  for (size_t i = 0; i < src.size(); ++i)
    v[i] = make_float2((float)src[i].real(), (float)src[i].imag());
  float2* d = nullptr;
  const int rc = upload_to(allocs, &d, v);
  *dst = d;
  return rc;
}

int s2b::build_fft_set(const int* lengths, int count, bool fp64, std::vector<void*>* allocs,
                       FFTSet* out) {
  FFTBuild fb;
  out->host.clear();
  std::vector<int> idx(count);
  for (int i = 0; i < count; ++i) {
    if (lengths[i] < 2) return fail(S2B_ERR_INVALID, "FFT length must be >= 2");
    idx[i] = fb.add(lengths[i]);
  }
  for (int i = 0; i < count; ++i) out->host.push_back(fb.descs[idx[i]]);
  int rc;
  if ((rc = upload_complex_to(allocs, fp64, &out->tw, fb.tw))) return rc;
  if ((rc = upload_complex_to(allocs, fp64, &out->chirp, fb.chirp))) return rc;
  if ((rc = upload_complex_to(allocs, fp64, &out->bf, fb.bf))) return rc;
  return S2B_OK;
}

// ----------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------
extern "C" {

int s2b_version(void) { return 100; }

const char* s2b_last_error(void) { return g_last_error.c_str(); }

int s2b_plan_create(const s2b_desc* desc, s2b_plan** out) {
  g_last_error.clear();
  if (!desc || !out) return fail(S2B_ERR_INVALID, "desc and plan must be non-NULL");
  const s2b_desc& d = *desc;
  if (d.L < 2) return fail(S2B_ERR_INVALID, "L must be >= 2");
  if (d.sampling < S2B_MW || d.sampling > S2B_HEALPIX)
    return fail(S2B_ERR_INVALID, "unknown sampling");
  if (d.sampling == S2B_HEALPIX) {
    if (d.nside < 1) return fail(S2B_ERR_INVALID, "healpix sampling needs nside >= 1");
    if (d.L < 2 * d.nside) return fail(S2B_ERR_INVALID, "healpix requires L >= 2*nside");
  }
  if (d.precision != S2B_F64 && d.precision != S2B_F32 && d.precision != S2B_BF16X3)
    return fail(S2B_ERR_INVALID, "unknown precision");
  if (d.precision == S2B_BF16X3 && d.N > 0)
    return fail(S2B_ERR_INVALID, "BF16x3 plans support the precompute path of spin transforms");
  if (d.reality && d.spin != 0) return fail(S2B_ERR_INVALID, "reality requires spin 0");
  if (std::abs(d.spin) >= d.L) return fail(S2B_ERR_INVALID, "|spin| must be < L");
  if (d.L_lower < 0 || d.L_lower >= d.L) return fail(S2B_ERR_INVALID, "0 <= L_lower < L");
  if (d.batch < 1) return fail(S2B_ERR_INVALID, "batch must be >= 1");
  if (d.iter < 0) return fail(S2B_ERR_INVALID, "iter must be >= 0");
  if (d.L > 8192) return fail(S2B_ERR_INVALID, "L > 8192 not supported");
  if (d.N < 0 || d.N > d.L) return fail(S2B_ERR_INVALID, "0 <= N <= L required");
  if (d.N > 0 && d.iter != 0) return fail(S2B_ERR_INVALID, "iter is not used by Wigner plans");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(S2B_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  s2b_plan* p = new s2b_plan();
  p->d = d;
  p->device = dev;
  int rc = d.N > 0 ? build_wigner(p) : build_plan(p);
  if (rc) {
    s2b_plan_destroy(p);
    return rc;
  }
  *out = p;
  return S2B_OK;
}

int s2b_plan_destroy(s2b_plan* p) {
  if (!p) return S2B_OK;
  for (s2b_plan* sp : p->subs) s2b_plan_destroy(sp);
  for (void* a : p->allocs) cudaFree(a);
  if (p->aux) cudaStreamDestroy(p->aux);
  if (p->aux_fork) cudaEventDestroy(p->aux_fork);
  if (p->aux_join) cudaEventDestroy(p->aux_join);
  for (int k = 0; k < s2b_plan::kMaxWStreams; ++k) {
    if (p->wstream[k]) cudaStreamDestroy(p->wstream[k]);
    if (p->wjoin[k]) cudaEventDestroy(p->wjoin[k]);
  }
  if (p->wfork) cudaEventDestroy(p->wfork);
  delete p;
  return S2B_OK;
}

int s2b_workspace_size(const s2b_plan* p, int forward, size_t* bytes) {
  if (!p || !bytes) return fail(S2B_ERR_INVALID, "plan and bytes must be non-NULL");
  if (forward < 0 || forward > 3) return fail(S2B_ERR_INVALID, "direction must be 0..3");
  if (p->d.N > 0)
    *bytes = wigner_ws(p);
  else
    *bytes = ws_of(p, forward);
  return S2B_OK;
}

int s2b_inverse(s2b_plan* p, const void* flm, void* f, void* ws, size_t ws_bytes, void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "plan is NULL or a Wigner plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(flm, "flm")) || (rc = check_ptr(f, "f")) || (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < ws_of(p, 0)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  return exec_call(p, 0, flm, f, (char*)ws, reinterpret_cast<cudaStream_t>(stream));
}

int s2b_forward(s2b_plan* p, const void* f, void* flm, void* ws, size_t ws_bytes, void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "plan is NULL or a Wigner plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(flm, "flm")) || (rc = check_ptr(f, "f")) || (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < ws_of(p, 1)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  return exec_call(p, 1, f, flm, (char*)ws, reinterpret_cast<cudaStream_t>(stream));
}

int s2b_inverse_adjoint(s2b_plan* p, const void* g_f, void* g_flm, void* ws, size_t ws_bytes,
                        void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "plan is NULL or a Wigner plan");
  if (p->d.reality) return fail(S2B_ERR_INVALID, "adjoints are defined for complex plans (reality = 0)");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(g_f, "g_f")) || (rc = check_ptr(g_flm, "g_flm")) ||
      (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < ws_of(p, 2)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  return exec_call(p, 2, g_f, g_flm, (char*)ws, reinterpret_cast<cudaStream_t>(stream));
}

int s2b_forward_adjoint(s2b_plan* p, const void* g_flm, void* g_f, void* ws, size_t ws_bytes,
                        void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "plan is NULL or a Wigner plan");
  if (p->d.reality) return fail(S2B_ERR_INVALID, "adjoints are defined for complex plans (reality = 0)");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(g_flm, "g_flm")) || (rc = check_ptr(g_f, "g_f")) ||
      (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < ws_of(p, 3)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  return exec_call(p, 3, g_flm, g_f, (char*)ws, reinterpret_cast<cudaStream_t>(stream));
}

int s2b_batch_create(s2b_plan* const* plans, int nplans, s2b_batch** out) {
  g_last_error.clear();
  if (!plans || !out) return fail(S2B_ERR_INVALID, "plans and batch must be non-NULL");
  if (nplans < 1) return fail(S2B_ERR_INVALID, "a batch needs at least one plan");
  for (int k = 0; k < nplans; ++k) {
    const s2b_plan* p = plans[k];
    if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "batch entries must be spin plans");
    if (p->device != plans[0]->device)
      return fail(S2B_ERR_INVALID, "the plans of a batch must share one device");
    if (p->fp64 != plans[0]->fp64)
      return fail(S2B_ERR_INVALID, "the plans of a batch must share one precision");
  }
  int rc;
  if ((rc = check_device(plans[0]))) return rc;
  s2b_batch* b = new s2b_batch();
  b->device = plans[0]->device;
  b->fp64 = plans[0]->fp64;
  b->plans.assign(plans, plans + nplans);
  b->ncounters = 8;
  cudaError_t e = dev_malloc(&b->counters, sizeof(int) * b->ncounters);
  b->nstreams = nplans > 1 ? std::min(nplans, s2b_batch::kMaxStreams) : 0;
  for (int w = 0; e == cudaSuccess && w < s2b_batch::kMaxWaves; ++w)
    e = cudaEventCreateWithFlags(&b->wave_done[w], cudaEventDisableTiming);
  if (e == cudaSuccess && b->nstreams > 1) {
    e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int k = 0; e == cudaSuccess && k < b->nstreams; ++k) {
      e = cudaStreamCreateWithFlags(&b->stream[k], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming);
    }
  }
  if (e != cudaSuccess) {
    s2b_batch_destroy(b);
    return fail(S2B_ERR_CUDA, std::string("s2b_batch_create: ") + cudaGetErrorString(e));
  }
  *out = b;
  return S2B_OK;
}

int s2b_batch_destroy(s2b_batch* b) {
  if (!b) return S2B_OK;
  if (b->counters) cudaFree(b->counters);
  for (int k = 0; k < s2b_batch::kMaxStreams; ++k) {
    if (b->stream[k]) cudaStreamDestroy(b->stream[k]);
    if (b->join[k]) cudaEventDestroy(b->join[k]);
  }
  for (int w = 0; w < s2b_batch::kMaxWaves; ++w)
    if (b->wave_done[w]) cudaEventDestroy(b->wave_done[w]);
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
  return S2B_OK;
}

int s2b_batch_set_option(s2b_batch* b, int key, int value) {
  if (!b) return fail(S2B_ERR_INVALID, "batch must be non-NULL");
  if (key == 0 && value >= 1 && value <= s2b_batch::kMaxWaves)
    b->waves = value;
  else if (key == 1 && value >= 0 && value <= 32)
    b->per_sm = value;
  else
    return fail(S2B_ERR_INVALID, "key 0 (waves) takes 1 to 4, key 1 (CTAs per SM of the "
                                 "persistent launches, 0 = as many as fit) 0 to 32");
  return S2B_OK;
}

static int batch_check(s2b_batch* b, int kind, const void* const* in, void* const* out,
                       void* const* ws, const size_t* ws_bytes) {
  if (!b) return fail(S2B_ERR_INVALID, "batch is NULL");
  if (!in || !out || !ws || !ws_bytes)
    return fail(S2B_ERR_INVALID, "pointer arrays must be non-NULL");
  int rc;
  if ((rc = check_device(b->plans[0]))) return rc;
  for (size_t k = 0; k < b->plans.size(); ++k) {
    if ((rc = check_ptr(in[k], kind ? "f" : "flm")) || (rc = check_ptr(out[k], kind ? "flm" : "f")) ||
        (rc = check_ptr(ws[k], "workspace")))
      return rc;
    if (ws_bytes[k] < ws_of(b->plans[k], kind))
      return fail(S2B_ERR_WORKSPACE, "workspace of entry " + std::to_string(k) + " too small");
  }
  return S2B_OK;
}

int s2b_batch_inverse(s2b_batch* b, const void* const* flm, void* const* f, void* const* ws,
                      const size_t* ws_bytes, void* stream) {
  int rc;
  if ((rc = batch_check(b, 0, flm, f, ws, ws_bytes))) return rc;
  std::vector<int> idx(b->plans.size());
  for (size_t k = 0; k < idx.size(); ++k) idx[k] = (int)k;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* const* w = reinterpret_cast<char* const*>(ws);
  return b->fp64 ? batch_run_inverse<double>(b, idx, flm, f, w, s)
                 : batch_run_inverse<float>(b, idx, flm, f, w, s);
}

int s2b_batch_forward(s2b_batch* b, const void* const* f, void* const* flm, void* const* ws,
                      const size_t* ws_bytes, void* stream) {
  int rc;
  if ((rc = batch_check(b, 1, f, flm, ws, ws_bytes))) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* const* w = reinterpret_cast<char* const*>(ws);
  return b->fp64 ? batch_run_forward<double>(b, f, flm, w, s)
                 : batch_run_forward<float>(b, f, flm, w, s);
}

int s2b_healpix_fft(s2b_plan* p, const void* f, void* ftm, void* stream) {
  if (!p || p->d.N > 0 || p->d.sampling != S2B_HEALPIX)
    return fail(S2B_ERR_INVALID, "plan must be a HEALPix spin plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(f, "f")) || (rc = check_ptr(ftm, "ftm"))) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->fp64 ? run_healpix_fft<double>(p, f, ftm, s) : run_healpix_fft<float>(p, f, ftm, s);
}

int s2b_healpix_ifft(s2b_plan* p, const void* ftm, void* f, void* stream) {
  if (!p || p->d.N > 0 || p->d.sampling != S2B_HEALPIX)
    return fail(S2B_ERR_INVALID, "plan must be a HEALPix spin plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(f, "f")) || (rc = check_ptr(ftm, "ftm"))) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->fp64 ? run_healpix_ifft<double>(p, ftm, f, s) : run_healpix_ifft<float>(p, ftm, f, s);
}

int s2b_kernel_size(const s2b_plan* p, int forward, size_t* bytes) {
  if (!p || !bytes || p->d.N > 0) return fail(S2B_ERR_INVALID, "bad plan or bytes");
  *bytes = kernel_bytes(p, forward != 0);
  return S2B_OK;
}

int s2b_kernel_build(s2b_plan* p, int forward, void* K, void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "bad plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(K, "kernel"))) return rc;
  return build_kernel(p, forward != 0, K, reinterpret_cast<cudaStream_t>(stream));
}

int s2b_precompute_inverse(s2b_plan* p, const void* K, const void* flm, void* f, void* ws,
                           size_t ws_bytes, void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "bad plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(K, "kernel")) || (rc = check_ptr(flm, "flm")) || (rc = check_ptr(f, "f")) ||
      (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < inv_ws(p)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->fp64 ? run_pre_inverse<double>(p, K, flm, f, (char*)ws, s)
                 : run_pre_inverse<float>(p, K, flm, f, (char*)ws, s);
}

int s2b_precompute_forward(s2b_plan* p, const void* K, const void* f, void* flm, void* ws,
                           size_t ws_bytes, void* stream) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "bad plan");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(K, "kernel")) || (rc = check_ptr(flm, "flm")) || (rc = check_ptr(f, "f")) ||
      (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < pre_fwd_ws(p)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->fp64 ? run_pre_forward<double>(p, K, f, flm, (char*)ws, s)
                 : run_pre_forward<float>(p, K, f, flm, (char*)ws, s);
}

static int check_pre_adjoint(const s2b_plan* p) {
  if (!p || p->d.N > 0) return fail(S2B_ERR_INVALID, "bad plan");
  if (p->d.reality) return fail(S2B_ERR_INVALID, "adjoints are defined for complex plans (reality = 0)");
  if (p->tc) return fail(S2B_ERR_INVALID, "adjoints need a float or double kernel table (not BF16x3)");
  return check_device(p);
}

int s2b_precompute_inverse_adjoint(s2b_plan* p, const void* K, const void* g_f, void* g_flm,
                                   void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_pre_adjoint(p))) return rc;
  if ((rc = check_ptr(K, "kernel")) || (rc = check_ptr(g_f, "g_f")) ||
      (rc = check_ptr(g_flm, "g_flm")) || (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < inv_ws(p)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->fp64 ? run_pre_inverse_adjoint<double>(p, K, g_f, g_flm, (char*)ws, s)
                 : run_pre_inverse_adjoint<float>(p, K, g_f, g_flm, (char*)ws, s);
}

int s2b_precompute_forward_adjoint(s2b_plan* p, const void* K, const void* g_flm, void* g_f,
                                   void* ws, size_t ws_bytes, void* stream) {
  int rc;
  if ((rc = check_pre_adjoint(p))) return rc;
  if ((rc = check_ptr(K, "kernel")) || (rc = check_ptr(g_flm, "g_flm")) ||
      (rc = check_ptr(g_f, "g_f")) || (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < pre_fwd_ws(p)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->fp64 ? run_pre_forward_adjoint<double>(p, K, g_flm, g_f, (char*)ws, s)
                 : run_pre_forward_adjoint<float>(p, K, g_flm, g_f, (char*)ws, s);
}

int s2b_wigner_inverse(s2b_plan* p, const void* flmn, void* f, void* ws, size_t ws_bytes,
                       void* stream) {
  if (!p || p->d.N < 1) return fail(S2B_ERR_INVALID, "plan is not a Wigner plan (desc.N > 0)");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(flmn, "flmn")) || (rc = check_ptr(f, "f")) || (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < wigner_ws(p)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  return run_wigner(p, false, flmn, f, (char*)ws, reinterpret_cast<cudaStream_t>(stream));
}

int s2b_wigner_forward(s2b_plan* p, const void* f, void* flmn, void* ws, size_t ws_bytes,
                       void* stream) {
  if (!p || p->d.N < 1) return fail(S2B_ERR_INVALID, "plan is not a Wigner plan (desc.N > 0)");
  int rc;
  if ((rc = check_device(p))) return rc;
  if ((rc = check_ptr(flmn, "flmn")) || (rc = check_ptr(f, "f")) || (rc = check_ptr(ws, "workspace")))
    return rc;
  if (ws_bytes < wigner_ws(p)) return fail(S2B_ERR_WORKSPACE, "workspace too small");
  return run_wigner(p, true, f, flmn, (char*)ws, reinterpret_cast<cudaStream_t>(stream));
}

static int plan_status_word(const s2b_plan* p, int* out) {
  int st = 0;
  if (p->status) S2B_CK(cudaMemcpy(&st, p->status, sizeof(int), cudaMemcpyDeviceToHost));
  *out |= st;
  int rc;
  for (const s2b_plan* sp : p->subs)
    if ((rc = plan_status_word(sp, out))) return rc;
  return S2B_OK;
}

int s2b_plan_status(s2b_plan* p, int* status) {
  if (!p || !status) return fail(S2B_ERR_INVALID, "plan and status must be non-NULL");
  *status = 0;
  const int rc = plan_status_word(p, status);
  if (rc) return rc;
  if (*status) return fail(S2B_ERR_TIMEOUT, "a bounded device wait gave up");
  return S2B_OK;
}

int s2b_plan_set_tuning(s2b_plan* p, int key, int value) {
  if (!p) return fail(S2B_ERR_INVALID, "plan must be non-NULL");
  const bool tile = (key == 0 && (value == 0 || value == 1)) || (key == 1 && value >= 0 && value <= 3);
  const bool seg = (key == 2 || key == 3) && (value == 1 || value == 2 || value == 4 || value == 8);
  if (!tile && !seg)
    return fail(S2B_ERR_INVALID,
                "key 0 (forward tile) takes 0 or 1, key 1 (inverse tile) 0 to 3, keys 2 and 3 "
                "(inverse / forward segments along m) 1, 2, 4 or 8");
  if (key == 0)
    p->tile_fwd = value;
  else if (key == 1)
    p->tile_inv = value;
  else if (key == 2)
    p->inv_nseg = value;
  else
    p->fwd_nseg = value;
  for (s2b_plan* sp : p->subs) s2b_plan_set_tuning(sp, key, value);
  return S2B_OK;
}

long long s2b_device_alloc_count(void) { return g_dev_allocs.load(std::memory_order_relaxed); }

int s2b_plan_device(const s2b_plan* p, int* device) {
  if (!p || !device) return fail(S2B_ERR_INVALID, "plan and device must be non-NULL");
  *device = p->device;
  return S2B_OK;
}

int s2b_debug_set_plan_device(s2b_plan* p, int device) {
  if (!p) return fail(S2B_ERR_INVALID, "plan must be non-NULL");
  p->device = device;
  for (s2b_plan* sp : p->subs) s2b_debug_set_plan_device(sp, device);
  return S2B_OK;
}

int s2b_plan_set_events(s2b_plan* p, int forward, void* ev_begin, void* ev_end) {
  if (!p || (forward != 0 && forward != 1)) return fail(S2B_ERR_INVALID, "bad plan or direction");
  p->ev_begin[forward] = reinterpret_cast<cudaEvent_t>(ev_begin);
  p->ev_end[forward] = reinterpret_cast<cudaEvent_t>(ev_end);
  return S2B_OK;
}

}  // extern "C"
