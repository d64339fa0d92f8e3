// Rotation of spherical-harmonic coefficients by Euler angles (alpha, beta, gamma):
//   flm'[l, m] = exp(-i m alpha) sum_n d^l_{m,n}(beta) exp(-i n gamma) flm[l, n]
// (upstream s2fft/utils/rotation.py:9-64, rotate_flms), with the Wigner-d planes at beta
// generated degree by degree by Risbo's recursion (upstream s2fft/recursions/risbo.py:4-120;
// T. Risbo, J. Geodesy 70 (1996) 383-396).
//
// Own formulation: each degree takes two half-degree steps, l-1 -> l-1/2 -> l, each written
// as a gather. With c = cos(beta/2), s = sin(beta/2), a plane S of size j x j becomes H of
// size (j+1) x (j+1):
//   H[h][K] = sqrt(j-h) (c A S[h][K] + s B S[h][K-1]) + sqrt(h) (-s A S[h-1][K] + c B S[h-1][K-1]),
//   A = sqrt(j-K) / j, B = sqrt(K) / j, terms outside S dropped;
// from D_0 = [1], two steps per degree give D_l[l+m][l+n] = d^l_{m,n}(beta) (standard
// convention, checked against Wigner's explicit sum).
//
// Schedule: one cooperative launch (all CTAs resident) walks every degree. The rows of a
// plane are cut into row blocks of at most kRotRowsMax rows; a CTA owns fixed row blocks
// for all degrees. Row I of D_l needs rows I-2..I of D_{l-1}, so row block rb at degree l
// waits only for its two neighbours to have finished degree l-1 (flags with release /
// acquire, bounded polls) -- no grid-wide barrier. Inside a CTA each warp takes chunks of
// 31 columns (lane 0 computes the column to the left, which lane 1 needs) and walks the
// rows of the block, carrying the half-step row H[I-1] in registers, so the intermediate
// plane is never stored. The contraction with flm runs on the values as they are made;
// the planes themselves (two of (2L-1) x 2L doubles, 33 MB each at L = 1024) stay in L2.
// All arithmetic is double.
#include <cuda_runtime.h>

#include <cstdint>

#include "s2b.h"
#include "s2b_internal.h"
#include "s2b_rotation.h"

namespace s2b {
namespace {

constexpr int kChunk = 31;  // plane columns a warp produces per chunk

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

__device__ __forceinline__ int load_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// exp(-i n gamma) flm[b][l][L-1+n] for plane column K = l + n (zero outside the plane)
template <typename R2>
__device__ __forceinline__ double2 weighted_coef(const RotParams& p, int b, int l, int K,
                                                 bool valid) {
  if (!valid) return make_double2(0.0, 0.0);
  const int L = p.L, col = L - 1 - l + K;
  const double2 x = RotIO<R2>::get(p.flm, ((size_t)b * L + l) * (2 * L - 1) + col);
  const double2 g = p.eg[col];
  return make_double2(x.x * g.x - x.y * g.y, x.x * g.y + x.y * g.x);
}

// thread 0 polls the flags of the neighbouring row blocks until both have finished
// degree l-1 (when they existed then); false for every thread when a bound ran out
__device__ bool wait_neighbours(const RotParams& p, int rb, int l) {
  int ok = 1;
  if (threadIdx.x == 0) {
#pragma unroll 1
    for (int d = -1; d <= 1 && ok; d += 2) {
      const int nb = rb + d;
      if (nb < 0 || nb >= p.nrb || nb * p.rows >= 2 * l - 1) continue;
      long it = 0;
      while (load_acquire(p.done + nb) < l) {
        if (*reinterpret_cast<volatile int*>(p.err) != 0 || ++it > kRotSpinLimit) {
          atomicOr(p.err, 1);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
    }
  }
  return __syncthreads_and(ok) != 0;
}

// the rows of a block reduced over the CTA's warps, phased and written to out
template <typename R2>
__device__ void flush_rows(const RotParams& p, const double2 (*red)[kRotRowsMax], int b, int l,
                           int r0, int nrows) {
  const int t = threadIdx.x;
  if (t < nrows) {
    double re = 0.0, im = 0.0;
#pragma unroll 1
    for (int w = 0; w < kRotThreads / 32; ++w) {
      re += red[w][t].x;
      im += red[w][t].y;
    }
    const int L = p.L, m = r0 + t - l;
    const double2 a = p.ea[L - 1 + m];
    RotIO<R2>::put(p.out, ((size_t)b * L + l) * (2 * L - 1) + L - 1 + m,
                   make_double2(re * a.x - im * a.y, re * a.y + im * a.x));
  }
}

// one half-degree step at one entry: row factors u0 = sqrt(j-h), u1 = sqrt(h); column
// factors cA, sA, cB, sB; S[h][K], S[h][K-1], S[h-1][K], S[h-1][K-1]
__device__ __forceinline__ double risbo_entry(double u0, double u1, double cA, double sA,
                                              double cB, double sB, double s00, double s01,
                                              double s10, double s11) {
  return u0 * (cA * s00 + sB * s01) + u1 * (cB * s11 - sA * s10);
}

// Row block [r0, r0 + nrows) of D_l from D_{l-1}; the contraction of each row with map 0
// is left per warp in red[warp][row].
template <typename R2>
__device__ void risbo_block(const RotParams& p, int l, int r0, int nrows, double c, double s,
                            double2 (*red)[kRotRowsMax]) {
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = p.L, W = 2 * L - 1, ld = p.ld;
  const int j = 2 * l - 1, jp = 2 * l;  // sizes of D_{l-1} and of the half-step plane
  const double ij = 1.0 / j, ijp = 1.0 / jp;
  const double* __restrict__ S = (l & 1) ? p.plane0 : p.plane1;
  double* __restrict__ D = (l & 1) ? p.plane1 : p.plane0;
  const double* __restrict__ sq = p.sq;
  const bool contract = p.flm != nullptr;
  double2 acc[kRotRowsMax];
#pragma unroll
  for (int r = 0; r < kRotRowsMax; ++r) acc[r] = make_double2(0.0, 0.0);

  const int nchunks = (2 * l + 1 + kChunk - 1) / kChunk;
#pragma unroll 1
  for (int ch = warp; ch < nchunks; ch += kRotThreads / 32) {
    const int K = ch * kChunk - 1 + lane;
    const bool hcol = K >= 0 && K <= j;  // column of the half-step plane
    const bool dcol = lane > 0 && K <= jp;  // column of D_l made by this lane
    double cA = 0.0, sA = 0.0, cB = 0.0, sB = 0.0;
    if (hcol) {
      const double A = sq[j - K] * ij, B = sq[K] * ij;
      cA = c * A, sA = s * A, cB = c * B, sB = s * B;
    }
    double cA2 = 0.0, sA2 = 0.0, cB2 = 0.0, sB2 = 0.0;
    if (K >= 0 && K <= jp) {
      const double A = sq[jp - K] * ijp, B = sq[K] * ijp;
      cA2 = c * A, sA2 = s * A, cB2 = c * B, sB2 = s * B;
    }
    const double2 y = contract ? weighted_coef<R2>(p, 0, l, K, dcol) : make_double2(0.0, 0.0);

    // rows r0-2 .. r0+nrows-1 of D_{l-1} at columns K and K-1, all loads in flight at once
    double sk[kRotRowsMax + 2], skm[kRotRowsMax + 2];
#pragma unroll
    for (int i = 0; i < kRotRowsMax + 2; ++i) {
      const int h = r0 - 2 + i;
      const bool row = i < nrows + 2 && h >= 0 && h < j;
      sk[i] = (row && K >= 0 && K < j) ? __ldcg(S + (size_t)h * ld + K) : 0.0;
      skm[i] = (row && lane == 0 && K >= 1 && K <= j) ? __ldcg(S + (size_t)h * ld + K - 1) : 0.0;
    }
#pragma unroll
    for (int i = 0; i < kRotRowsMax + 2; ++i) {
      const double left = __shfl_up_sync(full, sk[i], 1);
      if (lane > 0) skm[i] = left;
    }

    // half-step row h = r0 - 2 + i from rows i-1, i of the loads
#define S2B_HROW(i)                                                                        \
  ((hcol && (r0 - 2 + (i)) >= 0 && (r0 - 2 + (i)) <= j)                                    \
       ? risbo_entry(sq[j - (r0 - 2 + (i))], sq[r0 - 2 + (i)], cA, sA, cB, sB, sk[i], skm[i], \
                     sk[(i)-1], skm[(i)-1])                                                \
       : 0.0)
    double hprev = S2B_HROW(1);
    double hprevL = __shfl_up_sync(full, hprev, 1);
#pragma unroll
    for (int r = 0; r < kRotRowsMax; ++r) {
      if (r < nrows) {
        const int I = r0 + r;
        const double hcur = S2B_HROW(r + 2);
        const double hcurL = __shfl_up_sync(full, hcur, 1);
        const double d =
            risbo_entry(sq[jp - I], sq[I], cA2, sA2, cB2, sB2, hcur, hcurL, hprev, hprevL);
        if (dcol) {
          D[(size_t)I * ld + K] = d;
          if (p.dl_out) p.dl_out[((size_t)l * W + L - 1 - l + I) * W + L - 1 - l + K] = d;
          acc[r].x += d * y.x;
          acc[r].y += d * y.y;
        }
        hprev = hcur;
        hprevL = hcurL;
      }
    }
#undef S2B_HROW
  }
  if (contract) {
#pragma unroll
    for (int r = 0; r < kRotRowsMax; ++r) {
      if (r < nrows) {
        const double re = warp_sum(acc[r].x), im = warp_sum(acc[r].y);
        if (lane == 0) red[warp][r] = make_double2(re, im);
      }
    }
  }
}

// the contraction of rows [r0, r0 + nrows) of D_l (already stored by this thread's own
// pass over the same columns) with map b
template <typename R2>
__device__ void reread_block(const RotParams& p, int b, int l, int r0, int nrows,
                             double2 (*red)[kRotRowsMax]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* __restrict__ D = (l & 1) ? p.plane1 : p.plane0;
  double2 acc[kRotRowsMax];
#pragma unroll
  for (int r = 0; r < kRotRowsMax; ++r) acc[r] = make_double2(0.0, 0.0);
  const int nchunks = (2 * l + 1 + kChunk - 1) / kChunk;
#pragma unroll 1
  for (int ch = warp; ch < nchunks; ch += kRotThreads / 32) {
    const int K = ch * kChunk - 1 + lane;
    const bool dcol = lane > 0 && K <= 2 * l;
    const double2 y = weighted_coef<R2>(p, b, l, K, dcol);
#pragma unroll
    for (int r = 0; r < kRotRowsMax; ++r) {
      if (r < nrows && dcol) {
        const double d = __ldcg(D + (size_t)(r0 + r) * p.ld + K);
        acc[r].x += d * y.x;
        acc[r].y += d * y.y;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kRotRowsMax; ++r) {
    if (r < nrows) {
      const double re = warp_sum(acc[r].x), im = warp_sum(acc[r].y);
      if (lane == 0) red[warp][r] = make_double2(re, im);
    }
  }
}

template <typename R2>
__global__ void __launch_bounds__(kRotThreads, 2) rotate_risbo_kernel(RotParams p) {
  __shared__ double2 red[kRotThreads / 32][kRotRowsMax];
  const int L = p.L, W = 2 * L - 1;
  double s, c;
  sincos(0.5 * p.beta, &s, &c);
  if (p.flm) {  // entries |m| > l of out are zero
    const long total = (long)p.batch * L * W;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
         e += (long)gridDim.x * blockDim.x) {
      const int m = (int)(e % W) - (L - 1), l = (int)((e / W) % L);
      if (m < -l || m > l) RotIO<R2>::put(p.out, e, make_double2(0.0, 0.0));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // degree 0: D_0 = [1], row block 0
    p.plane0[0] = 1.0;
    if (p.dl_out) p.dl_out[(size_t)(L - 1) * W + L - 1] = 1.0;
    for (int b = 0; p.flm && b < p.batch; ++b)
      RotIO<R2>::put(p.out, (size_t)b * L * W + L - 1,
                     RotIO<R2>::get(p.flm, (size_t)b * L * W + L - 1));
    __threadfence();
    store_release(p.done, 1);
  }
#pragma unroll 1
  for (int l = 1; l < L; ++l) {
#pragma unroll 1
    for (int rb = blockIdx.x; rb < p.nrb; rb += gridDim.x) {
      const int r0 = rb * p.rows;
      if (r0 >= 2 * l + 1) break;  // this block and the CTA's later ones start at higher degrees
      const int nrows = min(p.rows, 2 * l + 1 - r0);
      if (!wait_neighbours(p, rb, l)) return;
      risbo_block<R2>(p, l, r0, nrows, c, s, red);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        store_release(p.done + rb, l + 1);
      }
      if (p.flm) {
        flush_rows<R2>(p, red, 0, l, r0, nrows);
#pragma unroll 1
        for (int b = 1; b < p.batch; ++b) {
          __syncthreads();
          reread_block<R2>(p, b, l, r0, nrows, red);
          __syncthreads();
          flush_rows<R2>(p, red, b, l, r0, nrows);
        }
      }
    }
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

// exp(-i m alpha), exp(-i n gamma) and sqrt(k), k in [0, 2L]
__global__ void rotate_tables_kernel(RotParams p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= 2 * p.L; i += gridDim.x * blockDim.x) {
    p.sq[i] = sqrt((double)i);
    if (i < 2 * p.L - 1) {
      const double k = (double)(i - (p.L - 1));
      double s, c;
      sincos(-k * p.alpha, &s, &c);
      p.ea[i] = make_double2(c, s);
      sincos(-k * p.gamma, &s, &c);
      p.eg[i] = make_double2(c, s);
    }
  }
}

template <typename R2>
cudaError_t rotate_launch(RotParams p, cudaStream_t s) {
  rotate_tables_kernel<<<(2 * p.L + 1 + 255) / 256, 256, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (p.dl_in) {
    const long warps = (long)p.batch * p.L * (2 * p.L - 1);
    long blocks = (warps + 7) / 8;
    if (blocks > 65535L * 16) blocks = 65535L * 16;
    rotate_planes_kernel<R2><<<(unsigned)blocks, 256, 0, s>>>(p);
    return cudaGetLastError();
  }
  int dev = 0, sms = 0, per_sm = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rotate_risbo_kernel<R2>,
                                                      kRotThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  // every row block has a resident owner (cooperative launch); at most kRotRowsMax rows a
  // block, at least 2 (a row block's inputs then come from its two neighbours only)
  const long gmax = (long)sms * (per_sm < 2 ? per_sm : 2);
  const int rows_all = 2 * p.L - 1;
  int rows = (int)((rows_all + gmax - 1) / gmax);
  rows = rows < 2 ? 2 : (rows > kRotRowsMax ? kRotRowsMax : rows);
  p.rows = rows;
  p.nrb = (rows_all + rows - 1) / rows;
  const long grid = p.nrb < gmax ? p.nrb : gmax;
  e = cudaMemsetAsync(p.done, 0, (size_t)(p.L + 1) * sizeof(int), s);  // flags and err
  if (e != cudaSuccess) return e;
  void* args[] = {&p};
  return cudaLaunchCooperativeKernel((const void*)rotate_risbo_kernel<R2>, dim3((unsigned)grid),
                                     dim3(kRotThreads), args, 0, s);
}

}  // namespace

static size_t rot_align(size_t b) { return (b + 255) & ~(size_t)255; }
static size_t rot_plane_bytes(int L) { return rot_align((size_t)(2 * L - 1) * 2 * L * sizeof(double)); }
static size_t rot_sq_bytes(int L) { return rot_align((size_t)(2 * L + 1) * sizeof(double)); }
static size_t rot_phase_bytes(int L) { return rot_align((size_t)(2 * L - 1) * sizeof(double2)); }
static size_t rot_flag_bytes(int L) { return rot_align((size_t)(L + 1) * sizeof(int)); }

size_t rotate_workspace_bytes(int L) {
  return 2 * rot_plane_bytes(L) + rot_sq_bytes(L) + 2 * rot_phase_bytes(L) + rot_flag_bytes(L);
}

void rotate_bind_workspace(RotParams& p, void* ws) {
  char* c = static_cast<char*>(ws);
  const int L = p.L;
  p.ld = 2 * L;
  p.plane0 = reinterpret_cast<double*>(c);
  c += rot_plane_bytes(L);
  p.plane1 = reinterpret_cast<double*>(c);
  c += rot_plane_bytes(L);
  p.sq = reinterpret_cast<double*>(c);
  c += rot_sq_bytes(L);
  p.ea = reinterpret_cast<double2*>(c);
  c += rot_phase_bytes(L);
  p.eg = reinterpret_cast<double2*>(c);
  c += rot_phase_bytes(L);
  p.done = reinterpret_cast<int*>(c);  // L row-block flags at most, then the error word
  p.err = p.done + L;
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
  if (ws_bytes < s2b::rotate_workspace_bytes(L))
    return s2b::set_last_error(S2B_ERR_WORKSPACE, "rotate_dls: workspace too small");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(dl, 0, (size_t)L * (2 * L - 1) * (2 * L - 1) * sizeof(double), s);
  if (e != cudaSuccess) return s2b::set_last_error(S2B_ERR_CUDA, cudaGetErrorString(e));
  s2b::RotParams p{};
  p.L = L;
  p.batch = 0;
  p.beta = beta;
  p.dl_out = dl;
  s2b::rotate_bind_workspace(p, ws);
  e = s2b::launch_rotate(true, p, s);
  if (e != cudaSuccess) return s2b::set_last_error(S2B_ERR_CUDA, cudaGetErrorString(e));
  return S2B_OK;
}

}  // extern "C"
