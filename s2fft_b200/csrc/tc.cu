// Batched precompute-kernel forward contraction on the 5th-generation tensor
// cores (tcgen05), with 3-term BF16 split operands and FP32 accumulation.
//
// For every m column the forward precompute transform is a dense product
//   flm[b][l][m] = (-1)^s sum_t K[t][l][m] ftm[b][t][m]
// (s2fft/precompute_transforms/spherical.py:314-380, einsum "tlm,tm->lm"),
// which over a batch of maps is a GEMM D[l][n] = sum_t A[l][t] B[n][t] with
// n = 2 b + {re, im}. Each operand x is split as x = hi + lo (both bf16) and
//   D ~= A_hi B_hi + A_hi B_lo + A_lo B_hi,
// accumulated in FP32 in tensor memory.
//
// Operands are packed once into the no-swizzle K-major core-matrix layout the
// MMA reads directly (8 rows x 16 bytes per core matrix; tile [r/8][k/8][r%8][k%8]),
// so every pipeline stage is four contiguous 1-D bulk copies (TMA engine, no
// multicast). CTA = 4 consecutive m columns x 128 l rows; 4 accumulators of
// 128 x 128 FP32 occupy the 512 TMEM columns. One thread produces and issues;
// all waits are bounded and TMEM is always released.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "s2b_tc.h"

namespace s2b {

namespace {

constexpr int kTileR = 128;              // rows of a tile (l for A, n for B)
constexpr int kTileK = 64;               // K (t) per stage
constexpr int kBlk = kTileR * kTileK;    // elements per operand block
constexpr int kBlkBytes = kBlk * 2;      // 16 KB (bf16)
constexpr int kStageBytes = 4 * kBlkBytes;  // A_hi, A_lo, B_hi, B_lo
constexpr int kStages = 3;
constexpr int kMPerCta = 4;
constexpr unsigned kTmemCols = 512;

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (r, k) inside a packed block
__host__ __device__ __forceinline__ int core_off(int r, int k) {
  return (((r >> 3) * (kTileK / 8) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7)) * 2;
}

__device__ __forceinline__ void mb_init(uint64_t* mb, unsigned c) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(mb)), "r"(c) : "memory");
}
__device__ __forceinline__ void mb_expect(uint64_t* mb, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(mb)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mb_wait(uint64_t* mb, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(mb)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* mb) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          su32(dst)),
      "l"(src), "r"(bytes), "r"(su32(mb))
      : "memory");
}

// shared-memory matrix descriptor: no swizzle, K-major, LBO = 128 B (next 8 k),
// SBO = 1024 B (next 8 rows), Blackwell descriptor version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((128u >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((1024u >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D f32, A/B bf16, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* mb) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(mb))
               : "memory");
}

}  // namespace

// ---------------------------------------------------------------------------
// packing: K[t][l][mi] (float) -> Ap[mi][rt][kc][hi/lo][block]; forward: rows l, k = t;
// transposed (inverse): rows t, k = l
// ---------------------------------------------------------------------------
__global__ void pack_kernel_a(const float* __restrict__ K, int nth, int L, int M, int nlt, int ntc,
                              int transposed, int cplx, __nv_bfloat16* __restrict__ out) {
  // cplx: K is complex (float2) and the K dimension is doubled: chunks tc < ntc / 2 hold
  // Re K, chunks tc >= ntc / 2 hold Im K of the same summation indices
  const int nth_c = cplx ? ntc / 2 : ntc;
  const long total = (long)M * nlt * ntc * kBlk;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int e = (int)(i % kBlk);
    long rest = i / kBlk;
    const int tc = (int)(rest % ntc);
    rest /= ntc;
    const int lt = (int)(rest % nlt);
    const int mi = (int)(rest / nlt);
    const int r = e / kTileK, k = e % kTileK;
    const int part = tc >= nth_c ? 1 : 0;  // 0: real, 1: imaginary (cplx only)
    const int row = lt * kTileR + r, kk = (tc - part * nth_c) * kTileK + k;
    const int l = transposed ? kk : row, t = transposed ? row : kk;
    float x = 0.f;
    if (l < L && t < nth) {
      const size_t o = ((size_t)t * L + l) * M + mi;
      x = cplx ? (part ? reinterpret_cast<const float2*>(K)[o].y
                       : reinterpret_cast<const float2*>(K)[o].x)
               : K[o];
    }
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
    __nv_bfloat16* blk = out + (((size_t)mi * nlt + lt) * ntc + tc) * 2 * kBlk;
    const int off = core_off(r, k) / 2;
    blk[off] = hi;
    blk[kBlk + off] = lo;
  }
}


// data (map b, summation index t, column mi; complex float) -> Bp[mi][bg][tc][hi/lo][block],
// row n = 2 (b - 64 bg) + (0: real, 1: imaginary part), through shared memory: a CTA takes
// 16 columns mi, one t chunk (64) and 4 maps (8 rows n, one core row group), reads the
// spectra in 128-byte segments (the 16 columns of a (b, t) pair), and writes every column
// as 1 KB of contiguous 16-byte stores (8 consecutive k of one row per store, hi and lo).
constexpr int kPackMaps = 4;
constexpr int kPackCols = 16;
constexpr int kPackTP = kTileK + 2;  // padded t row (float2)
// float2 per column slice: padded so that 16 consecutive columns fall 2 float2 (4 banks)
// apart modulo 16 (32 banks) while staying 16-byte aligned for the float4 reads
constexpr int kPackSC = kPackMaps * kPackTP + 10;
static_assert(kPackSC % 16 == 2, "column slices 4 banks apart");

__global__ void __launch_bounds__(256) pack_kernel_b2(const float2* __restrict__ X, int B,
                                                      int kdim, int M, long in_map, int in_row,
                                                      int in_col0, int nbg, int ntc, int cplx,
                                                      __nv_bfloat16* __restrict__ out) {
  // cplx: chunks tc >= ntc / 2 repeat the summation indices of chunk tc - ntc / 2 with the
  // rows (re, im) replaced by (-im, re), so that [Re K | Im K] x this gives the complex product
  __shared__ __align__(16) float2 S[kPackCols * kPackSC];
  const int tid = threadIdx.x;
  const int mi0 = blockIdx.x * kPackCols;
  const int tc = blockIdx.y;
  const int half = cplx ? ntc / 2 : ntc;
  const int part = tc >= half ? 1 : 0;
  const int tq = tc - part * half;  // chunk of summation indices
  const int bg = blockIdx.z / (64 / kPackMaps), sub = blockIdx.z % (64 / kPackMaps);
  const int bl0 = bg * 64 + sub * kPackMaps;  // first map of the CTA
  for (int e = tid; e < kPackCols * kPackMaps * kTileK; e += 256) {
    const int c = e % kPackCols, tl = (e / kPackCols) % kTileK, bl = e / (kPackCols * kTileK);
    const int b = bl0 + bl, t = tq * kTileK + tl, mi = mi0 + c;
    float2 v = make_float2(0.f, 0.f);
    if (b < B && t < kdim && mi < M) v = X[(size_t)b * in_map + (size_t)t * in_row + in_col0 + mi];
    S[c * kPackSC + bl * kPackTP + tl] = v;
  }
  __syncthreads();
  // unit = 8 consecutive k of one row n of one column: id -> (c, u), u = 8 kg + row fastest
  constexpr int kU = 8 * (kTileK / 8);
  for (int id = tid; id < kPackCols * kU; id += 256) {
    const int u = id % kU, c = id / kU;
    const int mi = mi0 + c;
    if (mi >= M) continue;
    const int nl = u & 7;  // row within the CTA's 8 rows
    const int kg = u >> 3;
    const float4* src =
        reinterpret_cast<const float4*>(&S[c * kPackSC + (nl >> 1) * kPackTP + kg * 8]);
    float x[8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float4 w = src[j];  // two complex values
      if (part == 0) {
        x[2 * j] = (nl & 1) ? w.y : w.x;
        x[2 * j + 1] = (nl & 1) ? w.w : w.z;
      } else {  // rows (-im, re)
        x[2 * j] = (nl & 1) ? w.x : -w.y;
        x[2 * j + 1] = (nl & 1) ? w.z : -w.w;
      }
    }
    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      hi[j] = __float2bfloat16_rn(x[j]);
      lo[j] = __float2bfloat16_rn(x[j] - __bfloat162float(hi[j]));
    }
    const int n = sub * 8 + nl;
    __nv_bfloat16* blk = out + (((size_t)mi * nbg + bg) * ntc + tc) * 2 * kBlk;
    const int off = core_off(n, kg * 8) / 2;
    *reinterpret_cast<uint4*>(blk + off) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(blk + kBlk + off) = *reinterpret_cast<const uint4*>(lo);
  }
}

// ---------------------------------------------------------------------------
// the MMA kernel: grid (nlt, ceil(M/4), nbg), 128 threads
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) tc_forward_kernel(TcParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* done = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // l tiles vary fastest: the CTAs of one m group run side by side and read the same
  // data blocks (B), which L2 then serves to all but the first
  const int lt = blockIdx.x, mg = blockIdx.y, bg = blockIdx.z;
  const int mi0 = mg * kMPerCta;
  const int nm = min(kMPerCta, p.M - mi0);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mb_init(&full[s], 1);
      mb_init(&empty[s], 1);
    }
    mb_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // work items: (j, tc) for j < nm, tc < ntc; skip m columns whose l tile is all zero
  const int ntc = p.ntc;
  const int niter = nm * ntc;
  bool ok = true;
  if (tid == 0) {
    auto produce = [&](int it) {
      const int j = it / ntc, tc = it % ntc;
      const int s = it % kStages;
      unsigned char* st = smem + (size_t)s * kStageBytes;
      const __nv_bfloat16* a =
          p.Ap + ((((size_t)(mi0 + j) * p.nlt + lt) * ntc + tc) * 2 * kBlk);
      const __nv_bfloat16* b =
          p.Bp + ((((size_t)(mi0 + j) * p.nbg + bg) * ntc + tc) * 2 * kBlk);
      mb_expect(&full[s], kStageBytes);
      bulk_copy(st, a, 2 * kBlkBytes, &full[s]);
      bulk_copy(st + 2 * kBlkBytes, b, 2 * kBlkBytes, &full[s]);
    };
    for (int it = 0; it < niter + kStages - 1 && ok; ++it) {
      if (it < niter) {
        const int s = it % kStages;
        if (it >= kStages) ok = mb_wait(&empty[s], ((it / kStages) - 1) & 1);
        if (!ok) break;
        produce(it);
      }
      const int k = it - (kStages - 1);
      if (k >= 0 && k < niter) {
        const int s = k % kStages;
        ok = mb_wait(&full[s], (k / kStages) & 1);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int j = k / ntc, tc = k % ntc;
        const uint32_t d = tmem + (uint32_t)(j * 128);
        const uint32_t st = su32(smem + (size_t)s * kStageBytes);
        const uint32_t ahi = st, alo = st + kBlkBytes, bhi = st + 2 * kBlkBytes,
                       blo = st + 3 * kBlkBytes;
#pragma unroll
        for (int kk = 0; kk < kTileK / 16; ++kk) {
          const uint32_t o = kk * 256;  // two core matrices (16 k) per MMA
          mma_bf16(d, sdesc(ahi + o), sdesc(bhi + o), (tc > 0 || kk > 0) ? 1u : 0u);
          mma_bf16(d, sdesc(ahi + o), sdesc(blo + o), 1u);
          mma_bf16(d, sdesc(alo + o), sdesc(bhi + o), 1u);
        }
        mma_commit(&empty[s]);
      }
    }
    if (ok) mma_commit(done);
    if (!ok) atomicExch(p.status, 1);
  }
  __syncwarp();
  // everyone waits for the accumulators (bounded); on failure skip the epilogue
  bool good = mb_wait(done, 0);
  good = __syncthreads_and(good) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (good) {
    // lane (row l) of this warp's TMEM quarter; 32 columns per load
    const int l = lt * kTileR + warp * 32 + lane;
    for (int q = 0; q < 4; ++q) {  // 16 maps per pass
      float v[kMPerCta][32];
#pragma unroll
      for (int j = 0; j < kMPerCta; ++j) {
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * 128 + q * 32);
        uint32_t r[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
            "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
              "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
              "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
              "=r"(r[31])
            : "r"(addr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int x = 0; x < 32; ++x) v[j][x] = __uint_as_float(r[x]);
      }
      if (l < p.rows) {
        for (int x = 0; x < 16; ++x) {
          const int b = bg * 64 + q * 16 + x;
          if (b >= p.B) break;
          float2* row = p.out + (size_t)b * p.out_map + (size_t)l * p.out_row + p.out_col0 + mi0;
#pragma unroll
          for (int j = 0; j < kMPerCta; ++j)
            if (j < nm) row[j] = make_float2(p.sign * v[j][2 * x], p.sign * v[j][2 * x + 1]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
}

size_t tc_packed_a_bytes(int kdim, int rows, int M, int cplx) {
  const int nlt = (rows + kTileR - 1) / kTileR, ntc = (kdim + kTileK - 1) / kTileK;
  return (size_t)M * nlt * ntc * (cplx ? 2 : 1) * 2 * kBlkBytes;
}
size_t tc_packed_b_bytes(int kdim, int B, int M, int cplx) {
  const int nbg = (B + 63) / 64, ntc = (kdim + kTileK - 1) / kTileK;
  return (size_t)M * nbg * ntc * (cplx ? 2 : 1) * 2 * kBlkBytes;
}

static int tgrid(long n) {
  long b = (n + 255) / 256;
  if (b > 1048576) b = 1048576;
  return b < 1 ? 1 : (int)b;
}

cudaError_t launch_tc_pack_a(const float* K, int nth, int L, int M, int transposed, int cplx,
                             void* out, cudaStream_t s) {
  const int rows = transposed ? nth : L, kdim = transposed ? L : nth;
  const int nlt = (rows + kTileR - 1) / kTileR;
  const int ntc = ((kdim + kTileK - 1) / kTileK) * (cplx ? 2 : 1);
  const long total = (long)M * nlt * ntc * kBlk;
  pack_kernel_a<<<tgrid(total), 256, 0, s>>>(K, nth, L, M, nlt, ntc, transposed, cplx,
                                             (__nv_bfloat16*)out);
  return cudaGetLastError();
}

cudaError_t launch_tc_pack_b(const void* X, int B, int kdim, int M, long in_map, int in_row,
                             int in_col0, int cplx, void* out, cudaStream_t s) {
  const int nbg = (B + 63) / 64, ntc = ((kdim + kTileK - 1) / kTileK) * (cplx ? 2 : 1);
  const dim3 grid((M + kPackCols - 1) / kPackCols, ntc, nbg * (64 / kPackMaps));
  if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidConfiguration;
  pack_kernel_b2<<<grid, 256, 0, s>>>((const float2*)X, B, kdim, M, in_map, in_row, in_col0,
                                      nbg, ntc, cplx, (__nv_bfloat16*)out);
  return cudaGetLastError();
}

cudaError_t launch_tc_forward(TcParams p, cudaStream_t s) {
  p.nlt = (p.rows + kTileR - 1) / kTileR;
  p.ntc = ((p.kdim + kTileK - 1) / kTileK) * (p.cplx ? 2 : 1);
  p.nbg = (p.B + 63) / 64;
  const size_t smem = (size_t)kStages * kStageBytes + 1024;
  cudaError_t e = cudaFuncSetAttribute(tc_forward_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(p.nlt, (p.M + kMPerCta - 1) / kMPerCta, p.nbg);
  if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidConfiguration;
  tc_forward_kernel<<<grid, 128, smem, s>>>(p);
  return cudaGetLastError();
}

}  // namespace s2b
