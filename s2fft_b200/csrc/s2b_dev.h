// Device helpers shared by the latitudinal kernels: vector accumulators,
// global reductions, and 1-D bulk asynchronous copies global -> shared
// completed on an mbarrier (no multicast). Waits are bounded.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>
#include <utility>

namespace s2b {

template <typename Real>
struct Vec;
template <>
struct Vec<float> {
  using t2 = float2;
  using t4 = float4;
};
template <>
struct Vec<double> {
  using t2 = double2;
  using t4 = double4;
};

// hint: bring the 128-byte line holding p (global memory) into L1
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <typename T2>
__device__ __forceinline__ void red_add(T2* addr, T2 v);
template <>
__device__ __forceinline__ void red_add<float2>(float2* addr, float2 v) {
  atomicAdd(addr, v);  // red.global.add.v2.f32 (sm_90+)
}
template <>
__device__ __forceinline__ void red_add<double2>(double2* addr, double2 v) {
  atomicAdd(&addr->x, v.x);
  atomicAdd(&addr->y, v.y);
}
template <>
__device__ __forceinline__ void red_add<float4>(float4* addr, float4 v) {
  atomicAdd(addr, v);  // red.global.add.v4.f32 (sm_90+)
}
template <>
__device__ __forceinline__ void red_add<double4>(double4* addr, double4 v) {
  atomicAdd(&addr->x, v.x);
  atomicAdd(&addr->y, v.y);
  atomicAdd(&addr->z, v.z);
  atomicAdd(&addr->w, v.w);
}

template <typename A>
__device__ __forceinline__ A zero_acc() {
  A a;
  a.x = 0;
  a.y = 0;
  if constexpr (sizeof(A) == 4 * sizeof(a.x)) {
    a.z = 0;
    a.w = 0;
  }
  return a;
}

template <typename A>
__device__ __forceinline__ void acc_add(A& a, const A& b) {
  a.x += b.x;
  a.y += b.y;
  if constexpr (sizeof(A) == 4 * sizeof(a.x)) {
    a.z += b.z;
    a.w += b.w;
  }
}

// a += x * f (component-wise)
template <typename A, typename Real>
__device__ __forceinline__ void acc_fma(A& a, Real x, const A& f) {
  a.x = fma(x, f.x, a.x);
  a.y = fma(x, f.y, a.y);
  if constexpr (sizeof(A) == 4 * sizeof(Real)) {
    a.z = fma(x, f.z, a.z);
    a.w = fma(x, f.w, a.w);
  }
}

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint64_t* mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mb)), "r"(count)
               : "memory");
}
// Invalidates an initialised mbarrier (no pending arrivals or transactions), so that the
// location can be initialised again (a persistent kernel reusing it for its next tile).
__device__ __forceinline__ void mbar_inval(uint64_t* mb) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(mb)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mb, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mb)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* mb) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(mb))
      : "memory");
}
// Per-thread asynchronous global -> shared copy of B (8 or 16) bytes to the shared-space
// address d (zero-filled when !valid: the source is not read), and its group fences.
template <int B>
__device__ __forceinline__ void cp_async(unsigned d, const void* src, bool valid) {
  static_assert(B == 8 || B == 16, "cp.async of 8 or 16 bytes");
  if constexpr (B == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Programmatic dependent launch along a stream's chain of kernels: a kernel launched by
// launch_chained may have its CTAs made resident while its predecessor's last CTAs still run.
// Every such kernel calls chain_enter() before its first global-memory access: it waits until
// the predecessor has completed and its writes are visible, then lets the next kernel of the
// chain launch, so that at most one grid waits ahead of the running one (without the launch
// attribute both are no-ops).
__device__ __forceinline__ void chain_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                  cudaStream_t s, Args&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Bounded wait for the phase with the given parity; false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mb, unsigned parity) {
  const uint32_t a = smem_u32(mb);
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

}  // namespace s2b
