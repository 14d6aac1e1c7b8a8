// sb_common.cuh -- shared helpers of libsparse_b200.so: status handling,
// dtype dispatch, streaming-load intrinsics and launch sizing for sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>
#include <nvtx3/nvToolsExt.h>

#include "sparse_b200.h"

namespace sb {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
int ensure_device();  // SB_OK when a CUDA device is usable, else SB_ENODEV

#define SB_CHECK_CUDA(call)                                   \
  do {                                                        \
    cudaError_t e__ = (call);                                 \
    if (e__ != cudaSuccess) return ::sb::cuda_status(e__, #call); \
  } while (0)

#define SB_REQUIRE(cond, ...)                                 \
  do {                                                        \
    if (!(cond)) {                                            \
      ::sb::set_error(__VA_ARGS__);                           \
      return SB_EINVAL;                                       \
    }                                                         \
  } while (0)

// Launch check: a failed launch reports SB_ECUDA with the kernel name.
#define SB_CHECK_LAUNCH(name) SB_CHECK_CUDA(cudaGetLastError())

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------- tracing
// An NVTX range over a public entry point (header-only NVTX v3: with no
// profiler attached a push/pop costs a few instructions), so that a trace
// (ncu --nvtx, Nsight Systems) attributes each launch to the C-ABI call
// that made it.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};
#define SB_TRACE(name) ::sb::TraceRange sb_trace_range__(name)

// Number of SMs of the current device (148 on B200), cached per device.
int sm_count();

// Per-device status word (device pointer) that kernels set on a bounded-wait
// timeout; read and cleared by sb_device_status().
int* device_status_word();

// Scratch allocation ordered on a stream (stream-ordered pool).
int scratch_alloc(void** p, size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);

// ---------------------------------------------------------------- loads
// Streaming loads for matrix arrays that are read exactly once per call: do
// not allocate in L1 (keep L1 for the gathered x) and tag the L2 lines
// evict-first through an L2 cache policy.
__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// Read-only loads that allocate in L1, for arrays whose 32-byte sectors are
// read by several load instructions of the same warp in a row (lanes that
// interleave over a row's entries).  Measured on B200 against the streaming
// form (no L1 allocation, L2 evict-first) in the CSR row-block kernel:
// banded 4M FP64 0.125 -> 0.110 ms, Laplacian 4096^2 FP32 0.202 -> 0.175 ms,
// power-law 2M FP64 0.242 -> 0.223 ms; keeping the L2 evict-first hint with
// L1 allocation was slower than the default policy.
__device__ __forceinline__ int ld_reuse(const int* p) { return __ldg(p); }
__device__ __forceinline__ float ld_reuse(const float* p) { return __ldg(p); }
__device__ __forceinline__ double ld_reuse(const double* p) { return __ldg(p); }
__device__ __forceinline__ unsigned short ld_reuse(const unsigned short* p) { return __ldg(p); }
__device__ __forceinline__ int4 ld_stream_v4(const int* p) {
  int4 r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ int ld_stream(const int* p) {
  int r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
               : "=r"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ float4 ld_stream_v4(const float* p) {
  float4 r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
               : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ float ld_stream(const float* p) {
  float r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ double2 ld_stream_v2(const double* p) {
  double2 r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
               : "=d"(r.x), "=d"(r.y)
               : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ double ld_stream(const double* p) {
  double r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ unsigned short ld_stream(const unsigned short* p) {
  unsigned short r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;"
               : "=h"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ uint2 ld_stream_v4(const unsigned short* p) {
  uint2 r;
  const uint64_t pol = evict_first_policy();
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
               : "=r"(r.x), "=r"(r.y)
               : "l"(p), "l"(pol));
  return r;
}

// Read-only cached load (x vectors: reused across rows).
template <typename T>
__device__ __forceinline__ T ld_ro(const T* p) {
  return __ldg(p);
}

// ---------------------------------------------------------------- async copy
// Bulk (non-tensor) async copies global -> shared completed on an mbarrier.
// Only this GPU's own memory is read and no multicast form is used.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after ~2^31 SM cycles (about a second) and returns
// false so that the caller can record an error status and leave.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > (1LL << 31)) return false;
  }
  return true;
}

// Device status codes written by kernels whose bounded waits ran out.
#define SB_DEV_OK 0
#define SB_DEV_TIMEOUT_BULK 1
#define SB_DEV_TIMEOUT_DEP 2

// Value-type traits: storage type S, accumulation type A.
template <int DT> struct vt;
template <> struct vt<SB_F32> { using S = float; using A = float; };
template <> struct vt<SB_F64> { using S = double; using A = double; };

inline size_t dtype_size(int dt) { return dt == SB_F64 ? 8 : (dt == SB_F32 ? 4 : 2); }

}  // namespace sb
