// sb_runtime.cu -- device memory, streams and error reporting of the C ABI.
// Stands in for MatMachJS's _malloc/_free over wasm linear memory
// (src/sequential/libs/matmachjs.wat:46-48) with device memory.
#include <mutex>
#include <string.h>

#include "sb_common.cuh"

namespace sb {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return SB_ENOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SB_ENODEV;
  return SB_ECUDA;
}

int ensure_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device available (%s)", e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    return SB_ENODEV;
  }
  return SB_OK;
}

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = n > 0 ? n : 148;
  }
  return cache[dev];
}

int* device_status_word() {
  static std::mutex mu;
  static int* words[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!words[dev]) {
    int* p = nullptr;
    if (cudaMalloc(&p, 64) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cudaMemset(p, 0, 64);
    words[dev] = p;
  }
  return words[dev];
}

// Stream-ordered scratch comes from the device's default memory pool.  By
// default the pool hands freed memory back to the driver at every
// synchronisation, so each call that needs scratch would map fresh pages;
// keeping up to kPoolKeep bytes of freed scratch lets later calls reuse it.
constexpr uint64_t kPoolKeep = 2ull << 30;

static void keep_pool_memory() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = kPoolKeep;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done[dev] = true;
}

int scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  keep_pool_memory();
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) return cuda_status(e, "cudaMallocAsync(scratch)");
  return SB_OK;
}

void scratch_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_version(void) { return 10000; }

const char* sb_last_error(void) { return g_err; }

const char* sb_status_string(int s) {
  switch (s) {
    case SB_OK: return "ok";
    case SB_EINVAL: return "invalid argument";
    case SB_ENOMEM: return "out of device memory";
    case SB_EREFUSED: return "refused by the format admission test";
    case SB_ETIMEOUT: return "bounded device wait timed out";
    case SB_ECUDA: return "CUDA error";
    case SB_ENODEV: return "no CUDA device";
    case SB_EALIGN: return "misaligned pointer";
    default: return "unknown status";
  }
}

int sb_device_count(int* count) {
  SB_REQUIRE(count, "sb_device_count: null output");
  *count = 0;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
  }
  return SB_OK;
}

int sb_set_device(int device) {
  int r = ensure_device();
  if (r) return r;
  SB_CHECK_CUDA(cudaSetDevice(device));
  return SB_OK;
}

int sb_malloc(void** ptr, size_t bytes) {
  SB_REQUIRE(ptr, "sb_malloc: null output");
  *ptr = nullptr;
  int r = ensure_device();
  if (r) return r;
  if (bytes == 0) bytes = 16;
  SB_CHECK_CUDA(cudaMalloc(ptr, bytes));
  return SB_OK;
}

int sb_free(void* ptr) {
  if (!ptr) return SB_OK;
  SB_CHECK_CUDA(cudaFree(ptr));
  return SB_OK;
}

int sb_host_alloc(void** ptr, size_t bytes) {
  SB_REQUIRE(ptr, "sb_host_alloc: null output");
  *ptr = nullptr;
  int r = ensure_device();
  if (r) return r;
  if (bytes == 0) bytes = 16;
  SB_CHECK_CUDA(cudaMallocHost(ptr, bytes));
  return SB_OK;
}

int sb_host_free(void* ptr) {
  if (!ptr) return SB_OK;
  SB_CHECK_CUDA(cudaFreeHost(ptr));
  return SB_OK;
}

int sb_memcpy_htod(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return SB_OK;
  SB_REQUIRE(dst && src, "sb_memcpy_htod: null pointer");
  SB_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream)));
  return SB_OK;
}

int sb_memcpy_dtoh(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return SB_OK;
  SB_REQUIRE(dst && src, "sb_memcpy_dtoh: null pointer");
  SB_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
  return SB_OK;
}

int sb_memcpy_dtod(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return SB_OK;
  SB_REQUIRE(dst && src, "sb_memcpy_dtod: null pointer");
  SB_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)));
  return SB_OK;
}

int sb_memset(void* dst, int value, size_t bytes, void* stream) {
  if (bytes == 0) return SB_OK;
  SB_REQUIRE(dst, "sb_memset: null pointer");
  SB_CHECK_CUDA(cudaMemsetAsync(dst, value, bytes, as_stream(stream)));
  return SB_OK;
}

int sb_stream_create(void** stream) {
  SB_REQUIRE(stream, "sb_stream_create: null output");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t s;
  SB_CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  *stream = reinterpret_cast<void*>(s);
  return SB_OK;
}

int sb_stream_create_priority(void** stream, int priority) {
  SB_REQUIRE(stream, "sb_stream_create_priority: null output");
  int r = ensure_device();
  if (r) return r;
  int least = 0, greatest = 0;
  SB_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  // clamp into [greatest, least] (numerically lower is more urgent)
  const int p = priority < greatest ? greatest : (priority > least ? least : priority);
  cudaStream_t s;
  SB_CHECK_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, p));
  *stream = reinterpret_cast<void*>(s);
  return SB_OK;
}

int sb_stream_priority_range(int* least, int* greatest) {
  SB_REQUIRE(least && greatest, "sb_stream_priority_range: null output");
  int r = ensure_device();
  if (r) return r;
  SB_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(least, greatest));
  return SB_OK;
}

int sb_stream_destroy(void* stream) {
  if (!stream) return SB_OK;
  SB_CHECK_CUDA(cudaStreamDestroy(as_stream(stream)));
  return SB_OK;
}

int sb_stream_synchronize(void* stream) {
  SB_CHECK_CUDA(cudaStreamSynchronize(as_stream(stream)));
  return SB_OK;
}

int sb_event_create(void** ev) {
  SB_REQUIRE(ev, "sb_event_create: null output");
  int r = ensure_device();
  if (r) return r;
  cudaEvent_t e;
  SB_CHECK_CUDA(cudaEventCreate(&e));
  *ev = reinterpret_cast<void*>(e);
  return SB_OK;
}

int sb_event_destroy(void* ev) {
  if (!ev) return SB_OK;
  SB_CHECK_CUDA(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(ev)));
  return SB_OK;
}

int sb_event_record(void* ev, void* stream) {
  SB_REQUIRE(ev, "sb_event_record: null event");
  SB_CHECK_CUDA(cudaEventRecord(reinterpret_cast<cudaEvent_t>(ev), as_stream(stream)));
  return SB_OK;
}

int sb_event_query(void* ev) {
  SB_REQUIRE(ev, "sb_event_query: null event");
  cudaError_t e = cudaEventQuery(reinterpret_cast<cudaEvent_t>(ev));
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) {
    cudaGetLastError();
    return 0;
  }
  return cuda_status(e, "cudaEventQuery");
}

int sb_event_synchronize(void* ev) {
  SB_REQUIRE(ev, "sb_event_synchronize: null event");
  SB_CHECK_CUDA(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(ev)));
  return SB_OK;
}

int sb_stream_wait_event(void* stream, void* ev) {
  SB_REQUIRE(ev, "sb_stream_wait_event: null event");
  SB_CHECK_CUDA(cudaStreamWaitEvent(as_stream(stream), reinterpret_cast<cudaEvent_t>(ev), 0));
  return SB_OK;
}

int sb_event_elapsed_ms(void* start, void* end, float* ms) {
  SB_REQUIRE(start && end && ms, "sb_event_elapsed_ms: null argument");
  SB_CHECK_CUDA(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(start),
                                     reinterpret_cast<cudaEvent_t>(end)));
  return SB_OK;
}

int sb_device_status(int* code) {
  SB_REQUIRE(code, "sb_device_status: null output");
  *code = 0;
  int r = ensure_device();
  if (r) return r;
  int* w = device_status_word();
  if (!w) return SB_OK;
  SB_CHECK_CUDA(cudaDeviceSynchronize());
  SB_CHECK_CUDA(cudaMemcpy(code, w, sizeof(int), cudaMemcpyDeviceToHost));
  SB_CHECK_CUDA(cudaMemset(w, 0, sizeof(int)));
  return SB_OK;
}

int sb_mem_info(size_t* free_bytes, size_t* total_bytes) {
  SB_REQUIRE(free_bytes && total_bytes, "sb_mem_info: null output");
  int r = ensure_device();
  if (r) return r;
  SB_CHECK_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
  return SB_OK;
}

}  // extern "C"
