// sb_batch.cu -- batched CSR SpMV: many matrices and right-hand sides in one
// persistent launch, replayed from a captured CUDA graph.
//
// No counterpart in the reference (it calls spmv once per matrix and vector,
// src/sequential/src/sparse32.js:1232-1286).  Work is a flat list of 32-row
// blocks over all matrices of the batch (block_offsets = exclusive scan of
// ceil(N_i/32)); persistent warps take blocks from a device counter, map a
// block index to its matrix by binary search, and reduce each row with V
// lanes (V per matrix from its mean row length: the "rows per warp"
// autotuning), accumulating all of the matrix's nrhs (1..8) right-hand sides
// at once (x and y are N x nrhs, row-major).  Values are stored f32, f64 or
// BF16 (f32 vectors and sums for f32/BF16).  The executor keeps descriptors
// in pinned host and device buffers; one run = the graph [copy descriptors,
// reset the counter, kernel] launched on the caller's stream.
#include <algorithm>
#include <vector>

#include "sb_common.cuh"

struct sb_batch_exec {
  int dtype = 0;
  int capacity = 0;
  int device = 0;
  int grid = 0;
  sb_batch_item* h_items = nullptr;  // pinned
  long long* h_offsets = nullptr;    // pinned, capacity + 1
  int* h_count = nullptr;            // pinned: [0] = items in the current run
  sb_batch_item* d_items = nullptr;
  long long* d_offsets = nullptr;
  int* d_count = nullptr;            // [0] items, [1] work counter
  cudaGraphExec_t graph = nullptr;
  cudaStream_t capture_stream = nullptr;
  cudaEvent_t done = nullptr;
  bool pending = false;
};

namespace sb {

constexpr int kBT = 256;
constexpr int kMaxRhs = 8;

__device__ __forceinline__ float ldv(const float* p, long long i) { return ld_stream(p + i); }
__device__ __forceinline__ double ldv(const double* p, long long i) { return ld_stream(p + i); }
__device__ __forceinline__ float ldv(const __nv_bfloat16* p, long long i) {
  return __bfloat162float(
      __ushort_as_bfloat16(ld_stream(reinterpret_cast<const unsigned short*>(p) + i)));
}

// One 32-row block of one matrix, V lanes per row, K right-hand sides.
template <typename SV, typename T, int V>
__device__ __forceinline__ void batch_block(const sb_batch_item& it, int r0, int lane) {
  constexpr int RPB = 32 / V;
  const int g = lane / V, q = lane - (lane / V) * V;
  const int* __restrict__ rp = it.row_ptr;
  const int* __restrict__ col = it.col;
  const SV* __restrict__ val = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  T* __restrict__ y = (T*)it.y;
  const int K = it.nrhs;
  const bool overwrite = (it.flags & 1) != 0;
  for (int b = 0; b < V; ++b) {
    const int row = r0 + b * RPB + g;
    const bool ok = row < it.N && row < r0 + 32;
    const int s = ok ? __ldg(rp + row) : 0;
    const int e = ok ? __ldg(rp + row + 1) : 0;
    T acc[kMaxRhs];
#pragma unroll
    for (int j = 0; j < kMaxRhs; ++j) acc[j] = 0;
    for (int k = s + q; k < e; k += V) {
      const long long c = (long long)ld_stream(col + k) * K;
      const T v = (T)ldv(val, k);
#pragma unroll
      for (int j = 0; j < kMaxRhs; ++j)
        if (j < K) acc[j] += v * __ldg(x + c + j);
    }
#pragma unroll
    for (int j = 0; j < kMaxRhs; ++j) {
      if (j < K) {
        T a = acc[j];
        for (int off = V >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
        if (ok && q == 0) {
          if (overwrite) y[(long long)row * K + j] = a;
          else if (e > s) y[(long long)row * K + j] += a;
        }
      }
    }
  }
}

template <typename SV, typename T>
__global__ void __launch_bounds__(kBT)
    batch_kernel(const sb_batch_item* __restrict__ items, const long long* __restrict__ offsets,
                 int* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int M = count[0];
  if (M <= 0) return;
  const long long total = offsets[M];
  while (true) {
    long long w = 0;
    if (lane == 0) w = atomicAdd((unsigned long long*)(count + 2), 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= total) return;
    // matrix of block w: last m with offsets[m] <= w
    int lo = 0, hi = M - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (offsets[mid] <= w) lo = mid; else hi = mid - 1;
    }
    const sb_batch_item it = items[lo];
    const int r0 = (int)((w - offsets[lo]) * 32);
    switch (it.lanes) {
      case 1: batch_block<SV, T, 1>(it, r0, lane); break;
      case 2: batch_block<SV, T, 2>(it, r0, lane); break;
      case 4: batch_block<SV, T, 4>(it, r0, lane); break;
      case 8: batch_block<SV, T, 8>(it, r0, lane); break;
      case 16: batch_block<SV, T, 16>(it, r0, lane); break;
      default: batch_block<SV, T, 32>(it, r0, lane); break;
    }
  }
}

static const void* batch_kernel_for(int dtype) {
  if (dtype == SB_F64) return (const void*)batch_kernel<double, double>;
  if (dtype == SB_BF16) return (const void*)batch_kernel<__nv_bfloat16, float>;
  return (const void*)batch_kernel<float, float>;
}

static int lanes_for(long long nnz, int N) {
  const double avg = N ? (double)nnz / N : 0.0;
  if (avg <= 3) return 1;
  if (avg <= 6) return 2;
  if (avg <= 14) return 4;
  if (avg <= 28) return 8;
  if (avg <= 56) return 16;
  return 32;
}

static void exec_release(sb_batch_exec* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->capture_stream) cudaStreamDestroy(e->capture_stream);
  if (e->done) cudaEventDestroy(e->done);
  if (e->h_items) cudaFreeHost(e->h_items);
  if (e->h_offsets) cudaFreeHost(e->h_offsets);
  if (e->h_count) cudaFreeHost(e->h_count);
  if (e->d_items) cudaFree(e->d_items);
  if (e->d_offsets) cudaFree(e->d_offsets);
  if (e->d_count) cudaFree(e->d_count);
  delete e;
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_batch_exec_create(int dtype, int32_t capacity, sb_batch_exec** out) {
  SB_REQUIRE(out, "sb_batch_exec_create: null output");
  *out = nullptr;
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64 || dtype == SB_BF16,
             "sb_batch_exec_create: bad dtype");
  SB_REQUIRE(capacity > 0, "sb_batch_exec_create: capacity must be positive");
  int r = ensure_device();
  if (r) return r;
  sb_batch_exec* e = new sb_batch_exec();
  e->dtype = dtype;
  e->capacity = capacity;
  cudaGetDevice(&e->device);
  cudaError_t ce = cudaSuccess;
#define SB_E(call)                                \
  if ((ce = (call)) != cudaSuccess) {             \
    r = cuda_status(ce, #call);                   \
    exec_release(e);                              \
    return r;                                     \
  }
  SB_E(cudaMallocHost(&e->h_items, sizeof(sb_batch_item) * capacity));
  SB_E(cudaMallocHost(&e->h_offsets, sizeof(long long) * (capacity + 1)));
  SB_E(cudaMallocHost(&e->h_count, sizeof(int) * 4));
  SB_E(cudaMalloc(&e->d_items, sizeof(sb_batch_item) * capacity));
  SB_E(cudaMalloc(&e->d_offsets, sizeof(long long) * (capacity + 1)));
  SB_E(cudaMalloc(&e->d_count, sizeof(int) * 4));
  SB_E(cudaStreamCreateWithFlags(&e->capture_stream, cudaStreamNonBlocking));
  SB_E(cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming));
  const void* kern = batch_kernel_for(dtype);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kBT, 0);
  e->grid = std::max(1, per) * sm_count();
  // capture: descriptors + offsets + item count (host -> device), reset the
  // work counter, persistent kernel
  cudaGraph_t g = nullptr;
  SB_E(cudaStreamBeginCapture(e->capture_stream, cudaStreamCaptureModeThreadLocal));
  cudaMemcpyAsync(e->d_items, e->h_items, sizeof(sb_batch_item) * capacity,
                  cudaMemcpyHostToDevice, e->capture_stream);
  cudaMemcpyAsync(e->d_offsets, e->h_offsets, sizeof(long long) * (capacity + 1),
                  cudaMemcpyHostToDevice, e->capture_stream);
  cudaMemcpyAsync(e->d_count, e->h_count, sizeof(int) * 4, cudaMemcpyHostToDevice,
                  e->capture_stream);
  void* args[] = {(void*)&e->d_items, (void*)&e->d_offsets, (void*)&e->d_count};
  cudaLaunchKernel(kern, dim3(e->grid), dim3(kBT), args, 0, e->capture_stream);
  SB_E(cudaStreamEndCapture(e->capture_stream, &g));
  ce = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    r = cuda_status(ce, "cudaGraphInstantiate");
    exec_release(e);
    return r;
  }
#undef SB_E
  *out = e;
  return SB_OK;
}

int sb_batch_exec_destroy(sb_batch_exec* e) {
  if (!e) return SB_OK;
  if (e->pending) cudaEventSynchronize(e->done);
  exec_release(e);
  return SB_OK;
}

int sb_batch_exec_run(sb_batch_exec* e, const sb_batch_item* items, int32_t n, void* stream) {
  SB_REQUIRE(e, "sb_batch_exec_run: null executor");
  SB_REQUIRE(n >= 0 && n <= e->capacity, "sb_batch_exec_run: %d items exceed capacity %d", n,
             e->capacity);
  SB_REQUIRE(n == 0 || items, "sb_batch_exec_run: null items");
  // the pinned staging buffers are read by the previous run's first node
  if (e->pending) SB_CHECK_CUDA(cudaEventSynchronize(e->done));
  long long acc = 0;
  for (int i = 0; i < n; ++i) {
    sb_batch_item it = items[i];
    SB_REQUIRE(it.N >= 0 && it.nrhs >= 1 && it.nrhs <= kMaxRhs,
               "sb_batch_exec_run: item %d: N >= 0 and 1 <= nrhs <= 8 required", i);
    SB_REQUIRE(it.N == 0 || (it.row_ptr && it.x && it.y && (it.nnz == 0 || (it.col && it.val))),
               "sb_batch_exec_run: item %d: null pointer", i);
    if (it.lanes <= 0) it.lanes = lanes_for(it.nnz, it.N);
    it.lanes = it.lanes > 32 ? 32 : it.lanes;
    e->h_items[i] = it;
    e->h_offsets[i] = acc;
    acc += ((long long)it.N + 31) / 32;
  }
  e->h_offsets[n] = acc;
  e->h_count[0] = n;
  e->h_count[1] = 0;
  e->h_count[2] = 0;
  e->h_count[3] = 0;
  cudaStream_t st = as_stream(stream);
  SB_CHECK_CUDA(cudaGraphLaunch(e->graph, st));
  SB_CHECK_CUDA(cudaEventRecord(e->done, st));
  e->pending = true;
  return SB_OK;
}

}  // extern "C"
