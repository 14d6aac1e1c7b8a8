// sb_spts.cu -- level-set analysis and sparse triangular solves.
//
// Analysis: CSR_create_level_sets_with_reorder
// (src/parallel/src/sparse32.js:3010-3181).  level[i] = 0 when row i holds
// exactly one entry, otherwise 1 + the maximum (starting at 0) of level[c]
// over all entries but the last, where only columns c < i contribute (the
// reference reads the still-zero level of rows it has not reached).  Rows are
// stably counting-sorted by level (permutation, its inverse `order`), and a
// reordered CSR with columns relabelled by order[] is built.  All integer
// outputs are bit-exact.  Levels are computed by one thread per row, rows
// handed out in increasing order through a warp ticket so that every row a
// thread waits for has already been claimed by a running warp; each wait is
// an acquire load with a clock bound.
//
// Solves (one thread per row, storage order, separately rounded mul/add, so
// the results are bit-identical to the reference's row kernels):
//   SB_SPTS_LEVEL    level by level on the reordered matrix, the row kernel
//                    of src/parallel/src/sparse_opt_32.wat:11679-11757
//                    (t = 0; t += L_ij*y_j; y_i = (b_i - t)/L_ii)
//   SB_SPTS_SYNCFREE natural order with per-row ready flags, the kernel of
//                    src/parallel/src/spts_opt_32.wat:8-117
//                    (t = b_i; t -= L_ij*y_j; y_i = t/L_ii)
//   SB_SPTS_HYBRID   level order with ready flags (no per-level barrier), the
//                    row kernel's arithmetic, as the level/sync-free hybrid of
//                    src/parallel/src/sparse_opt_32.wat:12846-13445
#include <algorithm>
#include <mutex>
#include <vector>

#include "sb_common.cuh"
#include "sb_prims.cuh"

struct sb_spts_plan {
  int dtype = 0;
  int N = 0;
  long long nnz = 0;
  int nlevels = 0;
  int solvable = 0;
  int device = 0;
  const int* row_ptr = nullptr;  // caller's arrays (must outlive the plan)
  const int* col = nullptr;
  const void* val = nullptr;
  int* level = nullptr;
  int* level_ptr = nullptr;
  int* perm = nullptr;
  int* order = nullptr;
  int* rrow = nullptr;
  int* rcol = nullptr;
  void* rval = nullptr;
  void* ywork = nullptr;
  unsigned* flags = nullptr;
  int* ticket = nullptr;
  std::vector<int> h_level_ptr;
  std::vector<void*> owned;
};

namespace sb {

constexpr int kT = 256;
constexpr long long kDefaultSpin = 1LL << 31;  // SM cycles (about a second)

static unsigned grid1(long long n) {
  long long g = (n + kT - 1) / kT;
  return (unsigned)std::max(1LL, std::min(g, 0x7fffffffLL));
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Wait until flags[c] != 0 or the clock bound passes (then record a timeout
// in the status word and carry on, so that the kernel always terminates).
__device__ __forceinline__ void wait_ready(const unsigned* flags, int c, long long limit,
                                           int* status) {
  if (ld_acquire(flags + c)) return;
  const long long t0 = clock64();
  while (!ld_acquire(flags + c)) {
    if (clock64() - t0 > limit) {
      atomicExch(status, SB_DEV_TIMEOUT_DEP);
      return;
    }
    __nanosleep(64);
  }
}

// Rows in increasing order, 32 per warp ticket.
__device__ __forceinline__ int next_rows(int* ticket) {
  int base = 0;
  if ((threadIdx.x & 31) == 0) base = atomicAdd(ticket, 32);
  return __shfl_sync(0xffffffffu, base, 0);
}

template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T sub_rn(T a, T b);
template <> __device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
template <> __device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
template <typename T> __device__ __forceinline__ T div_rn(T a, T b);
template <> __device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
template <> __device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// ------------------------------------------------------------ analysis

// flags[0] = 1 unless every row is non-empty, ends with its diagonal and has
// all other columns in [0, i) (the structure the solves require).
__global__ void lower_check(const int* __restrict__ row_ptr, const int* __restrict__ col, int N,
                            int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = row_ptr[i], e = row_ptr[i + 1];
  bool ok = e > s && col[e - 1] == i;
  for (int j = s; ok && j < e - 1; ++j) ok = col[j] >= 0 && col[j] < i;
  if (!ok) flags[0] = 1;
}

__global__ void level_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col, int N,
                             int* __restrict__ level, unsigned* __restrict__ done,
                             int* __restrict__ ticket, long long limit, int* __restrict__ status) {
  while (true) {
    const int base = next_rows(ticket);
    if (base >= N) return;
    const int i = base + (threadIdx.x & 31);
    if (i < N) {
      const int s = row_ptr[i], e = row_ptr[i + 1];
      int lv;
      if (e - s == 1) {
        lv = 0;
      } else {
        int m = 0;
        for (int j = s; j < e - 1; ++j) {
          const int c = col[j];
          if (c >= 0 && c < i) {
            wait_ready(done, c, limit, status);
            const int lc = *(volatile const int*)(level + c);
            m = lc > m ? lc : m;
          }
        }
        lv = 1 + m;
      }
      level[i] = lv;
      st_release(done + i, 1u);
    }
  }
}

__global__ void max_kernel(const int* __restrict__ a, int n, int* __restrict__ out) {
  int m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    m = max(m, a[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void level_hist(const int* __restrict__ level, int N, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) atomicAdd(counts + level[i], 1);
}

__global__ void level_keys(const int* __restrict__ level, int N, unsigned long long* __restrict__ k,
                           unsigned* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    k[i] = (unsigned long long)(unsigned)level[i];
    v[i] = (unsigned)i;
  }
}

__global__ void perm_order(const unsigned* __restrict__ sorted_rows, int N, int* __restrict__ perm,
                           int* __restrict__ order) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) {
    const int i = (int)sorted_rows[p];
    perm[p] = i;
    order[i] = p;
  }
}

__global__ void gather_lengths(const int* __restrict__ row_ptr, const int* __restrict__ perm,
                               int N, int* __restrict__ lens) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) lens[p] = row_ptr[perm[p] + 1] - row_ptr[perm[p]];
}

template <typename T>
__global__ void reorder_rows(const int* __restrict__ row_ptr, const int* __restrict__ col,
                             const T* __restrict__ val, const int* __restrict__ perm,
                             const int* __restrict__ order, const int* __restrict__ rrow, int N,
                             int* __restrict__ rcol, T* __restrict__ rval) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int src = perm[p];
  int o = rrow[p];
  for (int j = row_ptr[src]; j < row_ptr[src + 1]; ++j, ++o) {
    const int c = col[j];
    rcol[o] = (c >= 0 && c < N) ? order[c] : c;
    rval[o] = val[j];
  }
}

// ------------------------------------------------------------ solves

// Row kernel of the level-set solve on rows [r0, r1) of the reordered matrix;
// b is read through the permutation, y is kept in level order.
template <typename T, typename A>
__global__ void spts_level_rows(const int* __restrict__ rrow, const int* __restrict__ rcol,
                                const T* __restrict__ rval, int r0, int r1,
                                const int* __restrict__ perm, const T* __restrict__ b,
                                T* __restrict__ yw) {
  const int i = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r1) return;
  const int s = rrow[i], end = rrow[i + 1] - 1;
  const A bi = (A)b[perm[i]];
  if (end > s) {
    A t = 0;
    for (int j = s; j < end; ++j) t = add_rn(t, mul_rn((A)rval[j], (A)yw[rcol[j]]));
    yw[i] = (T)div_rn(sub_rn(bi, t), (A)rval[end]);
  } else {
    yw[i] = (T)div_rn(bi, (A)rval[end]);
  }
}

// Level-ordered rows with ready flags (hybrid): same arithmetic as above.
template <typename T, typename A>
__global__ void spts_hybrid_rows(const int* __restrict__ rrow, const int* __restrict__ rcol,
                                 const T* __restrict__ rval, int N, const int* __restrict__ perm,
                                 const T* __restrict__ b, T* yw, unsigned* __restrict__ done,
                                 int* __restrict__ ticket, long long limit, int* status) {
  while (true) {
    const int base = next_rows(ticket);
    if (base >= N) return;
    const int i = base + (threadIdx.x & 31);
    if (i < N) {
      const int s = rrow[i], end = rrow[i + 1] - 1;
      const A bi = (A)b[perm[i]];
      T yi;
      if (end > s) {
        A t = 0;
        for (int j = s; j < end; ++j) {
          const int c = rcol[j];
          wait_ready(done, c, limit, status);
          t = add_rn(t, mul_rn((A)rval[j], (A)*(volatile const T*)(yw + c)));
        }
        yi = (T)div_rn(sub_rn(bi, t), (A)rval[end]);
      } else {
        yi = (T)div_rn(bi, (A)rval[end]);
      }
      yw[i] = yi;
      st_release(done + i, 1u);
    }
  }
}

// Sync-free solve in natural order (t = b_i; t -= L_ij*y_j; y_i = t/L_ii).
template <typename T, typename A>
__global__ void spts_syncfree_rows(const int* __restrict__ row_ptr, const int* __restrict__ col,
                                   const T* __restrict__ val, int N, const T* __restrict__ b, T* y,
                                   unsigned* __restrict__ done, int* __restrict__ ticket,
                                   long long limit, int* status) {
  while (true) {
    const int base = next_rows(ticket);
    if (base >= N) return;
    const int i = base + (threadIdx.x & 31);
    if (i < N) {
      const int s = row_ptr[i], e = row_ptr[i + 1];
      A t = (A)b[i];
      T yi;
      if (e > s + 1) {
        for (int j = s; j < e - 1; ++j) {
          const int c = col[j];
          if (c >= 0 && c < N) {
            wait_ready(done, c, limit, status);
            t = sub_rn(t, mul_rn((A)val[j], (A)*(volatile const T*)(y + c)));
          }
        }
        yi = (T)div_rn(t, (A)val[e - 1]);
      } else {
        yi = (e > s) ? (T)div_rn(t, (A)val[s]) : (T)t;
      }
      y[i] = yi;
      st_release(done + i, 1u);
    }
  }
}

template <typename T>
__global__ void scatter_by_perm(const T* __restrict__ yw, const int* __restrict__ perm, int N,
                                T* __restrict__ y) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) y[perm[p]] = yw[p];
}

static int resident_grid(const void* kern) {
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kT, 0);
  return std::max(1, per) * sm_count();
}

static int plan_alloc(sb_spts_plan* p, void** out, size_t bytes) {
  *out = nullptr;
  cudaError_t e = cudaMalloc(out, bytes ? bytes : 16);
  if (e != cudaSuccess) return cuda_status(e, "sb_spts_analyze: cudaMalloc");
  p->owned.push_back(*out);
  return SB_OK;
}

static void plan_release(sb_spts_plan* p) {
  for (void* q : p->owned) cudaFree(q);
  p->owned.clear();
}

template <typename T>
static int analyze_impl(sb_spts_plan* p, cudaStream_t st) {
  const int N = p->N;
  const long long nnz = p->nnz;
  int r;
  void* m;
#define SB_PA(ptr, bytes)                       \
  if ((r = plan_alloc(p, &m, (bytes)))) return r; \
  ptr = (decltype(ptr))m;
  SB_PA(p->level, sizeof(int) * N);
  SB_PA(p->perm, sizeof(int) * N);
  SB_PA(p->order, sizeof(int) * N);
  SB_PA(p->rrow, sizeof(int) * ((size_t)N + 1));
  SB_PA(p->rcol, sizeof(int) * (size_t)nnz);
  SB_PA(p->rval, sizeof(T) * (size_t)nnz);
  SB_PA(p->ywork, sizeof(T) * N);
  SB_PA(p->flags, sizeof(unsigned) * N);
  SB_PA(p->ticket, sizeof(int) * 4);
#undef SB_PA
  int* status = device_status_word();
  if (!status) {
    set_error("sb_spts_analyze: device status word unavailable");
    return SB_ENOMEM;
  }
  int* tmp = nullptr;  // [0] lower-check flag, [1] max level
  if ((r = scratch_alloc((void**)&tmp, 4 * sizeof(int), st))) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(tmp, 0, 4 * sizeof(int), st));
  lower_check<<<grid1(N), kT, 0, st>>>(p->row_ptr, p->col, N, tmp);
  SB_CHECK_LAUNCH("lower_check");
  SB_CHECK_CUDA(cudaMemsetAsync(p->flags, 0, sizeof(unsigned) * N, st));
  SB_CHECK_CUDA(cudaMemsetAsync(p->ticket, 0, sizeof(int), st));
  level_kernel<<<resident_grid((const void*)level_kernel), kT, 0, st>>>(
      p->row_ptr, p->col, N, p->level, p->flags, p->ticket, kDefaultSpin, status);
  SB_CHECK_LAUNCH("level_kernel");
  max_kernel<<<std::min<unsigned>(grid1(N), (unsigned)sm_count() * 4), kT, 0, st>>>(p->level, N,
                                                                                    tmp + 1);
  SB_CHECK_LAUNCH("max_kernel");
  int h[2] = {0, 0};
  SB_CHECK_CUDA(cudaMemcpyAsync(h, tmp, sizeof(h), cudaMemcpyDeviceToHost, st));
  int dstat = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&dstat, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(tmp, st);
  if (dstat) {
    cudaMemsetAsync(status, 0, sizeof(int), st);
    set_error("sb_spts_analyze: a level dependency wait timed out");
    return SB_ETIMEOUT;
  }
  p->solvable = h[0] ? 0 : 1;
  p->nlevels = N ? h[1] + 1 : 0;
  const int L = p->nlevels;
  {
    void* lp = nullptr;
    if ((r = plan_alloc(p, &lp, sizeof(int) * ((size_t)L + 1)))) return r;
    p->level_ptr = (int*)lp;
  }
  // level_ptr = exclusive scan of the per-level counts
  SB_CHECK_CUDA(cudaMemsetAsync(p->level_ptr, 0, sizeof(int) * ((size_t)L + 1), st));
  level_hist<<<grid1(N), kT, 0, st>>>(p->level, N, p->level_ptr);
  SB_CHECK_LAUNCH("level_hist");
  if ((r = prim::exclusive_scan(p->level_ptr, p->level_ptr, L + 1, st))) return r;
  // stable counting sort of rows by level
  prim::RadixBuffers rb;
  void* mem = nullptr;
  const size_t kb = sizeof(unsigned long long) * N, vb = sizeof(unsigned) * N;
  if ((r = scratch_alloc(&mem, 2 * kb + 2 * vb, st))) return r;
  rb.k[0] = (unsigned long long*)mem;
  rb.k[1] = (unsigned long long*)((char*)mem + kb);
  rb.v[0] = (unsigned*)((char*)mem + 2 * kb);
  rb.v[1] = (unsigned*)((char*)mem + 2 * kb + vb);
  level_keys<<<grid1(N), kT, 0, st>>>(p->level, N, rb.k[0], rb.v[0]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "level_keys");
  const int ranges[2] = {0, prim::bits_for(L - 1)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(rb, N, ranges, 1, &which, st);
  if (!r) {
    perm_order<<<grid1(N), kT, 0, st>>>(rb.v[which], N, p->perm, p->order);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "perm_order");
  }
  if (!r) {
    // reordered CSR: row lengths in level order, scanned into rrow
    int* lens = (int*)rb.k[0];
    gather_lengths<<<grid1(N), kT, 0, st>>>(p->row_ptr, p->perm, N, lens);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "gather_lengths");
    if (!r) r = prim::exclusive_scan(lens, p->rrow, N, st);
    if (!r) {
      const int nz = (int)nnz;
      e = cudaMemcpyAsync(p->rrow + N, &nz, sizeof(int), cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) r = cuda_status(e, "rrow");
    }
    if (!r) {
      reorder_rows<T><<<grid1(N), kT, 0, st>>>(p->row_ptr, p->col, (const T*)p->val, p->perm,
                                                p->order, p->rrow, N, p->rcol, (T*)p->rval);
      e = cudaGetLastError();
      if (e != cudaSuccess) r = cuda_status(e, "reorder_rows");
    }
  }
  if (!r) {
    p->h_level_ptr.resize((size_t)L + 1);
    e = cudaMemcpyAsync(p->h_level_ptr.data(), p->level_ptr, sizeof(int) * ((size_t)L + 1),
                        cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_spts_analyze");
  }
  scratch_free(mem, st);
  return r;
}

template <typename T, typename A>
static int solve_impl(const sb_spts_plan* p, int algo, const T* b, T* y, long long limit,
                      cudaStream_t st) {
  const int N = p->N;
  int* status = device_status_word();
  if (!status) {
    set_error("sb_spts_solve: device status word unavailable");
    return SB_ENOMEM;
  }
  if (algo == SB_SPTS_SYNCFREE) {
    SB_CHECK_CUDA(cudaMemsetAsync(p->flags, 0, sizeof(unsigned) * N, st));
    SB_CHECK_CUDA(cudaMemsetAsync(p->ticket, 0, sizeof(int), st));
    auto k = spts_syncfree_rows<T, A>;
    k<<<resident_grid((const void*)k), kT, 0, st>>>(p->row_ptr, p->col, (const T*)p->val, N, b, y,
                                                     p->flags, p->ticket, limit, status);
    SB_CHECK_LAUNCH("spts_syncfree_rows");
    return SB_OK;
  }
  T* yw = (T*)p->ywork;
  if (algo == SB_SPTS_HYBRID) {
    SB_CHECK_CUDA(cudaMemsetAsync(p->flags, 0, sizeof(unsigned) * N, st));
    SB_CHECK_CUDA(cudaMemsetAsync(p->ticket, 0, sizeof(int), st));
    auto k = spts_hybrid_rows<T, A>;
    k<<<resident_grid((const void*)k), kT, 0, st>>>(p->rrow, p->rcol, (const T*)p->rval, N,
                                                     p->perm, b, yw, p->flags, p->ticket, limit,
                                                     status);
    SB_CHECK_LAUNCH("spts_hybrid_rows");
  } else {
    for (int l = 0; l < p->nlevels; ++l) {
      const int r0 = p->h_level_ptr[l], r1 = p->h_level_ptr[l + 1];
      if (r1 <= r0) continue;
      spts_level_rows<T, A><<<grid1(r1 - r0), kT, 0, st>>>(p->rrow, p->rcol, (const T*)p->rval,
                                                           r0, r1, p->perm, b, yw);
      SB_CHECK_LAUNCH("spts_level_rows");
    }
  }
  scatter_by_perm<T><<<grid1(N), kT, 0, st>>>(yw, p->perm, N, y);
  SB_CHECK_LAUNCH("scatter_by_perm");
  return SB_OK;
}

// ------------------------------------------------------------ no-allocation variant
// Scratch of sb_spts_syncfree_csr_noalloc: one ready flag per row for up to
// kNoAllocMaxRows rows, then the row ticket and the status word on their own
// 128-byte lines.  It is a file-scope device array, so every GPU that loads
// this library holds these 16 MiB until the process exits, and every call
// shares them.
constexpr int kNoAllocMaxRows = 1 << 22;  // 4,194,304 rows
constexpr int kNoAllocTail = 64;          // ticket at +0, status at +32 (words)
static __device__ __align__(256) unsigned g_noalloc_scratch[kNoAllocMaxRows + kNoAllocTail];

// Device address of g_noalloc_scratch for the current device, looked up once
// per device (with that device current) and cached.  The host-side symbol is
// only a stand-in and must never be handed to a kernel.
static unsigned* noalloc_scratch(int* status) {
  static std::mutex mu;
  static unsigned* addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    *status = cuda_status(e == cudaSuccess ? cudaErrorInvalidDevice : e, "cudaGetDevice");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      *status = cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
      return nullptr;
    }
    addr[dev] = (unsigned*)p;
  }
  return addr[dev];
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_spts_syncfree_csr_noalloc(int dtype, const int32_t* row_ptr, const int32_t* col,
                                 const void* val, int32_t N, const void* b, void* y,
                                 int64_t spin_limit_cycles, void* stream) {
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_spts_syncfree_csr_noalloc: bad dtype");
  SB_REQUIRE(N >= 0, "sb_spts_syncfree_csr_noalloc: negative size");
  if (N > kNoAllocMaxRows) {
    set_error("sb_spts_syncfree_csr_noalloc: N = %d exceeds the fixed scratch limit of %d rows "
              "(use sb_spts_syncfree_csr)", N, kNoAllocMaxRows);
    return SB_EINVAL;
  }
  if (N == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col && val && b && y, "sb_spts_syncfree_csr_noalloc: null pointer");
  int r = ensure_device();
  if (r) return r;
  unsigned* scratch = noalloc_scratch(&r);
  if (!scratch) return r;
  cudaStream_t st = as_stream(stream);
  unsigned* flags = scratch;
  int* ticket = (int*)(scratch + kNoAllocMaxRows);
  int* status = (int*)(scratch + kNoAllocMaxRows + 32);
  // the array keeps the previous call's contents: clear what must start at 0
  SB_CHECK_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned) * (size_t)N, st));
  SB_CHECK_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * kNoAllocTail, st));
  const long long limit = spin_limit_cycles > 0 ? spin_limit_cycles : kDefaultSpin;
  if (dtype == SB_F64) {
    auto k = spts_syncfree_rows<double, double>;
    k<<<resident_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const double*)val, N,
                                                     (const double*)b, (double*)y, flags, ticket,
                                                     limit, status);
  } else {
    auto k = spts_syncfree_rows<float, float>;
    k<<<resident_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const float*)val, N,
                                                     (const float*)b, (float*)y, flags, ticket,
                                                     limit, status);
  }
  SB_CHECK_LAUNCH("spts_syncfree_rows");
  int dstat = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&dstat, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  if (dstat) {
    set_error("sb_spts_syncfree_csr_noalloc: a dependency wait ran out (row never became ready)");
    return SB_ETIMEOUT;
  }
  return SB_OK;
}

int sb_spts_analyze(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                    int32_t N, int64_t nnz, void* stream, sb_spts_plan** plan) {
  SB_REQUIRE(plan, "sb_spts_analyze: null plan output");
  *plan = nullptr;
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_spts_analyze: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_spts_analyze: bad size");
  SB_REQUIRE(row_ptr && (nnz == 0 || (col && val)), "sb_spts_analyze: null pointer");
  int r = ensure_device();
  if (r) return r;
  sb_spts_plan* p = new sb_spts_plan();
  p->dtype = dtype;
  p->N = N;
  p->nnz = nnz;
  p->row_ptr = row_ptr;
  p->col = col;
  p->val = val;
  cudaGetDevice(&p->device);
  cudaStream_t st = as_stream(stream);
  if (N == 0) {
    *plan = p;
    return SB_OK;
  }
  r = dtype == SB_F32 ? analyze_impl<float>(p, st) : analyze_impl<double>(p, st);
  if (r) {
    cudaStreamSynchronize(st);
    plan_release(p);
    delete p;
    return r;
  }
  *plan = p;
  return SB_OK;
}

int sb_spts_plan_destroy(sb_spts_plan* plan) {
  if (!plan) return SB_OK;
  cudaDeviceSynchronize();
  plan_release(plan);
  delete plan;
  return SB_OK;
}

int sb_spts_plan_info(const sb_spts_plan* plan, int32_t* nlevels, int32_t* solvable) {
  SB_REQUIRE(plan && nlevels && solvable, "sb_spts_plan_info: null argument");
  *nlevels = plan->nlevels;
  *solvable = plan->solvable;
  return SB_OK;
}

int sb_spts_plan_levels(const sb_spts_plan* plan, int32_t* level, int32_t* level_ptr,
                        int32_t* permutation, int32_t* order, void* stream) {
  SB_REQUIRE(plan, "sb_spts_plan_levels: null plan");
  const size_t n = sizeof(int) * (size_t)plan->N;
  cudaStream_t st = as_stream(stream);
  if (plan->N == 0) return SB_OK;
  if (level) SB_CHECK_CUDA(cudaMemcpyAsync(level, plan->level, n, cudaMemcpyDeviceToDevice, st));
  if (level_ptr)
    SB_CHECK_CUDA(cudaMemcpyAsync(level_ptr, plan->level_ptr,
                                  sizeof(int) * ((size_t)plan->nlevels + 1),
                                  cudaMemcpyDeviceToDevice, st));
  if (permutation)
    SB_CHECK_CUDA(cudaMemcpyAsync(permutation, plan->perm, n, cudaMemcpyDeviceToDevice, st));
  if (order) SB_CHECK_CUDA(cudaMemcpyAsync(order, plan->order, n, cudaMemcpyDeviceToDevice, st));
  return SB_OK;
}

int sb_spts_plan_reordered(const sb_spts_plan* plan, int32_t* row_ptr, int32_t* col, void* val,
                           void* stream) {
  SB_REQUIRE(plan, "sb_spts_plan_reordered: null plan");
  cudaStream_t st = as_stream(stream);
  if (plan->N == 0) return SB_OK;
  if (row_ptr)
    SB_CHECK_CUDA(cudaMemcpyAsync(row_ptr, plan->rrow, sizeof(int) * ((size_t)plan->N + 1),
                                  cudaMemcpyDeviceToDevice, st));
  if (col)
    SB_CHECK_CUDA(cudaMemcpyAsync(col, plan->rcol, sizeof(int) * (size_t)plan->nnz,
                                  cudaMemcpyDeviceToDevice, st));
  if (val)
    SB_CHECK_CUDA(cudaMemcpyAsync(val, plan->rval, dtype_size(plan->dtype) * (size_t)plan->nnz,
                                  cudaMemcpyDeviceToDevice, st));
  return SB_OK;
}

int sb_spts_solve(const sb_spts_plan* plan, int algo, int policy, const void* b, void* y,
                  void* stream) {
  SB_REQUIRE(plan, "sb_spts_solve: null plan");
  SB_REQUIRE(algo == SB_SPTS_LEVEL || algo == SB_SPTS_SYNCFREE || algo == SB_SPTS_HYBRID,
             "sb_spts_solve: unknown algorithm %d", algo);
  if (plan->N == 0) return SB_OK;
  SB_REQUIRE(b && y, "sb_spts_solve: null vector");
  if (!plan->solvable) {
    set_error("sb_spts_solve: matrix is not lower triangular with its diagonal stored last");
    return SB_EINVAL;
  }
  cudaStream_t st = as_stream(stream);
  if (plan->dtype == SB_F64)
    return solve_impl<double, double>(plan, algo, (const double*)b, (double*)y, kDefaultSpin, st);
  if (policy == SB_SPTS_ACC_F64)
    return solve_impl<float, double>(plan, algo, (const float*)b, (float*)y, kDefaultSpin, st);
  return solve_impl<float, float>(plan, algo, (const float*)b, (float*)y, kDefaultSpin, st);
}

int sb_spts_syncfree_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                         int32_t N, const void* b, void* y, int64_t spin_limit_cycles,
                         void* stream) {
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_spts_syncfree_csr: bad dtype");
  SB_REQUIRE(N >= 0, "sb_spts_syncfree_csr: negative size");
  if (N == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col && val && b && y, "sb_spts_syncfree_csr: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  int* status = device_status_word();
  if (!status) return SB_ENOMEM;
  unsigned* flags = nullptr;
  if ((r = scratch_alloc((void**)&flags, sizeof(unsigned) * ((size_t)N + 8), st))) return r;
  int* ticket = (int*)(flags + N);
  SB_CHECK_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned) * ((size_t)N + 8), st));
  const long long limit = spin_limit_cycles > 0 ? spin_limit_cycles : kDefaultSpin;
  if (dtype == SB_F64) {
    auto k = spts_syncfree_rows<double, double>;
    k<<<resident_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const double*)val, N,
                                                     (const double*)b, (double*)y, flags, ticket,
                                                     limit, status);
  } else {
    auto k = spts_syncfree_rows<float, float>;
    k<<<resident_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const float*)val, N,
                                                     (const float*)b, (float*)y, flags, ticket,
                                                     limit, status);
  }
  SB_CHECK_LAUNCH("spts_syncfree_rows");
  int dstat = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&dstat, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(flags, st);
  if (dstat) {
    SB_CHECK_CUDA(cudaMemset(status, 0, sizeof(int)));
    set_error("sb_spts_syncfree_csr: a dependency wait ran out (row never became ready)");
    return SB_ETIMEOUT;
  }
  return SB_OK;
}

}  // extern "C"
