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
//                    (t = 0; t += L_ij*y_j; y_i = (b_i - t)/L_ii), in one
//                    cooperative launch with a grid barrier per level
//   SB_SPTS_SYNCFREE natural order with per-row ready flags, the kernel of
//                    src/parallel/src/spts_opt_32.wat:8-117
//                    (t = b_i; t -= L_ij*y_j; y_i = t/L_ii)
//   SB_SPTS_HYBRID   level order with ready flags (no per-level barrier), the
//                    row kernel's arithmetic, as the level/sync-free hybrid of
//                    src/parallel/src/sparse_opt_32.wat:12846-13445
#include <algorithm>
#include <cstring>
#include <type_traits>
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
  int* ticket = nullptr;
  std::vector<int> h_level_ptr;
  std::vector<void*> owned;
  cudaEvent_t ev[2] = {nullptr, nullptr};  // bracket the analysis's device work
  float analysis_ms = 0.f;
};

namespace sb {

constexpr int kT = 256;
constexpr long long kDefaultSpin = 1LL << 31;  // SM cycles (about a second)

// Polling back-off of the dependency waits: the sleep between two polls of a
// ready flag starts at SB_SPTS_SLEEP_MIN_NS and doubles up to
// SB_SPTS_SLEEP_MAX_NS.  Measured on B200 over maxima of 64 to 2048 ns (and no
// sleep), the wake-up delay of the longer sleeps costs more per level than
// the extra polling traffic of the short ones, from 190-level to 100,000-level
// factors; 64 ns was best or within 5% of best on every matrix tried.
#ifndef SB_SPTS_SLEEP_MIN_NS
#define SB_SPTS_SLEEP_MIN_NS 32u
#endif
#ifndef SB_SPTS_SLEEP_MAX_NS
#define SB_SPTS_SLEEP_MAX_NS 64u
#endif

static unsigned grid1(long long n) {
  long long g = (n + kT - 1) / kT;
  return (unsigned)std::max(1LL, std::min(g, 0x7fffffffLL));
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void fence_acquire() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Wait until flags[c] != 0 or the clock bound passes (then record a timeout
// in the status word and carry on, so that the kernel always terminates).
// Polls with relaxed loads: the caller issues an acquire fence before it
// reads what the flag publishes.
__device__ __noinline__ void wait_ready(const unsigned* flags, int c, long long limit,
                                        int* status) {
  const long long t0 = clock64();
  unsigned ns = SB_SPTS_SLEEP_MIN_NS;
  while (!ld_relaxed_u32(flags + c)) {
    // once any wait has given up, the others give up at once
    if (clock64() - t0 > limit || *(volatile const int*)status) {
      atomicExch(status, SB_DEV_TIMEOUT_DEP);
      return;
    }
    __nanosleep(ns);
    ns = ns < SB_SPTS_SLEEP_MAX_NS ? 2 * ns : ns;
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

// ------------------------------------------------------------ pending values
// The plan-based solves and the level analysis publish each row's result in a
// work array that starts filled with all-one bits ("pending").  One relaxed
// load of a dependency then gives both its readiness and its value: no ready
// flag, no fence, and the loads of a row's dependencies go out together
// (kG per round trip).  A result that happens to have the pending bits is
// stored as a canonical NaN instead, so a written result is never pending.
__device__ __forceinline__ float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_relaxed(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(int* p, int v) {
  asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ bool pending(float v) { return __float_as_uint(v) == 0xffffffffu; }
__device__ __forceinline__ bool pending(double v) { return __double_as_longlong(v) == -1LL; }
__device__ __forceinline__ bool pending(int v) { return v < 0; }
__device__ __forceinline__ float settled(float v) {
  return pending(v) ? __uint_as_float(0x7fffffffu) : v;
}
__device__ __forceinline__ double settled(double v) {
  return pending(v) ? __longlong_as_double(0x7fffffffffffffffLL) : v;
}

constexpr int kG = 8;  // dependencies loaded per round trip

// Wait until none of v[k] (k < n, loaded from p[c[k]]) is pending: every
// poll reloads all still-pending entries of the group at once (one round
// trip).  The sleep between polls backs off; past the clock bound (or once
// any other wait has given up) the wait records a timeout in the status
// word and returns with the entries still pending, so that the kernel
// always terminates.
template <typename V>
__device__ __forceinline__ void wait_group(const V* p, const int (&c)[kG], V (&v)[kG], int n,
                                           long long limit, int* status) {
  unsigned mask = 0;
#pragma unroll
  for (int k = 0; k < kG; ++k)
    if (k < n && pending(v[k])) mask |= 1u << k;
  if (!mask) return;
  const long long t0 = clock64();
  unsigned ns = SB_SPTS_SLEEP_MIN_NS;
  while (true) {
    __nanosleep(ns);
    ns = ns < SB_SPTS_SLEEP_MAX_NS ? 2 * ns : ns;
#pragma unroll
    for (int k = 0; k < kG; ++k)
      if (mask & (1u << k)) v[k] = ld_relaxed(p + c[k]);
    unsigned still = 0;
#pragma unroll
    for (int k = 0; k < kG; ++k)
      if ((mask & (1u << k)) && pending(v[k])) still |= 1u << k;
    mask = still;
    if (!mask) return;
    if (clock64() - t0 > limit || *(volatile const int*)status) {
      atomicExch(status, SB_DEV_TIMEOUT_DEP);
      return;
    }
  }
}

// acc (+|-)= val[j] * w[col[j]] for j in [s, e), in storage order, waiting
// for each w[col[j]] to be published (SUB selects the sync-free form).
template <typename T, typename A, bool SUB>
__device__ __forceinline__ A dot_published(const int* __restrict__ col, const T* __restrict__ val,
                                           int s, int e, const T* w, A acc, long long limit,
                                           int* status) {
  for (int j0 = s; j0 < e; j0 += kG) {
    const int n = e - j0 < kG ? e - j0 : kG;
    int c[kG];
    A a[kG];
    T v[kG];
#pragma unroll
    for (int k = 0; k < kG; ++k)
      if (k < n) {
        c[k] = col[j0 + k];
        a[k] = (A)val[j0 + k];
      }
#pragma unroll
    for (int k = 0; k < kG; ++k)
      if (k < n) v[k] = ld_relaxed(w + c[k]);
    wait_group(w, c, v, n, limit, status);
#pragma unroll
    for (int k = 0; k < kG; ++k)
      if (k < n) acc = SUB ? sub_rn(acc, mul_rn(a[k], (A)v[k])) : add_rn(acc, mul_rn(a[k], (A)v[k]));
  }
  return acc;
}

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
                             int* level, int* __restrict__ ticket, long long limit,
                             int* __restrict__ status) {
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
        for (int j0 = s; j0 < e - 1; j0 += kG) {
          int c[kG], v[kG];
#pragma unroll
          for (int k = 0; k < kG; ++k) {
            // columns outside [0, i) read as level 0 (row 0's slot, never pending)
            const int cc = (j0 + k < e - 1) ? col[j0 + k] : -1;
            c[k] = (cc >= 0 && cc < i) ? cc : -1;
          }
#pragma unroll
          for (int k = 0; k < kG; ++k) v[k] = c[k] >= 0 ? ld_relaxed(level + c[k]) : 0;
          wait_group(level, c, v, kG, limit, status);
#pragma unroll
          for (int k = 0; k < kG; ++k) m = v[k] > m ? v[k] : m;
        }
        lv = 1 + m;
      }
      st_relaxed(level + i, lv);
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

// Grid barrier of a cooperative launch (every block resident) on one
// monotonic arrival counter: at the barrier that closes level l, thread 0 of
// each block adds 1 with an acquire-release add (ordered after the block's
// stores, which bar.sync made visible to it) and waits until the counter reaches
// gridDim.x * (l + 1), polling with acquire loads and a short sleep, bounded
// by `limit` SM cycles (or by a timeout already recorded in the status
// word).  One atomic per block and level: no reset and no generation word
// (the earlier form's last arrival reset the counter and advanced a
// generation, two more dependent atomics per level).  The comparison is
// wrap-safe: the counter never runs more than gridDim.x ahead of a waiter.
// Returns false after a timeout, which it records; the caller then returns.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;"
               : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, long long limit,
                                             int* status) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    // acq_rel: the last block to arrive goes on at once, so its add also
    // acquires the other blocks' released stores
    if (atom_add_acq_rel(bar, 1u) + 1u != target) {
      const long long t0 = clock64();
      unsigned ns = SB_SPTS_SLEEP_MIN_NS;
      while ((int)(ld_acquire_u32(bar) - target) < 0) {
        if (clock64() - t0 > limit || *(volatile const int*)status) {
          atomicExch(status, SB_DEV_TIMEOUT_DEP);
          ok = 0;
          break;
        }
        __nanosleep(ns);
        ns = ns < SB_SPTS_SLEEP_MAX_NS ? 2 * ns : ns;
      }
    }
  }
  __syncthreads();
  return ok != 0;
}

// A thread's first row of a level, read ahead of the barrier that opens the
// level: its structure, b, diagonal and up to kG off-diagonal columns and
// values (the values of the columns are read after the barrier).
template <typename T, typename A>
struct LevelRow {
  int i = -1, s = 0, end = 0, pi = 0;
  A bi = 0, diag = 0;
  int c[kG];
  A v[kG];
};

// A thread's first row of the level after next: where its entries are and
// where its output goes (the first of the two dependent load rounds of a
// row, issued one level earlier than the second).
struct LevelHead {
  int i = -1, s = 0, end = 0, pi = 0;
};

__device__ __forceinline__ void level_head_load(LevelHead& h, int i, const int* rrow,
                                                const int* perm) {
  h.i = i;
  h.s = rrow[i];
  h.end = rrow[i + 1] - 1;
  h.pi = perm[i];
}

// The second round: b, the diagonal and up to kG off-diagonal columns and
// values of the row a head describes.
template <typename T, typename A>
__device__ __forceinline__ void level_row_from_head(LevelRow<T, A>& r, const LevelHead& h,
                                                    const int* rcol, const T* rval, const T* b) {
  r.i = h.i;
  if (h.i < 0) return;
  r.s = h.s;
  r.end = h.end;
  r.pi = h.pi;
  r.bi = (A)b[r.pi];
  r.diag = (A)rval[r.end];
#pragma unroll
  for (int k = 0; k < kG; ++k) {
    const int j = r.s + k;
    r.c[k] = j < r.end ? rcol[j] : 0;
    r.v[k] = j < r.end ? (A)rval[j] : A(0);
  }
}

template <typename T, typename A>
__device__ __forceinline__ void level_row_load(LevelRow<T, A>& r, int i, const int* rrow,
                                               const int* rcol, const T* rval, const int* perm,
                                               const T* b) {
  r.i = i;
  r.s = rrow[i];
  r.end = rrow[i + 1] - 1;
  r.pi = perm[i];
  r.bi = (A)b[r.pi];
  r.diag = (A)rval[r.end];
#pragma unroll
  for (int k = 0; k < kG; ++k) {
    const int j = r.s + k;
    r.c[k] = j < r.end ? rcol[j] : 0;
    r.v[k] = j < r.end ? (A)rval[j] : A(0);
  }
}

// The level-set solve in one cooperative launch: the levels in order, the
// rows of a level spread over all threads with the arithmetic of
// spts_level_rows, a grid barrier after every level (the reference's
// structure, src/parallel/src/spts_opt_32.wat:339-546).  Values of earlier
// levels are read from L2 (__ldcg), since L1 is not kept coherent with other
// SMs' stores inside a launch; each row also writes its natural-order
// output, so no scatter pass follows.  Each thread reads its first row of
// a level in two rounds ahead of time: its row pointers and permutation two
// levels before, its columns, values, b and diagonal one level before, so
// that only the y reads after each barrier lie on the level's critical
// path.  When every level fits in
// one block of kLevelBlock1 threads, the launch is that one block and the
// barrier is __syncthreads.
constexpr int kLevelBlock1 = 512;  // threads of the single-block form

template <typename T, typename A, bool TWO>
__global__ void __launch_bounds__(kLevelBlock1, 1)
    spts_level_coop(const int* __restrict__ rrow, const int* __restrict__ rcol,
                    const T* __restrict__ rval, const int* __restrict__ level_ptr, int nlevels,
                    const int* __restrict__ perm, const T* __restrict__ b, T* yw,
                    T* __restrict__ y, unsigned* bar, long long limit, int* status) {
  const int nthreads = gridDim.x * blockDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  LevelRow<T, A> nx;
  LevelHead hd;  // the first row of the level after the next one
  {
    const int r0 = __ldg(level_ptr), r1 = __ldg(level_ptr + 1);
    if (r0 + gt < r1) level_row_load(nx, r0 + gt, rrow, rcol, rval, perm, b);
    if (TWO && nlevels > 1) {
      const int q0 = r1, q1 = __ldg(level_ptr + 2);
      if (q0 + gt < q1) level_head_load(hd, q0 + gt, rrow, perm);
    }
  }
  for (int l = 0; l < nlevels; ++l) {
    const int r0 = __ldg(level_ptr + l), r1 = __ldg(level_ptr + l + 1);
    if (nx.i >= 0) {  // the prefetched first row (index r0 + gt)
      A t = 0;
      const int n = nx.end - nx.s;
      T w[kG];
#pragma unroll
      for (int k = 0; k < kG; ++k)
        if (k < n) w[k] = __ldcg(yw + nx.c[k]);
#pragma unroll
      for (int k = 0; k < kG; ++k)
        if (k < n) t = add_rn(t, mul_rn(nx.v[k], (A)w[k]));
      for (int j = nx.s + kG; j < nx.end; ++j)
        t = add_rn(t, mul_rn((A)rval[j], (A)__ldcg(yw + rcol[j])));
      const T yi = n > 0 ? (T)div_rn(sub_rn(nx.bi, t), nx.diag) : (T)div_rn(nx.bi, nx.diag);
      __stcg(yw + nx.i, yi);
      y[nx.pi] = yi;
    }
    for (int i = r0 + gt + nthreads; i < r1; i += nthreads) {
      const int s = rrow[i], end = rrow[i + 1] - 1;
      const int pi = perm[i];
      const A bi = (A)b[pi];
      T yi;
      if (end > s) {
        A t = 0;
        for (int j = s; j < end; ++j) t = add_rn(t, mul_rn((A)rval[j], (A)__ldcg(yw + rcol[j])));
        yi = (T)div_rn(sub_rn(bi, t), (A)rval[end]);
      } else {
        yi = (T)div_rn(bi, (A)rval[end]);
      }
      __stcg(yw + i, yi);
      y[pi] = yi;
    }
    if (l + 1 < nlevels) {
      if constexpr (TWO) {
        // the next level's first row from the head read one level ago, and
        // the head of the level after it: neither depends on y, so both load
        // rounds overlap the barrier and the next level's y reads
        level_row_from_head(nx, hd, rcol, rval, b);
        hd.i = -1;
        if (l + 2 < nlevels) {
          const int q0 = __ldg(level_ptr + l + 2), q1 = __ldg(level_ptr + l + 3);
          if (q0 + gt < q1) level_head_load(hd, q0 + gt, rrow, perm);
        }
      } else {
        // both rounds of the next level's first row, before the barrier
        const int q0 = r1, q1 = __ldg(level_ptr + l + 2);
        nx.i = -1;
        if (q0 + gt < q1) level_row_load(nx, q0 + gt, rrow, rcol, rval, perm, b);
      }
      if (gridDim.x == 1) __syncthreads();  // one block: its barrier orders the L2 accesses
      else if (!grid_barrier(bar, gridDim.x * (unsigned)(l + 1), limit, status)) return;
    }
  }
}

// Level-ordered rows (hybrid): same arithmetic as above, dependencies read
// from the pending-initialised work vector yw (level order); each row also
// writes its natural-order output y[perm[i]].
template <typename T, typename A>
__global__ void spts_hybrid_rows(const int* __restrict__ rrow, const int* __restrict__ rcol,
                                 const T* __restrict__ rval, int N, const int* __restrict__ perm,
                                 const T* __restrict__ b, T* yw, T* __restrict__ y,
                                 int* __restrict__ ticket, long long limit, int* status) {
  while (true) {
    const int base = next_rows(ticket);
    if (base >= N) return;
    const int i = base + (threadIdx.x & 31);
    if (i < N) {
      const int s = rrow[i], end = rrow[i + 1] - 1;
      const int pi = perm[i];
      const A bi = (A)b[pi];
      T yi;
      if (end > s) {
        const A t = dot_published<T, A, false>(rcol, rval, s, end, yw, A(0), limit, status);
        yi = (T)div_rn(sub_rn(bi, t), (A)rval[end]);
      } else {
        yi = (T)div_rn(bi, (A)rval[end]);
      }
      st_relaxed(yw + i, settled(yi));
      y[pi] = yi;
    }
  }
}

// Sync-free solve of an analysed (lower, diagonal last) matrix in natural
// order, the sync-free kernel's arithmetic (t = b_i; t -= L_ij*y_j;
// y_i = t/L_ii), dependencies read from the pending-initialised yw.
template <typename T, typename A>
__global__ void spts_syncfree_plan_rows(const int* __restrict__ row_ptr,
                                        const int* __restrict__ col, const T* __restrict__ val,
                                        int N, const T* __restrict__ b, T* yw, T* __restrict__ y,
                                        int* __restrict__ ticket, long long limit, int* status) {
  while (true) {
    const int base = next_rows(ticket);
    if (base >= N) return;
    const int i = base + (threadIdx.x & 31);
    if (i < N) {
      const int s = row_ptr[i], e = row_ptr[i + 1];
      const A t = dot_published<T, A, true>(col, val, s, e - 1, yw, (A)b[i], limit, status);
      const T yi = (T)div_rn(t, (A)val[e - 1]);
      st_relaxed(yw + i, settled(yi));
      y[i] = yi;
    }
  }
}

// Sync-free solve in natural order (t = b_i; t -= L_ij*y_j; y_i = t/L_ii) on
// the caller's arrays with ready flags: a row first waits for the flags of
// all its in-range dependencies (kG relaxed loads per round trip), then one
// acquire fence orders the value loads after them.
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
        for (int j0 = s; j0 < e - 1; j0 += kG) {
          int c[kG];
          unsigned f[kG];
#pragma unroll
          for (int k = 0; k < kG; ++k) c[k] = (j0 + k < e - 1) ? col[j0 + k] : -1;
#pragma unroll
          for (int k = 0; k < kG; ++k) f[k] = (c[k] >= 0 && c[k] < N) ? ld_relaxed_u32(done + c[k]) : 1u;
#pragma unroll
          for (int k = 0; k < kG; ++k)
            if (!f[k]) wait_ready(done, c[k], limit, status);
        }
        fence_acquire();
        for (int j0 = s; j0 < e - 1; j0 += kG) {
          int c[kG];
          T v[kG];
#pragma unroll
          for (int k = 0; k < kG; ++k) c[k] = (j0 + k < e - 1) ? col[j0 + k] : -1;
#pragma unroll
          for (int k = 0; k < kG; ++k)
            if (c[k] >= 0 && c[k] < N) v[k] = ld_relaxed(y + c[k]);
#pragma unroll
          for (int k = 0; k < kG; ++k)
            if (c[k] >= 0 && c[k] < N) t = sub_rn(t, mul_rn((A)val[j0 + k], (A)v[k]));
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

// ------------------------------------------------------------ batched solves
// Many independent systems in one launch of one warp per 32-row chunk (not
// persistent: warps exit after their chunk, and the hardware dispatches the
// blocks as SM slots free up).  Warps are laid out in rounds of one chunk per
// unfinished system, so all systems of a batch advance at the same time and
// the launch takes about the deepest system's time, not the sum.  A warp
// takes its chunk from its system's ticket counter, i.e. chunks of a system
// are claimed in level order by running warps; a row waits only on rows of
// its own system with a smaller level-order index, all claimed by running
// warps, so the launch always makes progress whatever order the hardware
// runs the blocks in.  Rows are solved as in spts_hybrid_rows.
constexpr int kTB = 128;  // threads per block of the batched solve

struct SptsDesc {
  const int* rrow;
  const int* rcol;
  const void* rval;
  const int* perm;
  void* yw;
  const void* b;
  void* y;
  int N;
  int pad;
};

// Schedule of one batch: systems sorted by chunk count (order[]), and the
// warps in rounds of one chunk per system still unfinished.  Segment k holds
// the rounds [nch(order[k-1]), nch(order[k])) of the M - k systems
// order[k..M-1]; seg[k] is the first warp of segment k and `warps` the
// number of warps (one per chunk of the batch).
struct SptsSched {
  int M;
  int pad;
  long long warps;
};

// Every item's work vector to the pending bits.
template <typename T>
__global__ void spts_batch_reset(const SptsDesc* __restrict__ items,
                                 const SptsSched* __restrict__ sched) {
  using U = typename std::conditional<sizeof(T) == 4, unsigned, unsigned long long>::type;
  const int M = sched->M;
  for (int k = 0; k < M; ++k) {
    U* w = (U*)items[k].yw;
    const long long N = items[k].N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
      w[i] = ~U(0);
  }
}

// The chunk of warp slot gw of the round layout: its system from the
// segment table, the chunk itself from the system's ticket (claimed in level
// order by a running warp), then one row per lane as in spts_hybrid_rows.
template <typename T, typename A>
__device__ __forceinline__ void batch_chunk(const SptsDesc* __restrict__ items,
                                            const int* __restrict__ order,
                                            const long long* __restrict__ seg,
                                            int* __restrict__ tickets, int M, long long gw,
                                            int lane, long long limit, int* status) {
  int lo = 0, hi = M - 1;  // last segment starting at or before gw
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid] <= gw) lo = mid; else hi = mid - 1;
  }
  const int sys = order[lo + (int)((gw - seg[lo]) % (M - lo))];
  int t = 0;
  if (lane == 0) t = atomicAdd(tickets + sys, 1);
  t = __shfl_sync(0xffffffffu, t, 0);
  const SptsDesc d = items[sys];
  const int i = t * 32 + lane;
  if (i >= d.N) return;
  const T* __restrict__ rval = (const T*)d.rval;
  T* yw = (T*)d.yw;
  const int s = d.rrow[i], end = d.rrow[i + 1] - 1;
  const int pi = d.perm[i];
  const A bi = (A)((const T*)d.b)[pi];
  T yi;
  if (end > s) {
    const A acc = dot_published<T, A, false>(d.rcol, rval, s, end, yw, A(0), limit, status);
    yi = (T)div_rn(sub_rn(bi, acc), (A)rval[end]);
  } else {
    yi = (T)div_rn(bi, (A)rval[end]);
  }
  st_relaxed(yw + i, settled(yi));
  ((T*)d.y)[pi] = yi;
}

// persistent == 0: one warp per warp slot (the grid covers the layout).
// persistent != 0: a capped grid whose warps take warp slots from *work
// until the layout is done, so that the launch leaves SMs to other work (a
// concurrent batch on another stream).  Either way a chunk is claimed only
// by a running warp, and a row waits only on rows of its own system claimed
// earlier, so the launch always makes progress.
template <typename T, typename A>
__global__ void __launch_bounds__(kTB)
    spts_batch_kernel(const SptsDesc* __restrict__ items, const SptsSched* __restrict__ sched,
                      const int* __restrict__ order, const long long* __restrict__ seg,
                      int* __restrict__ tickets, long long limit, int* status,
                      unsigned long long* __restrict__ work, int persistent) {
  const int lane = threadIdx.x & 31;
  const int M = sched->M;
  const long long warps = sched->warps;
  if (M <= 0) return;
  if (!persistent) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw < warps) batch_chunk<T, A>(items, order, seg, tickets, M, gw, lane, limit, status);
    return;
  }
  while (true) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(work, 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if ((long long)w >= warps) return;
    batch_chunk<T, A>(items, order, seg, tickets, M, (long long)w, lane, limit, status);
    __syncwarp();
  }
}

// max over rows of sum_{j < diag} |L_ij| / |L_ii| (inf for a zero diagonal),
// as the bits of a non-negative double so that an integer max orders them.
template <typename T>
__global__ void growth_kernel(const int* __restrict__ row_ptr, const T* __restrict__ val, int N,
                              unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = row_ptr[i], e = row_ptr[i + 1];
    if (e <= s) continue;
    double off = 0.0;
    for (int j = s; j < e - 1; ++j) off += fabs((double)val[j]);
    const double dg = fabs((double)val[e - 1]);
    const double r = off / dg;  // 0/0 -> NaN, x/0 -> inf
    const double rr = (r != r) ? __longlong_as_double(0x7ff0000000000000LL) : r;
    m = rr > m ? rr : m;
  }
  unsigned long long b = (unsigned long long)__double_as_longlong(m);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, b, o);
    b = v > b ? v : b;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, b);
}

// flags[0] = 1 unless every column j of a CSC lower triangle is non-empty,
// starts with its diagonal (row j) and has all other rows in (j, N).
__global__ void csc_lower_check(const int* __restrict__ col_ptr, const int* __restrict__ row,
                                int N, int* __restrict__ flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const int s = col_ptr[j], e = col_ptr[j + 1];
  bool ok = e > s && row[s] == j;
  for (int q = s + 1; ok && q < e; ++q) ok = row[q] > j && row[q] < N;
  if (!ok) flags[0] = 1;
}

static int resident_grid(const void* kern) {
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kT, 0);
  return std::max(1, per) * sm_count();
}

// Grid of the plan-based polling solves.  Every warp that holds rows ahead
// of the dependency frontier polls, and polling warps take issue slots and
// L2 round trips from the warps at the frontier.  Measured on B200 from 74 to
// 592 CTAs, on factors with 1 to 10^6 rows per level:
//  * the level-ordered hybrid solve was fastest, or within 3%, with one CTA
//    per SM on every factor (3-D Laplacian 64^3: 0.295 -> 0.246 ms; 1M-row
//    random factor with 3470 levels: 9.5 -> 4.6 ms);
//  * the natural-order sync-free solve needs the full resident grid when
//    levels are wide (3-D Laplacians, >= 1380 rows per level: 5.6 ms at 444
//    CTAs, 9.5 ms at 148 on 128^3) and one CTA per SM when they are narrow
//    (288 rows per level: 9.5 -> 4.4 ms).
// Grid of the natural-order polling kernels that run without level
// information (the analysis itself and the sync-free solve on caller
// arrays): two CTAs per SM.  Measured on B200 against the resident grid
// (analysis / caller-array sync-free, ms): 3-D Laplacian 64^3 3.35 -> 3.16 /
// 1.51 -> 1.50; 128^3 8.58 -> 8.15 / 15.2 -> 15.4; 1M-row random factor
// 18.1 -> 8.1 / 41.0 -> 25.9; band-50 1M 425 -> 224 / 2048 -> 1368;
// bidiagonal 100k 122 -> 81 / 265 -> 259.  One CTA per SM was faster still on
// the narrow factors and 30-50% slower on the Laplacians.
static int natural_order_grid(const void* kern) {
  return std::min(resident_grid(kern), 2 * sm_count());
}

static int polling_grid(const void* kern, int algo, int N, int nlevels) {
  const int full = resident_grid(kern);
  const bool wide = nlevels > 0 && (long long)N >= 1024LL * nlevels;
  if (algo == SB_SPTS_SYNCFREE && wide) return full;
  return std::min(full, sm_count());
}

// The plan's device arrays live in one allocation (one cudaMalloc per plan,
// not one per array); level_ptr is sized for the largest possible level
// count, N + 1 (a row's level is at most its index + 1).
static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

static void plan_release(sb_spts_plan* p) {
  for (void* q : p->owned) cudaFree(q);
  p->owned.clear();
  if (p->ev[0]) cudaEventDestroy(p->ev[0]);
  if (p->ev[1]) cudaEventDestroy(p->ev[1]);
  p->ev[0] = p->ev[1] = nullptr;
}

template <typename T>
static int analyze_impl(sb_spts_plan* p, cudaStream_t st) {
  const int N = p->N;
  const long long nnz = p->nnz;
  int r;
  {
    const size_t sizes[9] = {sizeof(int) * (size_t)N,           sizeof(int) * (size_t)N,
                             sizeof(int) * (size_t)N,           sizeof(int) * ((size_t)N + 1),
                             sizeof(int) * (size_t)nnz,         sizeof(T) * (size_t)nnz,
                             sizeof(T) * (size_t)N,             sizeof(int) * 4,
                             sizeof(int) * ((size_t)N + 2)};
    size_t total = 0;
    for (size_t b : sizes) total += align256(b);
    void* slab = nullptr;
    cudaError_t e = cudaMalloc(&slab, total);
    if (e != cudaSuccess) return cuda_status(e, "sb_spts_analyze: cudaMalloc");
    p->owned.push_back(slab);
    char* q = (char*)slab;
    void* part[9];
    for (int k = 0; k < 9; ++k) {
      part[k] = q;
      q += align256(sizes[k]);
    }
    p->level = (int*)part[0];
    p->perm = (int*)part[1];
    p->order = (int*)part[2];
    p->rrow = (int*)part[3];
    p->rcol = (int*)part[4];
    p->rval = part[5];
    p->ywork = part[6];
    p->ticket = (int*)part[7];
    p->level_ptr = (int*)part[8];
    SB_CHECK_CUDA(cudaEventCreate(&p->ev[0]));
    SB_CHECK_CUDA(cudaEventCreate(&p->ev[1]));
  }
  int* status = device_status_word();
  if (!status) {
    set_error("sb_spts_analyze: device status word unavailable");
    return SB_ENOMEM;
  }
  SB_CHECK_CUDA(cudaEventRecord(p->ev[0], st));
  int* tmp = nullptr;  // [0] lower-check flag, [1] max level
  if ((r = scratch_alloc((void**)&tmp, 4 * sizeof(int), st))) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(tmp, 0, 4 * sizeof(int), st));
  lower_check<<<grid1(N), kT, 0, st>>>(p->row_ptr, p->col, N, tmp);
  SB_CHECK_LAUNCH("lower_check");
  SB_CHECK_CUDA(cudaMemsetAsync(p->level, 0xff, sizeof(int) * N, st));
  SB_CHECK_CUDA(cudaMemsetAsync(p->ticket, 0, sizeof(int), st));
  level_kernel<<<natural_order_grid((const void*)level_kernel), kT, 0, st>>>(
      p->row_ptr, p->col, N, p->level, p->ticket, kDefaultSpin, status);
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
    e = cudaEventRecord(p->ev[1], st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->h_level_ptr.data(), p->level_ptr, sizeof(int) * ((size_t)L + 1),
                          cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&p->analysis_ms, p->ev[0], p->ev[1]);
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
  T* yw = (T*)p->ywork;
  if (algo == SB_SPTS_SYNCFREE || algo == SB_SPTS_HYBRID) {
    SB_CHECK_CUDA(cudaMemsetAsync(yw, 0xff, sizeof(T) * N, st));
    SB_CHECK_CUDA(cudaMemsetAsync(p->ticket, 0, sizeof(int), st));
    if (algo == SB_SPTS_SYNCFREE) {
      auto k = spts_syncfree_plan_rows<T, A>;
      k<<<polling_grid((const void*)k, algo, N, p->nlevels), kT, 0, st>>>(
          p->row_ptr, p->col, (const T*)p->val, N, b, yw, y, p->ticket, limit, status);
      SB_CHECK_LAUNCH("spts_syncfree_plan_rows");
    } else {
      auto k = spts_hybrid_rows<T, A>;
      k<<<polling_grid((const void*)k, algo, N, p->nlevels), kT, 0, st>>>(
          p->rrow, p->rcol, (const T*)p->rval, N, p->perm, b, yw, y, p->ticket, limit, status);
      SB_CHECK_LAUNCH("spts_hybrid_rows");
    }
    return SB_OK;
  }
  {
    // one cooperative launch: a single block of kLevelBlock1 threads when
    // every level fits in it (no grid barrier), else blocks of kT threads for
    // the widest level, at most one per SM (fewer blocks make each barrier
    // cheaper), all of them resident
    int widest = 0;
    for (int l = 0; l < p->nlevels; ++l)
      widest = std::max(widest, p->h_level_ptr[l + 1] - p->h_level_ptr[l]);
    const int threads = widest <= kLevelBlock1 ? kLevelBlock1 : kT;
    // the two-round prefetch except for the one-block FP32 form, where the
    // one-round form measured faster (1M-row random factor, 3470 levels:
    // 6.54 against 7.27 ms; FP64 10.2 -> 9.40 ms and every grid form
    // faster with two rounds)
    const bool two = !(threads == kLevelBlock1 && sizeof(T) == 4 && sizeof(A) == 4);
    auto k = two ? spts_level_coop<T, A, true> : spts_level_coop<T, A, false>;
    int per = 0, coop = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k, threads, 0);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, p->device);
    const int blocks =
        threads == kLevelBlock1
            ? std::min(1, per * sm_count())
            : std::min(std::min((widest + kT - 1) / kT, sm_count()), std::max(per, 0) * sm_count());
    if (coop && blocks >= 1) {
      unsigned* bar = (unsigned*)(p->ticket + 2);
      SB_CHECK_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st));
      const int* rrow = p->rrow;
      const int* rcol = p->rcol;
      const T* rval = (const T*)p->rval;
      const int* lptr = p->level_ptr;
      int nl = p->nlevels;
      const int* perm = p->perm;
      void* args[] = {(void*)&rrow, (void*)&rcol, (void*)&rval, (void*)&lptr, (void*)&nl,
                      (void*)&perm, (void*)&b,    (void*)&yw,   (void*)&y,    (void*)&bar,
                      (void*)&limit, (void*)&status};
      SB_CHECK_CUDA(
          cudaLaunchCooperativeKernel((const void*)k, dim3(blocks), dim3(threads), args, 0, st));
      return SB_OK;
    }
  }
  for (int l = 0; l < p->nlevels; ++l) {
    const int r0 = p->h_level_ptr[l], r1 = p->h_level_ptr[l + 1];
    if (r1 <= r0) continue;
    spts_level_rows<T, A><<<grid1(r1 - r0), kT, 0, st>>>(p->rrow, p->rcol, (const T*)p->rval,
                                                         r0, r1, p->perm, b, yw);
    SB_CHECK_LAUNCH("spts_level_rows");
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

struct sb_spts_batch {
  int dtype = 0;
  int policy = 0;
  int capacity = 0;
  int device = 0;
  SptsDesc* h_items = nullptr;   // pinned staging of the descriptors...
  SptsSched* h_sched = nullptr;  // ...the schedule header...
  int* h_order = nullptr;        // ...systems by chunk count...
  long long* h_seg = nullptr;    // ...and segment starts (capacity + 1)
  SptsDesc* d_items = nullptr;
  SptsSched* d_sched = nullptr;
  int* d_order = nullptr;
  long long* d_seg = nullptr;
  int* d_tickets = nullptr;      // one chunk counter per item
  unsigned long long* d_work = nullptr;  // warp-slot counter of the capped grid
  int persistent = 0;            // capped grid: blocks per SM (0 = one warp per slot)
  cudaGraph_t graph_def = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaGraphNode_t solve_node = nullptr;
  cudaKernelNodeParams solve_params = {};
  void* solve_args[9] = {};
  long long limit = 0;
  int* status = nullptr;
  cudaStream_t capture_stream = nullptr;
  cudaEvent_t done = nullptr;
  bool pending = false;
  int full_per_sm = 1;     // resident blocks per SM of the solve kernel without a cap
  int smem_per_sm = 0;     // shared memory of an SM, bytes
  int smem_reserved = 0;   // shared memory the runtime reserves per block
  int smem_optin = 0;      // largest dynamic shared memory a block may request
};

static void spts_batch_release(sb_spts_batch* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->graph_def) cudaGraphDestroy(e->graph_def);
  if (e->capture_stream) cudaStreamDestroy(e->capture_stream);
  if (e->done) cudaEventDestroy(e->done);
  for (void* h : {(void*)e->h_items, (void*)e->h_sched, (void*)e->h_order, (void*)e->h_seg})
    if (h) cudaFreeHost(h);
  for (void* d : {(void*)e->d_items, (void*)e->d_sched, (void*)e->d_order, (void*)e->d_seg,
                  (void*)e->d_tickets, (void*)e->d_work})
    if (d) cudaFree(d);
  delete e;
}

static const void* spts_batch_kernel_for(int dtype, int policy) {
  if (dtype == SB_F64) return (const void*)spts_batch_kernel<double, double>;
  if (policy == SB_SPTS_ACC_F64) return (const void*)spts_batch_kernel<float, double>;
  return (const void*)spts_batch_kernel<float, float>;
}

extern "C" {

int sb_spts_plan_growth(const sb_spts_plan* plan, double* growth, void* stream) {
  SB_TRACE("sb_spts_plan_growth");
  SB_REQUIRE(plan && growth, "sb_spts_plan_growth: null argument");
  *growth = 0.0;
  if (plan->N == 0) return SB_OK;
  cudaStream_t st = as_stream(stream);
  unsigned long long* d = nullptr;
  int r = scratch_alloc((void**)&d, sizeof(unsigned long long), st);
  if (r) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), st));
  const unsigned g = std::min<unsigned>(grid1(plan->N), (unsigned)sm_count() * 8);
  if (plan->dtype == SB_F64)
    growth_kernel<double><<<g, kT, 0, st>>>(plan->row_ptr, (const double*)plan->val, plan->N, d);
  else
    growth_kernel<float><<<g, kT, 0, st>>>(plan->row_ptr, (const float*)plan->val, plan->N, d);
  SB_CHECK_LAUNCH("growth_kernel");
  unsigned long long h = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(d, st);
  double v;
  memcpy(&v, &h, sizeof(v));
  *growth = v;
  return SB_OK;
}

int sb_spts_batch_create(int dtype, int policy, int32_t capacity, sb_spts_batch** out) {
  SB_TRACE("sb_spts_batch_create");
  SB_REQUIRE(out, "sb_spts_batch_create: null output");
  *out = nullptr;
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_spts_batch_create: dtype must be F32 or F64");
  SB_REQUIRE(policy == SB_SPTS_ACC_NATIVE || policy == SB_SPTS_ACC_F64,
             "sb_spts_batch_create: bad accumulation policy");
  SB_REQUIRE(capacity > 0, "sb_spts_batch_create: capacity must be positive");
  int r = ensure_device();
  if (r) return r;
  int* status = device_status_word();
  if (!status) {
    set_error("sb_spts_batch_create: device status word unavailable");
    return SB_ENOMEM;
  }
  sb_spts_batch* e = new sb_spts_batch();
  e->dtype = dtype;
  e->policy = dtype == SB_F64 ? SB_SPTS_ACC_F64 : policy;
  e->capacity = capacity;
  cudaGetDevice(&e->device);
  cudaError_t ce = cudaSuccess;
#define SB_E(call)                    \
  if ((ce = (call)) != cudaSuccess) { \
    r = cuda_status(ce, #call);       \
    spts_batch_release(e);            \
    return r;                         \
  }
  SB_E(cudaMallocHost(&e->h_items, sizeof(SptsDesc) * capacity));
  SB_E(cudaMallocHost(&e->h_sched, sizeof(SptsSched)));
  SB_E(cudaMallocHost(&e->h_order, sizeof(int) * capacity));
  SB_E(cudaMallocHost(&e->h_seg, sizeof(long long) * (capacity + 1)));
  SB_E(cudaMalloc(&e->d_items, sizeof(SptsDesc) * capacity));
  SB_E(cudaMalloc(&e->d_sched, sizeof(SptsSched)));
  SB_E(cudaMalloc(&e->d_order, sizeof(int) * capacity));
  SB_E(cudaMalloc(&e->d_seg, sizeof(long long) * (capacity + 1)));
  SB_E(cudaMalloc(&e->d_tickets, sizeof(int) * capacity));
  SB_E(cudaMalloc(&e->d_work, sizeof(unsigned long long)));
  SB_E(cudaStreamCreateWithFlags(&e->capture_stream, cudaStreamNonBlocking));
  SB_E(cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming));
  e->h_sched->M = 0;
  e->h_sched->warps = 0;
  e->limit = kDefaultSpin;
  e->status = status;
  // graph: descriptors and schedule (host -> device), tickets to 0, work
  // vectors to pending, the solve (its grid is set per run)
  SB_E(cudaStreamBeginCapture(e->capture_stream, cudaStreamCaptureModeThreadLocal));
  const cudaStream_t cs = e->capture_stream;
  cudaMemcpyAsync(e->d_items, e->h_items, sizeof(SptsDesc) * capacity, cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(e->d_sched, e->h_sched, sizeof(SptsSched), cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(e->d_order, e->h_order, sizeof(int) * capacity, cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(e->d_seg, e->h_seg, sizeof(long long) * (capacity + 1), cudaMemcpyHostToDevice,
                  cs);
  cudaMemsetAsync(e->d_tickets, 0, sizeof(int) * capacity, cs);
  cudaMemsetAsync(e->d_work, 0, sizeof(unsigned long long), cs);
  {
    const void* reset = dtype == SB_F64 ? (const void*)spts_batch_reset<double>
                                        : (const void*)spts_batch_reset<float>;
    void* rargs[] = {(void*)&e->d_items, (void*)&e->d_sched};
    cudaLaunchKernel(reset, dim3(sm_count() * 4), dim3(kT), rargs, 0, cs);
  }
  e->solve_args[0] = (void*)&e->d_items;
  e->solve_args[1] = (void*)&e->d_sched;
  e->solve_args[2] = (void*)&e->d_order;
  e->solve_args[3] = (void*)&e->d_seg;
  e->solve_args[4] = (void*)&e->d_tickets;
  e->solve_args[5] = (void*)&e->limit;
  e->solve_args[6] = (void*)&e->status;
  e->solve_args[7] = (void*)&e->d_work;
  e->solve_args[8] = (void*)&e->persistent;
  const void* kern = spts_batch_kernel_for(dtype, e->policy);
  cudaLaunchKernel(kern, dim3(1), dim3(kTB), e->solve_args, 0, cs);
  SB_E(cudaStreamEndCapture(cs, &e->graph_def));
  {
    size_t nn = 0;
    SB_E(cudaGraphGetNodes(e->graph_def, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    SB_E(cudaGraphGetNodes(e->graph_def, nodes.data(), &nn));
    for (cudaGraphNode_t nd : nodes) {
      cudaGraphNodeType ty;
      SB_E(cudaGraphNodeGetType(nd, &ty));
      if (ty != cudaGraphNodeTypeKernel) continue;
      cudaKernelNodeParams kp = {};
      SB_E(cudaGraphKernelNodeGetParams(nd, &kp));
      if (kp.func == kern) {
        e->solve_node = nd;
        e->solve_params = kp;
      }
    }
    if (!e->solve_node) {
      set_error("sb_spts_batch_create: solve node not found in the captured graph");
      spts_batch_release(e);
      return SB_ECUDA;
    }
    e->solve_params.kernelParams = e->solve_args;
    e->solve_params.extra = nullptr;
  }
  SB_E(cudaGraphInstantiate(&e->graph, e->graph_def, 0));
  // residency cap of the solve (see sb_spts_batch_run): dynamic shared memory
  // that no solve uses, requested only to limit the blocks per SM
  SB_E(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e->full_per_sm, kern, kTB, 0));
  e->full_per_sm = std::max(1, e->full_per_sm);
  SB_E(cudaDeviceGetAttribute(&e->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                              e->device));
  SB_E(cudaDeviceGetAttribute(&e->smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock,
                              e->device));
  SB_E(cudaDeviceGetAttribute(&e->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                              e->device));
  SB_E(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem_optin));
#undef SB_E
  *out = e;
  return SB_OK;
}

int sb_spts_batch_set_grid(sb_spts_batch* e, int32_t blocks_per_sm) {
  SB_TRACE("sb_spts_batch_set_grid");
  SB_REQUIRE(e, "sb_spts_batch_set_grid: null executor");
  SB_REQUIRE(blocks_per_sm >= 0, "sb_spts_batch_set_grid: negative block count");
  if (e->pending) SB_CHECK_CUDA(cudaEventSynchronize(e->done));
  e->persistent = blocks_per_sm;
  return SB_OK;
}

int sb_spts_batch_destroy(sb_spts_batch* e) {
  SB_TRACE("sb_spts_batch_destroy");
  if (!e) return SB_OK;
  if (e->pending) cudaEventSynchronize(e->done);
  spts_batch_release(e);
  return SB_OK;
}

int sb_spts_batch_run(sb_spts_batch* e, const sb_spts_batch_item* items, int32_t n,
                      void* stream) {
  SB_TRACE("sb_spts_batch_run");
  SB_REQUIRE(e, "sb_spts_batch_run: null executor");
  SB_REQUIRE(n >= 0 && n <= e->capacity, "sb_spts_batch_run: %d items exceed capacity %d", n,
             e->capacity);
  SB_REQUIRE(n == 0 || items, "sb_spts_batch_run: null items");
  for (int i = 0; i < n; ++i) {
    const sb_spts_plan* p = items[i].plan;
    SB_REQUIRE(p, "sb_spts_batch_run: item %d: null plan", i);
    SB_REQUIRE(p->dtype == e->dtype, "sb_spts_batch_run: item %d: plan dtype differs", i);
    SB_REQUIRE(p->device == e->device, "sb_spts_batch_run: item %d: plan on another device", i);
    SB_REQUIRE(p->N == 0 || (items[i].b && items[i].y), "sb_spts_batch_run: item %d: null vector",
               i);
    if (p->N > 0 && !p->solvable) {
      set_error("sb_spts_batch_run: item %d: matrix is not lower triangular with its diagonal "
                "stored last", i);
      return SB_EINVAL;
    }
    const size_t vs = p->dtype == SB_F64 ? 8 : 4;
    SB_REQUIRE(reinterpret_cast<uintptr_t>(items[i].work) % vs == 0,
               "sb_spts_batch_run: item %d: work vector not aligned to the value size", i);
  }
  {
    // a plan's own work vector serves one solve per run
    std::vector<const sb_spts_plan*> ps;
    for (int i = 0; i < n; ++i)
      if (!items[i].work) ps.push_back(items[i].plan);
    std::sort(ps.begin(), ps.end());
    for (size_t i = 1; i < ps.size(); ++i)
      SB_REQUIRE(ps[i] != ps[i - 1],
                 "sb_spts_batch_run: a plan appears twice in one batch with its own work vector");
  }
  // the pinned staging buffers are read by the previous run's first nodes
  if (e->pending) SB_CHECK_CUDA(cudaEventSynchronize(e->done));
  cudaStream_t st = as_stream(stream);
  std::vector<std::pair<int, int>> by_chunks(n);
  for (int i = 0; i < n; ++i) {
    sb_spts_plan* p = items[i].plan;
    SptsDesc& d = e->h_items[i];
    d.rrow = p->rrow;
    d.rcol = p->rcol;
    d.rval = p->rval;
    d.perm = p->perm;
    d.yw = items[i].work ? items[i].work : p->ywork;
    d.b = items[i].b;
    d.y = items[i].y;
    d.N = p->N;
    d.pad = 0;
    by_chunks[i] = {(p->N + 31) / 32, i};
  }
  std::sort(by_chunks.begin(), by_chunks.end());
  long long warps = 0;
  int prev = 0;
  for (int k = 0; k < n; ++k) {
    e->h_order[k] = by_chunks[k].second;
    e->h_seg[k] = warps;
    warps += (long long)(by_chunks[k].first - prev) * (n - k);
    prev = by_chunks[k].first;
  }
  e->h_seg[n] = warps;
  e->h_sched->M = n;
  e->h_sched->warps = warps;
  const long long per_block = kTB / 32;
  long long blocks = std::max(1LL, (warps + per_block - 1) / per_block);
  if (e->persistent > 0)
    blocks = std::min(blocks, (long long)std::min(e->persistent, e->full_per_sm) * sm_count());
  SB_REQUIRE(blocks <= 0x7fffffffLL, "sb_spts_batch_run: batch too large");
  e->solve_params.gridDim = dim3((unsigned)blocks);
  // Resident blocks per SM: one per 8 systems, up to the occupancy limit.
  // Every resident warp that holds rows ahead of its system's frontier
  // polls, so a batch of few systems runs faster with few blocks per SM and
  // a batch of many with all of them (measured on B200: one 100k-row factor
  // 0.95 -> 0.52 ms at one block per SM, 64 of them 0.83 ms at full
  // occupancy and 1.73 ms at one block per SM).  The cap is dynamic shared
  // memory that the solve does not use, rounded down to whole KiB, kept only
  // where the occupancy query confirms at least one block still fits.
  unsigned smem = 0;
  const int bps = std::min(e->full_per_sm, std::max(1, (n + 7) / 8));
  if (e->persistent == 0 && bps < e->full_per_sm && e->smem_per_sm > 0) {
    long long want = (long long)e->smem_per_sm / bps - e->smem_reserved;
    want = std::min<long long>(want, e->smem_optin) / 1024 * 1024;
    int fit = 0;
    if (want > 0 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                        &fit, e->solve_params.func, kTB, (size_t)want) == cudaSuccess &&
        fit >= 1)
      smem = (unsigned)want;
  }
  e->solve_params.sharedMemBytes = smem;
  SB_CHECK_CUDA(cudaGraphExecKernelNodeSetParams(e->graph, e->solve_node, &e->solve_params));
  SB_CHECK_CUDA(cudaGraphLaunch(e->graph, st));
  SB_CHECK_CUDA(cudaEventRecord(e->done, st));
  e->pending = true;
  return SB_OK;
}


int sb_spts_syncfree_csr_noalloc(int dtype, const int32_t* row_ptr, const int32_t* col,
                                 const void* val, int32_t N, const void* b, void* y,
                                 int64_t spin_limit_cycles, void* stream) {
  SB_TRACE("sb_spts_syncfree_csr_noalloc");
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
    k<<<natural_order_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const double*)val, N,
                                                          (const double*)b, (double*)y, flags,
                                                          ticket, limit, status);
  } else {
    auto k = spts_syncfree_rows<float, float>;
    k<<<natural_order_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const float*)val, N,
                                                          (const float*)b, (float*)y, flags,
                                                          ticket, limit, status);
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
  SB_TRACE("sb_spts_analyze");
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
  SB_TRACE("sb_spts_plan_destroy");
  if (!plan) return SB_OK;
  cudaDeviceSynchronize();
  plan_release(plan);
  delete plan;
  return SB_OK;
}

int sb_spts_plan_info(const sb_spts_plan* plan, int32_t* nlevels, int32_t* solvable) {
  SB_TRACE("sb_spts_plan_info");
  SB_REQUIRE(plan && nlevels && solvable, "sb_spts_plan_info: null argument");
  *nlevels = plan->nlevels;
  *solvable = plan->solvable;
  return SB_OK;
}

int sb_spts_plan_analysis_ms(const sb_spts_plan* plan, float* ms) {
  SB_TRACE("sb_spts_plan_analysis_ms");
  SB_REQUIRE(plan && ms, "sb_spts_plan_analysis_ms: null argument");
  *ms = plan->analysis_ms;
  return SB_OK;
}

int sb_spts_plan_levels(const sb_spts_plan* plan, int32_t* level, int32_t* level_ptr,
                        int32_t* permutation, int32_t* order, void* stream) {
  SB_TRACE("sb_spts_plan_levels");
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
  SB_TRACE("sb_spts_plan_reordered");
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
  SB_TRACE("sb_spts_solve");
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
  SB_TRACE("sb_spts_syncfree_csr");
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
    k<<<natural_order_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const double*)val, N,
                                                     (const double*)b, (double*)y, flags, ticket,
                                                     limit, status);
  } else {
    auto k = spts_syncfree_rows<float, float>;
    k<<<natural_order_grid((const void*)k), kT, 0, st>>>(row_ptr, col, (const float*)val, N,
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

int sb_spts_csc(int dtype, const int32_t* col_ptr, const int32_t* row, const void* val,
                int32_t N, int64_t nnz, const void* x, void* y, void* stream) {
  SB_TRACE("sb_spts_csc");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_spts_csc: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_spts_csc: bad size");
  if (N == 0) return SB_OK;
  SB_REQUIRE(col_ptr && row && val && x && y, "sb_spts_csc: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  const size_t vb = dtype_size(dtype);
  void* mem = nullptr;
  // [flag] [CSR row_ptr N+1] [CSR col nnz] [CSR val nnz]
  const size_t off_rp = 16, off_col = off_rp + sizeof(int) * ((size_t)N + 1);
  const size_t off_val = (off_col + sizeof(int) * (size_t)nnz + 15) / 16 * 16;
  if ((r = scratch_alloc(&mem, off_val + vb * (size_t)nnz, st))) return r;
  char* p = (char*)mem;
  int* flag = (int*)p;
  int* rp = (int*)(p + off_rp);
  int* col = (int*)(p + off_col);
  void* cval = p + off_val;
  SB_CHECK_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
  csc_lower_check<<<grid1(N), kT, 0, st>>>(col_ptr, row, N, flag);
  SB_CHECK_LAUNCH("csc_lower_check");
  int h = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  if (h) {
    scratch_free(mem, st);
    set_error("sb_spts_csc: every column must start with its diagonal, the other rows below it");
    return SB_EINVAL;
  }
  // the CSC arrays are the CSR of L^T; its transpose is L in CSR with each
  // row's entries in increasing column order (diagonal last)
  r = sb_transpose_csr(dtype, col_ptr, row, val, N, nnz, rp, col, cval, stream);
  if (!r) r = sb_spts_syncfree_csr(dtype, rp, col, cval, N, x, y, 0, stream);
  scratch_free(mem, st);
  return r;
}

}  // extern "C"
