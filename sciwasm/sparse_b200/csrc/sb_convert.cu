// sb_convert.cu -- format conversions on the device, bit-exact with the
// reference's JavaScript loops:
//   coo_csr   src/sequential/src/sparse32.js:1674-1720 (+ sort :1612-1627)
//   num_cols  :1436-1447 and csr_ell :1449-1484
//   num_diags :1486-1512 and csr_dia :1515-1574
// coo_csr's per-row stable bubble sort makes the result a stable sort of the
// COO entries by (row, col).  Sorted input (the reference's mmread always
// quick-sorts by (row, col)) is detected and takes a copy-speed path; other
// input goes into row buckets whose rows are each sorted by (col, original
// position) when no row holds more than 2048 entries, and is otherwise
// ordered by a stable LSD radix sort of packed (row, col) keys whose payload
// is the original position; either way equal keys keep their COO order.
#include <algorithm>

#include <climits>

#include "sb_common.cuh"
#include "sb_prims.cuh"

namespace sb {

constexpr int kThreads = 256;

static unsigned grid_for(long long n, int per = kThreads) {
  long long g = (n + per - 1) / per;
  if (g < 1) g = 1;
  if (g > 0x7fffffffLL) g = 0x7fffffffLL;
  return (unsigned)g;
}

// flags[0] |= 1: index out of range; flags[1] |= 1: not sorted by (row, col).
// Each thread checks kCheckItems entries (strided by the block size, so every
// load is coalesced) and a block stores its findings once, and only while the
// flag still reads 0: in a shuffled COO nearly every entry is out of order,
// and one store per entry to the same word serialised (0.79 ms for 44M
// entries).
constexpr int kCheckItems = 8;

__global__ void coo_check(const int* __restrict__ row, const int* __restrict__ col, long long nnz,
                          int N, int* __restrict__ flags) {
  const long long base = (long long)blockIdx.x * blockDim.x * kCheckItems + threadIdx.x;
  int bad = 0, unsorted = 0;
#pragma unroll
  for (int u = 0; u < kCheckItems; ++u) {
    const long long i = base + (long long)u * blockDim.x;
    if (i < nnz) {
      const int r = row[i], c = col[i];
      bad |= (r < 0 || r >= N || c < 0 || c >= N);
      if (i + 1 < nnz) {
        const int r1 = row[i + 1], c1 = col[i + 1];
        unsorted |= (r1 < r || (r1 == r && c1 < c));
      }
    }
  }
  bad = __syncthreads_or(bad);
  unsorted = __syncthreads_or(unsorted);
  if (threadIdx.x == 0) {
    if (bad && __ldcg(flags) == 0) flags[0] = 1;
    if (unsorted && __ldcg(flags + 1) == 0) flags[1] = 1;
  }
}

__global__ void pack_keys(const int* __restrict__ row, const int* __restrict__ col,
                          long long nnz, unsigned long long* __restrict__ keys,
                          unsigned* __restrict__ idx) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  keys[i] = ((unsigned long long)(unsigned)row[i] << 32) | (unsigned)col[i];
  idx[i] = (unsigned)i;
}

template <typename T>
__global__ void unpack_sorted(const unsigned long long* __restrict__ keys,
                              const unsigned* __restrict__ idx, const T* __restrict__ val,
                              long long nnz, int* __restrict__ row_out, int* __restrict__ col_out,
                              T* __restrict__ val_out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  const unsigned long long k = keys[i];
  row_out[i] = (int)(k >> 32);
  col_out[i] = (int)(k & 0xffffffffu);
  val_out[i] = val[idx[i]];
}

// max row length (num_cols)
__global__ void max_row_len(const int* __restrict__ row_ptr, int N, int* __restrict__ out) {
  __shared__ int sm[32];
  int m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    m = max(m, row_ptr[i + 1] - row_ptr[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomicMax(out, m);
  }
}

// csr_ell: thread per row writes all nc slots of its row (entries in storage
// order, then zero padding with index 0), column-major slot k*N + i.
template <typename T>
__global__ void csr_to_ell(const int* __restrict__ row_ptr, const int* __restrict__ col,
                           const T* __restrict__ val, int N, int nc, int* __restrict__ indices,
                           T* __restrict__ data) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = row_ptr[i], e = row_ptr[i + 1];
  for (int k = 0; k < nc; ++k) {
    const long long o = (long long)k * N + i;
    const int j = s + k;
    if (j < e) {
      indices[o] = col[j];
      data[o] = val[j];
    } else {
      indices[o] = 0;
      data[o] = (T)0;
    }
  }
}

// Presence of diagonal c - i, stored at index N + c - i - 1 as in the
// reference (:1498); stores of 1 from several threads are benign.  Rows
// [r0, r1).  CHECK: a flag is stored only while it reads 0 (a stale 0 costs
// one more idempotent store).  Every row of a band marks the same few
// flags, and those repeated stores to a handful of addresses dominated a
// 4M-row band's conversion (csr_dia 1.17 -> 0.56 ms with the check); with
// random columns the check is a load round trip in front of every store
// (a 2M-row power-law num_diags 0.39 -> 0.90 ms), so it is used only where
// a prefix of the rows spans few diagonals.  SPAN: the prefix pass, which
// also reduces the smallest and largest N + c - i it marks into span[0]
// (min) and span[1] (max): one reduction per warp, no returning atomics.
template <bool CHECK, bool SPAN>
__global__ void mark_diagonals(const int* __restrict__ row_ptr, const int* __restrict__ col,
                               int N, int r0, int r1, int* __restrict__ ind,
                               unsigned* __restrict__ span) {
  const int i = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r1) return;
  unsigned lo = 0xffffffffu, hi = 0;
  for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
    const int c = col[j];
    if (c < 0 || c >= N) continue;
    const long long d = (long long)N + c - i - 1;
    int* f = ind + d;
    if (!CHECK || *f == 0) *f = 1;
    if (SPAN) {
      lo = min(lo, (unsigned)d);
      hi = max(hi, (unsigned)d);
    }
  }
  if (SPAN) {
    const unsigned m = __activemask();
    lo = __reduce_min_sync(m, lo);
    hi = __reduce_max_sync(m, hi);
    if ((threadIdx.x & 31) == __ffs(m) - 1) {
      atomicMin(span, lo);
      atomicMax(span + 1, hi);
    }
  }
}

// Compact the present diagonals: slot[d] = rank of d among present ones
// (from the exclusive scan), offset[slot] = d - (N - 1) ascending.
__global__ void compact_diagonals(const int* __restrict__ present, const int* __restrict__ rank,
                                  long long nd_all, int N, int* __restrict__ offset) {
  const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nd_all) return;
  if (present[d]) offset[rank[d]] = (int)(d - (N - 1));
}

// csr_dia fill for at most kDiaGather diagonals: thread per row; slot k of
// row i receives the row's LAST entry in column i + offset[k] (the
// reference's row-major loop, :1559-1571, lets a later duplicate overwrite
// an earlier one), else +0, so every slot is written exactly once with
// writes coalesced across rows, and no zero fill or scatter is needed.  Rows
// of up to kDiaRowRegs entries are held in registers.
constexpr int kDiaGather = 64;
constexpr int kDiaRowRegs = 16;

template <typename T>
__global__ void csr_to_dia_rows(const int* __restrict__ row_ptr, const int* __restrict__ col,
                                const T* __restrict__ val, int N, int nd,
                                const int* __restrict__ offset, T* __restrict__ data) {
  __shared__ int off_s[kDiaGather];
  for (int k = threadIdx.x; k < nd; k += blockDim.x) off_s[k] = offset[k];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = row_ptr[i], e = row_ptr[i + 1];
  if (e - s <= kDiaRowRegs) {
    int rel[kDiaRowRegs];
    T v[kDiaRowRegs];
#pragma unroll
    for (int u = 0; u < kDiaRowRegs; ++u) {
      const bool in = s + u < e;
      const int c = in ? col[s + u] : -1;
      // out-of-range columns are not stored (the reference skips them)
      rel[u] = (in && c >= 0 && c < N) ? c - i : INT_MIN;
      v[u] = in ? val[s + u] : T(0);
    }
    for (int k = 0; k < nd; ++k) {
      const int want = off_s[k];
      T out = T(0);
#pragma unroll
      for (int u = 0; u < kDiaRowRegs; ++u)
        if (rel[u] == want) out = v[u];
      data[(long long)k * N + i] = out;
    }
    return;
  }
  for (int k = 0; k < nd; ++k) {
    const int want = off_s[k];
    T out = T(0);
    for (int j = s; j < e; ++j) {
      const int c = col[j];
      if (c >= 0 && c < N && c - i == want) out = val[j];
    }
    data[(long long)k * N + i] = out;
  }
}

// csr_dia fill: thread per row, entries in storage order so a later
// duplicate (i, c) overwrites an earlier one exactly as the reference's
// row-major loop does (:1559-1571).  data is zero-filled beforehand.
template <typename T>
__global__ void csr_to_dia(const int* __restrict__ row_ptr, const int* __restrict__ col,
                           const T* __restrict__ val, int N, int stride,
                           const int* __restrict__ rank, T* __restrict__ data) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const long long move = (long long)N - stride;
  for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
    const int c = col[j];
    if (c < 0 || c >= N) continue;
    const int k = rank[(long long)N + c - i - 1];
    const long long o = (long long)k * stride + i - ((c - i) < 0 ? move : 0);
    data[o] = val[j];
  }
}

static int check_dt(int dtype, const char* fn) {
  if (dtype != SB_F32 && dtype != SB_F64) {
    set_error("%s: dtype %d not supported", fn, dtype);
    return SB_EINVAL;
  }
  return SB_OK;
}

// Host-side admission test of csr_ell / csr_dia, evaluated in doubles as in
// JavaScript: admit iff w*N < 2^27 and (w*N)/nnz <= 5 (0/0 is NaN: refused).
static bool admitted(long long w, long long N, long long nnz) {
  const double wn = (double)w * (double)N;
  const double ratio = wn / (double)nnz;
  return (wn < 134217728.0) && (ratio <= 5.0);
}

// ------------------------------------------------------------ coo_csr by row buckets
// Unsorted COO whose rows hold at most kBucketMaxRow entries: a counting sort
// by row (an atomic cursor per row hands every entry a slot of its row, in no
// particular order), then a sort of each row by the key (col << 32 | original
// position).  The position breaks ties between equal columns, so each row ends
// up in (col, COO order) -- the stable (row, col) order of the reference's
// per-row bubble sort -- whatever order the atomics handed out the slots in.
// One pass over the COO to count, one to scatter 16-byte items, one to sort
// and store: about 3.5 GB moved for 44M FP64 entries, against the six
// 8-bit digit passes of the general radix sort.

constexpr int kBucketMaxRow = 2048;   // longer rows: the radix sort
constexpr int kRowThreadMax = 16;     // rows up to this long: one thread, registers
constexpr int kRowRankMax = 64;       // up to this long: one warp, registers
constexpr int kRowWarpMax = 256;      // up to this long: one warp, shared memory
constexpr int kSortWarps = 8;         // warps per block of the warp-per-row kernel

struct BucketItem {
  unsigned long long key;   // col << 32 | position in the COO
  unsigned long long bits;  // the value's bits (FP32 in the low half)
};

__device__ __forceinline__ unsigned long long val_bits(float v) { return __float_as_uint(v); }
__device__ __forceinline__ unsigned long long val_bits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}
template <typename T> __device__ __forceinline__ T bits_val(unsigned long long b);
template <> __device__ __forceinline__ float bits_val<float>(unsigned long long b) {
  return __uint_as_float((unsigned)b);
}
template <> __device__ __forceinline__ double bits_val<double>(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

__global__ void count_rows(const int* __restrict__ row, long long nnz, int* __restrict__ cnt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nnz) atomicAdd(&cnt[row[i]], 1);
}

__global__ void max_count(const int* __restrict__ cnt, int N, int* __restrict__ out) {
  int m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    m = max(m, cnt[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}

template <typename T>
__global__ void scatter_rows(const int* __restrict__ row, const int* __restrict__ col,
                             const T* __restrict__ val, long long nnz, int* __restrict__ cursor,
                             BucketItem* __restrict__ items) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  const int pos = atomicAdd(&cursor[row[i]], 1);
  BucketItem it;
  it.key = ((unsigned long long)(unsigned)col[i] << 32) | (unsigned long long)i;
  it.bits = val_bits(val[i]);
  items[pos] = it;
}

template <typename T>
__device__ __forceinline__ void store_entry(int* col_out, T* val_out, long long p,
                                            unsigned long long key, unsigned long long bits) {
  col_out[p] = (int)(key >> 32);
  val_out[p] = bits_val<T>(bits);
}

// Bitonic sorting network over registers (n a power of two; indices are
// compile-time constants after unrolling, so the arrays stay in registers).
template <int n>
__device__ __forceinline__ void bitonic_regs(unsigned long long (&k)[n],
                                             unsigned long long (&b)[n]) {
#pragma unroll
  for (int size = 2; size <= n; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
      for (int i = 0; i < n; ++i) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const unsigned long long ki = k[i], kj = k[j], bi = b[i], bj = b[j];
          const bool sw = (ki > kj) == up;
          k[i] = sw ? kj : ki;
          k[j] = sw ? ki : kj;
          b[i] = sw ? bj : bi;
          b[j] = sw ? bi : bj;
        }
      }
    }
  }
}

// One thread per row: rows of up to kRowThreadMax entries are sorted in
// registers and stored; longer rows are listed for the kernels below, each
// list read only by the kernel that sorts its rows: up to kRowRankMax entries
// in lists[0], up to kRowWarpMax in lists[1], longer in lists[2] (counts in
// n_listed[0..2]).
template <typename T>
__global__ void sort_short_rows(const int* __restrict__ row_ptr, int N,
                                const BucketItem* __restrict__ items, int* __restrict__ col_out,
                                T* __restrict__ val_out, int* __restrict__ lists, int list_len,
                                int* __restrict__ n_listed) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int s = row_ptr[r], len = row_ptr[r + 1] - s;
  if (len == 0) return;
  if (len > kRowThreadMax) {
    // one counter add per list and warp (lanes bound for the same list share it)
    const int which = len <= kRowRankMax ? 0 : (len <= kRowWarpMax ? 1 : 2);
    const unsigned peers = __match_any_sync(__activemask(), which);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(n_listed + which, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    lists[(long long)which * list_len + base + __popc(peers & ((1u << lane) - 1u))] = r;
    return;
  }
  if (len == 1) {
    const BucketItem it = items[s];
    store_entry<T>(col_out, val_out, s, it.key, it.bits);
    return;
  }
  if (len <= 8) {
    unsigned long long k[8], b[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j < len) {
        const BucketItem it = items[s + j];
        k[j] = it.key;
        b[j] = it.bits;
      } else {
        k[j] = ~0ull;
        b[j] = 0;
      }
    }
    bitonic_regs<8>(k, b);
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (j < len) store_entry<T>(col_out, val_out, (long long)s + j, k[j], b[j]);
    return;
  }
  unsigned long long k[kRowThreadMax], b[kRowThreadMax];
#pragma unroll
  for (int j = 0; j < kRowThreadMax; ++j) {
    if (j < len) {
      const BucketItem it = items[s + j];
      k[j] = it.key;
      b[j] = it.bits;
    } else {
      k[j] = ~0ull;  // above every real key (columns are below 2^31)
      b[j] = 0;
    }
  }
  bitonic_regs<kRowThreadMax>(k, b);
#pragma unroll
  for (int j = 0; j < kRowThreadMax; ++j)
    if (j < len) store_entry<T>(col_out, val_out, (long long)s + j, k[j], b[j]);
}

// Bitonic sort of m (a power of two) keys with their bits in shared memory by
// `nt` cooperating threads numbered t; `sync` orders the steps.  A step's m/2
// compare-exchange pairs (i, i + stride), i with its stride bit clear, are
// disjoint; pair p is done by thread p mod nt, so no thread idles in a step.
struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

template <typename Sync>
__device__ __forceinline__ void bitonic_shared(unsigned long long* sk, unsigned long long* sb,
                                               int m, int t, int nt, Sync sync) {
  const int half = m >> 1;
  for (int size = 2; size <= m; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int p = t; p < half; p += nt) {
        const int i = ((p & ~(stride - 1)) << 1) | (p & (stride - 1));
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const unsigned long long ki = sk[i], kj = sk[j];
        if ((ki > kj) == up) {
          sk[i] = kj;
          sk[j] = ki;
          const unsigned long long bi = sb[i];
          sb[i] = sb[j];
          sb[j] = bi;
        }
      }
      sync();
    }
  }
}

// One warp per row of kRowThreadMax+1 .. kRowRankMax entries: each lane holds
// entries lane and lane + 32 in registers and counts, over all the row's keys
// broadcast by shuffles, how many are smaller; that count is the entry's slot
// (keys are distinct: they hold the position).  No shared memory, so every
// warp slot of an SM can hold a row in flight.
template <typename T>
__global__ void __launch_bounds__(256)
    sort_rank_rows(const int* __restrict__ row_ptr, const BucketItem* __restrict__ items,
                   const int* __restrict__ rows, const int* __restrict__ n_rows,
                   int* __restrict__ col_out, T* __restrict__ val_out) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const int n = *n_rows;
  for (int q = blockIdx.x * wpb + (threadIdx.x >> 5); q < n; q += gridDim.x * wpb) {
    const int r = rows[q];
    const int s = row_ptr[r], len = row_ptr[r + 1] - s;
    unsigned long long k0 = ~0ull, b0 = 0, k1 = ~0ull, b1 = 0;
    if (lane < len) {
      const BucketItem it = items[s + lane];
      k0 = it.key;
      b0 = it.bits;
    }
    if (lane + 32 < len) {
      const BucketItem it = items[s + 32 + lane];
      k1 = it.key;
      b1 = it.bits;
    }
    int r0 = 0, r1 = 0;
    if (len <= 32) {
      for (int j = 0; j < len; ++j) r0 += __shfl_sync(0xffffffffu, k0, j) < k0;
    } else {
#pragma unroll 4
      for (int j = 0; j < 32; ++j) {
        const unsigned long long a = __shfl_sync(0xffffffffu, k0, j);
        const unsigned long long c = __shfl_sync(0xffffffffu, k1, j);
        r0 += (a < k0) + (c < k0);
        r1 += (a < k1) + (c < k1);
      }
    }
    if (lane < len) store_entry<T>(col_out, val_out, (long long)s + r0, k0, b0);
    if (lane + 32 < len) store_entry<T>(col_out, val_out, (long long)s + r1, k1, b1);
  }
}

// One warp per row of kRowRankMax+1 .. kRowWarpMax entries: a bitonic sort in
// the warp's shared memory.
template <typename T>
__global__ void __launch_bounds__(kSortWarps * 32)
    sort_warp_rows(const int* __restrict__ row_ptr, const BucketItem* __restrict__ items,
                   const int* __restrict__ rows, const int* __restrict__ n_rows,
                   int* __restrict__ col_out, T* __restrict__ val_out) {
  __shared__ unsigned long long sk[kSortWarps][kRowWarpMax];
  __shared__ unsigned long long sb[kSortWarps][kRowWarpMax];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = *n_rows;
  for (int q = blockIdx.x * kSortWarps + warp; q < n; q += gridDim.x * kSortWarps) {
    const int r = rows[q];
    const int s = row_ptr[r], len = row_ptr[r + 1] - s;
    int m = 128;
    while (m < len) m <<= 1;
    for (int t = lane; t < m; t += 32) {
      if (t < len) {
        const BucketItem it = items[s + t];
        sk[warp][t] = it.key;
        sb[warp][t] = it.bits;
      } else {
        sk[warp][t] = ~0ull;
        sb[warp][t] = 0;
      }
    }
    __syncwarp();
    bitonic_shared(sk[warp], sb[warp], m, lane, 32, WarpSync());
    for (int t = lane; t < len; t += 32)
      store_entry<T>(col_out, val_out, (long long)s + t, sk[warp][t], sb[warp][t]);
    __syncwarp();
  }
}

// One block per listed row of kRowWarpMax+1 .. kBucketMaxRow entries.
constexpr int kBlockSortThreads = 512;

template <typename T>
__global__ void __launch_bounds__(kBlockSortThreads)
    sort_block_rows(const int* __restrict__ row_ptr, const BucketItem* __restrict__ items,
                    const int* __restrict__ long_rows, const int* __restrict__ n_long,
                    int* __restrict__ col_out, T* __restrict__ val_out) {
  __shared__ unsigned long long sk[kBucketMaxRow];
  __shared__ unsigned long long sb[kBucketMaxRow];
  const int n = *n_long;
  for (int q = blockIdx.x; q < n; q += gridDim.x) {
    const int r = long_rows[q];
    const int s = row_ptr[r], len = row_ptr[r + 1] - s;
    int m = 512;
    while (m < len) m <<= 1;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
      if (t < len) {
        const BucketItem it = items[s + t];
        sk[t] = it.key;
        sb[t] = it.bits;
      } else {
        sk[t] = ~0ull;
        sb[t] = 0;
      }
    }
    __syncthreads();
    bitonic_shared(sk, sb, m, threadIdx.x, blockDim.x, BlockSync());
    for (int t = threadIdx.x; t < len; t += blockDim.x)
      store_entry<T>(col_out, val_out, (long long)s + t, sk[t], sb[t]);
    __syncthreads();
  }
}

static int device_sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
    return 148;
  return n;
}

// Returns SB_OK, an error, or kBucketFallBack when a row is longer than
// kBucketMaxRow (nothing has been written then).
constexpr int kBucketFallBack = 1;

template <typename T>
static int coo_csr_buckets(const int* row, const int* col, const T* val, int N, long long nnz,
                           int* csr_row, int* csr_col, T* csr_val, cudaStream_t st) {
  // cnt[N + 1], lists[3][N] (rows for the rank, warp and block sorts),
  // misc[4] = {max row, rows listed for each of the three sorts}
  int* small = nullptr;
  const size_t small_ints = 4 * (size_t)N + 5;
  int r = scratch_alloc((void**)&small, sizeof(int) * small_ints, st);
  if (r) return r;
  int* cnt = small;
  int* lists = small + N + 1;
  int* misc = small + 4 * (size_t)N + 1;
  BucketItem* items = nullptr;
  const int sms = device_sm_count();
  cudaError_t e = cudaMemsetAsync(small, 0, sizeof(int) * small_ints, st);
  if (e == cudaSuccess) {
    count_rows<<<grid_for(nnz), kThreads, 0, st>>>(row, nnz, cnt);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    max_count<<<std::min<unsigned>(grid_for(N), 4u * sms), kThreads, 0, st>>>(cnt, N, misc);
    e = cudaGetLastError();
  }
  int maxlen = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&maxlen, misc, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) r = cuda_status(e, "coo_csr (row counts)");
  if (!r && maxlen > kBucketMaxRow) r = kBucketFallBack;
  if (!r) r = prim::exclusive_scan(cnt, csr_row, (long long)N + 1, st);  // cnt[N] = 0
  if (!r) r = scratch_alloc((void**)&items, sizeof(BucketItem) * (size_t)nnz, st);
  if (!r) {
    e = cudaMemcpyAsync(cnt, csr_row, sizeof(int) * (size_t)N, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) {
      scatter_rows<T><<<grid_for(nnz), kThreads, 0, st>>>(row, col, val, nnz, cnt, items);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      sort_short_rows<T><<<grid_for(N), kThreads, 0, st>>>(csr_row, N, items, csr_col, csr_val,
                                                           lists, N, misc + 1);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && maxlen > kRowThreadMax) {
      sort_rank_rows<T><<<8 * sms, 256, 0, st>>>(csr_row, items, lists, misc + 1, csr_col,
                                                 csr_val);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && maxlen > kRowRankMax) {
      sort_warp_rows<T><<<4 * sms, kSortWarps * 32, 0, st>>>(csr_row, items, lists + N, misc + 2,
                                                             csr_col, csr_val);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && maxlen > kRowWarpMax) {
      sort_block_rows<T><<<4 * sms, kBlockSortThreads, 0, st>>>(
          csr_row, items, lists + 2 * (size_t)N, misc + 3, csr_col, csr_val);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "coo_csr (row buckets)");
  }
  if (items) scratch_free(items, st);
  scratch_free(small, st);
  return r;
}

template <typename T>
static int coo_csr_impl(const int* row, const int* col, const T* val, int N, long long nnz,
                        int* csr_row, int* csr_col, T* csr_val, cudaStream_t st) {
  int* flags = nullptr;
  int r = scratch_alloc((void**)&flags, 2 * sizeof(int), st);
  if (r) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(int), st));
  coo_check<<<grid_for(nnz, kThreads * kCheckItems), kThreads, 0, st>>>(row, col, nnz, N, flags);
  SB_CHECK_LAUNCH("coo_check");
  int hf[2] = {0, 0};
  SB_CHECK_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(flags, st);
  if (hf[0]) {
    set_error("coo_csr: row or column index outside [0, N)");
    return SB_EINVAL;
  }
  if (!hf[1]) {
    // already in (row, col) order: the stable sort is the identity
    SB_CHECK_CUDA(cudaMemcpyAsync(csr_col, col, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, st));
    SB_CHECK_CUDA(cudaMemcpyAsync(csr_val, val, sizeof(T) * nnz, cudaMemcpyDeviceToDevice, st));
    prim::row_ptr_from_sorted<<<grid_for(nnz + 1), kThreads, 0, st>>>(row, nnz, N, csr_row);
    SB_CHECK_LAUNCH("row_ptr_from_sorted");
    return SB_OK;
  }
  // general order, rows of at most kBucketMaxRow entries: row buckets
  r = coo_csr_buckets<T>(row, col, val, N, nnz, csr_row, csr_col, csr_val, st);
  if (r != kBucketFallBack) return r;
  // longer rows: stable radix sort of (row << 32 | col) with positions
  prim::RadixBuffers b;
  void* mem = nullptr;
  const size_t kb = sizeof(unsigned long long) * (size_t)nnz, vb = sizeof(unsigned) * (size_t)nnz;
  r = scratch_alloc(&mem, 2 * kb + 2 * vb + sizeof(int) * (size_t)nnz, st);
  if (r) return r;
  char* p = (char*)mem;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* rows_sorted = (int*)(p + 2 * kb + 2 * vb);
  pack_keys<<<grid_for(nnz), kThreads, 0, st>>>(row, col, nnz, b.k[0], b.v[0]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "pack_keys");
  const int nb = prim::bits_for(N > 0 ? N - 1 : 0);
  const int ranges[4] = {0, nb, 32, 32 + nb};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, nnz, ranges, 2, &which, st);
  if (!r) {
    unpack_sorted<T><<<grid_for(nnz), kThreads, 0, st>>>(b.k[which], b.v[which], val, nnz,
                                                         rows_sorted, csr_col, csr_val);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "unpack_sorted");
  }
  if (!r) {
    prim::row_ptr_from_sorted<<<grid_for(nnz + 1), kThreads, 0, st>>>(rows_sorted, nnz, N, csr_row);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "row_ptr_from_sorted");
  }
  if (!r) {
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "coo_csr");
  }
  scratch_free(mem, st);
  return r;
}

constexpr int kDiaPrefixRows = 4096;   // rows of the counting prefix pass
constexpr int kDiaFewDiagonals = 64;   // prefix span below this many diagonals: check before storing

static int num_diags_impl(const int* row_ptr, const int* col, int N, int** present_out,
                          int** rank_out, int* nd, cudaStream_t st) {
  const long long nall = 2LL * N - 1;
  int* present = nullptr;
  int r = scratch_alloc((void**)&present, sizeof(int) * (size_t)(2 * nall + 2), st);
  if (r) return r;
  int* rank = present + nall;
  unsigned* span = reinterpret_cast<unsigned*>(rank + nall);  // the allocation's last 2 ints
  SB_CHECK_CUDA(cudaMemsetAsync(present, 0, sizeof(int) * (size_t)nall, st));
  SB_CHECK_CUDA(cudaMemsetAsync(span, 0xff, sizeof(unsigned), st));
  SB_CHECK_CUDA(cudaMemsetAsync(span + 1, 0, sizeof(unsigned), st));
  // a prefix of the rows, measuring the span of the diagonals it marks: a
  // narrow span (a band) makes the rest check before storing, a wide one
  // store plainly
  const int pre = std::min(N, kDiaPrefixRows);
  mark_diagonals<false, true><<<grid_for(pre), kThreads, 0, st>>>(row_ptr, col, N, 0, pre,
                                                                  present, span);
  SB_CHECK_LAUNCH("mark_diagonals");
  unsigned hs[2] = {0xffffffffu, 0};
  SB_CHECK_CUDA(cudaMemcpyAsync(hs, span, sizeof(hs), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  if (N > pre) {
    const bool narrow = hs[1] >= hs[0] && hs[1] - hs[0] < (unsigned)kDiaFewDiagonals;
    if (narrow)
      mark_diagonals<true, false><<<grid_for(N - pre), kThreads, 0, st>>>(row_ptr, col, N, pre, N,
                                                                        present, span);
    else
      mark_diagonals<false, false><<<grid_for(N - pre), kThreads, 0, st>>>(row_ptr, col, N, pre,
                                                                         N, present, span);
    SB_CHECK_LAUNCH("mark_diagonals");
  }
  r = prim::exclusive_scan(present, rank, nall, st);
  if (r) {
    scratch_free(present, st);
    return r;
  }
  int last[2] = {0, 0};
  SB_CHECK_CUDA(cudaMemcpyAsync(&last[0], present + nall - 1, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaMemcpyAsync(&last[1], rank + nall - 1, sizeof(int), cudaMemcpyDeviceToHost,
                                st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  *nd = last[0] + last[1];
  *present_out = present;
  *rank_out = rank;
  return SB_OK;
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_coo_csr(int dtype, const int32_t* row, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t* csr_row_ptr, int32_t* csr_col, void* csr_val,
               void* stream) {
  SB_TRACE("sb_coo_csr");
  int r = check_dt(dtype, "sb_coo_csr");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0, "sb_coo_csr: negative size");
  SB_REQUIRE(nnz <= 0x7fffffffLL, "sb_coo_csr: nnz exceeds int32 row_ptr range");
  SB_REQUIRE(csr_row_ptr, "sb_coo_csr: null row_ptr");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  if (nnz == 0) {
    SB_CHECK_CUDA(cudaMemsetAsync(csr_row_ptr, 0, sizeof(int) * ((size_t)N + 1), st));
    SB_CHECK_CUDA(cudaStreamSynchronize(st));
    return SB_OK;
  }
  SB_REQUIRE(row && col && val && csr_col && csr_val, "sb_coo_csr: null pointer");
  if (dtype == SB_F32)
    return coo_csr_impl<float>(row, col, (const float*)val, N, nnz, csr_row_ptr, csr_col,
                               (float*)csr_val, st);
  return coo_csr_impl<double>(row, col, (const double*)val, N, nnz, csr_row_ptr, csr_col,
                              (double*)csr_val, st);
}

int sb_num_cols(const int32_t* row_ptr, int32_t N, int32_t* nc, void* stream) {
  SB_TRACE("sb_num_cols");
  SB_REQUIRE(nc && N >= 0, "sb_num_cols: bad argument");
  *nc = 0;
  if (N == 0) return SB_OK;
  SB_REQUIRE(row_ptr, "sb_num_cols: null row_ptr");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  int* out = nullptr;
  if ((r = scratch_alloc((void**)&out, sizeof(int), st))) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(int), st));
  const unsigned g = std::min<unsigned>(grid_for(N), (unsigned)sm_count() * 8);
  max_row_len<<<g, kThreads, 0, st>>>(row_ptr, N, out);
  SB_CHECK_LAUNCH("max_row_len");
  SB_CHECK_CUDA(cudaMemcpyAsync(nc, out, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(out, st);
  return SB_OK;
}

int sb_ell_admitted(int64_t ncols, int32_t N, int64_t nnz) {
  return admitted(ncols, N, nnz) ? 1 : 0;
}

int sb_csr_ell(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t nc, int32_t* indices, void* data, void* stream) {
  SB_TRACE("sb_csr_ell");
  int r = check_dt(dtype, "sb_csr_ell");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && nc >= 0, "sb_csr_ell: negative size");
  if (!admitted(nc, N, nnz)) {
    set_error("csr_ell: not efficient to store this matrix in ELL (nc*N=%lld, nnz=%lld)",
              (long long)nc * N, (long long)nnz);
    return SB_EREFUSED;
  }
  SB_REQUIRE(row_ptr && indices && data && (nnz == 0 || (col && val)), "sb_csr_ell: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    csr_to_ell<float><<<grid_for(N), kThreads, 0, st>>>(row_ptr, col, (const float*)val, N, nc,
                                                        indices, (float*)data);
  else
    csr_to_ell<double><<<grid_for(N), kThreads, 0, st>>>(row_ptr, col, (const double*)val, N, nc,
                                                         indices, (double*)data);
  SB_CHECK_LAUNCH("csr_to_ell");
  return SB_OK;
}

int sb_num_diags(const int32_t* row_ptr, const int32_t* col, int32_t N, int32_t* nd,
                 int32_t* stride, void* stream) {
  SB_TRACE("sb_num_diags");
  SB_REQUIRE(nd && stride && N >= 0, "sb_num_diags: bad argument");
  *nd = 0;
  *stride = N;
  if (N == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col, "sb_num_diags: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  int *present = nullptr, *rank = nullptr;
  if ((r = num_diags_impl(row_ptr, col, N, &present, &rank, nd, st))) return r;
  scratch_free(present, st);
  return SB_OK;
}

int sb_dia_admitted(int64_t ndiags, int32_t stride, int64_t nnz) {
  return admitted(ndiags, stride, nnz) ? 1 : 0;
}

int sb_csr_dia(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t nd, int32_t stride, int32_t* offset, void* data,
               void* stream) {
  SB_TRACE("sb_csr_dia");
  int r = check_dt(dtype, "sb_csr_dia");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && nd >= 0, "sb_csr_dia: negative size");
  SB_REQUIRE(stride == N, "sb_csr_dia: stride must equal N (reference :1510)");
  if (!admitted(nd, stride, nnz)) {
    set_error("csr_dia: not efficient to store this matrix in DIA (nd*stride=%lld, nnz=%lld)",
              (long long)nd * stride, (long long)nnz);
    return SB_EREFUSED;
  }
  SB_REQUIRE(row_ptr && col && val && offset && data, "sb_csr_dia: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  int *present = nullptr, *rank = nullptr;
  int nd_found = 0;
  if ((r = num_diags_impl(row_ptr, col, N, &present, &rank, &nd_found, st))) return r;
  if (nd_found != nd) {
    scratch_free(present, st);
    set_error("sb_csr_dia: nd=%d does not match the matrix (%d diagonals)", nd, nd_found);
    return SB_EINVAL;
  }
  const long long nall = 2LL * N - 1;
  compact_diagonals<<<grid_for(nall), kThreads, 0, st>>>(present, rank, nall, N, offset);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && nd <= kDiaGather) {
    // gather: every slot written once (stride == N)
    if (dtype == SB_F32)
      csr_to_dia_rows<float><<<grid_for(N), kThreads, 0, st>>>(
          row_ptr, col, (const float*)val, N, nd, offset, (float*)data);
    else
      csr_to_dia_rows<double><<<grid_for(N), kThreads, 0, st>>>(
          row_ptr, col, (const double*)val, N, nd, offset, (double*)data);
    e = cudaGetLastError();
  } else if (e == cudaSuccess) {
    e = cudaMemsetAsync(data, 0, dtype_size(dtype) * (size_t)nd * (size_t)stride, st);
    if (e == cudaSuccess) {
      if (dtype == SB_F32)
        csr_to_dia<float><<<grid_for(N), kThreads, 0, st>>>(row_ptr, col, (const float*)val, N,
                                                            stride, rank, (float*)data);
      else
        csr_to_dia<double><<<grid_for(N), kThreads, 0, st>>>(row_ptr, col, (const double*)val, N,
                                                             stride, rank, (double*)data);
      e = cudaGetLastError();
    }
  }
  scratch_free(present, st);
  if (e != cudaSuccess) return cuda_status(e, "sb_csr_dia");
  return SB_OK;
}

int sb_coo_csc(int dtype, const int32_t* row, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t* csc_col_ptr, int32_t* csc_row, void* csc_val,
               void* stream) {
  SB_TRACE("sb_coo_csc");
  // coo_csc is coo_csr with the roles of rows and columns swapped
  return sb_coo_csr(dtype, col, row, val, N, nnz, csc_col_ptr, csc_row, csc_val, stream);
}

}  // extern "C"
