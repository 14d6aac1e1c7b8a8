// sb_batch.cu -- batched SpMV: many matrices (CSR, DIA or ELL) and
// right-hand sides in one persistent launch, replayed from a captured CUDA
// graph.
//
// No counterpart in the reference (it calls spmv once per matrix and vector,
// src/sequential/src/sparse32.js:1232-1286).  Work is a flat list of 32-row
// blocks over all matrices of the batch (block_offsets = exclusive scan of
// ceil(N_i/32)); persistent warps take four blocks at a time from a device
// counter, map a block index to its matrix by binary search, and reduce each
// short row with V lanes (V per matrix from its mean row length: the "rows
// per warp" autotuning) and each long row with the whole warp (compensated
// f32 sums); with several right-hand sides (x and y are N x nrhs, row-major,
// nrhs <= 8) the right-hand sides go across lanes instead, so that one load
// gathers all of a column's x values.  DIA and ELL items take one row per
// lane in the reference's per-row order (bit-identical to sb_spmv_dia /
// sb_spmv_ell).  Values are stored f32, f64 or BF16
// (f32 vectors and sums for f32/BF16).  The executor keeps descriptors
// in pinned host and device buffers; one run = the graph [copy descriptors,
// reset the counter, kernel] launched on the caller's stream.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "sb_common.cuh"

// One of the executor's two descriptor sets: runs alternate between them, so
// that a run does not wait for the previous one to finish before staging its
// descriptors (only for the run before that, which used the same set).
struct sb_batch_slot {
  sb_batch_item* h_items = nullptr;  // pinned
  long long* h_offsets = nullptr;    // pinned, capacity + 1
  int* h_count = nullptr;            // pinned: [0] = items in the current run
  sb_batch_item* d_items = nullptr;
  long long* d_offsets = nullptr;
  int* d_count = nullptr;            // [0] items, [2] work counter
  cudaGraphExec_t graph = nullptr;   // [descriptors, offsets, count up; kernel]
  cudaEvent_t done = nullptr;
  bool pending = false;
};

struct sb_batch_exec {
  int dtype = 0;
  int capacity = 0;
  int device = 0;
  int grid = 0;
  int next = 0;                      // the set the next run uses
  sb_batch_slot slot[2];
  cudaStream_t capture_stream = nullptr;
};

namespace sb {

constexpr int kBT = 256;
constexpr int kMaxRhs = 8;
constexpr int kBlocksPerTicket = 4;  // 32-row blocks a warp takes per work-counter update
constexpr int kLaneRows = 1 << 30;   // internal item flag: one row per lane (set by the run)
constexpr int kX32 = 1 << 29;        // internal item flag: x 32-byte aligned (set by the run)

__device__ __forceinline__ float ldv(const float* p, long long i) { return ld_reuse(p + i); }
__device__ __forceinline__ double ldv(const double* p, long long i) { return ld_reuse(p + i); }
__device__ __forceinline__ float ldv(const __nv_bfloat16* p, long long i) {
  return __bfloat162float(
      __ushort_as_bfloat16(ld_reuse(reinterpret_cast<const unsigned short*>(p) + i)));
}

// Neumaier-compensated accumulation (long rows with f32 sums).
template <typename T>
__device__ __forceinline__ void comp_add(T& s, T& c, T v) {
  const T t = s + v;
  c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
  s = t;
}

// y[row*K + j] for one finished row sum: y = A x (overwrite) or y += A x,
// where a row without entries keeps y unless it is overwritten with 0.
template <typename T>
__device__ __forceinline__ void put_y(T* y, long long at, T sum, bool overwrite, bool nonempty) {
  if (overwrite) y[at] = sum;
  else if (nonempty) y[at] += sum;
}

// One 32-row block of one matrix, V lanes per row, K right-hand sides: the
// block's row_ptr entries are read once (one per lane); rows of up to kLong
// entries are reduced in batches of 32/V rows, each lane issuing UNROLL
// independent col/val loads per pass before the x gathers (K consecutive
// values per column), then one shuffle reduction per right-hand side; longer
// rows are reduced by the whole warp, one right-hand side at a time, with
// compensated f32 sums.
constexpr int kLong = 128;

// Rows of a block longer than kLong: the whole warp per row, one right-hand
// side at a time, compensated f32 sums.
template <typename SV, typename T>
__device__ __forceinline__ void batch_long_rows(const sb_batch_item& it, int r0, int lane, int s_l,
                                                int e_l, int len_l) {
  constexpr int UNROLL = 4;
  constexpr bool COMP = sizeof(T) == 4;
  const int* __restrict__ col = it.col;
  const SV* __restrict__ val = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  T* __restrict__ y = (T*)it.y;
  const int K = it.nrhs;
  const int N = it.N;
  const bool overwrite = (it.flags & 1) != 0;
  const int rr = r0 + lane;
  unsigned longm = __ballot_sync(0xffffffffu, rr < N && len_l > kLong);
  while (longm) {
    const int j = __ffs(longm) - 1;
    longm &= longm - 1;
    const int s = __shfl_sync(0xffffffffu, s_l, j);
    const int e = __shfl_sync(0xffffffffu, e_l, j);
    for (int h = 0; h < K; ++h) {
      T sum = 0, comp = 0;
      for (int k0 = s; k0 < e; k0 += 32 * UNROLL) {
        int cc[UNROLL];
        T vv[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int k = k0 + lane + u * 32;
          cc[u] = k < e ? ld_reuse(col + k) : 0;
          vv[u] = k < e ? ldv(val, k) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int k = k0 + lane + u * 32;
          if (k < e) {
            const T p = vv[u] * __ldg(x + (long long)cc[u] * K + h);
            if (COMP) comp_add(sum, comp, p);
            else sum += p;
          }
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const T o = __shfl_xor_sync(0xffffffffu, sum, off);
        if (COMP) {
          comp += __shfl_xor_sync(0xffffffffu, comp, off);
          comp_add(sum, comp, o);
        } else {
          sum += o;
        }
      }
      if (lane == 0) put_y(y, (long long)(r0 + j) * K + h, COMP ? sum + comp : sum, overwrite, true);
    }
  }
}

template <typename SV, typename T, int V>
__device__ __forceinline__ void batch_block(const sb_batch_item& it, int r0, int lane) {
  constexpr int UNROLL = 4;
  constexpr int RPB = 32 / V;
  const int g = lane / V, q = lane - (lane / V) * V;
  const int* __restrict__ rp = it.row_ptr;
  const int* __restrict__ col = it.col;
  const SV* __restrict__ val = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  T* __restrict__ y = (T*)it.y;
  const int K = it.nrhs;
  const int N = it.N;
  const bool overwrite = (it.flags & 1) != 0;
  const int rr = r0 + lane;
  const int s_l = rr < N ? __ldg(rp + rr) : 0;
  const int e_l = rr < N ? __ldg(rp + rr + 1) : 0;
  const int len_l = e_l - s_l;
#pragma unroll
  for (int b = 0; b < V; ++b) {
    const int j = b * RPB + g;
    const int s = __shfl_sync(0xffffffffu, s_l, j);
    const int e = __shfl_sync(0xffffffffu, e_l, j);
    const int len = e - s;
    T acc[kMaxRhs];
#pragma unroll
    for (int h = 0; h < kMaxRhs; ++h) acc[h] = 0;
    if (len <= kLong) {
      for (int k0 = s + q; k0 < e; k0 += V * UNROLL) {
        int cc[UNROLL];
        T vv[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int k = k0 + u * V;
          cc[u] = k < e ? ld_reuse(col + k) : 0;
          vv[u] = k < e ? ldv(val, k) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          if (k0 + u * V < e) {
            const T* xc = x + (long long)cc[u] * K;
#pragma unroll
            for (int h = 0; h < kMaxRhs; ++h)
              if (h < K) acc[h] += vv[u] * __ldg(xc + h);
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < kMaxRhs; ++h) {
      if (h < K) {
        T a = acc[h];
#pragma unroll
        for (int off = V >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
        if (q == 0 && len <= kLong && r0 + j < N)
          put_y(y, (long long)(r0 + j) * K + h, a, overwrite, len > 0);
      }
    }
  }
  batch_long_rows<SV, T>(it, r0, lane, s_l, e_l, len_l);
}

// Several right-hand sides (K = 2..8): one 32-row block, the right-hand
// sides across lanes.  KP = K rounded up to a power of two lanes share a row,
// lane h of the group accumulating right-hand side h over the row's entries
// in storage order (UNROLL entries per pass), so one load instruction gathers
// the K consecutive x values of 32/KP columns (one L1 tag per nonzero instead
// of K) and the col/val loads of a row are shared by its KP lanes.  Rows
// longer than kLong go to the whole-warp path of batch_block.
template <typename SV, typename T, int KP>
__device__ __forceinline__ void batch_block_rhs(const sb_batch_item& it, int r0, int lane) {
  constexpr int UNROLL = 4;
  constexpr int R = 32 / KP;  // rows per pass
  constexpr bool COMP = sizeof(T) == 4;
  const int r = lane / KP, h = lane - (lane / KP) * KP;
  const int* __restrict__ rp = it.row_ptr;
  const int* __restrict__ col = it.col;
  const SV* __restrict__ val = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  T* __restrict__ y = (T*)it.y;
  const int K = it.nrhs;
  const int N = it.N;
  const bool overwrite = (it.flags & 1) != 0;
  const int rr = r0 + lane;
  const int s_l = rr < N ? __ldg(rp + rr) : 0;
  const int e_l = rr < N ? __ldg(rp + rr + 1) : 0;
  const int len_l = e_l - s_l;
#pragma unroll
  for (int b = 0; b < KP; ++b) {
    const int j = b * R + r;
    const int s = __shfl_sync(0xffffffffu, s_l, j);
    const int e = __shfl_sync(0xffffffffu, e_l, j);
    const int len = e - s;
    if (len <= kLong) {
      T acc = 0;
      for (int k0 = s; k0 < e; k0 += UNROLL) {
        int cc[UNROLL];
        T vv[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          cc[u] = k0 + u < e ? ld_reuse(col + k0 + u) : 0;
          vv[u] = k0 + u < e ? ldv(val, k0 + u) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
          if (k0 + u < e && h < K) acc += vv[u] * __ldg(x + (long long)cc[u] * K + h);
      }
      if (h < K && r0 + j < N) put_y(y, (long long)(r0 + j) * K + h, acc, overwrite, len > 0);
    }
  }
  unsigned longm = __ballot_sync(0xffffffffu, rr < N && len_l > kLong);
  while (longm) {
    const int j = __ffs(longm) - 1;
    longm &= longm - 1;
    const int s = __shfl_sync(0xffffffffu, s_l, j);
    const int e = __shfl_sync(0xffffffffu, e_l, j);
    for (int hh = 0; hh < K; ++hh) {
      T sum = 0, comp = 0;
      for (int k0 = s; k0 < e; k0 += 32 * 4) {
        int cc[4];
        T vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + lane + u * 32;
          cc[u] = k < e ? ld_reuse(col + k) : 0;
          vv[u] = k < e ? ldv(val, k) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + lane + u * 32;
          if (k < e) {
            const T p = vv[u] * __ldg(x + (long long)cc[u] * K + hh);
            if (COMP) comp_add(sum, comp, p);
            else sum += p;
          }
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const T o = __shfl_xor_sync(0xffffffffu, sum, off);
        if (COMP) {
          comp += __shfl_xor_sync(0xffffffffu, comp, off);
          comp_add(sum, comp, o);
        } else {
          sum += o;
        }
      }
      if (lane == 0) put_y(y, (long long)(r0 + j) * K + hh, COMP ? sum + comp : sum, overwrite, true);
    }
  }
}

// The K-value x row at xr (x 16-byte aligned, xr = x + c*K) when K values are
// not a whole number of aligned vectors (FP32 K = 3, 5, 6, 7): the aligned
// 16-byte blocks that cover the row are loaded (one to three random gathers
// instead of K, or of three float2), and the row is picked out of them by its
// offset in the first block.  Every block holds bytes of the row, so none
// starts before x; a row whose last block would run past x's end (the last
// row or two) is loaded value by value instead, so that no byte outside x
// is read.
template <typename T, int K>
__device__ __forceinline__ void load_xrow_blocks(const T* __restrict__ xr,
                                                 const T* __restrict__ xend, T (&v)[K]) {
  constexpr int E = 16 / (int)sizeof(T);        // values per 16-byte block
  constexpr int NB = (K + 2 * E - 2) / E;       // blocks at the worst offset
  using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const uintptr_t a = reinterpret_cast<uintptr_t>(xr);
  const int r = (int)((a & 15u) / sizeof(T));   // the row's offset in block 0
  const T* blk = reinterpret_cast<const T*>(a & ~(uintptr_t)15);
  const int nb = (r + K + E - 1) / E;
  if (blk + nb * E > xend) {
#pragma unroll
    for (int h = 0; h < K; ++h) v[h] = __ldg(xr + h);
    return;
  }
  T w[NB * E];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if (b < nb) {
      const V4 q = __ldg(reinterpret_cast<const V4*>(blk) + b);
      if constexpr (sizeof(T) == 4) {
        w[b * 4] = q.x; w[b * 4 + 1] = q.y; w[b * 4 + 2] = q.z; w[b * 4 + 3] = q.w;
      } else {
        w[b * 2] = q.x; w[b * 2 + 1] = q.y;
      }
    } else {
#pragma unroll
      for (int t = 0; t < E; ++t) w[b * E + t] = (T)0;
    }
  }
#pragma unroll
  for (int h = 0; h < K; ++h) {
    T t = w[h];
#pragma unroll
    for (int rr = 1; rr < E; ++rr)
      if (r == rr) t = w[h + rr];
    v[h] = t;
  }
}

// Eight FP32 values from a 32-byte aligned address: one 256-bit load
// (sm_100), i.e. one gather request where two 16-byte loads took two.
__device__ __forceinline__ void ld_v8(const float* __restrict__ p, float* w) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3]), "=f"(w[4]), "=f"(w[5]), "=f"(w[6]),
        "=f"(w[7])
      : "l"(p));
}

template <typename T, int K>
__device__ __forceinline__ void load_xrow(const T* __restrict__ xr, T (&v)[K]);

// x row loader of the several-right-hand-side paths: with x 32-byte aligned
// (X32) an FP32 row of 8 values is one 256-bit load; otherwise aligned
// vectors when K values are whole vectors, the covering 16-byte blocks when
// not.  Measured on B200 (512-matrix batch, ns per 1000 nonzeros): K = 8
// 10.2 -> 9.3 with the 256-bit load.  The same 32-byte blocks for K = 3, 5,
// 6, 7 (1.25-1.75 loads per row instead of 1.5-2.5 16-byte ones) were
// slower (K = 7: 10.7 -> 11.4): a random gather costs by the bytes it
// returns, and the second block plus the pick by offset outweighed the
// fewer requests.
template <typename T, int K, bool X32>
__device__ __forceinline__ void load_xrow_any(const T* __restrict__ xr, const T* __restrict__ xend,
                                              T (&v)[K]) {
  // FP64 keeps value-by-value loads for odd K: its covering blocks need
  // more registers than the batch kernel's 48 (ptxas spilled)
  constexpr bool whole = sizeof(T) == 4 ? (K % 4 == 0 || K <= 2) : true;
  if constexpr (X32 && sizeof(T) == 4 && K == 8) ld_v8(xr, v);
  else if constexpr (whole) load_xrow<T, K>(xr, v);
  else load_xrow_blocks<T, K>(xr, xend, v);
}

// Several right-hand sides (K = 2..8), one row per lane (the path taken when
// x is 16-byte aligned; measured on B200 on the 512-matrix batch, FP32 1.99 ->
// 1.87 ms and BF16 2.15 -> 1.83 ms against K lanes per row, same bits): the 32
// rows of the block are walked together, each lane over its own row in storage order,
// UNROLL entries per pass (their col/val loads first, then the K-value x
// rows), with the K sums in registers and no shuffles.  x rows are loaded
// as float4 / float2 (double2) vectors when K times the value size is a
// multiple of the vector size, so that every vector load is aligned (x is
// 16-byte aligned and row c starts at c*K values); otherwise value by value.
template <typename T, int K>
__device__ __forceinline__ void load_xrow(const T* __restrict__ xr, T (&v)[K]) {
  if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
    for (int h = 0; h < K; h += 4) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(xr + h));
      v[h] = q.x; v[h + 1] = q.y; v[h + 2] = q.z; v[h + 3] = q.w;
    }
  } else if constexpr (sizeof(T) == 4 && K % 2 == 0) {
#pragma unroll
    for (int h = 0; h < K; h += 2) {
      const float2 q = __ldg(reinterpret_cast<const float2*>(xr + h));
      v[h] = q.x; v[h + 1] = q.y;
    }
  } else if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
    for (int h = 0; h < K; h += 2) {
      const double2 q = __ldg(reinterpret_cast<const double2*>(xr + h));
      v[h] = q.x; v[h + 1] = q.y;
    }
  } else {
#pragma unroll
    for (int h = 0; h < K; ++h) v[h] = __ldg(xr + h);
  }
}

template <typename SV, typename T, int K, bool X32>
__device__ __forceinline__ void batch_block_lane_rows(const sb_batch_item& it, int r0, int lane) {
  constexpr int UNROLL = 4;
  const int i = r0 + lane;
  const int N = it.N;
  const bool overwrite = (it.flags & 1) != 0;
  if (i >= N) return;
  const int s = __ldg(it.row_ptr + i), e = __ldg(it.row_ptr + i + 1);
  const int* __restrict__ col = it.col;
  const SV* __restrict__ val = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  const T* __restrict__ xend = x + (long long)it.N * K;
  T* __restrict__ y = (T*)it.y;
  T acc[K];
#pragma unroll
  for (int h = 0; h < K; ++h) acc[h] = 0;
  for (int k0 = s; k0 < e; k0 += UNROLL) {
    int cc[UNROLL];
    T vv[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      cc[u] = k0 + u < e ? ld_reuse(col + k0 + u) : 0;
      vv[u] = k0 + u < e ? ldv(val, k0 + u) : (T)0;
    }
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      if (k0 + u < e) {
        T xv[K];
        load_xrow_any<T, K, X32>(x + (long long)cc[u] * K, xend, xv);
#pragma unroll
        for (int h = 0; h < K; ++h) acc[h] += vv[u] * xv[h];
      }
    }
  }
#pragma unroll
  for (int h = 0; h < K; ++h) put_y(y, (long long)i * K + h, acc[h], overwrite, e > s);
}

// Several right-hand sides (K = 2..8), V lanes per row (V = the item's lanes,
// 2..16): the lanes of a row interleave over its entries, so that the col
// and val loads stay coalesced as in batch_block; each lane keeps K partial
// sums fed by vector loads of the K-value x rows (x 16-byte aligned), and one
// shuffle reduction per right-hand side combines the V lanes.  Rows longer
// than kLong go to the whole warp.
template <typename SV, typename T, int V, int K, bool X32>
__device__ __forceinline__ void batch_block_vk(const sb_batch_item& it, int r0, int lane) {
  constexpr int UNROLL = K <= 4 ? 4 : 2;
  constexpr int RPB = 32 / V;
  const int g = lane / V, q = lane - (lane / V) * V;
  const int* __restrict__ rp = it.row_ptr;
  const int* __restrict__ col = it.col;
  const SV* __restrict__ val = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  const T* __restrict__ xend = x + (long long)it.N * K;
  T* __restrict__ y = (T*)it.y;
  const int N = it.N;
  const bool overwrite = (it.flags & 1) != 0;
  const int rr = r0 + lane;
  const int s_l = rr < N ? __ldg(rp + rr) : 0;
  const int e_l = rr < N ? __ldg(rp + rr + 1) : 0;
  const int len_l = e_l - s_l;
#pragma unroll 1
  for (int b = 0; b < V; ++b) {
    const int j = b * RPB + g;
    const int s = __shfl_sync(0xffffffffu, s_l, j);
    const int e = __shfl_sync(0xffffffffu, e_l, j);
    const int len = e - s;
    T acc[K];
#pragma unroll
    for (int h = 0; h < K; ++h) acc[h] = 0;
    if (len <= kLong) {
      for (int k0 = s + q; k0 < e; k0 += V * UNROLL) {
        int cc[UNROLL];
        T vv[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int k = k0 + u * V;
          cc[u] = k < e ? ld_reuse(col + k) : 0;
          vv[u] = k < e ? ldv(val, k) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          if (k0 + u * V < e) {
            T xv[K];
            load_xrow_any<T, K, X32>(x + (long long)cc[u] * K, xend, xv);
#pragma unroll
            for (int h = 0; h < K; ++h) acc[h] += vv[u] * xv[h];
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < K; ++h) {
      T a = acc[h];
#pragma unroll
      for (int off = V >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      if (q == 0 && len <= kLong && r0 + j < N)
        put_y(y, (long long)(r0 + j) * K + h, a, overwrite, len > 0);
    }
  }
  batch_long_rows<SV, T>(it, r0, lane, s_l, e_l, len_l);
}

// K = 8 with x 32-byte aligned: FP32 x rows as one 256-bit load
template <typename SV, typename T, int V>
__device__ __forceinline__ void batch_block_vk_k(const sb_batch_item& it, int r0, int lane) {
  switch (it.nrhs) {
    case 2: batch_block_vk<SV, T, V, 2, false>(it, r0, lane); break;
    case 3: batch_block_vk<SV, T, V, 3, false>(it, r0, lane); break;
    case 4: batch_block_vk<SV, T, V, 4, false>(it, r0, lane); break;
    case 5: batch_block_vk<SV, T, V, 5, false>(it, r0, lane); break;
    case 6: batch_block_vk<SV, T, V, 6, false>(it, r0, lane); break;
    case 7: batch_block_vk<SV, T, V, 7, false>(it, r0, lane); break;
    default:
      if (sizeof(T) == 4 && (it.flags & kX32)) batch_block_vk<SV, T, V, 8, true>(it, r0, lane);
      else batch_block_vk<SV, T, V, 8, false>(it, r0, lane);
      break;
  }
}

template <typename SV, typename T>
__device__ __forceinline__ void batch_block_lane_rows_k(const sb_batch_item& it, int r0, int lane) {
  switch (it.nrhs) {
    case 2: batch_block_lane_rows<SV, T, 2, false>(it, r0, lane); break;
    case 3: batch_block_lane_rows<SV, T, 3, false>(it, r0, lane); break;
    case 4: batch_block_lane_rows<SV, T, 4, false>(it, r0, lane); break;
    case 5: batch_block_lane_rows<SV, T, 5, false>(it, r0, lane); break;
    case 6: batch_block_lane_rows<SV, T, 6, false>(it, r0, lane); break;
    case 7: batch_block_lane_rows<SV, T, 7, false>(it, r0, lane); break;
    default:
      if (sizeof(T) == 4 && (it.flags & kX32)) batch_block_lane_rows<SV, T, 8, true>(it, r0, lane);
      else batch_block_lane_rows<SV, T, 8, false>(it, r0, lane);
      break;
  }
}

template <typename T> __device__ __forceinline__ T bmul_rn(T a, T b);
template <> __device__ __forceinline__ float bmul_rn(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double bmul_rn(double a, double b) { return __dmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T badd_rn(T a, T b);
template <> __device__ __forceinline__ float badd_rn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double badd_rn(double a, double b) { return __dadd_rn(a, b); }

// One 32-row block of a DIA item, one row per lane: for each diagonal in
// stored order, the separately rounded product of the in-band entry and x is
// added to the row's running value (the order and rounding of sb_spmv_dia,
// src/sequential/src/sparse_opt_32.wat:290-407), for every right-hand side.
template <typename SV, typename T>
__device__ __forceinline__ void batch_block_dia(const sb_batch_item& it, int r0, int lane) {
  const int i = r0 + lane;
  const int N = it.N;
  if (i >= N) return;
  const int K = it.nrhs;
  const int nd = it.width;
  const int* __restrict__ off = it.row_ptr;
  const SV* __restrict__ data = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  T* __restrict__ y = (T*)it.y;
  const bool overwrite = (it.flags & 1) != 0;
  // one right-hand side at a time (few registers); the data re-reads of the
  // later ones hit L1
  for (int h = 0; h < K; ++h) {
    T t = overwrite ? (T)0 : y[(long long)i * K + h];
    for (int d = 0; d < nd; ++d) {
      const int k = __ldg(off + d);
      if ((unsigned)(i + k) >= (unsigned)N) continue;
      t = badd_rn(bmul_rn((T)ldv(data, (long long)d * N + i), __ldg(x + (long long)(i + k) * K + h)),
                  t);
    }
    y[(long long)i * K + h] = t;
  }
}

// One 32-row block of an ELL item, one row per lane, slots in stored order
// (padding included), as sb_spmv_ell (src/sequential/src/sparse_opt_32.wat:427-479).
template <typename SV, typename T>
__device__ __forceinline__ void batch_block_ell(const sb_batch_item& it, int r0, int lane) {
  const int i = r0 + lane;
  const int N = it.N;
  if (i >= N) return;
  const int K = it.nrhs;
  const int nc = it.width;
  const int* __restrict__ idx = it.col;
  const SV* __restrict__ data = (const SV*)it.val;
  const T* __restrict__ x = (const T*)it.x;
  T* __restrict__ y = (T*)it.y;
  const bool overwrite = (it.flags & 1) != 0;
  for (int h = 0; h < K; ++h) {
    T t = overwrite ? (T)0 : y[(long long)i * K + h];
    for (int s = 0; s < nc; ++s) {
      const long long o = (long long)s * N + i;
      t = badd_rn(bmul_rn((T)ldv(data, o), __ldg(x + (long long)__ldg(idx + o) * K + h)), t);
    }
    y[(long long)i * K + h] = t;
  }
}

template <typename SV, typename T>
__global__ void __launch_bounds__(kBT, 5)
    batch_kernel(const sb_batch_item* __restrict__ items, const long long* __restrict__ offsets,
                 int* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int M = count[0];
  if (M <= 0) return;
  const long long total = offsets[M];
  while (true) {
    long long w0 = 0;
    if (lane == 0) w0 = (long long)atomicAdd((unsigned long long*)(count + 2), 1ull) * kBlocksPerTicket;
    w0 = __shfl_sync(0xffffffffu, w0, 0);
    if (w0 >= total) return;
    const long long w1 = min(w0 + kBlocksPerTicket, total);
    for (long long w = w0; w < w1; ++w) {
      // matrix of block w: last m with offsets[m] <= w
      int lo = 0, hi = M - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offsets + mid) <= w) lo = mid; else hi = mid - 1;
      }
      const sb_batch_item it = items[lo];
      const int r0 = (int)((w - __ldg(offsets + lo)) * 32);
      if (it.format == SB_FMT_DIA) {
        batch_block_dia<SV, T>(it, r0, lane);
        continue;
      }
      if (it.format == SB_FMT_ELL) {
        batch_block_ell<SV, T>(it, r0, lane);
        continue;
      }
      if (it.nrhs > 1 && (it.flags & kLaneRows) && it.lanes >= 2) {
        switch (it.lanes) {
          case 2: batch_block_vk_k<SV, T, 2>(it, r0, lane); break;
          case 4: batch_block_vk_k<SV, T, 4>(it, r0, lane); break;
          case 8: batch_block_vk_k<SV, T, 8>(it, r0, lane); break;
          default: batch_block_vk_k<SV, T, 16>(it, r0, lane); break;
        }
        continue;
      }
      if (it.nrhs > 1 && (it.flags & kLaneRows)) {
        batch_block_lane_rows_k<SV, T>(it, r0, lane);
        continue;
      }
      if (it.nrhs > 1) {
        if (it.nrhs == 2) batch_block_rhs<SV, T, 2>(it, r0, lane);
        else if (it.nrhs <= 4) batch_block_rhs<SV, T, 4>(it, r0, lane);
        else batch_block_rhs<SV, T, 8>(it, r0, lane);
        continue;
      }
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
}

static const void* batch_kernel_for(int dtype) {
  if (dtype == SB_F64) return (const void*)batch_kernel<double, double>;
  if (dtype == SB_BF16) return (const void*)batch_kernel<__nv_bfloat16, float>;
  return (const void*)batch_kernel<float, float>;
}

// Lanes per row of a several-right-hand-side item: each lane does K
// multiply-adds per entry, so a lane takes about 6-12 entries of a row
// (measured on 512 matrices of mean row length 13, K = 1..8: 2 lanes 1.77 ms,
// 4 lanes 1.83, row per lane 1.90).
static int lanes_for_rhs(long long nnz, int N) {
  const double avg = N ? (double)nnz / N : 0.0;
  if (avg <= 3) return 1;
  if (avg <= 24) return 2;
  if (avg <= 48) return 4;
  if (avg <= 96) return 8;
  return 16;
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
  for (sb_batch_slot& b : e->slot) {
    if (b.graph) cudaGraphExecDestroy(b.graph);
    if (b.done) cudaEventDestroy(b.done);
    if (b.h_items) cudaFreeHost(b.h_items);
    if (b.h_offsets) cudaFreeHost(b.h_offsets);
    if (b.h_count) cudaFreeHost(b.h_count);
    if (b.d_items) cudaFree(b.d_items);
    if (b.d_offsets) cudaFree(b.d_offsets);
    if (b.d_count) cudaFree(b.d_count);
  }
  if (e->capture_stream) cudaStreamDestroy(e->capture_stream);
  delete e;
}

// The gather floor of several right-hand sides: sum over entries of
// val[k] * (sum over h of x[col[k]*K + h]), streaming col and val (8
// entries per thread, coalesced) and gathering each entry's K-value x row
// with the loaders of the batch kernel (aligned vectors, covering 16-byte
// blocks, or one 256-bit load for 8 FP32 values with x 32-byte aligned);
// no row structure and no y.  The floor a batched SpMV over the same
// entries and right-hand sides is measured against.
template <typename SV, typename T, int K, bool VEC, bool X32>
__global__ void __launch_bounds__(256)
    gather_rows_kernel(const int* __restrict__ col, const SV* __restrict__ val,
                       const T* __restrict__ x, long long x_rows, long long nnz,
                       double* __restrict__ out) {
  constexpr int kItems = 8;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const T* __restrict__ xend = x + x_rows * K;
  T acc = 0;
  for (long long k0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kItems; k0 < nnz;
       k0 += nthreads * kItems) {
    int c[kItems];
    T v[kItems];
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      c[e] = k0 + e < nnz ? ld_reuse(col + k0 + e) : 0;
      v[e] = k0 + e < nnz ? (T)ldv(val, k0 + e) : (T)0;
    }
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      if (k0 + e < nnz) {
        T xv[K];
        if constexpr (VEC) {
          load_xrow_any<T, K, X32>(x + (long long)c[e] * K, xend, xv);
        } else {
#pragma unroll
          for (int h = 0; h < K; ++h) xv[h] = __ldg(x + (long long)c[e] * K + h);
        }
        T t = 0;
#pragma unroll
        for (int h = 0; h < K; ++h) t += xv[h];
        acc += v[e] * t;
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, (double)acc);
}

template <typename SV, typename T, int K>
static void launch_gather_rows(const int* col, const void* val, const void* x, long long x_rows,
                               long long nnz, double* out, cudaStream_t st) {
  const uintptr_t xa = reinterpret_cast<uintptr_t>(x);
  const bool vec = (xa & 15u) == 0, x32 = (xa & 31u) == 0;
  const long long steps = (nnz + 7) / 8;
  const unsigned ctas = (unsigned)std::max(
      1LL, std::min((steps + 255) / 256, (long long)sm_count() * 8));
  if (vec && x32 && K == 8 && sizeof(T) == 4)
    gather_rows_kernel<SV, T, K, true, true><<<ctas, 256, 0, st>>>(
        col, (const SV*)val, (const T*)x, x_rows, nnz, out);
  else if (vec)
    gather_rows_kernel<SV, T, K, true, false><<<ctas, 256, 0, st>>>(
        col, (const SV*)val, (const T*)x, x_rows, nnz, out);
  else
    gather_rows_kernel<SV, T, K, false, false><<<ctas, 256, 0, st>>>(
        col, (const SV*)val, (const T*)x, x_rows, nnz, out);
}

template <typename SV, typename T>
static void gather_rows_k(int K, const int* col, const void* val, const void* x,
                          long long x_rows, long long nnz, double* out, cudaStream_t st) {
  switch (K) {
    case 1: launch_gather_rows<SV, T, 1>(col, val, x, x_rows, nnz, out, st); break;
    case 2: launch_gather_rows<SV, T, 2>(col, val, x, x_rows, nnz, out, st); break;
    case 3: launch_gather_rows<SV, T, 3>(col, val, x, x_rows, nnz, out, st); break;
    case 4: launch_gather_rows<SV, T, 4>(col, val, x, x_rows, nnz, out, st); break;
    case 5: launch_gather_rows<SV, T, 5>(col, val, x, x_rows, nnz, out, st); break;
    case 6: launch_gather_rows<SV, T, 6>(col, val, x, x_rows, nnz, out, st); break;
    case 7: launch_gather_rows<SV, T, 7>(col, val, x, x_rows, nnz, out, st); break;
    default: launch_gather_rows<SV, T, 8>(col, val, x, x_rows, nnz, out, st); break;
  }
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_batch_exec_create(int dtype, int32_t capacity, sb_batch_exec** out) {
  SB_TRACE("sb_batch_exec_create");
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
  SB_E(cudaStreamCreateWithFlags(&e->capture_stream, cudaStreamNonBlocking));
  const void* kern = batch_kernel_for(dtype);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kBT, 0);
  e->grid = std::max(1, per) * sm_count();
  for (sb_batch_slot& b : e->slot) {
    SB_E(cudaMallocHost(&b.h_items, sizeof(sb_batch_item) * capacity));
    SB_E(cudaMallocHost(&b.h_offsets, sizeof(long long) * (capacity + 1)));
    SB_E(cudaMallocHost(&b.h_count, sizeof(int) * 4));
    SB_E(cudaMalloc(&b.d_items, sizeof(sb_batch_item) * capacity));
    SB_E(cudaMalloc(&b.d_offsets, sizeof(long long) * (capacity + 1)));
    SB_E(cudaMalloc(&b.d_count, sizeof(int) * 4));
    SB_E(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    // capture: descriptors + offsets + item count (host -> device, the
    // count's copy also resets the work counter), persistent kernel
    cudaGraph_t g = nullptr;
    SB_E(cudaStreamBeginCapture(e->capture_stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(b.d_items, b.h_items, sizeof(sb_batch_item) * capacity,
                    cudaMemcpyHostToDevice, e->capture_stream);
    cudaMemcpyAsync(b.d_offsets, b.h_offsets, sizeof(long long) * (capacity + 1),
                    cudaMemcpyHostToDevice, e->capture_stream);
    cudaMemcpyAsync(b.d_count, b.h_count, sizeof(int) * 4, cudaMemcpyHostToDevice,
                    e->capture_stream);
    void* args[] = {(void*)&b.d_items, (void*)&b.d_offsets, (void*)&b.d_count};
    cudaLaunchKernel(kern, dim3(e->grid), dim3(kBT), args, 0, e->capture_stream);
    SB_E(cudaStreamEndCapture(e->capture_stream, &g));
    ce = cudaGraphInstantiate(&b.graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      r = cuda_status(ce, "cudaGraphInstantiate");
      exec_release(e);
      return r;
    }
  }
#undef SB_E
  *out = e;
  return SB_OK;
}

int sb_batch_exec_destroy(sb_batch_exec* e) {
  SB_TRACE("sb_batch_exec_destroy");
  if (!e) return SB_OK;
  for (sb_batch_slot& b : e->slot)
    if (b.pending) cudaEventSynchronize(b.done);
  exec_release(e);
  return SB_OK;
}

int sb_batch_exec_run(sb_batch_exec* e, const sb_batch_item* items, int32_t n, void* stream) {
  SB_TRACE("sb_batch_exec_run");
  SB_REQUIRE(e, "sb_batch_exec_run: null executor");
  SB_REQUIRE(n >= 0 && n <= e->capacity, "sb_batch_exec_run: %d items exceed capacity %d", n,
             e->capacity);
  SB_REQUIRE(n == 0 || items, "sb_batch_exec_run: null items");
  // this set's pinned staging buffers were read by the run before the
  // previous one (its first nodes): wait for that run only
  sb_batch_slot& b = e->slot[e->next];
  if (b.pending) SB_CHECK_CUDA(cudaEventSynchronize(b.done));
  b.pending = false;
  long long acc = 0;
  for (int i = 0; i < n; ++i) {
    sb_batch_item it = items[i];
    SB_REQUIRE(it.N >= 0 && it.nrhs >= 1 && it.nrhs <= kMaxRhs,
               "sb_batch_exec_run: item %d: N >= 0 and 1 <= nrhs <= 8 required", i);
    SB_REQUIRE(it.format == SB_FMT_CSR || it.format == SB_FMT_DIA || it.format == SB_FMT_ELL,
               "sb_batch_exec_run: item %d: unknown format %d", i, it.format);
    if (it.format == SB_FMT_CSR) {
      SB_REQUIRE(it.N == 0 || (it.row_ptr && it.x && it.y && (it.nnz == 0 || (it.col && it.val))),
                 "sb_batch_exec_run: item %d: null pointer", i);
      // several right-hand sides with x 16-byte aligned: x rows loaded as
      // vectors, by one row per lane (lanes 1) or lanes per row (otherwise
      // the right-hand sides go across lanes)
      it.flags &= ~(kLaneRows | kX32);
      if (it.nrhs > 1 && (reinterpret_cast<uintptr_t>(it.x) & 15u) == 0) it.flags |= kLaneRows;
      if (it.nrhs == 8 && (reinterpret_cast<uintptr_t>(it.x) & 31u) == 0) it.flags |= kX32;
      if (it.lanes <= 0)
        it.lanes = it.nrhs > 1 ? lanes_for_rhs(it.nnz, it.N) : lanes_for(it.nnz, it.N);
      it.lanes = it.lanes > 32 ? 32 : it.lanes;
    } else {
      SB_REQUIRE(it.width >= 0, "sb_batch_exec_run: item %d: negative width", i);
      const bool need_idx = it.width > 0 && it.N > 0;
      SB_REQUIRE(it.N == 0 || (it.x && it.y), "sb_batch_exec_run: item %d: null vector", i);
      SB_REQUIRE(!need_idx || (it.val && (it.format == SB_FMT_DIA ? it.row_ptr != nullptr
                                                                 : it.col != nullptr)),
                 "sb_batch_exec_run: item %d: null pointer", i);
    }
    b.h_items[i] = it;
    b.h_offsets[i] = acc;
    acc += ((long long)it.N + 31) / 32;
  }
  b.h_offsets[n] = acc;
  b.h_count[0] = n;
  b.h_count[1] = 0;
  b.h_count[2] = 0;
  b.h_count[3] = 0;
  cudaStream_t st = as_stream(stream);
  SB_CHECK_CUDA(cudaGraphLaunch(b.graph, st));
  SB_CHECK_CUDA(cudaEventRecord(b.done, st));
  b.pending = true;
  e->next ^= 1;
  return SB_OK;
}

int sb_gather_dot_rows(int dtype, const int32_t* col, const void* val, const void* x,
                       int64_t x_rows, int32_t nrhs, int64_t nnz, double* out, void* stream) {
  SB_TRACE("sb_gather_dot_rows");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64 || dtype == SB_BF16,
             "sb_gather_dot_rows: bad dtype");
  SB_REQUIRE(nrhs >= 1 && nrhs <= kMaxRhs && nnz >= 0 && x_rows >= 0,
             "sb_gather_dot_rows: 1 <= nrhs <= 8 and non-negative sizes required");
  SB_REQUIRE(out, "sb_gather_dot_rows: null output");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  SB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
  if (nnz == 0) return SB_OK;
  SB_REQUIRE(col && val && x, "sb_gather_dot_rows: null pointer");
  if (dtype == SB_F64)
    gather_rows_k<double, double>(nrhs, col, val, x, x_rows, nnz, out, st);
  else if (dtype == SB_BF16)
    gather_rows_k<__nv_bfloat16, float>(nrhs, col, val, x, x_rows, nnz, out, st);
  else
    gather_rows_k<float, float>(nrhs, col, val, x, x_rows, nnz, out, st);
  SB_CHECK_LAUNCH("gather_rows_kernel");
  return SB_OK;
}

}  // extern "C"
