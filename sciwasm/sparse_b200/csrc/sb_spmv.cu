// sb_spmv.cu -- SpMV kernels (y <- y + A x) for COO, CSR, DIA and ELL.
//
// Reference loops: src/sequential/src/sparse_opt_32.wat:175-498 (f32) and
// src/sequential/src/sparse_opt_64.wat:187-515 (f64).  The reference walks
// storage order on one core (or splits rows / nnz over Web Workers,
// src/parallel/src/sparse32.js:2637-2821).  Here:
//   * CSR (default) is a row-block kernel: a warp owns 32 consecutive rows,
//     reduces the short ones V lanes per row (V from the mean row length:
//     adaptive rows per warp) with unrolled independent loads and shuffle
//     reductions, and the long ones with the whole warp.  An alternative
//     streams fixed-size nonzero tiles into a shared-memory ring with bulk
//     async copies (option kernel 1); a third cuts the nonzeros into
//     row-aligned warp ranges walked in 256-nonzero tiles (kernel 2).
//   * COO walks 256-entry tiles, 8 entries per lane; every row segment is
//     added with one atomic, so unsorted input is accepted.  With rows the
//     caller declares sorted (and short on average), rows inside a tile are
//     added without atomics.
//   * DIA and ELL assign one row per thread and keep the reference's per-row
//     addition order (separately rounded mul and add), so their results are
//     bit-identical to the reference's serial loops; DIA with up to 16
//     diagonals runs a kernel with the count fixed at compile time.
#include <algorithm>
#include <climits>

#include "sb_common.cuh"

namespace sb {

constexpr int kWarp = 32;
constexpr int kItems = 8;                  // COO items per lane per tile
constexpr int kTile = kWarp * kItems;      // 256 COO items per warp tile
constexpr int kWarpsPerCta = 8;
constexpr unsigned kFull = 0xffffffffu;

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename K>
static int resident_ctas(K kernel, int threads) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (per_sm < 1) per_sm = 1;
  return per_sm * sm_count();
}

// ------------------------------------------------------------ CSR (merge)

// ------------------------------------------------------------ CSR (stream)

// Smallest a in [0, N] with a == N or row_ptr[a+1] > b: the row holding
// nonzero b (rows ending at or before b are skipped).  32-ary warp search.
__device__ __forceinline__ int row_of_item(const int* __restrict__ row_ptr, int N, long long b,
                                           int lane) {
  int lo = 0, hi = N;
  while (hi - lo > kWarp) {
    int step = (hi - lo) / kWarp;
    int p = lo + lane * step;
    bool pred = (long long)__ldg(row_ptr + p + 1) > b;
    unsigned m = __ballot_sync(kFull, pred);
    if (m == 0) {
      lo = lo + (kWarp - 1) * step + 1;
    } else {
      int f = __ffs(m) - 1;
      hi = lo + f * step;
      if (f > 0) lo = lo + (f - 1) * step + 1;
    }
  }
  int p = lo + lane;
  bool pred = (p >= hi) || ((long long)__ldg(row_ptr + p + 1) > b);
  unsigned m = __ballot_sync(kFull, pred);
  return lo + __ffs(m) - 1;
}

constexpr int kStreamThreads = 256;
template <typename S, int T, int STAGES>
struct CsrStreamSmem {
  int col[STAGES][T];
  S val[STAGES][T];  // values, overwritten in place by the products
  int re[2][kStreamThreads];
  S ys[2][kStreamThreads];  // y of the chunk's rows, prefetched
  // (row, lo, hi, atomic) of rows left to whole warps: a deferred row holds
  // more than 16 items, so at most T/17 of them fit in one tile
  int4 lrow[2][T / 16 + 2];
  uint64_t bar[STAGES];
  int lcount[2];
  int rfirst;
};

// Products of 4 consecutive staged items (col int4, values as 16-byte words).
template <typename S>
__device__ __forceinline__ void prod4(int* pc, S* pv, const S* __restrict__ x) {
  const int4 c = *reinterpret_cast<const int4*>(pc);
  if constexpr (sizeof(S) == 8) {
    double2 v0 = reinterpret_cast<const double2*>(pv)[0];
    double2 v1 = reinterpret_cast<const double2*>(pv)[1];
    v0.x *= ld_ro(x + c.x);
    v0.y *= ld_ro(x + c.y);
    v1.x *= ld_ro(x + c.z);
    v1.y *= ld_ro(x + c.w);
    reinterpret_cast<double2*>(pv)[0] = v0;
    reinterpret_cast<double2*>(pv)[1] = v1;
  } else {
    float4 v = *reinterpret_cast<const float4*>(pv);
    v.x *= ld_ro(x + c.x);
    v.y *= ld_ro(x + c.y);
    v.z *= ld_ro(x + c.z);
    v.w *= ld_ro(x + c.w);
    *reinterpret_cast<float4*>(pv) = v;
  }
}

// Streaming CSR: a persistent CTA walks a contiguous range of T-nonzero
// tiles through a STAGES-deep shared-memory ring.  One elected thread keeps
// STAGES-1 tiles of col/val in flight with bulk async copies completed on
// per-stage mbarriers, while the CTA multiplies the current tile (x gathers,
// 4 items per thread per pass) and reduces its rows with groups of V lanes,
// V = 256 / next_pow2(rows in the tile) capped at a warp (adaptive rows per
// CTA), warp-shuffle reductions inside each group.  A row much longer than
// its group's share is deferred to a whole warp.  Rows wholly inside a tile
// are written with a plain y += sum (y prefetched with the row ends); rows cut
// by a tile boundary are added atomically.
template <typename S, int T, int STAGES>
__global__ void __launch_bounds__(kStreamThreads)
    csr_stream_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                      const S* __restrict__ val, const S* __restrict__ x, S* __restrict__ y,
                      int N, long long nnz, long long ntiles, long long tpc, int* status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  CsrStreamSmem<S, T, STAGES>& sm = *reinterpret_cast<CsrStreamSmem<S, T, STAGES>*>(smem_raw);
  const int tid = threadIdx.x;
  const int lane = tid & (kWarp - 1);
  const int warp = tid >> 5;
  const long long t0 = (long long)blockIdx.x * tpc;
  const long long t_end = min(t0 + tpc, ntiles);
  if (t0 >= t_end) return;
  const int ntile = (int)(t_end - t0);

  auto issue = [&](long long tt, int st) {
    const long long b0 = tt * T;
    const int n = (int)min((long long)T, nnz - b0);
    const int nal = n & ~3;
    mbar_expect_tx(&sm.bar[st], (uint32_t)nal * (uint32_t)(sizeof(int) + sizeof(S)));
    if (nal > 0) {
      bulk_g2s(sm.col[st], col + b0, (uint32_t)nal * sizeof(int), &sm.bar[st]);
      bulk_g2s(sm.val[st], val + b0, (uint32_t)nal * sizeof(S), &sm.bar[st]);
    }
  };

  if (tid == 0) {
    for (int st = 0; st < STAGES; ++st) mbar_init(&sm.bar[st], 1);
    mbar_fence_init();
    sm.lcount[0] = sm.lcount[1] = 0;
  }
  __syncthreads();
  if (tid == 0) {
    for (int st = 0; st < STAGES && st < ntile; ++st) issue(t0 + st, st);
  }
  if (warp == 0) {
    int r = row_of_item(row_ptr, N, t0 * (long long)T, lane);
    if (lane == 0) sm.rfirst = r;
  }
  __syncthreads();
  int r = sm.rfirst;
  int cp = 0;  // chunk parity (double-buffered row ends / y / long-row lists)

  for (int k = 0; k < ntile; ++k) {
    const long long t = t0 + k;
    const int st = k % STAGES;
    const uint32_t par = (uint32_t)((k / STAGES) & 1);
    const long long b0 = t * T;
    const int n = (int)min((long long)T, nnz - b0);
    const int nal = n & ~3;
    // first chunk of row ends and y, issued before the wait
    int e = (r + tid < N) ? (int)(__ldg(row_ptr + r + tid + 1) - b0) : 0x7fffffff;
    S yp = (r + tid < N) ? y[r + tid] : (S)0;
    int prev_end = (r < N) ? (int)max((long long)__ldg(row_ptr + r) - b0, -1LL) : n;

    const bool ok = mbar_wait_bounded(&sm.bar[st], par);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(status, SB_DEV_TIMEOUT_BULK);
        for (int j = k + 1; j < ntile && j < k + STAGES; ++j)
          mbar_wait_bounded(&sm.bar[j % STAGES], (uint32_t)((j / STAGES) & 1));
      }
      return;
    }

    S* pv = sm.val[st];
    int* pc = sm.col[st];
#pragma unroll
    for (int base = 0; base < T; base += 4 * kStreamThreads) {
      const int i = base + 4 * tid;
      if (i + 4 <= nal) {
        prod4<S>(pc + i, pv + i, x);
      } else if (i < n) {
        for (int q = i; q < n && q < i + 4; ++q) {
          int c;
          S v;
          if (q < nal) {
            c = pc[q];
            v = pv[q];
          } else {
            c = ld_stream(col + b0 + q);
            v = ld_stream(val + b0 + q);
          }
          pv[q] = v * ld_ro(x + c);
        }
      }
    }

    bool first_chunk = true;
    while (true) {
      sm.re[cp][tid] = e;
      sm.ys[cp][tid] = yp;
      const int c = __syncthreads_count(e <= n);
      if (first_chunk) {
        // every thread is past tile k-1: refill its stage with tile k-1+STAGES
        if (tid == 0 && k >= 1 && k - 1 + STAGES < ntile) {
          fence_proxy_async_smem();
          issue(t0 + k - 1 + STAGES, (k - 1) % STAGES);
        }
        first_chunk = false;
      }
      const bool last_chunk = c < kStreamThreads;
      // rows of this pass: c rows ending in the tile, plus the cut row
      const bool has_cut = last_chunk && (r + c < N);
      const int nrows = c + (has_cut ? 1 : 0);
      if (nrows > 0) {
        const int p2 = nrows <= 1 ? 1 : (1 << (32 - __clz(nrows - 1)));
        const int V = min(kWarp, max(1, kStreamThreads / p2));
        const int G = kStreamThreads / V;
        const int g = tid / V;
        const int q = tid - g * V;
        for (int j0 = 0; j0 < nrows; j0 += G) {
          const int j = j0 + g;
          int lo = 0, hi = 0;
          bool atom = false;
          if (j < nrows) {
            const int s0 = (j == 0) ? prev_end : sm.re[cp][j - 1];
            hi = (j < c) ? sm.re[cp][j] : n;
            lo = max(s0, 0);
            atom = (s0 < 0) || (j >= c);
          }
          const bool longrow = (V < kWarp) && (hi - lo > 16 * V);
          S sum = 0;
          if (!longrow) {
            for (int qq = lo + q; qq < hi; qq += V) sum += pv[qq];
          }
          for (int off = V >> 1; off > 0; off >>= 1) sum += __shfl_xor_sync(kFull, sum, off);
          if (q == 0 && j < nrows && hi > lo) {
            const int row = r + j;
            if (longrow) {
              const int slot = atomicAdd(&sm.lcount[cp], 1);
              sm.lrow[cp][slot] = make_int4(row, lo, hi, atom ? 1 : 0);
            } else if (atom) {
              atomicAdd(y + row, sum);
            } else {
              y[row] = sm.ys[cp][j] + sum;
            }
          }
        }
      }
      __syncthreads();
      const int L = sm.lcount[cp];
      for (int j = warp; j < L; j += kStreamThreads / kWarp) {
        const int4 w = sm.lrow[cp][j];
        S sum = 0;
        for (int qq = w.y + lane; qq < w.z; qq += kWarp) sum += pv[qq];
        for (int off = kWarp / 2; off > 0; off >>= 1) sum += __shfl_xor_sync(kFull, sum, off);
        if (lane == 0) {
          if (w.w) atomicAdd(y + w.x, sum);
          else y[w.x] = sm.ys[cp][w.x - r] + sum;
        }
      }
      if (c > 0) prev_end = sm.re[cp][c - 1];
      if (tid == 0) sm.lcount[cp ^ 1] = 0;
      r += c;
      cp ^= 1;
      if (last_chunk) break;
      e = (r + tid < N) ? (int)(__ldg(row_ptr + r + tid + 1) - b0) : 0x7fffffff;
      yp = (r + tid < N) ? y[r + tid] : (S)0;
    }
  }
}

// ------------------------------------------------------------ CSR (rows)

// Stored value -> accumulation type (BF16 storage widens exactly to f32).
template <typename T> __device__ __forceinline__ T widen(float v) { return (T)v; }
__device__ __forceinline__ float ld_val(const float* p) { return ld_stream(p); }
__device__ __forceinline__ double ld_val(const double* p) { return ld_stream(p); }
__device__ __forceinline__ float ld_val_reuse(const float* p) { return ld_reuse(p); }
__device__ __forceinline__ double ld_val_reuse(const double* p) { return ld_reuse(p); }
__device__ __forceinline__ float ld_val_reuse(const __nv_bfloat16* p) {
  return __bfloat162float(__ushort_as_bfloat16(ld_reuse(reinterpret_cast<const unsigned short*>(p))));
}
__device__ __forceinline__ float ld_val(const __nv_bfloat16* p) {
  return __bfloat162float(__ushort_as_bfloat16(ld_stream(reinterpret_cast<const unsigned short*>(p))));
}

// Neumaier-compensated accumulation (used for long rows with f32 sums).
template <typename T>
__device__ __forceinline__ void comp_add(T& s, T& c, T v) {
  const T t = s + v;
  c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
  s = t;
}

// Row-block CSR: each warp owns 32 consecutive rows.  It reads their row_ptr
// entries once (one per lane), then reduces the short rows in batches of
// 32/V rows, V lanes per row, each lane issuing UNROLL independent col/val
// loads before the dependent x gathers and one shuffle reduction per batch;
// rows longer than the short limit are reduced afterwards by the whole warp
// (with compensated f32 sums when the accumulation type is f32).  V is picked
// per matrix from its mean row length.  No shared memory and no block
// barrier: occupancy and unrolled loads keep the loads in flight.  The V
// lanes of a row interleave over its entries, so a 32-byte sector of col or
// val is read by several consecutive load instructions: those loads
// allocate in L1 (ld_reuse).  SV is the stored value type (f32, f64 or
// BF16); x, y and the sums are T.
// Where the row kernel's sums go.  YOut: y itself (rows without entries
// keep their y, as in the reference).  YScatter: the value of every row,
// also of rows without entries (whose y is passed on unchanged), to up to 8
// destination vectors at the row's global index -- this GPU's own buffers
// or other GPUs' buffers mapped over NVLink (plain stores, no multicast), so
// that a row-sharded SpMV leaves the whole y in every rank's buffer without
// a separate all-gather.
template <typename T>
struct YOut {
  static constexpr bool kAll = false;
  // 0: no minimum (the compiler's own choice, 32 registers for the kernels
  // the tuner picks).  An explicit minimum of 1 let ptxas take 48-62
  // registers, 4 blocks per SM (format sweep: banded CSR 0.114 -> 0.1345 ms,
  // 4096^2 Laplacian FP32 0.176 -> 0.215 ms); 6 blocks (at most 42) only
  // recovered part of it.
  template <typename V>
  static constexpr int min_blocks() { return 0; }
  T* y;
  __device__ __forceinline__ void put(long long i, T v) const { y[i] = v; }
};
constexpr int kMaxScatter = 8;
template <typename T>
struct YScatter {
  static constexpr bool kAll = true;
  template <typename V>
  static constexpr int min_blocks() { return 8; }  // 32 registers
  const unsigned long long* d;  // device array of n destination addresses
  int n;
  long long r0;
  __device__ __forceinline__ void put(long long i, T v) const {
    for (int k = 0; k < n; ++k) {
      // read at each store (an L1 hit): held in registers, the 8
      // addresses took the kernel from 32 to 48 registers and cut its
      // resident warps from 64 to 40 per SM
      unsigned long long a;
      asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(a) : "l"(d + k));
      reinterpret_cast<T*>(a)[r0 + i] = v;
    }
  }
};

template <typename SV, typename T, int V, int UNROLL, class Out>
__global__ void __launch_bounds__(256, Out::template min_blocks<T>())
    csr_rows_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                    const SV* __restrict__ val, const T* __restrict__ x, const T* y_in,
                    Out out, int N) {
  constexpr int RPB = kWarp / V;           // rows per batch
  constexpr int SHORT = V * UNROLL;        // a short row needs one unrolled pass
  constexpr bool COMP = sizeof(T) == 4;    // compensate long f32 sums
  const int lane = threadIdx.x & (kWarp - 1);
  const int g = lane / V;
  const int q = lane - g * V;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
       w * kWarp < N; w += warps) {
    const int r0 = (int)(w * kWarp);
    const int rr = r0 + lane;
    const int s_l = rr < N ? __ldg(row_ptr + rr) : 0;
    const int e_l = rr < N ? __ldg(row_ptr + rr + 1) : 0;
    const int len_l = e_l - s_l;
    const T y_l = (rr < N && (len_l > 0 || Out::kAll)) ? y_in[rr] : (T)0;
#pragma unroll
    for (int b = 0; b < V; ++b) {
      const int j = b * RPB + g;  // row of this group within the block
      const int s = __shfl_sync(kFull, s_l, j);
      const int e = __shfl_sync(kFull, e_l, j);
      const int len = e - s;
      T sum = 0;
      if (len <= SHORT) {
        int cc[UNROLL];
        T vv[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int k = s + q + u * V;
          cc[u] = k < e ? ld_reuse(col + k) : 0;
          vv[u] = k < e ? (T)ld_val_reuse(val + k) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int k = s + q + u * V;
          if (k < e) sum += vv[u] * ld_ro(x + cc[u]);
        }
      }
#pragma unroll
      for (int off = V >> 1; off > 0; off >>= 1) sum += __shfl_xor_sync(kFull, sum, off);
      const T yj = __shfl_sync(kFull, y_l, j);
      if (q == 0 && len > 0 && len <= SHORT && r0 + j < N) out.put(r0 + j, yj + sum);
      else if (Out::kAll && q == 0 && len == 0 && r0 + j < N) out.put(r0 + j, yj);
    }
    // long rows of the block: whole warp each
    unsigned longm = __ballot_sync(kFull, rr < N && len_l > SHORT);
    while (longm) {
      const int j = __ffs(longm) - 1;
      longm &= longm - 1;
      const int s = __shfl_sync(kFull, s_l, j);
      const int e = __shfl_sync(kFull, e_l, j);
      T sum = 0, comp = 0;
      for (int k0 = s; k0 < e; k0 += kWarp * 4) {
        int cc[4];
        T vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + lane + u * kWarp;
          cc[u] = k < e ? ld_reuse(col + k) : 0;
          vv[u] = k < e ? (T)ld_val_reuse(val + k) : (T)0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + lane + u * kWarp;
          if (k < e) {
            if (COMP) comp_add(sum, comp, vv[u] * ld_ro(x + cc[u]));
            else sum += vv[u] * ld_ro(x + cc[u]);
          }
        }
      }
#pragma unroll
      for (int off = kWarp / 2; off > 0; off >>= 1) {
        const T o = __shfl_xor_sync(kFull, sum, off);
        if (COMP) {
          comp += __shfl_xor_sync(kFull, comp, off);
          comp_add(sum, comp, o);
        } else {
          sum += o;
        }
      }
      const T yj = __shfl_sync(kFull, y_l, j);
      if (lane == 0) out.put(r0 + j, COMP ? yj + (sum + comp) : yj + sum);
    }
  }
}

// grid 0: a resident grid whose warps stride over the 32-row blocks (best for
// regular rows); grid 1: one warp per block, the hardware handing blocks to
// SMs as they free up, so blocks holding long rows do not hold back a fixed
// share of the others (best for skewed row lengths).
template <typename SV, typename T, int V, int UNROLL, class Out>
static int launch_csr_rows_v(const int* row_ptr, const int* col, const SV* val, const T* x,
                             const T* y_in, Out out, int N, int grid, cudaStream_t st) {
  auto kern = csr_rows_kernel<SV, T, V, UNROLL, Out>;
  const long long warps_needed = ((long long)N + kWarp - 1) / kWarp;
  const long long warps =
      grid == 1 ? warps_needed
                : std::min(warps_needed, (long long)resident_ctas(kern, 256) * 8);
  const unsigned ctas = (unsigned)((warps + 7) / 8);
  kern<<<ctas, 256, 0, st>>>(row_ptr, col, val, x, y_in, out, N);
  SB_CHECK_LAUNCH("csr_rows_kernel");
  return SB_OK;
}

template <typename SV, typename T, int V, class Out>
static int launch_csr_rows_u(const int* row_ptr, const int* col, const SV* val, const T* x,
                             const T* y_in, Out out, int N, int unroll, int grid,
                             cudaStream_t st) {
  if (unroll <= 2)
    return launch_csr_rows_v<SV, T, V, 2>(row_ptr, col, val, x, y_in, out, N, grid, st);
  if (unroll >= 8)
    return launch_csr_rows_v<SV, T, V, 8>(row_ptr, col, val, x, y_in, out, N, grid, st);
  return launch_csr_rows_v<SV, T, V, 4>(row_ptr, col, val, x, y_in, out, N, grid, st);
}

// Default lanes per row from the mean row length (about three items per lane).
static int default_lanes(int N, long long nnz) {
  const double avg = N ? (double)nnz / N : 0.0;
  if (avg <= 6) return 2;
  if (avg <= 14) return 4;
  if (avg <= 28) return 8;
  return 16;
}

template <typename SV, typename T, class Out>
static int launch_csr_rows_out(const int* row_ptr, const int* col, const SV* val, const T* x,
                               const T* y_in, Out out, int N, long long nnz, int lanes,
                               int unroll, int grid, cudaStream_t st) {
  if (lanes <= 0) lanes = default_lanes(N, nnz);
  if (unroll <= 0) unroll = 4;
#define SB_CSR_L(v) \
  return launch_csr_rows_u<SV, T, v>(row_ptr, col, val, x, y_in, out, N, unroll, grid, st)
  switch (lanes) {
    case 1: SB_CSR_L(1);
    case 2: SB_CSR_L(2);
    case 4: SB_CSR_L(4);
    case 8: SB_CSR_L(8);
    case 16: SB_CSR_L(16);
    default: SB_CSR_L(32);
  }
#undef SB_CSR_L
}

template <typename SV, typename T>
static int launch_csr_rows(const int* row_ptr, const int* col, const SV* val, const T* x, T* y,
                           int N, long long nnz, int lanes, int unroll, int grid,
                           cudaStream_t st) {
  return launch_csr_rows_out<SV, T>(row_ptr, col, val, x, y, YOut<T>{y}, N, nnz, lanes, unroll,
                                    grid, st);
}

// ------------------------------------------------------------ COO

// SORTED: the caller guarantees non-decreasing rows.  A row that touches
// neither end of a tile then has all its entries in that tile, so its sum
// is added with a plain read-modify-write; only the rows of the tile's first
// and last entries, which other tiles may share, keep the atomic.
template <typename S, typename A, bool VEC, bool SORTED>
__global__ void __launch_bounds__(kWarpsPerCta * kWarp)
    coo_tile_kernel(const int* __restrict__ row, const int* __restrict__ col,
                    const S* __restrict__ val, const S* __restrict__ x, S* __restrict__ y,
                    long long nnz, long long ntiles, long long tiles_per_warp) {
  const int lane = threadIdx.x & (kWarp - 1);
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  long long tile = gw * tiles_per_warp;
  const long long tile_end = min(tile + tiles_per_warp, ntiles);
  for (; tile < tile_end; ++tile) {
    const long long k0 = tile * kTile + (long long)lane * kItems;
    int r[kItems];
    A p[kItems];
    int cnt = 0;
    if (VEC && k0 + kItems <= nnz) {
      cnt = kItems;
#pragma unroll
      for (int h = 0; h < kItems; h += 4) {
        int4 rr = ld_stream_v4(row + k0 + h);
        int4 cc = ld_stream_v4(col + k0 + h);
        r[h + 0] = rr.x; r[h + 1] = rr.y; r[h + 2] = rr.z; r[h + 3] = rr.w;
        if constexpr (sizeof(S) == 4) {
          float4 w = ld_stream_v4(reinterpret_cast<const float*>(val) + k0 + h);
          p[h + 0] = (A)w.x * (A)ld_ro(x + cc.x);
          p[h + 1] = (A)w.y * (A)ld_ro(x + cc.y);
          p[h + 2] = (A)w.z * (A)ld_ro(x + cc.z);
          p[h + 3] = (A)w.w * (A)ld_ro(x + cc.w);
        } else {
          double2 w0 = ld_stream_v2(reinterpret_cast<const double*>(val) + k0 + h);
          double2 w1 = ld_stream_v2(reinterpret_cast<const double*>(val) + k0 + h + 2);
          p[h + 0] = (A)w0.x * (A)ld_ro(x + cc.x);
          p[h + 1] = (A)w0.y * (A)ld_ro(x + cc.y);
          p[h + 2] = (A)w1.x * (A)ld_ro(x + cc.z);
          p[h + 3] = (A)w1.y * (A)ld_ro(x + cc.w);
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < kItems; ++e) {
        const long long k = k0 + e;
        if (k < nnz) {
          r[e] = ld_stream(row + k);
          p[e] = (A)ld_stream(val + k) * (A)ld_ro(x + ld_stream(col + k));
          cnt = e + 1;
        } else {
          r[e] = -1;
          p[e] = 0;
        }
      }
    }
    // lane-local runs
    const int start_row = cnt ? r[0] : -1;
    int cur = start_row;
    A acc = 0;
    bool internal = false;
    A first_val = 0;
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      if (e < cnt) {
        if (r[e] != cur) {
          if (!internal) { internal = true; first_val = acc; }
          else if (SORTED) y[cur] += (S)acc;  // strictly inside one lane: a whole row
          else atomicAdd(y + cur, (S)acc);
          cur = r[e];
          acc = 0;
        }
        acc += p[e];
      }
    }
    const int end_row = cur;
    int tile_first = -1, tile_last = -1;
    if (SORTED) {
      tile_first = __shfl_sync(kFull, start_row, 0);
      const unsigned have = __ballot_sync(kFull, cnt > 0);
      tile_last = __shfl_sync(kFull, end_row, 31 - __clz(have));
    }
    const int prev_end = __shfl_up_sync(kFull, end_row, 1);
    const bool cont_prev = lane > 0 && cnt > 0 && start_row == prev_end;
    // segment head for the scan: lane does not simply continue the previous one
    bool hf = internal || !cont_prev;
    A S_ = acc;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      A v = __shfl_up_sync(kFull, S_, off);
      bool f = __shfl_up_sync(kFull, hf, off);
      if (lane >= off) {
        if (!hf) S_ += v;
        hf = hf || f;
      }
    }
    A carry = __shfl_up_sync(kFull, S_, 1);
    if (internal) {
      A v = first_val + (cont_prev ? carry : (A)0);
      if (SORTED && start_row != tile_first) y[start_row] += (S)v;
      else atomicAdd(y + start_row, (S)v);
    }
    // tail run: emitted unless the next lane continues it
    const int next_start = __shfl_down_sync(kFull, start_row, 1);
    const int next_cnt = __shfl_down_sync(kFull, cnt, 1);
    const bool next_internal_or_diff = (lane == kWarp - 1) || next_cnt == 0 || next_start != end_row;
    if (cnt > 0 && next_internal_or_diff) {
      if (SORTED && end_row != tile_first && end_row != tile_last) y[end_row] += (S)S_;
      else atomicAdd(y + end_row, (S)S_);
    }
  }
}

// ------------------------------------------------------------ CSR (nonzero tiles)

// 8 consecutive stored values from a 16-byte aligned index k0 (a multiple of
// 8), widened to the accumulation type.
template <typename SV, typename T>
__device__ __forceinline__ void load_vals8(const SV* __restrict__ val, long long k0, T (&v)[kItems]) {
  if constexpr (sizeof(SV) == 8) {
#pragma unroll
    for (int h = 0; h < kItems; h += 2) {
      const double2 w = ld_stream_v2(reinterpret_cast<const double*>(val) + k0 + h);
      v[h] = w.x;
      v[h + 1] = w.y;
    }
  } else if constexpr (sizeof(SV) == 4) {
#pragma unroll
    for (int h = 0; h < kItems; h += 4) {
      const float4 w = ld_stream_v4(reinterpret_cast<const float*>(val) + k0 + h);
      v[h] = w.x;
      v[h + 1] = w.y;
      v[h + 2] = w.z;
      v[h + 3] = w.w;
    }
  } else {  // BF16: 8 values in one 16-byte word, element 2i in the low half of word i
    const int4 w = ld_stream_v4(reinterpret_cast<const int*>(val) + k0 / 2);
    const int ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      v[2 * h] = __uint_as_float((unsigned)ws[h] << 16);
      v[2 * h + 1] = __uint_as_float((unsigned)ws[h] & 0xffff0000u);
    }
  }
}

// Nonzero-tile CSR: the nonzeros are cut into ranges of `items` (whole
// 256-item warp tiles) and every cut is moved forward to the next row start,
// so each row lies in exactly one warp's range and is written once, without
// atomics, in an order fixed by the matrix and the range size
// (y[row] += sum; rows without entries are not written).  A warp walks its
// range in tiles of 256 nonzeros, 8 consecutive ones per lane loaded with
// 16-byte vector loads and their 8 x gathers in flight together.  Each
// item's row comes from row_ptr: the starts of the rows that begin inside
// the tile are marked in a per-warp shared array (the largest row index wins
// a position, which skips empty rows) and a prefix maximum over the
// positions gives every item its row.  Row sums are combined by a segmented
// scan across the lanes; the tile's last run is carried in registers into
// the next tile.
template <typename SV, typename T, bool VEC>
__global__ void __launch_bounds__(kWarpsPerCta * kWarp)
    csr_tile_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                    const SV* __restrict__ val, const T* __restrict__ x, T* __restrict__ y, int N,
                    long long nnz, long long items) {
  __shared__ __align__(16) int mark_all[kWarpsPerCta][kTile];
  const int lane = threadIdx.x & (kWarp - 1);
  int* mark = mark_all[threadIdx.x >> 5];
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long b_lo = gw * items;
  if (b_lo >= nnz) return;
  const long long b_hi = b_lo + items;
  // The warp owns the rows whose start lies in [b_lo, b_hi): from r_lo, the
  // first row starting at or after b_lo, up to the first row starting at or
  // after b_hi, which is found while walking (its start is k_hi).
  const int r_lo = b_lo == 0 ? 0 : row_of_item(row_ptr, N, b_lo - 1, lane) + 1;
  if (r_lo >= N) return;
  const long long k_lo = __ldg(row_ptr + r_lo);
  if (k_lo >= b_hi || k_lo >= nnz) return;
  long long k_hi = nnz;
  bool hi_known = false;
  int next_row = r_lo;  // first row whose start is not yet marked
  int base_row = -1;    // row of the item before the tile
  int carry_row = -1;   // row of the previous tile's last run, still open
  T carry = 0;
  for (long long kt = k_lo & ~7LL; kt < k_hi; kt += kTile) {
    // the tile's col/val and x gathers first, so that they are in flight
    // while the row starts are read (items found below to lie past the
    // range end get a zero product)
    const long long k0 = kt + (long long)kItems * lane;
    int c[kItems];
    T v[kItems];
    if (VEC && k0 + kItems <= nnz) {
      const int4 c0 = ld_stream_v4(col + k0), c1 = ld_stream_v4(col + k0 + 4);
      c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
      c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
      load_vals8<SV, T>(val, k0, v);
    } else {
#pragma unroll
      for (int e = 0; e < kItems; ++e) {
        const long long k = k0 + e;
        c[e] = k < nnz ? ld_stream(col + k) : 0;
        v[e] = k < nnz ? (T)ld_val(val + k) : (T)0;
      }
    }
    T p[kItems];
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      const long long k = k0 + e;
      p[e] = (k >= k_lo && k < k_hi) ? v[e] * ld_ro(x + c[e]) : (T)0;
    }
    *reinterpret_cast<int4*>(mark + kItems * lane) = make_int4(-1, -1, -1, -1);
    *reinterpret_cast<int4*>(mark + kItems * lane + 4) = make_int4(-1, -1, -1, -1);
    __syncwarp();
    const long long lim = min(kt + kTile, k_hi);
    while (true) {  // row starts are non-decreasing: the rows inside form a prefix
      const int j = next_row + lane;
      const long long s = j < N ? (long long)__ldg(row_ptr + j) : LLONG_MAX;
      if (!hi_known) {
        const unsigned h = __ballot_sync(kFull, s >= b_hi);
        if (h) {
          hi_known = true;
          k_hi = min(__shfl_sync(kFull, s, __ffs(h) - 1), nnz);
        }
      }
      const bool in = s < min(lim, k_hi);
      if (in) atomicMax(mark + (int)(s - kt), j);
      const unsigned b = __ballot_sync(kFull, in);
      next_row += __popc(b);
      if (b != kFull) break;
    }
#pragma unroll
    for (int e = 0; e < kItems; ++e)
      if (k0 + e >= k_hi) p[e] = 0;
    __syncwarp();
    // rows: prefix maximum of the marks (items outside [k_lo, k_hi) join the
    // first or last row of the range with a zero product)
    const int4 m0 = *reinterpret_cast<const int4*>(mark + kItems * lane);
    const int4 m1 = *reinterpret_cast<const int4*>(mark + kItems * lane + 4);
    int r[kItems] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
    for (int e = 1; e < kItems; ++e) r[e] = max(r[e], r[e - 1]);
    int incl = r[kItems - 1];
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl = max(incl, t);
    }
    int before = __shfl_up_sync(kFull, incl, 1);
    before = max(lane == 0 ? -1 : before, base_row);
#pragma unroll
    for (int e = 0; e < kItems; ++e) r[e] = max(r[e], before);
    if (base_row < 0) {  // first tile: items before k_lo take the row that starts at k_lo
      const int fr = mark[(int)(k_lo - kt)];
#pragma unroll
      for (int e = 0; e < kItems; ++e)
        if (r[e] < 0) r[e] = fr;
    }
    __syncwarp();
    // the open row of the previous tile: continued by lane 0, or finished
    const int r00 = __shfl_sync(kFull, r[0], 0);
    if (carry_row >= 0 && r00 != carry_row) {
      if (lane == 0) y[carry_row] += carry;
      carry_row = -1;
    }
    if (lane == 0 && carry_row >= 0) p[0] = carry + p[0];
    // lane-local runs; the runs strictly inside a lane are whole rows
    const int start_row = r[0];
    int cur = start_row;
    T acc = 0, first_val = 0;
    bool internal = false;
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      if (r[e] != cur) {
        if (!internal) {
          internal = true;
          first_val = acc;
        } else {
          y[cur] += acc;
        }
        cur = r[e];
        acc = 0;
      }
      acc += p[e];
    }
    const int end_row = cur;
    const int prev_end = __shfl_up_sync(kFull, end_row, 1);
    const bool cont_prev = lane > 0 && start_row == prev_end;
    bool hf = internal || !cont_prev;  // this lane's last run does not continue the previous lane's
    T sum = acc;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      const T o = __shfl_up_sync(kFull, sum, off);
      const bool f = __shfl_up_sync(kFull, hf, off);
      if (lane >= off) {
        if (!hf) sum += o;
        hf = hf || f;
      }
    }
    const T from_prev = __shfl_up_sync(kFull, sum, 1);
    if (internal) y[start_row] += first_val + (cont_prev ? from_prev : (T)0);
    const int next_start = __shfl_down_sync(kFull, start_row, 1);
    if (lane < kWarp - 1 && next_start != end_row) y[end_row] += sum;
    carry_row = __shfl_sync(kFull, end_row, kWarp - 1);
    carry = __shfl_sync(kFull, sum, kWarp - 1);
    base_row = carry_row;
  }
  if (lane == 0 && carry_row >= 0) y[carry_row] += carry;
}

template <typename SV, typename T>
static int launch_csr_tiles(const int* row_ptr, const int* col, const SV* val, const T* x, T* y,
                            int N, long long nnz, int tiles_per_warp, cudaStream_t st) {
  const long long items = (long long)std::max(1, std::min(tiles_per_warp, 64)) * kTile;
  const long long warps = (nnz + items - 1) / items;
  const long long ctas = (warps + kWarpsPerCta - 1) / kWarpsPerCta;
  if (ctas > 0x7fffffffLL) {
    set_error("sb_spmv_csr: too many nonzero tiles");
    return SB_EINVAL;
  }
  const int threads = kWarpsPerCta * kWarp;
  if (aligned16(col) && aligned16(val))
    csr_tile_kernel<SV, T, true><<<(unsigned)ctas, threads, 0, st>>>(row_ptr, col, val, x, y, N,
                                                                     nnz, items);
  else
    csr_tile_kernel<SV, T, false><<<(unsigned)ctas, threads, 0, st>>>(row_ptr, col, val, x, y, N,
                                                                      nnz, items);
  SB_CHECK_LAUNCH("csr_tile_kernel");
  return SB_OK;
}

// ------------------------------------------------------------ CSR (block stream)

// Block-stream CSR: a warp owns 32 consecutive rows, as in the row-block
// kernel, but walks their nonzeros as one flat stream of 256-entry chunks:
// 8 consecutive entries per lane loaded with 16-byte vector loads and their
// 8 x gathers in flight together, whatever the row lengths.  Each entry's row
// is found among the block's row starts, which the lanes hold one each (a
// shuffle binary search for a lane's first entry, then shuffle steps across
// row ends).  Rows are summed by lane-local runs and a warp segmented scan;
// a row cut by a chunk boundary is carried into the next chunk.  Every
// complete row sum lands once in a per-warp shared array, and the block's
// rows are written at the end with one coalesced y[i] = y[i] + sum (rows
// without entries are not written).  The summation order is fixed by the
// matrix, so results are identical run to run.
template <typename SV, typename T, bool VEC>
__global__ void __launch_bounds__(kWarpsPerCta * kWarp)
    csr_block_stream_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                            const SV* __restrict__ val, const T* __restrict__ x,
                            T* __restrict__ y, int N, long long nnz) {
  __shared__ T rowsum_all[kWarpsPerCta][kWarp];
  const int lane = threadIdx.x & (kWarp - 1);
  T* rowsum = rowsum_all[threadIdx.x >> 5];
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w * kWarp >= N) return;
  const int r0 = (int)(w * kWarp);
  const int rr = r0 + lane;
  const int s_l = __ldg(row_ptr + min(rr, N));      // start of this lane's row
  const int n_l = __ldg(row_ptr + min(rr + 1, N));  // its end (next row's start)
  const bool has = rr < N && n_l > s_l;
  const T y_l = has ? y[rr] : (T)0;
  rowsum[lane] = (T)0;
  __syncwarp();
  const long long b_lo = __shfl_sync(kFull, s_l, 0);
  const long long b_hi = __shfl_sync(kFull, n_l, kWarp - 1);
  int carry_row = -1;
  T carry = 0;
  for (long long kb = b_lo & ~7LL; kb < b_hi; kb += kTile) {
    const long long k0 = kb + (long long)kItems * lane;
    int c[kItems];
    T v[kItems];
    if (VEC && k0 + kItems <= nnz) {
      const int4 c0 = ld_stream_v4(col + k0), c1 = ld_stream_v4(col + k0 + 4);
      c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
      c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
      load_vals8<SV, T>(val, k0, v);
    } else {
#pragma unroll
      for (int e = 0; e < kItems; ++e) {
        const long long k = k0 + e;
        c[e] = k < nnz ? ld_stream(col + k) : 0;
        v[e] = k < nnz ? (T)ld_val(val + k) : (T)0;
      }
    }
    T p[kItems];
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      const long long k = k0 + e;
      p[e] = (k >= b_lo && k < b_hi) ? v[e] * ld_ro(x + c[e]) : (T)0;
    }
    // row of each entry: the largest j with start_j <= k (empty rows share
    // their start with the next row and are skipped)
    int j = 0;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
      const long long sc = __shfl_sync(kFull, s_l, j + st);
      if (sc <= k0) j += st;
    }
    long long nb = __shfl_sync(kFull, n_l, j);
    int r[kItems];
    r[0] = j;
#pragma unroll
    for (int e = 1; e < kItems; ++e) {
      const long long k = k0 + e;
      bool need = k >= nb && j < kWarp - 1;
      while (__any_sync(kFull, need)) {
        const int j2 = need ? j + 1 : j;
        const long long nb2 = __shfl_sync(kFull, n_l, j2);
        if (need) {
          j = j2;
          nb = nb2;
        }
        need = k >= nb && j < kWarp - 1;
      }
      r[e] = j;
    }
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      const long long k = k0 + e;
      if (k < b_lo || k >= b_hi) r[e] = -1;  // not this block's entry (product 0)
    }
    // the open row of the previous chunk: continued by lane 0, or complete
    const int r00 = __shfl_sync(kFull, r[0], 0);
    if (carry_row >= 0 && r00 != carry_row) {
      if (lane == 0) rowsum[carry_row] = carry;
      carry_row = -1;
    }
    if (lane == 0 && carry_row >= 0) p[0] = carry + p[0];
    // lane-local runs; a run strictly inside a lane is a whole row
    const int start_row = r[0];
    int cur = start_row;
    T acc = 0, first_val = 0;
    bool internal = false;
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
      if (r[e] != cur) {
        if (!internal) {
          internal = true;
          first_val = acc;
        } else if (cur >= 0) {
          rowsum[cur] = acc;
        }
        cur = r[e];
        acc = 0;
      }
      acc += p[e];
    }
    const int end_row = cur;
    const int prev_end = __shfl_up_sync(kFull, end_row, 1);
    const bool cont_prev = lane > 0 && start_row == prev_end;
    bool hf = internal || !cont_prev;
    T sum = acc;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
      const T o = __shfl_up_sync(kFull, sum, off);
      const bool f = __shfl_up_sync(kFull, hf, off);
      if (lane >= off) {
        if (!hf) sum += o;
        hf = hf || f;
      }
    }
    const T from_prev = __shfl_up_sync(kFull, sum, 1);
    if (internal && start_row >= 0) rowsum[start_row] = first_val + (cont_prev ? from_prev : (T)0);
    const int next_start = __shfl_down_sync(kFull, start_row, 1);
    if (lane < kWarp - 1 && next_start != end_row && end_row >= 0) rowsum[end_row] = sum;
    carry_row = __shfl_sync(kFull, end_row, kWarp - 1);
    carry = __shfl_sync(kFull, sum, kWarp - 1);
  }
  if (lane == 0 && carry_row >= 0) rowsum[carry_row] = carry;
  __syncwarp();
  if (has) y[rr] = y_l + rowsum[lane];
}

template <typename SV, typename T>
static int launch_csr_block_stream(const int* row_ptr, const int* col, const SV* val, const T* x,
                                   T* y, int N, long long nnz, cudaStream_t st) {
  const long long warps = ((long long)N + kWarp - 1) / kWarp;
  const long long ctas = (warps + kWarpsPerCta - 1) / kWarpsPerCta;
  const int threads = kWarpsPerCta * kWarp;
  if (aligned16(col) && aligned16(val))
    csr_block_stream_kernel<SV, T, true><<<(unsigned)ctas, threads, 0, st>>>(row_ptr, col, val, x,
                                                                             y, N, nnz);
  else
    csr_block_stream_kernel<SV, T, false><<<(unsigned)ctas, threads, 0, st>>>(row_ptr, col, val,
                                                                              x, y, N, nnz);
  SB_CHECK_LAUNCH("csr_block_stream_kernel");
  return SB_OK;
}

// ------------------------------------------------------------ gather floor

// sum += val[k] * x[col[k]] over all entries: the column and value streams an
// SpMV must read and its x gathers, without any row structure.  8 entries
// per lane per step with vector loads, partial sums reduced per warp, one
// atomic per warp.
template <typename T>
__global__ void __launch_bounds__(256)
    gather_dot_kernel(const int* __restrict__ col, const T* __restrict__ val,
                      const T* __restrict__ x, long long nnz, double* __restrict__ out) {
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  T acc = 0;
  for (long long k0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kItems; k0 < nnz;
       k0 += nthreads * kItems) {
    int c[kItems];
    T v[kItems];
    if (k0 + kItems <= nnz) {
      const int4 c0 = ld_stream_v4(col + k0), c1 = ld_stream_v4(col + k0 + 4);
      c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
      c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
      load_vals8<T, T>(val, k0, v);
    } else {
#pragma unroll
      for (int e = 0; e < kItems; ++e) {
        c[e] = k0 + e < nnz ? ld_stream(col + k0 + e) : 0;
        v[e] = k0 + e < nnz ? ld_stream(val + k0 + e) : (T)0;
      }
    }
#pragma unroll
    for (int e = 0; e < kItems; ++e) acc += v[e] * ld_ro(x + c[e]);
  }
#pragma unroll
  for (int off = kWarp / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off);
  if ((threadIdx.x & (kWarp - 1)) == 0) atomicAdd(out, (double)acc);
}

// ------------------------------------------------------------ DIA / ELL

template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// One row per thread; diagonals in stored order, each added with a
// separately rounded product (src/sequential/src/sparse_opt_32.wat:290-407).
// The in-band test is a predicate so that the unrolled loop issues the data
// and x loads of several diagonals before their dependent additions.
template <typename SV, typename T>
__global__ void __launch_bounds__(256)
    dia_row_kernel(const int* __restrict__ offset, const SV* __restrict__ data, int N, int nd,
                   int stride, const T* __restrict__ x, T* __restrict__ y) {
  // smallest and largest offset (whatever their order), for the interior test
  __shared__ int kext[2];
  if (threadIdx.x == 0) {
    kext[0] = 0x7fffffff;
    kext[1] = -0x7fffffff - 1;
  }
  __syncthreads();
  for (int d = threadIdx.x; d < nd; d += blockDim.x) {
    const int k = __ldg(offset + d);
    atomicMin(&kext[0], k);
    atomicMax(&kext[1], k);
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T t = y[i];
  const long long move = (long long)N - stride;
  // interior rows (every diagonal in band) walk the diagonals with pointer
  // increments and no predicates
  const int kmin = kext[0], kmax = kext[1];
  if (move == 0 && (long long)i + kmin >= 0 && (long long)i + kmax < N) {
    const SV* dp = data + i;
    const T* xp = x + i;
#pragma unroll 4
    for (int d = 0; d < nd; ++d, dp += stride)
      t = add_rn(mul_rn((T)ld_val(dp), ld_ro(xp + __ldg(offset + d))), t);
    y[i] = t;
    return;
  }
#pragma unroll 4
  for (int d = 0; d < nd; ++d) {
    const int k = __ldg(offset + d);
    const bool in = (unsigned)(i + k) < (unsigned)N;
    const long long idx = (long long)d * stride + i - (k < 0 ? move : 0);
    T a = in ? (T)ld_val(data + idx) : (T)0;
    T b = in ? ld_ro(x + i + k) : (T)0;
    T p = mul_rn(a, b);
    t = in ? add_rn(p, t) : t;
  }
  y[i] = t;
}

// dia_row_kernel with the diagonal count ND fixed at compile time (1..16):
// the offsets and their extremes are held in registers (no shared memory, no
// block barrier), and a row's ND data loads and ND x loads are all issued
// before its additions, which keep the stored order (bit-identical to the
// runtime-count kernel).
template <typename SV, typename T, int ND>
__global__ void __launch_bounds__(256)
    dia_rows_nd(const int* __restrict__ offset, const SV* __restrict__ data, int N, int stride,
                const T* __restrict__ x, T* __restrict__ y) {
  int k[ND];
  int kmin = 0x7fffffff, kmax = -0x7fffffff - 1;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    k[d] = __ldg(offset + d);
    kmin = min(kmin, k[d]);
    kmax = max(kmax, k[d]);
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T t = y[i];
  const long long move = (long long)N - stride;
  T a[ND], b[ND];
  if (move == 0 && (long long)i + kmin >= 0 && (long long)i + kmax < N) {
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      a[d] = (T)ld_val(data + (long long)d * stride + i);
      b[d] = ld_ro(x + i + k[d]);
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) t = add_rn(mul_rn(a[d], b[d]), t);
    y[i] = t;
    return;
  }
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const bool in = (unsigned)(i + k[d]) < (unsigned)N;
    const long long idx = (long long)d * stride + i - (k[d] < 0 ? move : 0);
    a[d] = in ? (T)ld_val(data + idx) : (T)0;
    b[d] = in ? ld_ro(x + i + k[d]) : (T)0;
  }
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const bool in = (unsigned)(i + k[d]) < (unsigned)N;
    const T p = mul_rn(a[d], b[d]);
    t = in ? add_rn(p, t) : t;
  }
  y[i] = t;
}

// dia_rows_nd with R rows per thread (rows base + r*256, so that each load
// instruction of a warp stays coalesced): the R rows' data, x and y loads
// are all issued before their additions, which puts R times the bytes in
// flight per thread -- for 4-byte values and few diagonals one row per
// thread leaves too few loads in flight.  Every row is computed as in
// dia_rows_nd (bit-identical).
template <typename SV, typename T, int ND, int R>
__global__ void __launch_bounds__(256)
    dia_rows_multi(const int* __restrict__ offset, const SV* __restrict__ data, int N, int stride,
                   const T* __restrict__ x, T* __restrict__ y) {
  int k[ND];
  const SV* dp[ND];  // diagonal d's entry of row 0 (rows below the band shift by N - stride)
  const long long move = (long long)N - stride;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    k[d] = __ldg(offset + d);
    dp[d] = data + (long long)d * stride - (k[d] < 0 ? move : 0);
  }
  const int base = blockIdx.x * (256 * R) + threadIdx.x;
  T a[R][ND], b[R][ND], t[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = base + r * 256;
    const bool valid = i < N;
    t[r] = valid ? y[i] : (T)0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const bool in = valid && (unsigned)(i + k[d]) < (unsigned)N;
      a[r][d] = in ? (T)ld_val(dp[d] + i) : (T)0;
      b[r][d] = in ? ld_ro(x + i + k[d]) : (T)0;
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = base + r * 256;
    if (i >= N) continue;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const bool in = (unsigned)(i + k[d]) < (unsigned)N;
      const T p = mul_rn(a[r][d], b[r][d]);
      t[r] = in ? add_rn(p, t[r]) : t[r];
    }
    y[i] = t[r];
  }
}

// BF16 or FP32 data with f32 vectors, up to 16 diagonals: two adjacent rows
// per thread (rows 2j and 2j+1), so that one 4- or 8-byte load brings both
// rows' values of a diagonal (with stride == N and N even the pair is
// aligned in every diagonal), y moves as a float2 and x as a float2 where
// i + k is even.
// One row per thread with 2-byte loads left too few bytes in flight (ncu,
// 5-point Laplacian 4096^2: DRAM 43% of peak, long-scoreboard stalls 17.8
// per issue at 85% warps active).  A pair with a row outside the band's
// full range takes dia_rows_nd's per-row form.  Every row is computed as in
// dia_rows_nd (bit-identical: a bf16 value widens to f32 by a 16-bit shift).
__device__ __forceinline__ void ld_pair(const __nv_bfloat16* p, float& a0, float& a1) {
  const unsigned w = (unsigned)ld_stream(reinterpret_cast<const int*>(p));
  a0 = __uint_as_float(w << 16);
  a1 = __uint_as_float(w & 0xffff0000u);
}
__device__ __forceinline__ void ld_pair(const float* p, float& a0, float& a1) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  a0 = v.x;
  a1 = v.y;
}

template <typename SV, int ND>
__global__ void __launch_bounds__(256)
    dia_rows_pair(const int* __restrict__ offset, const SV* __restrict__ data,
                  int N, const float* __restrict__ x, float* __restrict__ y) {
  int k[ND];
  int kmin = 0x7fffffff, kmax = -0x7fffffff - 1;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    k[d] = __ldg(offset + d);
    kmin = min(kmin, k[d]);
    kmax = max(kmax, k[d]);
  }
  const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= N) return;
  if ((long long)i + kmin >= 0 && (long long)i + 1 + kmax < N) {
    float2 t = *reinterpret_cast<const float2*>(y + i);
    float a0[ND], a1[ND], b0[ND], b1[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      ld_pair(data + (long long)d * N + i, a0[d], a1[d]);
      if ((k[d] & 1) == 0) {
        const float2 xv = __ldg(reinterpret_cast<const float2*>(x + i + k[d]));
        b0[d] = xv.x;
        b1[d] = xv.y;
      } else {
        b0[d] = ld_ro(x + i + k[d]);
        b1[d] = ld_ro(x + i + 1 + k[d]);
      }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      t.x = add_rn(mul_rn(a0[d], b0[d]), t.x);
      t.y = add_rn(mul_rn(a1[d], b1[d]), t.y);
    }
    *reinterpret_cast<float2*>(y + i) = t;
    return;
  }
#pragma unroll 1
  for (int r = i; r < i + 2 && r < N; ++r) {
    float t = y[r];
    float a[ND], b[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const bool in = (unsigned)(r + k[d]) < (unsigned)N;
      a[d] = in ? (float)ld_val(data + (long long)d * N + r) : 0.f;
      b[d] = in ? ld_ro(x + r + k[d]) : 0.f;
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const bool in = (unsigned)(r + k[d]) < (unsigned)N;
      const float p = mul_rn(a[d], b[d]);
      t = in ? add_rn(p, t) : t;
    }
    y[r] = t;
  }
}

// BF16 data, up to 16 diagonals, N a multiple of 4: four adjacent rows per
// thread, one 8-byte load of a diagonal's four values, x as a float4 where
// i + k is a multiple of 4 (two float2 where it is even, else four
// values), y as a float4.  A quad with a row outside the band's full range
// takes the per-row form.  Every row is computed as in dia_rows_nd.
template <int ND>
__global__ void __launch_bounds__(256)
    dia_rows_quad_bf16(const int* __restrict__ offset, const __nv_bfloat16* __restrict__ data,
                       int N, const float* __restrict__ x, float* __restrict__ y) {
  int k[ND];
  int kmin = 0x7fffffff, kmax = -0x7fffffff - 1;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    k[d] = __ldg(offset + d);
    kmin = min(kmin, k[d]);
    kmax = max(kmax, k[d]);
  }
  const int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= N) return;
  if ((long long)i + kmin >= 0 && (long long)i + 3 + kmax < N) {
    float4 t = *reinterpret_cast<const float4*>(y + i);
    float a[ND][4], b[ND][4];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const uint2 w = ld_stream_v4(reinterpret_cast<const unsigned short*>(data) +
                                   (long long)d * N + i);
      a[d][0] = __uint_as_float(w.x << 16);
      a[d][1] = __uint_as_float(w.x & 0xffff0000u);
      a[d][2] = __uint_as_float(w.y << 16);
      a[d][3] = __uint_as_float(w.y & 0xffff0000u);
      const float* xp = x + i + k[d];
      if ((k[d] & 3) == 0) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(xp));
        b[d][0] = v.x; b[d][1] = v.y; b[d][2] = v.z; b[d][3] = v.w;
      } else if ((k[d] & 1) == 0) {
        const float2 v0 = __ldg(reinterpret_cast<const float2*>(xp));
        const float2 v1 = __ldg(reinterpret_cast<const float2*>(xp + 2));
        b[d][0] = v0.x; b[d][1] = v0.y; b[d][2] = v1.x; b[d][3] = v1.y;
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) b[d][u] = ld_ro(xp + u);
      }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      t.x = add_rn(mul_rn(a[d][0], b[d][0]), t.x);
      t.y = add_rn(mul_rn(a[d][1], b[d][1]), t.y);
      t.z = add_rn(mul_rn(a[d][2], b[d][2]), t.z);
      t.w = add_rn(mul_rn(a[d][3], b[d][3]), t.w);
    }
    *reinterpret_cast<float4*>(y + i) = t;
    return;
  }
#pragma unroll 1
  for (int r = i; r < i + 4 && r < N; ++r) {
    float t = y[r];
    float av[ND], bv[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const bool in = (unsigned)(r + k[d]) < (unsigned)N;
      av[d] = in ? ld_val(data + (long long)d * N + r) : 0.f;
      bv[d] = in ? ld_ro(x + r + k[d]) : 0.f;
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const bool in = (unsigned)(r + k[d]) < (unsigned)N;
      const float p = mul_rn(av[d], bv[d]);
      t = in ? add_rn(p, t) : t;
    }
    y[r] = t;
  }
}

template <typename SV, typename T>
static void launch_dia(const int* offset, const SV* data, int N, int nd, int stride, const T* x,
                       T* y, cudaStream_t st) {
  const unsigned blocks = (unsigned)((N + 255) / 256);
  if constexpr (sizeof(T) == 4) {
    // BF16 / FP32 data: two rows per thread where the pair loads are aligned
    const bool pair_ok = nd >= 1 && nd <= 16 && stride == N && (N % 2) == 0 &&
                         (reinterpret_cast<uintptr_t>(data) & (2 * sizeof(SV) - 1)) == 0 &&
                         (reinterpret_cast<uintptr_t>(x) & 7u) == 0 &&
                         (reinterpret_cast<uintptr_t>(y) & 7u) == 0;
    if constexpr (sizeof(SV) == 2) {
      const bool quad_ok = pair_ok && (N % 4) == 0 &&
                           (reinterpret_cast<uintptr_t>(data) & 7u) == 0 &&
                           (reinterpret_cast<uintptr_t>(x) & 15u) == 0 &&
                           (reinterpret_cast<uintptr_t>(y) & 15u) == 0;
      if (quad_ok) {
        const unsigned qblocks = (unsigned)((N / 4 + 255) / 256);
        switch (nd) {
#define SB_DIA_QUAD(n)                                                                   \
  case n:                                                                                \
    dia_rows_quad_bf16<n><<<qblocks, 256, 0, st>>>(offset, data, N, x, y);             \
    return;
          SB_DIA_QUAD(1) SB_DIA_QUAD(2) SB_DIA_QUAD(3) SB_DIA_QUAD(4) SB_DIA_QUAD(5)
          SB_DIA_QUAD(6) SB_DIA_QUAD(7) SB_DIA_QUAD(8)
#undef SB_DIA_QUAD
          default: break;
        }
      }
    }
    if (pair_ok) {
      const unsigned pblocks = (unsigned)((N / 2 + 255) / 256);
      switch (nd) {
#define SB_DIA_PAIR(n)                                                                   \
  case n:                                                                                \
    dia_rows_pair<SV, n><<<pblocks, 256, 0, st>>>(offset, data, N, x, y);              \
    return;
        SB_DIA_PAIR(1) SB_DIA_PAIR(2) SB_DIA_PAIR(3) SB_DIA_PAIR(4) SB_DIA_PAIR(5)
        SB_DIA_PAIR(6) SB_DIA_PAIR(7) SB_DIA_PAIR(8) SB_DIA_PAIR(9) SB_DIA_PAIR(10)
        SB_DIA_PAIR(11) SB_DIA_PAIR(12) SB_DIA_PAIR(13) SB_DIA_PAIR(14) SB_DIA_PAIR(15)
        SB_DIA_PAIR(16)
#undef SB_DIA_PAIR
        default: break;
      }
    }
  }
  // few diagonals of 4-byte values where the pair form does not apply: 4
  // rows per thread (2 for 5..8), strided by 256; the row index stays
  // 32-bit (N < 2^31 and the grid covers N rows).  Measured on B200,
  // 5-point Laplacian 4096^2: FP32 0.1068 (one row per thread) -> 0.1006
  // (this form) -> 0.0823 ms (the pair form); BF16 data 0.1016 -> 0.3035 ms
  // in this form, 0.0802 ms in the pair form.
  if constexpr (sizeof(SV) == 4) {
    if (nd <= 8 && (long long)N + 256LL * 4 < 0x7fffffffLL) {
    switch (nd) {
#define SB_DIA_MR(n, r)                                                                      \
  case n:                                                                                    \
    dia_rows_multi<SV, T, n, r><<<(unsigned)((N + 256 * r - 1) / (256 * r)), 256, 0, st>>>( \
        offset, data, N, stride, x, y);                                                      \
    return;
      SB_DIA_MR(1, 4) SB_DIA_MR(2, 4) SB_DIA_MR(3, 4) SB_DIA_MR(4, 4) SB_DIA_MR(5, 2)
      SB_DIA_MR(6, 2) SB_DIA_MR(7, 2) SB_DIA_MR(8, 2)
#undef SB_DIA_MR
      default: break;
    }
    }
  }
  switch (nd) {
#define SB_DIA_ND(n) \
  case n: dia_rows_nd<SV, T, n><<<blocks, 256, 0, st>>>(offset, data, N, stride, x, y); return;
    SB_DIA_ND(1) SB_DIA_ND(2) SB_DIA_ND(3) SB_DIA_ND(4) SB_DIA_ND(5) SB_DIA_ND(6) SB_DIA_ND(7)
    SB_DIA_ND(8) SB_DIA_ND(9) SB_DIA_ND(10) SB_DIA_ND(11) SB_DIA_ND(12) SB_DIA_ND(13)
    SB_DIA_ND(14) SB_DIA_ND(15) SB_DIA_ND(16)
#undef SB_DIA_ND
    default:
      dia_row_kernel<SV, T><<<blocks, 256, 0, st>>>(offset, data, N, nd, stride, x, y);
  }
}

// One row per thread over the nc column-major slots, padding included
// (src/sequential/src/sparse_opt_32.wat:427-479).
template <typename T>
__global__ void __launch_bounds__(256)
    ell_row_kernel(const int* __restrict__ indices, const T* __restrict__ data, int N, int nc,
                   const T* __restrict__ x, T* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T t = y[i];
  const T* dp = data + i;
  const int* ip = indices + i;
  for (int k = 0; k < nc; ++k) {
    const long long o = (long long)k * N;
    t = add_rn(mul_rn(ld_stream(dp + o), ld_ro(x + ld_stream(ip + o))), t);
  }
  y[i] = t;
}

// ------------------------------------------------------------ launchers


template <typename S, int T, int STAGES>
static int launch_csr_stream(const int* row_ptr, const int* col, const S* val, const S* x, S* y,
                             int N, long long nnz, cudaStream_t st) {
  const long long ntiles = (nnz + T - 1) / T;
  auto kern = csr_stream_kernel<S, T, STAGES>;
  const size_t smem = sizeof(CsrStreamSmem<S, T, STAGES>);
  static int configured[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    SB_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    configured[dev] = 1;
  }
  int per_sm = 0;
  SB_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads,
                                                              smem));
  if (per_sm < 1) per_sm = 1;
  const long long max_ctas = (long long)per_sm * sm_count();
  const long long ctas = std::min(ntiles, max_ctas);
  const long long tpc = (ntiles + ctas - 1) / ctas;
  const long long used = (ntiles + tpc - 1) / tpc;
  int* status = device_status_word();
  if (!status) {
    set_error("sb_spmv_csr: device status word unavailable");
    return SB_ENOMEM;
  }
  kern<<<(unsigned)used, kStreamThreads, smem, st>>>(row_ptr, col, val, x, y, N, nnz, ntiles,
                                                     tpc, status);
  SB_CHECK_LAUNCH("csr_stream_kernel");
  return SB_OK;
}

// CSR dispatch.  opts (may be null = row blocks with default options):
// kernel 0 = row blocks (lanes_per_row / unroll 0 = default), 1 = streamed
// tiles of 1024 nonzeros, or 2048 with unroll = 2048 (needs 16-byte aligned
// col/val, else row blocks), 2 = nonzero tiles (unroll = tiles per warp).
template <typename S, typename A>
static int launch_csr(const int* row_ptr, const int* col, const S* val, const S* x, S* y, int N,
                      long long nnz, const sb_csr_opts* opts, cudaStream_t st) {
  const int kernel = opts ? opts->kernel : 0;
  if (kernel == 2) return launch_csr_tiles<S, S>(row_ptr, col, val, x, y, N, nnz, opts->unroll, st);
  if (kernel == 3) return launch_csr_block_stream<S, S>(row_ptr, col, val, x, y, N, nnz, st);
  if (kernel == 1 && aligned16(col) && aligned16(val)) {
    if (opts->unroll == 2048) return launch_csr_stream<S, 2048, 3>(row_ptr, col, val, x, y, N, nnz, st);
    return launch_csr_stream<S, 1024, 4>(row_ptr, col, val, x, y, N, nnz, st);
  }
  return launch_csr_rows<S, S>(row_ptr, col, val, x, y, N, nnz, opts ? opts->lanes_per_row : 0,
                               opts ? opts->unroll : 0, opts ? opts->grid : 0, st);
}

template <typename S, typename A>
static int launch_coo(const int* row, const int* col, const S* val, const S* x, S* y,
                      long long nnz, bool sorted, cudaStream_t st) {
  const long long ntiles = (nnz + kTile - 1) / kTile;
  const bool vec = aligned16(row) && aligned16(col) && aligned16(val);
  auto kern = vec ? (sorted ? coo_tile_kernel<S, A, true, true> : coo_tile_kernel<S, A, true, false>)
                  : (sorted ? coo_tile_kernel<S, A, false, true> : coo_tile_kernel<S, A, false, false>);
  const int threads = kWarpsPerCta * kWarp;
  const long long max_warps = (long long)resident_ctas(kern, threads) * kWarpsPerCta;
  const long long warps = std::min(ntiles, max_warps);
  const long long tpw = (ntiles + warps - 1) / warps;
  const long long used_warps = (ntiles + tpw - 1) / tpw;
  const long long ctas = (used_warps + kWarpsPerCta - 1) / kWarpsPerCta;
  kern<<<(unsigned)ctas, threads, 0, st>>>(row, col, val, x, y, nnz, ntiles, tpw);
  SB_CHECK_LAUNCH("coo_tile_kernel");
  return SB_OK;
}

static int check_dtype(int dtype, const char* fn) {
  if (dtype != SB_F32 && dtype != SB_F64) {
    set_error("%s: dtype %d not supported (SB_F32=0, SB_F64=1)", fn, dtype);
    return SB_EINVAL;
  }
  return SB_OK;
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_spmv_csr_allgather(int dtype, const int32_t* row_ptr, const int32_t* col,
                          const void* val, const void* x, const void* y_in, int32_t rows,
                          int64_t nnz, int64_t row_offset, void* const* dst, int32_t ndst,
                          const sb_csr_opts* opts, void* stream) {
  SB_TRACE("sb_spmv_csr_allgather");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64 || dtype == SB_BF16,
             "sb_spmv_csr_allgather: bad dtype");
  SB_REQUIRE(rows >= 0 && nnz >= 0 && row_offset >= 0, "sb_spmv_csr_allgather: negative size");
  SB_REQUIRE(nnz <= 0x7fffffffLL, "sb_spmv_csr_allgather: nnz exceeds int32 row_ptr range");
  SB_REQUIRE(ndst >= 1 && ndst <= kMaxScatter && dst,
             "sb_spmv_csr_allgather: 1 <= ndst <= 8 destinations required");
  SB_REQUIRE((reinterpret_cast<uintptr_t>(dst) & 7u) == 0,
             "sb_spmv_csr_allgather: destination array not 8-byte aligned");
  if (opts) {
    const int l = opts->lanes_per_row;
    SB_REQUIRE(l == 0 || l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32,
               "sb_spmv_csr_allgather: lanes_per_row must be 0 or a power of two <= 32");
    SB_REQUIRE(opts->grid == 0 || opts->grid == 1, "sb_spmv_csr_allgather: grid must be 0 or 1");
  }
  if (rows == 0) return SB_OK;
  SB_REQUIRE(row_ptr && y_in && (nnz == 0 || (col && val && x)),
             "sb_spmv_csr_allgather: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  const int lanes = opts ? opts->lanes_per_row : 0, unroll = opts ? opts->unroll : 0;
  const int grid = opts ? opts->grid : 0;
  const unsigned long long* dd = reinterpret_cast<const unsigned long long*>(dst);
  if (dtype == SB_F64) {
    YScatter<double> out{};
    out.d = dd;
    out.n = ndst;
    out.r0 = row_offset;
    return launch_csr_rows_out<double, double>(row_ptr, col, (const double*)val,
                                               (const double*)x, (const double*)y_in, out, rows,
                                               nnz, lanes, unroll, grid, st);
  }
  YScatter<float> out{};
  out.d = dd;
  out.n = ndst;
  out.r0 = row_offset;
  if (dtype == SB_BF16)
    return launch_csr_rows_out<__nv_bfloat16, float>(row_ptr, col, (const __nv_bfloat16*)val,
                                                     (const float*)x, (const float*)y_in, out,
                                                     rows, nnz, lanes, unroll, grid, st);
  return launch_csr_rows_out<float, float>(row_ptr, col, (const float*)val, (const float*)x,
                                           (const float*)y_in, out, rows, nnz, lanes, unroll,
                                           grid, st);
}

int sb_spmv_csr_ex(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                   const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                   const sb_csr_opts* opts, void* stream) {
  SB_TRACE("sb_spmv_csr_ex");
  int r = dtype == SB_BF16 ? SB_OK : check_dtype(dtype, "sb_spmv_csr");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && inner_max >= 0, "sb_spmv_csr: negative size");
  SB_REQUIRE(nnz <= 0x7fffffffLL, "sb_spmv_csr: nnz exceeds int32 row_ptr range");
  if (opts) {
    SB_REQUIRE(opts->kernel >= 0 && opts->kernel <= 3, "sb_spmv_csr: unknown kernel %d",
               opts->kernel);
    const int l = opts->lanes_per_row;
    SB_REQUIRE(l == 0 || l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32,
               "sb_spmv_csr: lanes_per_row must be 0 or a power of two <= 32");
    SB_REQUIRE(opts->grid == 0 || opts->grid == 1, "sb_spmv_csr: grid must be 0 or 1");
  }
  if (N == 0 || nnz == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col && val && x && y, "sb_spmv_csr: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_BF16 && opts && opts->kernel == 2)
      r = launch_csr_tiles<__nv_bfloat16, float>(row_ptr, col, (const __nv_bfloat16*)val,
                                                 (const float*)x, (float*)y, N, nnz, opts->unroll,
                                                 st);
    else if (dtype == SB_BF16 && opts && opts->kernel == 3)
      r = launch_csr_block_stream<__nv_bfloat16, float>(row_ptr, col, (const __nv_bfloat16*)val,
                                                        (const float*)x, (float*)y, N, nnz, st);
    else if (dtype == SB_BF16)
      r = launch_csr_rows<__nv_bfloat16, float>(row_ptr, col, (const __nv_bfloat16*)val,
                                                (const float*)x, (float*)y, N, nnz,
                                                opts ? opts->lanes_per_row : 0,
                                                opts ? opts->unroll : 0, opts ? opts->grid : 0,
                                                st);
    else if (dtype == SB_F32)
      r = launch_csr<float, float>(row_ptr, col, (const float*)val, (const float*)x, (float*)y, N,
                                   nnz, opts, st);
    else
      r = launch_csr<double, double>(row_ptr, col, (const double*)val, (const double*)x,
                                     (double*)y, N, nnz, opts, st);
    if (r) return r;
  }
  return SB_OK;
}

int sb_spmv_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                void* stream) {
  SB_TRACE("sb_spmv_csr");
  return sb_spmv_csr_ex(dtype, row_ptr, col, val, x, y, N, nnz, inner_max, nullptr, stream);
}

int sb_csr_autotune(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                    const void* x, int32_t N, int64_t nnz, int32_t reps, sb_csr_opts* best,
                    float* best_ms, void* stream) {
  SB_TRACE("sb_csr_autotune");
  int r = dtype == SB_BF16 ? SB_OK : check_dtype(dtype, "sb_csr_autotune");
  if (r) return r;
  SB_REQUIRE(best && N >= 0 && nnz >= 0, "sb_csr_autotune: bad argument");
  best->kernel = 0;
  best->lanes_per_row = default_lanes(N, nnz);
  best->unroll = 4;
  best->grid = 0;
  if (best_ms) *best_ms = 0.f;
  if (N == 0 || nnz == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col && val && x, "sb_csr_autotune: null pointer");
  if ((r = ensure_device())) return r;
  if (reps <= 0) reps = 5;
  cudaStream_t st = as_stream(stream);
  // candidates around the mean row length: lanes in {d/4, d/2, d, 2d}, unroll {2, 4, 8},
  // both grids, plus the streamed-tile kernel and the nonzero-tile kernel with
  // 8 tiles per warp
  const int d = default_lanes(N, nnz);
  sb_csr_opts cand[32];
  int nc = 0;
  for (int lanes : {d / 4, d / 2, d, d * 2}) {
    if (lanes < 1 || lanes > 32) continue;
    for (int u : {2, 4, 8})
      for (int g : {0, 1}) cand[nc++] = sb_csr_opts{0, lanes, u, g};
  }
  cand[nc++] = sb_csr_opts{1, 0, 1024, 0};
  cand[nc++] = sb_csr_opts{2, 0, 8, 0};
  cand[nc++] = sb_csr_opts{3, 0, 0, 0};
  void* ywork = nullptr;
  const size_t ysize = dtype == SB_BF16 ? sizeof(float) : dtype_size(dtype);  // y is f32 for BF16
  if ((r = scratch_alloc(&ywork, ysize * (size_t)N, st))) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(ywork, 0, ysize * (size_t)N, st));
  cudaEvent_t e0, e1;
  SB_CHECK_CUDA(cudaEventCreate(&e0));
  SB_CHECK_CUDA(cudaEventCreate(&e1));
  float best_t = 3.0e38f;
  for (int c = 0; c < nc && !r; ++c) {
    r = sb_spmv_csr_ex(dtype, row_ptr, col, val, x, ywork, N, nnz, 1, &cand[c], stream);
    if (r) break;
    cudaEventRecord(e0, st);
    r = sb_spmv_csr_ex(dtype, row_ptr, col, val, x, ywork, N, nnz, reps, &cand[c], stream);
    cudaEventRecord(e1, st);
    if (r) break;
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) { r = cuda_status(e, "sb_csr_autotune"); break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= reps;
    if (ms < best_t) {
      best_t = ms;
      *best = cand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  scratch_free(ywork, st);
  if (best_ms) *best_ms = best_t;
  return r;
}

int sb_gather_dot(int dtype, const int32_t* col, const void* val, const void* x, int64_t nnz,
                  double* out, void* stream) {
  SB_TRACE("sb_gather_dot");
  int r = check_dtype(dtype, "sb_gather_dot");
  if (r) return r;
  SB_REQUIRE(nnz >= 0, "sb_gather_dot: negative size");
  if (nnz == 0) return SB_OK;
  SB_REQUIRE(col && val && x && out, "sb_gather_dot: null pointer");
  SB_REQUIRE(aligned16(col) && aligned16(val), "sb_gather_dot: col and val must be 16-byte aligned");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  const long long steps = (nnz + kItems - 1) / kItems;
  const long long per = 256;
  auto kf = gather_dot_kernel<float>;
  auto kd = gather_dot_kernel<double>;
  const long long maxc = dtype == SB_F32 ? resident_ctas(kf, 256) : resident_ctas(kd, 256);
  const unsigned ctas = (unsigned)std::max(1LL, std::min((steps + per - 1) / per, maxc));
  if (dtype == SB_F32)
    kf<<<ctas, 256, 0, st>>>(col, (const float*)val, (const float*)x, nnz, out);
  else
    kd<<<ctas, 256, 0, st>>>(col, (const double*)val, (const double*)x, nnz, out);
  SB_CHECK_LAUNCH("gather_dot_kernel");
  return SB_OK;
}

int sb_spmv_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                void* stream) {
  SB_TRACE("sb_spmv_coo");
  return sb_spmv_coo_ex(dtype, row, col, val, x, y, N, nnz, inner_max, 0, stream);
}

int sb_spmv_coo_ex(int dtype, const int32_t* row, const int32_t* col, const void* val,
                   const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                   int32_t flags, void* stream) {
  SB_TRACE("sb_spmv_coo_ex");
  int r = check_dtype(dtype, "sb_spmv_coo");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && inner_max >= 0, "sb_spmv_coo: negative size");
  if (N == 0 || nnz == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(row && col && val && x && y, "sb_spmv_coo: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  // A plain add reads y and waits for it; an atomic add is sent without a
  // reply.  Dropping the atomics pays where rows are short and many (banded,
  // 11 per row: 0.163 -> 0.130 ms) and costs where they are long and few
  // (power-law, 20.5 per row: 0.225 -> 0.232 ms), so the sorted-rows kernel
  // is taken for a mean row length of at most 16.  (Loading y of the lane's
  // rows while the gathers are in flight, then storing without a wait, was
  // measured: banded 0.1356 ms, power-law no faster than the atomics.)
  const bool sorted = (flags & SB_COO_ROWS_SORTED) != 0 && nnz <= 16LL * N;
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_F32)
      r = launch_coo<float, float>(row, col, (const float*)val, (const float*)x, (float*)y, nnz,
                                   sorted, st);
    else
      r = launch_coo<double, double>(row, col, (const double*)val, (const double*)x, (double*)y,
                                     nnz, sorted, st);
    if (r) return r;
  }
  return SB_OK;
}

int sb_spmv_dia(int dtype, const int32_t* offset, const void* data, int32_t N, int32_t nd,
                int32_t stride, const void* x, void* y, int32_t inner_max, void* stream) {
  SB_TRACE("sb_spmv_dia");
  int r = dtype == SB_BF16 ? SB_OK : check_dtype(dtype, "sb_spmv_dia");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nd >= 0 && inner_max >= 0, "sb_spmv_dia: negative size");
  SB_REQUIRE(stride >= N, "sb_spmv_dia: stride %d < N %d", stride, N);
  if (N == 0 || nd == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(offset && data && x && y, "sb_spmv_dia: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_F32)
      launch_dia<float, float>(offset, (const float*)data, N, nd, stride, (const float*)x,
                               (float*)y, st);
    else if (dtype == SB_BF16)
      launch_dia<__nv_bfloat16, float>(offset, (const __nv_bfloat16*)data, N, nd, stride,
                                       (const float*)x, (float*)y, st);
    else
      launch_dia<double, double>(offset, (const double*)data, N, nd, stride, (const double*)x,
                                 (double*)y, st);
    SB_CHECK_LAUNCH("dia_row_kernel");
  }
  return SB_OK;
}

int sb_spmv_ell(int dtype, const int32_t* indices, const void* data, int32_t N, int32_t nc,
                const void* x, void* y, int32_t inner_max, void* stream) {
  SB_TRACE("sb_spmv_ell");
  int r = check_dtype(dtype, "sb_spmv_ell");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nc >= 0 && inner_max >= 0, "sb_spmv_ell: negative size");
  if (N == 0 || nc == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(indices && data && x && y, "sb_spmv_ell: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  const unsigned blocks = (unsigned)((N + 255) / 256);
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_F32)
      ell_row_kernel<float><<<blocks, 256, 0, st>>>(indices, (const float*)data, N, nc,
                                                    (const float*)x, (float*)y);
    else
      ell_row_kernel<double><<<blocks, 256, 0, st>>>(indices, (const double*)data, N, nc,
                                                     (const double*)x, (double*)y);
    SB_CHECK_LAUNCH("ell_row_kernel");
  }
  return SB_OK;
}

}  // extern "C"
