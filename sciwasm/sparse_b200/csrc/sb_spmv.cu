// sb_spmv.cu -- SpMV kernels (y <- y + A x) for COO, CSR, DIA and ELL.
//
// Reference loops: src/sequential/src/sparse_opt_32.wat:175-498 (f32) and
// src/sequential/src/sparse_opt_64.wat:187-515 (f64).  The reference walks
// storage order on one core (or splits rows / nnz over Web Workers,
// src/parallel/src/sparse32.js:2637-2821).  Here:
//   * CSR is a merge-path kernel: every warp consumes a fixed number of
//     (row-end + nonzero) merge items, so rows of any length distribution
//     give equal work per warp; col/val are streamed with 128-bit loads into
//     shared memory and reduced with a per-lane walk plus a warp segmented
//     scan (rows per warp adapt to the row lengths by construction).
//   * COO is the same tile scheme keyed on the row array; every row segment
//     is added with one atomic, so unsorted input is accepted.
//   * DIA and ELL assign one row per thread and keep the reference's per-row
//     addition order (separately rounded mul and add), so their results are
//     bit-identical to the reference's serial loops.
#include <algorithm>

#include "sb_common.cuh"

namespace sb {

constexpr int kWarp = 32;
constexpr int kItems = 8;                  // merge items per lane per tile
constexpr int kTile = kWarp * kItems;      // 256 merge items per warp tile
constexpr int kPadTile = kTile + kTile / 8;
constexpr int kReCap = kTile + kWarp;      // row-end staging capacity
constexpr int kWarpsPerCta = 8;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }

// ------------------------------------------------------------ CSR (merge)

// Smallest a in [0, N] with a == N or a + row_ptr[a+1] >= D: the number of
// row-end markers among the first D merge items.  32-ary search by a warp.
__device__ __forceinline__ int merge_search(const int* __restrict__ row_ptr, int N, long long D,
                                            int lane) {
  int lo = 0, hi = N;
  while (hi - lo > kWarp) {
    int step = (hi - lo) / kWarp;
    int p = lo + lane * step;
    bool pred = ((long long)p + __ldg(row_ptr + p + 1)) >= D;
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
  bool pred = (p >= hi) || (((long long)p + __ldg(row_ptr + p + 1)) >= D);
  unsigned m = __ballot_sync(kFull, pred);
  return lo + __ffs(m) - 1;
}

template <typename S, typename A>
__device__ __forceinline__ void emit_row(S* __restrict__ y, int r, int rs, int re, long long b0,
                                         A p) {
  if (re <= rs) return;                 // empty row: y untouched (reference :243)
  if ((long long)re <= b0) return;      // no items of this row in this tile
  if ((long long)rs >= b0) {
    y[r] = (S)((A)y[r] + p);            // whole row inside this tile: exclusive
  } else {
    atomicAdd(y + r, (S)p);             // row continues from an earlier tile
  }
}

template <typename S, typename A, bool VEC>
__global__ void __launch_bounds__(kWarpsPerCta * kWarp)
    csr_merge_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                     const S* __restrict__ val, const S* __restrict__ x, S* __restrict__ y,
                     int N, long long total, long long ntiles, long long tiles_per_warp) {
  __shared__ A s_prod[kWarpsPerCta][kPadTile];
  __shared__ int s_re[kWarpsPerCta][kReCap];
  const int lane = threadIdx.x & (kWarp - 1);
  const int wib = threadIdx.x >> 5;
  A* prod = s_prod[wib];
  int* re = s_re[wib];
  const long long gw = (long long)blockIdx.x * kWarpsPerCta + wib;
  long long tile = gw * tiles_per_warp;
  const long long tile_end = min(tile + tiles_per_warp, ntiles);
  if (tile >= tile_end) return;

  long long D0 = tile * kTile;
  int a0 = merge_search(row_ptr, N, D0, lane);
  long long b0 = D0 - a0;

  for (; tile < tile_end; ++tile) {
    const long long D1 = min(D0 + kTile, total);
    // ---- rows whose end marker falls inside this tile
    int nr = 0;
    while (true) {
      int r = a0 + nr + lane;
      int e = (r < N) ? __ldg(row_ptr + r + 1) : 0x7fffffff;
      bool f = (r < N) && ((long long)r + e < D1);
      if (nr + lane < kReCap) re[nr + lane] = e;
      unsigned m = __ballot_sync(kFull, f);
      int c = __popc(m);
      nr += c;
      if (c < kWarp) break;
    }
    const int a1 = a0 + nr;
    const long long b1 = D1 - a1;
    const int ni = (int)(b1 - b0);
    const int M = nr + ni;
    const int rs0 = (a0 < N) ? __ldg(row_ptr + a0) : 0;

    // ---- stream col/val of items [b0, b1) and stage the products
    {
      const long long g0 = b0 & ~3LL;
      const int nvec = (int)((b1 - g0 + 3) >> 2);
#pragma unroll 2
      for (int v = lane; v < nvec; v += kWarp) {
        const long long g = g0 + 4LL * v;
        if (VEC && g >= b0 && g + 4 <= b1) {
          int4 c = ld_stream_v4(col + g);
          const int o = (int)(g - b0);
          if constexpr (sizeof(S) == 4) {
            float4 w = ld_stream_v4(reinterpret_cast<const float*>(val) + g);
            prod[pad8(o + 0)] = (A)w.x * (A)ld_ro(x + c.x);
            prod[pad8(o + 1)] = (A)w.y * (A)ld_ro(x + c.y);
            prod[pad8(o + 2)] = (A)w.z * (A)ld_ro(x + c.z);
            prod[pad8(o + 3)] = (A)w.w * (A)ld_ro(x + c.w);
          } else {
            double2 w0 = ld_stream_v2(reinterpret_cast<const double*>(val) + g);
            double2 w1 = ld_stream_v2(reinterpret_cast<const double*>(val) + g + 2);
            prod[pad8(o + 0)] = (A)w0.x * (A)ld_ro(x + c.x);
            prod[pad8(o + 1)] = (A)w0.y * (A)ld_ro(x + c.y);
            prod[pad8(o + 2)] = (A)w1.x * (A)ld_ro(x + c.z);
            prod[pad8(o + 3)] = (A)w1.y * (A)ld_ro(x + c.w);
          }
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const long long k = g + e;
            if (k >= b0 && k < b1) {
              int c = ld_stream(col + k);
              prod[pad8((int)(k - b0))] = (A)ld_stream(val + k) * (A)ld_ro(x + c);
            }
          }
        }
      }
    }
    __syncwarp();

    // ---- per-lane merge walk over ITEMS merge steps
    const int dl = min(lane * kItems, M);
    const int dh = min(dl + kItems, M);
    int lo = 0, hi = nr;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if ((long long)mid + (re[mid] - b0) < dl) lo = mid + 1; else hi = mid;
    }
    int ra = lo;
    int rb = dl - ra;
    A acc = 0;
    bool head = false;
    int first_ra = 0;
    A first_val = 0;
    for (int s = dl; s < dh; ++s) {
      const bool take_end = (ra < nr) && (rb >= ni || (long long)re[ra] <= b0 + rb);
      if (take_end) {
        if (!head) {
          head = true;
          first_ra = ra;
          first_val = acc;
        } else {
          emit_row<S, A>(y, a0 + ra, ra ? re[ra - 1] : rs0, re[ra], b0, acc);
        }
        acc = 0;
        ++ra;
      } else {
        acc += prod[pad8(rb)];
        ++rb;
      }
    }
    // ---- warp segmented inclusive scan of the lanes' trailing partials
    A S_ = acc;
    bool hf = head;
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
    if (lane == 0) carry = 0;
    if (head) {
      emit_row<S, A>(y, a0 + first_ra, first_ra ? re[first_ra - 1] : rs0, re[first_ra], b0,
                     first_val + carry);
    }
    // ---- row a1 continues past this tile: add its partial atomically
    if (lane == kWarp - 1 && a1 < N) {
      const int rs1 = nr ? re[nr - 1] : rs0;
      const long long lo_item = max((long long)rs1, b0);
      if (b1 > lo_item) atomicAdd(y + a1, (S)S_);
    }
    __syncwarp();
    a0 = a1;
    b0 = b1;
    D0 = D1;
  }
}

// ------------------------------------------------------------ COO

template <typename S, typename A, bool VEC>
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
          else atomicAdd(y + cur, (S)acc);
          cur = r[e];
          acc = 0;
        }
        acc += p[e];
      }
    }
    const int end_row = cur;
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
      atomicAdd(y + start_row, (S)v);
    }
    // tail run: emitted unless the next lane continues it
    const int next_start = __shfl_down_sync(kFull, start_row, 1);
    const int next_cnt = __shfl_down_sync(kFull, cnt, 1);
    const bool next_internal_or_diff = (lane == kWarp - 1) || next_cnt == 0 || next_start != end_row;
    if (cnt > 0 && next_internal_or_diff) atomicAdd(y + end_row, (S)S_);
  }
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
template <typename T>
__global__ void __launch_bounds__(256)
    dia_row_kernel(const int* __restrict__ offset, const T* __restrict__ data, int N, int nd,
                   int stride, const T* __restrict__ x, T* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T t = y[i];
  const long long move = (long long)N - stride;
  for (int d = 0; d < nd; ++d) {
    const int k = __ldg(offset + d);
    const int lo = k < 0 ? -k : 0;
    const int hi = (N < N - k) ? N : N - k;
    if (i >= lo && i < hi) {
      const long long idx = (long long)d * stride + i - (k < 0 ? move : 0);
      t = add_rn(mul_rn(ld_stream(data + idx), ld_ro(x + i + k)), t);
    }
  }
  y[i] = t;
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

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename K>
static int resident_ctas(K kernel, int threads) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (per_sm < 1) per_sm = 1;
  return per_sm * sm_count();
}

template <typename S, typename A>
static int launch_csr(const int* row_ptr, const int* col, const S* val, const S* x, S* y, int N,
                      long long nnz, cudaStream_t st) {
  const long long total = (long long)N + nnz;
  const long long ntiles = (total + kTile - 1) / kTile;
  const bool vec = aligned16(col) && aligned16(val);
  auto kern = vec ? csr_merge_kernel<S, A, true> : csr_merge_kernel<S, A, false>;
  const int threads = kWarpsPerCta * kWarp;
  const long long max_warps = (long long)resident_ctas(kern, threads) * kWarpsPerCta;
  const long long warps = std::min(ntiles, max_warps);
  const long long tpw = (ntiles + warps - 1) / warps;
  const long long used_warps = (ntiles + tpw - 1) / tpw;
  const long long ctas = (used_warps + kWarpsPerCta - 1) / kWarpsPerCta;
  kern<<<(unsigned)ctas, threads, 0, st>>>(row_ptr, col, val, x, y, N, total, ntiles, tpw);
  SB_CHECK_LAUNCH("csr_merge_kernel");
  return SB_OK;
}

template <typename S, typename A>
static int launch_coo(const int* row, const int* col, const S* val, const S* x, S* y,
                      long long nnz, cudaStream_t st) {
  const long long ntiles = (nnz + kTile - 1) / kTile;
  const bool vec = aligned16(row) && aligned16(col) && aligned16(val);
  auto kern = vec ? coo_tile_kernel<S, A, true> : coo_tile_kernel<S, A, false>;
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

int sb_spmv_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                void* stream) {
  int r = check_dtype(dtype, "sb_spmv_csr");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && inner_max >= 0, "sb_spmv_csr: negative size");
  SB_REQUIRE(nnz <= 0x7fffffffLL, "sb_spmv_csr: nnz exceeds int32 row_ptr range");
  if (N == 0 || nnz == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col && val && x && y, "sb_spmv_csr: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_F32)
      r = launch_csr<float, float>(row_ptr, col, (const float*)val, (const float*)x, (float*)y, N,
                                   nnz, st);
    else
      r = launch_csr<double, double>(row_ptr, col, (const double*)val, (const double*)x,
                                     (double*)y, N, nnz, st);
    if (r) return r;
  }
  return SB_OK;
}

int sb_spmv_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                void* stream) {
  int r = check_dtype(dtype, "sb_spmv_coo");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && inner_max >= 0, "sb_spmv_coo: negative size");
  if (N == 0 || nnz == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(row && col && val && x && y, "sb_spmv_coo: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_F32)
      r = launch_coo<float, float>(row, col, (const float*)val, (const float*)x, (float*)y, nnz,
                                   st);
    else
      r = launch_coo<double, double>(row, col, (const double*)val, (const double*)x, (double*)y,
                                     nnz, st);
    if (r) return r;
  }
  return SB_OK;
}

int sb_spmv_dia(int dtype, const int32_t* offset, const void* data, int32_t N, int32_t nd,
                int32_t stride, const void* x, void* y, int32_t inner_max, void* stream) {
  int r = check_dtype(dtype, "sb_spmv_dia");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nd >= 0 && inner_max >= 0, "sb_spmv_dia: negative size");
  SB_REQUIRE(stride >= N, "sb_spmv_dia: stride %d < N %d", stride, N);
  if (N == 0 || nd == 0 || inner_max == 0) return SB_OK;
  SB_REQUIRE(offset && data && x && y, "sb_spmv_dia: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  const unsigned blocks = (unsigned)((N + 255) / 256);
  for (int it = 0; it < inner_max; ++it) {
    if (dtype == SB_F32)
      dia_row_kernel<float><<<blocks, 256, 0, st>>>(offset, (const float*)data, N, nd, stride,
                                                    (const float*)x, (float*)y);
    else
      dia_row_kernel<double><<<blocks, 256, 0, st>>>(offset, (const double*)data, N, nd, stride,
                                                     (const double*)x, (double*)y);
    SB_CHECK_LAUNCH("dia_row_kernel");
  }
  return SB_OK;
}

int sb_spmv_ell(int dtype, const int32_t* indices, const void* data, int32_t N, int32_t nc,
                const void* x, void* y, int32_t inner_max, void* stream) {
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
