// sb_prims.cuh -- device primitives shared by the conversion, structure and
// level-set kernels: exclusive scan of int32 counts, max reduction, and a
// stable LSD radix sort of 64-bit keys carrying a 32-bit payload.
#pragma once

#include "sb_common.cuh"

namespace sb {
namespace prim {
// Internal linkage: each translation unit that includes this header gets its
// own copy of these kernels and helpers.
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one int per thread (returns the block total).
__device__ __forceinline__ int block_exclusive_scan(int v, int* smem_warp, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) smem_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? smem_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    smem_warp[lane] = w;
  }
  __syncthreads();
  const int before = warp ? smem_warp[warp - 1] : 0;
  total = smem_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

// Per-tile sums of `in` (tile = kScanTile items).
__global__ void __launch_bounds__(kScanThreads)
    scan_tile_sums(const int* __restrict__ in, long long n, int* __restrict__ sums) {
  __shared__ int sw[32];
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) s += in[base + j];
  int total;
  block_exclusive_scan(s, sw, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Exclusive scan of each tile plus its tile offset (offsets may be null).
__global__ void __launch_bounds__(kScanThreads)
    scan_tiles(const int* __restrict__ in, long long n, const int* __restrict__ offsets,
               int* __restrict__ out) {
  __shared__ int sw[32];
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = (base + j < n) ? in[base + j] : 0;
    s += v[j];
  }
  int total;
  int run = block_exclusive_scan(s, sw, total) + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    if (base + j < n) out[base + j] = run;
    run += v[j];
  }
}

// out[i] = sum of in[0..i), n items (in-place allowed); scratch is allocated
// on the stream.  Totals must fit in int32 (they count nonzeros here).
inline int exclusive_scan(const int* in, int* out, long long n, cudaStream_t st) {
  if (n <= 0) return SB_OK;
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    scan_tiles<<<1, kScanThreads, 0, st>>>(in, n, nullptr, out);
    SB_CHECK_LAUNCH("scan_tiles");
    return SB_OK;
  }
  int* sums = nullptr;
  int r = scratch_alloc((void**)&sums, sizeof(int) * (size_t)tiles, st);
  if (r) return r;
  scan_tile_sums<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums);
  SB_CHECK_LAUNCH("scan_tile_sums");
  r = exclusive_scan(sums, sums, tiles, st);
  if (!r) {
    scan_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "scan_tiles");
  }
  scratch_free(sums, st);
  return r;
}

// row_ptr from a row array sorted ascending: row_ptr[r] = first position of
// a row >= r.  Every row_ptr entry (0..N) is written exactly once.
__global__ void row_ptr_from_sorted(const int* __restrict__ row, long long nnz, int N,
                                    int* __restrict__ row_ptr) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nnz) return;
  const int prev = (i == 0) ? -1 : row[i - 1];
  const int cur = (i == nnz) ? N : row[i];
  for (int r = prev + 1; r <= cur; ++r) row_ptr[r] = (int)i;
}

// Row index of every CSR entry.
__global__ void expand_rows(const int* __restrict__ row_ptr, int N, int* __restrict__ row_of) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) row_of[j] = i;
}

// ------------------------------------------------------------ radix sort

constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 8;  // striped: item j of thread t is j*256 + t
constexpr int kRadixTile = kRadixThreads * kRadixItems;
constexpr int kRadixWarps = kRadixThreads / 32;

__global__ void __launch_bounds__(kRadixThreads)
    radix_hist(const unsigned long long* __restrict__ keys, long long n, int shift,
               long long ntiles, int* __restrict__ counts) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kRadixTile;
#pragma unroll
  for (int j = 0; j < kRadixItems; ++j) {
    const long long i = base + (long long)j * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1);
  }
  __syncthreads();
  counts[(long long)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter of one 8-bit digit: items keep their input order inside
// each digit (ranks from warp match + per-warp counters, slice by slice).
__global__ void __launch_bounds__(kRadixThreads)
    radix_scatter(const unsigned long long* __restrict__ kin, const unsigned* __restrict__ vin,
                  unsigned long long* __restrict__ kout, unsigned* __restrict__ vout, long long n,
                  int shift, long long ntiles, const int* __restrict__ offsets) {
  __shared__ int base[256];
  __shared__ int tot[256];
  __shared__ int wcnt[kRadixWarps][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  base[tid] = offsets[(long long)tid * ntiles + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kRadixWarps; ++w) wcnt[w][tid] = 0;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  const long long tbase = (long long)blockIdx.x * kRadixTile;
  for (int j = 0; j < kRadixItems; ++j) {
    const long long i = tbase + (long long)j * kRadixThreads + tid;
    const bool valid = i < n;
    const unsigned long long key = valid ? kin[i] : 0ull;
    const unsigned val = valid ? vin[i] : 0u;
    const int d = valid ? (int)((key >> shift) & 255u) : 256 + lane;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & lt);
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      int run = 0;
#pragma unroll
      for (int w = 0; w < kRadixWarps; ++w) {
        const int c = wcnt[w][tid];
        wcnt[w][tid] = run;
        run += c;
      }
      tot[tid] = run;
    }
    __syncthreads();
    if (valid) {
      const int pos = base[d] + wcnt[warp][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    base[tid] += tot[tid];
#pragma unroll
    for (int w = 0; w < kRadixWarps; ++w) wcnt[w][tid] = 0;
    __syncthreads();
  }
}

// Stable sort of (key, payload) pairs by the key bits [lo_bit, hi_bit) of the
// listed bit ranges, least significant range first.  Buffers are swapped
// between passes; *result points at the buffer holding the sorted data.
struct RadixBuffers {
  unsigned long long* k[2];
  unsigned* v[2];
};

inline int radix_sort_ranges(RadixBuffers& b, long long n, const int* ranges, int nranges,
                             int* which, cudaStream_t st) {
  *which = 0;
  if (n <= 1) return SB_OK;
  const long long ntiles = (n + kRadixTile - 1) / kRadixTile;
  int* counts = nullptr;
  int r = scratch_alloc((void**)&counts, sizeof(int) * 256 * (size_t)ntiles, st);
  if (r) return r;
  int cur = 0;
  for (int q = 0; q < nranges && !r; ++q) {
    for (int sh = ranges[2 * q]; sh < ranges[2 * q + 1] && !r; sh += 8) {
      radix_hist<<<(unsigned)ntiles, kRadixThreads, 0, st>>>(b.k[cur], n, sh, ntiles, counts);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) { r = cuda_status(e, "radix_hist"); break; }
      r = exclusive_scan(counts, counts, 256 * ntiles, st);
      if (r) break;
      radix_scatter<<<(unsigned)ntiles, kRadixThreads, 0, st>>>(b.k[cur], b.v[cur], b.k[cur ^ 1],
                                                               b.v[cur ^ 1], n, sh, ntiles,
                                                               counts);
      e = cudaGetLastError();
      if (e != cudaSuccess) { r = cuda_status(e, "radix_scatter"); break; }
      cur ^= 1;
    }
  }
  scratch_free(counts, st);
  *which = cur;
  return r;
}

inline int bits_for(long long maxval) {
  int b = 0;
  while (b < 62 && (1LL << b) <= maxval) ++b;
  return b;
}

}  // namespace
}  // namespace prim
}  // namespace sb
