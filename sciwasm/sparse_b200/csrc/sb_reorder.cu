// sb_reorder.cu -- row reordering by row length and the CSR locality index
// (src/parallel/src/sparse32.js:2148-2269).
//
// sort_rows_by_nnz is a stable counting sort of the rows by their number of
// nonzeros followed by a CSR whose rows are gathered in that order (columns
// unchanged); here the rows are stably radix-sorted by length on the device,
// the new row_ptr is a scan of the permuted lengths and one thread per row
// copies its entries.  sort_y_rows_by_nnz scatters y back to the original
// row order.  calculate_csr_locality_index walks the entries in storage
// order and counts the accesses whose 16-column line was last touched fewer
// than 16 rows earlier; each access's previous touch of its line is its
// predecessor after a stable sort of the accesses by line, so the count is
// one sort, one comparison per access and a reduction.
#include <algorithm>
#include <vector>

#include "sb_common.cuh"
#include "sb_prims.cuh"

namespace sb {
namespace {

constexpr int kT = 256;

unsigned grid_n(long long n) {
  const long long g = (n + kT - 1) / kT;
  return (unsigned)std::max(1LL, std::min(g, 0x7fffffffLL));
}

__global__ void length_keys(const int* __restrict__ rp, int N, unsigned long long* __restrict__ k,
                            unsigned* __restrict__ v, int* __restrict__ len,
                            int* __restrict__ small) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int l = rp[i + 1] - rp[i];
  k[i] = (unsigned long long)(unsigned)l;
  v[i] = (unsigned)i;
  len[i] = l;
  if (l < 4) atomicAdd(small + l, 1);
}

__global__ void perm_lengths(const unsigned* __restrict__ sorted, const int* __restrict__ len,
                             int N, int* __restrict__ perm, int* __restrict__ plen) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int i = (int)sorted[p];
  perm[p] = i;
  plen[p] = len[i];
}

template <typename T>
__global__ void gather_rows(const int* __restrict__ rp, const int* __restrict__ col,
                            const T* __restrict__ val, const int* __restrict__ perm,
                            const int* __restrict__ nrp, int N, int* __restrict__ ncol,
                            T* __restrict__ nval) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int src = perm[p];
  int o = nrp[p];
  for (int j = rp[src]; j < rp[src + 1]; ++j, ++o) {
    ncol[o] = col[j];
    nval[o] = val[j];
  }
}

template <typename T>
__global__ void scatter_rows(const int* __restrict__ perm, const T* __restrict__ in, int N,
                             T* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) out[perm[p]] = in[p];
}

__global__ void line_keys(const int* __restrict__ col, long long nnz,
                          unsigned long long* __restrict__ k, unsigned* __restrict__ v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x) {
    k[i] = (unsigned long long)(unsigned)(col[i] / 16);
    v[i] = (unsigned)i;
  }
}

// Accesses (in line order) whose previous touch of the same line is fewer
// than 16 rows back.
__global__ void near_reuse(const unsigned long long* __restrict__ k,
                           const unsigned* __restrict__ pos, const int* __restrict__ row_of,
                           long long nnz, unsigned long long* __restrict__ count) {
  unsigned c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x)
    if (i > 0 && k[i] == k[i - 1] && row_of[pos[i]] - row_of[pos[i - 1]] < 16) ++c;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

template <typename T>
int sort_rows_impl(const int* rp, const int* col, const T* val, int N, long long nnz, int* nrp,
                   int* ncol, T* nval, int* nnz_per_row, int* perm, int32_t* small_rows,
                   cudaStream_t st) {
  const size_t kb = sizeof(unsigned long long) * (size_t)N, vb = sizeof(unsigned) * (size_t)N;
  void* mem = nullptr;
  int r = scratch_alloc(&mem, 2 * kb + 2 * vb + sizeof(int) * ((size_t)N + 4), st);
  if (r) return r;
  char* p = (char*)mem;
  prim::RadixBuffers b;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* small = (int*)(p + 2 * kb + 2 * vb);
  int* len = small + 4;
  SB_CHECK_CUDA(cudaMemsetAsync(small, 0, 4 * sizeof(int), st));
  length_keys<<<grid_n(N), kT, 0, st>>>(rp, N, b.k[0], b.v[0], len, small);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "length_keys");
  const int ranges[2] = {0, prim::bits_for(nnz)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, N, ranges, 1, &which, st);
  if (!r) {
    perm_lengths<<<grid_n(N), kT, 0, st>>>(b.v[which], len, N, perm, nnz_per_row);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "perm_lengths");
  }
  if (!r) r = prim::exclusive_scan(nnz_per_row, nrp, N, st);
  if (!r) {
    const int nz = (int)nnz;
    e = cudaMemcpyAsync(nrp + N, &nz, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) r = cuda_status(e, "row_ptr");
  }
  if (!r) {
    gather_rows<T><<<grid_n(N), kT, 0, st>>>(rp, col, val, perm, nrp, N, ncol, nval);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "gather_rows");
  }
  int h[4] = {0, 0, 0, 0};
  if (!r) {
    e = cudaMemcpyAsync(h, small, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_sort_rows_by_nnz");
  }
  if (!r && small_rows) {  // cumulative: rows with at most 0, 1, 2, 3 nonzeros
    small_rows[0] = h[0];
    for (int q = 1; q < 4; ++q) small_rows[q] = small_rows[q - 1] + h[q];
  }
  scratch_free(mem, st);
  return r;
}

// ------------------------------------------------------------ reorder_NN
// src/parallel/src/sparse32.js:2271-2622.  The reference walks consecutive
// position ranges ("subsets", sized by the row-length histogram, at most
// 1024 rows) one after another; each walk only reads and writes its own
// range, so here one CTA walks one subset and all subsets run at once.
// Within a walk the steps are sequential, as in the reference: at each step
// the new window row's 16-column lines go into a shared-memory hash set,
// every unvisited row of the subset gets its Jaccard value in parallel, and
// warp 0 inserts them into the row's top-w list with the reference's exact
// sequential rule (float32 list values compared as doubles with the new
// value; see nn_insert), then the window's lists are scanned in slot order.

constexpr int kNNThreads = 256;
constexpr int kNNMaxRows = 1024;   // the reference's subset size B
constexpr int kNNMaxW = 32;
constexpr int kNNSmemTable = 16384;  // hash entries kept in shared memory
constexpr unsigned kNNEmpty = 0xffffffffu;

// Number of runs of equal 16-column line in each row (storage order), the
// reference's nlines (0 for empty rows); row length histogram.
__global__ void nn_row_stats(const int* __restrict__ rp, const int* __restrict__ col, int N,
                             int* __restrict__ nlines, int* __restrict__ freq,
                             int* __restrict__ first_nonempty) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = rp[i], e = rp[i + 1];
  int runs = 0;
  for (int j = s; j < e; ++j)
    if (j == s || (col[j - 1] >> 4) != (col[j] >> 4)) ++runs;
  nlines[i] = runs;
  atomicAdd(freq + (e - s), 1);
  if (e > s) atomicMin(first_nonempty, i);
}

// Largest row length of each subset (sizes its line hash set).
__global__ void nn_subset_maxlen(const int* __restrict__ rp, const int2* __restrict__ sub,
                                 int nsub, int* __restrict__ maxlen) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nsub) return;
  int m = 0;
  for (int i = sub[b].x; i < sub[b].y; ++i) m = max(m, rp[i + 1] - rp[i]);
  maxlen[b] = m;
}

__device__ __forceinline__ unsigned nn_hash(unsigned key, unsigned mask) {
  return (key * 2654435761u) & mask;
}

// Insertion of candidate `key` (value v) at position p < w of a list, the
// reference's assign_w_min_elems (src/parallel/src/sparse32.js:2271-2318):
// into an empty slot as is; otherwise entries p .. last-filled-1 move down
// one slot, overwriting the last filled one (a partly filled list does not
// grow on a middle insertion).  Values are stored as float32.
__device__ __forceinline__ void nn_insert(float* L, int* NI, int w, int p, double v, int key) {
  if (L[p] == -1.0f) {
    L[p] = (float)v;
    NI[p] = key;
    return;
  }
  int j = w - 1;
  while (L[j] == -1.0f) --j;
  while (j != p) {
    L[j] = L[j - 1];
    NI[j] = NI[j - 1];
    --j;
  }
  L[p] = (float)v;
  NI[p] = key;
}

__global__ void __launch_bounds__(kNNThreads)
    nn_walk_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                   const int* __restrict__ nlines, const int2* __restrict__ sub,
                   const int* __restrict__ subset_ids, int w, int table_size,
                   unsigned* __restrict__ gtable, int* __restrict__ walk) {
  extern __shared__ __align__(16) unsigned char nn_smem[];
  double* jd = reinterpret_cast<double*>(nn_smem);                      // [kNNMaxRows]
  float* Ls = reinterpret_cast<float*>(jd + kNNMaxRows);                 // [w*w]
  int* NI = reinterpret_cast<int*>(Ls + kNNMaxW * kNNMaxW);              // [w*w]
  int* win = NI + kNNMaxW * kNNMaxW;                                     // [w]
  int* ctl = win + kNNMaxW;                                              // index, count, nnb, next
  unsigned char* vis = reinterpret_cast<unsigned char*>(ctl + 8);        // [kNNMaxRows]
  unsigned* table = gtable ? gtable + (size_t)blockIdx.x * table_size
                           : reinterpret_cast<unsigned*>(vis + kNNMaxRows);
  const int b = subset_ids[blockIdx.x];
  const int start = sub[b].x, n = sub[b].y - sub[b].x;
  const unsigned mask = (unsigned)table_size - 1u;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < n; i += kNNThreads)
    vis[i] = rp[start + i + 1] == rp[start + i] ? 2 : 0;
  if (tid == 0) {
    ctl[0] = 0;  // index (local)
    ctl[1] = 0;  // count
    ctl[2] = 0;  // nnb
  }
  __syncthreads();
  for (int pos = 0; pos < n; ++pos) {
    const int index = ctl[0];
    int slot = 0;
    if (tid == 0) {
      slot = ctl[1];
      win[slot] = index;
      ctl[1] = slot + 1 == w ? 0 : slot + 1;
      ctl[2] = min(ctl[2] + 1, w);
      walk[start + pos] = start + index;
      vis[index] = 1;
    }
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (warp == 0) ctl[3] = slot;  // every lane of warp 0 writes the same value
    for (int q = tid; q < table_size; q += kNNThreads) table[q] = kNNEmpty;
    __syncthreads();
    slot = ctl[3];
    float* L = Ls + slot * w;
    int* NIs = NI + slot * w;
    if (tid < w) {
      L[tid] = -1.0f;
      NIs[tid] = -1;
    }
    // the new window row's lines
    const int gi = start + index;
    for (int j = rp[gi] + tid; j < rp[gi + 1]; j += kNNThreads) {
      const unsigned key = (unsigned)(col[j] >> 4);
      unsigned h = nn_hash(key, mask);
      while (true) {
        const unsigned old = atomicCAS(table + h, kNNEmpty, key);
        if (old == kNNEmpty || old == key) break;
        h = (h + 1) & mask;
      }
    }
    __syncthreads();
    // Jaccard value of every unvisited row against it
    const int nl_index = nlines[gi];
    for (int i = tid; i < n; i += kNNThreads) {
      double v = -2.0;  // not a candidate
      if (vis[i] == 0) {
        const int r = start + i, s = rp[r], e = rp[r + 1];
        int al = 0, prev = -1;
        for (int j = s; j < e; ++j) {
          const int line = col[j] >> 4;
          if (line == prev) continue;
          prev = line;
          unsigned h = nn_hash((unsigned)line, mask);
          while (true) {
            const unsigned t = table[h];
            if (t == (unsigned)line) {
              ++al;
              break;
            }
            if (t == kNNEmpty) break;
            h = (h + 1) & mask;
          }
        }
        v = (double)al / (double)(nl_index + nlines[r] - al);
      }
      jd[i] = v;
    }
    __syncthreads();
    if (warp == 0) {
      // insertion in increasing row order, exactly as one thread would do it:
      // each lane finds its candidate's position against the current list;
      // the first lane that would insert does so and the batch restarts
      // after it, so every candidate sees the list its predecessors left
      int base = 0;
      while (base < n) {
        const int i = base + lane;
        const double v = i < n ? jd[i] : -2.0;
        int p = w;
        if (v >= 0.0) {
          p = 0;
          while (p < w && (double)L[p] >= 0.0 && (double)L[p] >= v) ++p;
        }
        const unsigned m = __ballot_sync(0xffffffffu, p < w);
        if (!m) {
          base += 32;
          continue;
        }
        const int f = __ffs(m) - 1;
        if (lane == f) nn_insert(L, NIs, w, p, v, i);
        __syncwarp();
        base += f + 1;
      }
      // next row: each window slot's first unvisited candidate, then the
      // slots in order, a later slot winning a tie
      const int nnb = ctl[2];
      int nk = -1;
      double mk = 0.0;
      if (lane < nnb) {
        for (int q = 0; q < w; ++q) {
          const float lv = Ls[lane * w + q];
          if ((double)lv >= 0.0 && vis[NI[lane * w + q]] == 0) {
            nk = NI[lane * w + q];
            mk = (double)lv;
            break;
          }
        }
      }
      double mx = 0.0;
      int next = -1;
      for (int k = 0; k < nnb; ++k) {
        const int nkk = __shfl_sync(0xffffffffu, nk, k);
        const double mkk = __shfl_sync(0xffffffffu, mk, k);
        if (mx <= mkk && nkk >= 0) {
          mx = mkk;
          next = nkk;
        }
      }
      if (lane == 0) ctl[0] = next;
    }
    __syncthreads();
    if (ctl[0] < 0) break;
  }
}

// walk -> composed permutation (perm_in NULL: the identity) and new row lengths
__global__ void nn_compose(const int* __restrict__ walk, const int* __restrict__ perm_in,
                           const int* __restrict__ rp, int N, int* __restrict__ perm_out,
                           int* __restrict__ plen) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = walk[i];
  perm_out[i] = perm_in ? perm_in[s] : s;
  plen[i] = rp[s + 1] - rp[s];
}

__global__ void iota_kernel(int* __restrict__ a, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) a[i] = i;
}

template <typename T>
int reorder_nn_impl(const int* rp, const int* col, const T* val, int N, long long nnz, int w,
                    const int* perm_in, int* walk, int* perm_out, int* nrp, int* ncol, T* nval,
                    cudaStream_t st) {
  // scratch: nlines[N], freq[N+1], first_nonempty, lengths[N]
  int* mem = nullptr;
  int r = scratch_alloc((void**)&mem, sizeof(int) * (3 * (size_t)N + 4), st);
  if (r) return r;
  int* nlines = mem;
  int* freq = mem + N;
  int* first = freq + N + 1;
  int* plen = first + 1;
  std::vector<int> hfreq;
  int hfirst = N;
  cudaError_t e = cudaMemsetAsync(freq, 0, sizeof(int) * ((size_t)N + 1), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(first, &hfirst, sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    iota_kernel<<<grid_n(N), kT, 0, st>>>(walk, N);
    nn_row_stats<<<grid_n(N), kT, 0, st>>>(rp, col, N, nlines, freq, first);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    hfreq.resize((size_t)N + 1);
    e = cudaMemcpyAsync(hfreq.data(), freq, sizeof(int) * ((size_t)N + 1), cudaMemcpyDeviceToHost,
                        st);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hfirst, first, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    scratch_free(mem, st);
    return cuda_status(e, "sb_reorder_nn");
  }
  // the subsets: from the first non-empty row, ranges sized by the length
  // histogram (lengths 1, 2, ...), at most kNNMaxRows rows each
  std::vector<int2> hsub;
  int start = hfirst;
  if (start < N) {
    for (int len = 1; len <= N; ++len) {
      int f = hfreq[len];
      while (f >= kNNMaxRows) {
        hsub.push_back(make_int2(start, start + kNNMaxRows));
        start += kNNMaxRows;
        f -= kNNMaxRows;
      }
      if (f > 0) {
        hsub.push_back(make_int2(start, start + f));
        start += f;
      }
    }
  }
  const int nsub = (int)hsub.size();
  int2* dsub = nullptr;
  int* dmax = nullptr;
  int* dids = nullptr;
  unsigned* gtable = nullptr;
  if (nsub > 0) {
    void* sm = nullptr;
    r = scratch_alloc(&sm, (sizeof(int2) + 2 * sizeof(int)) * (size_t)nsub, st);
    if (!r) {
      dsub = (int2*)sm;
      dmax = (int*)(dsub + nsub);
      dids = dmax + nsub;
      e = cudaMemcpyAsync(dsub, hsub.data(), sizeof(int2) * nsub, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) {
        nn_subset_maxlen<<<grid_n(nsub), kT, 0, st>>>(rp, dsub, nsub, dmax);
        e = cudaGetLastError();
      }
      std::vector<int> hmax(nsub);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(hmax.data(), dmax, sizeof(int) * nsub, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) r = cuda_status(e, "sb_reorder_nn");
      // two launches: subsets whose line set fits a shared-memory hash table
      // (at most kNNSmemTable / 2 lines), and the rest with tables in global
      // memory sized for their longest row
      std::vector<int> small, large;
      int large_len = 0;
      for (int q = 0; q < nsub; ++q) {
        if (2 * hmax[q] <= kNNSmemTable) small.push_back(q);
        else {
          large.push_back(q);
          large_len = std::max(large_len, hmax[q]);
        }
      }
      std::vector<int> ids(small);
      ids.insert(ids.end(), large.begin(), large.end());
      if (!r) {
        e = cudaMemcpyAsync(dids, ids.data(), sizeof(int) * nsub, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) r = cuda_status(e, "sb_reorder_nn");
      }
      const size_t fixed = sizeof(double) * kNNMaxRows + 2 * sizeof(float) * kNNMaxW * kNNMaxW +
                           sizeof(int) * (kNNMaxW + 8) + kNNMaxRows;
      if (!r && !small.empty()) {
        int small_len = 0;
        for (int q : small) small_len = std::max(small_len, hmax[q]);
        int ts = 64;
        while (ts < 2 * small_len) ts <<= 1;
        const size_t smem = fixed + sizeof(unsigned) * ts;
        e = cudaFuncSetAttribute(nn_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess) {
          nn_walk_kernel<<<(unsigned)small.size(), kNNThreads, smem, st>>>(
              rp, col, nlines, dsub, dids, w, ts, nullptr, walk);
          e = cudaGetLastError();
        }
        if (e != cudaSuccess) r = cuda_status(e, "nn_walk_kernel");
      }
      if (!r && !large.empty()) {
        int ts = 64;
        while (ts < 2 * large_len) ts <<= 1;
        r = scratch_alloc((void**)&gtable, sizeof(unsigned) * (size_t)ts * large.size(), st);
        if (!r) {
          nn_walk_kernel<<<(unsigned)large.size(), kNNThreads, fixed, st>>>(
              rp, col, nlines, dsub, dids + small.size(), w, ts, gtable, walk);
          e = cudaGetLastError();
          if (e != cudaSuccess) r = cuda_status(e, "nn_walk_kernel");
        }
      }
    }
  }
  // the new CSR: rows in walk order; the permutation composed with perm_in
  if (!r) {
    nn_compose<<<grid_n(N), kT, 0, st>>>(walk, perm_in, rp, N, perm_out, plen);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "nn_compose");
  }
  if (!r) r = prim::exclusive_scan(plen, nrp, N, st);
  if (!r) {
    const int nz = (int)nnz;
    e = cudaMemcpyAsync(nrp + N, &nz, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
      gather_rows<T><<<grid_n(N), kT, 0, st>>>(rp, col, val, walk, nrp, N, ncol, nval);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_reorder_nn");
  } else {
    cudaStreamSynchronize(st);
  }
  if (gtable) scratch_free(gtable, st);
  if (dsub) scratch_free(dsub, st);
  scratch_free(mem, st);
  return r;
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

int sb_sort_rows_by_nnz(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                        int32_t N, int64_t nnz, int32_t* out_row_ptr, int32_t* out_col,
                        void* out_val, int32_t* nnz_per_row, int32_t* permutation,
                        int32_t* small_rows, void* stream) {
  SB_TRACE("sb_sort_rows_by_nnz");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_sort_rows_by_nnz: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_sort_rows_by_nnz: bad size");
  SB_REQUIRE(N == 0 || (row_ptr && out_row_ptr && nnz_per_row && permutation),
             "sb_sort_rows_by_nnz: null pointer");
  SB_REQUIRE(nnz == 0 || (col && val && out_col && out_val), "sb_sort_rows_by_nnz: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (N == 0) {
    if (small_rows) small_rows[0] = small_rows[1] = small_rows[2] = small_rows[3] = 0;
    if (out_row_ptr) SB_CHECK_CUDA(cudaMemsetAsync(out_row_ptr, 0, sizeof(int32_t), st));
    return SB_OK;
  }
  if (dtype == SB_F32)
    return sort_rows_impl<float>(row_ptr, col, (const float*)val, N, nnz, out_row_ptr, out_col,
                                 (float*)out_val, nnz_per_row, permutation, small_rows, st);
  return sort_rows_impl<double>(row_ptr, col, (const double*)val, N, nnz, out_row_ptr, out_col,
                                (double*)out_val, nnz_per_row, permutation, small_rows, st);
}

int sb_unpermute_rows(int dtype, const int32_t* permutation, const void* in, void* out,
                      int32_t N, void* stream) {
  SB_TRACE("sb_unpermute_rows");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_unpermute_rows: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0, "sb_unpermute_rows: bad size");
  if (N == 0) return SB_OK;
  SB_REQUIRE(permutation && in && out && in != out, "sb_unpermute_rows: bad pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    scatter_rows<float><<<grid_n(N), kT, 0, st>>>(permutation, (const float*)in, N, (float*)out);
  else
    scatter_rows<double><<<grid_n(N), kT, 0, st>>>(permutation, (const double*)in, N,
                                                   (double*)out);
  SB_CHECK_LAUNCH("scatter_rows");
  return SB_OK;
}

int sb_reorder_nn(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                  int32_t N, int64_t nnz, int32_t w, const int32_t* perm_in, int32_t* walk,
                  int32_t* perm_out, int32_t* out_row_ptr, int32_t* out_col, void* out_val,
                  void* stream) {
  SB_TRACE("sb_reorder_nn");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_reorder_nn: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_reorder_nn: bad size");
  SB_REQUIRE(w >= 1 && w <= kNNMaxW, "sb_reorder_nn: window %d outside 1..%d", w, kNNMaxW);
  SB_REQUIRE(N == 0 || (row_ptr && walk && perm_out && out_row_ptr),
             "sb_reorder_nn: null pointer");
  SB_REQUIRE(nnz == 0 || (col && val && out_col && out_val), "sb_reorder_nn: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (N == 0) {
    SB_CHECK_CUDA(cudaMemsetAsync(out_row_ptr, 0, sizeof(int32_t), st));
    return SB_OK;
  }
  if (dtype == SB_F32)
    return reorder_nn_impl<float>(row_ptr, col, (const float*)val, N, nnz, w, perm_in, walk,
                                  perm_out, out_row_ptr, out_col, (float*)out_val, st);
  return reorder_nn_impl<double>(row_ptr, col, (const double*)val, N, nnz, w, perm_in, walk,
                                 perm_out, out_row_ptr, out_col, (double*)out_val, st);
}

int sb_csr_locality_index(const int32_t* row_ptr, const int32_t* col, int32_t N, int64_t nnz,
                          double* index, void* stream) {
  SB_TRACE("sb_csr_locality_index");
  SB_REQUIRE(index, "sb_csr_locality_index: null output");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_csr_locality_index: bad size");
  *index = 0.0;
  if (nnz == 0) {  // the reference's 0 * 100 / 0
    *index = __builtin_nan("");
    return SB_OK;
  }
  SB_REQUIRE(row_ptr && col, "sb_csr_locality_index: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  const size_t kb = sizeof(unsigned long long) * (size_t)nnz, vb = sizeof(unsigned) * (size_t)nnz;
  void* mem = nullptr;
  // [count (8 bytes)] [keys 2 x nnz u64] [positions 2 x nnz u32] [row of each entry]
  if ((r = scratch_alloc(&mem, 8 + 2 * kb + 2 * vb + sizeof(int) * (size_t)nnz, st))) return r;
  char* p = (char*)mem;
  unsigned long long* count = (unsigned long long*)p;
  p += 8;
  prim::RadixBuffers b;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* row_of = (int*)(p + 2 * kb + 2 * vb);
  cudaError_t e = cudaSuccess;
  SB_CHECK_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
  prim::expand_rows<<<grid_n(N), kT, 0, st>>>(row_ptr, N, row_of);
  e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "expand_rows");
  if (!r) {
    line_keys<<<std::min(grid_n(nnz), 4096u), kT, 0, st>>>(col, nnz, b.k[0], b.v[0]);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "line_keys");
  }
  const int ranges[2] = {0, prim::bits_for(N / 16)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, nnz, ranges, 1, &which, st);
  if (!r) {
    near_reuse<<<std::min(grid_n(nnz), 4096u), kT, 0, st>>>(b.k[which], b.v[which], row_of, nnz,
                                                            count);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "near_reuse");
  }
  unsigned long long h = 0;
  if (!r) {
    e = cudaMemcpyAsync(&h, count, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_csr_locality_index");
  }
  scratch_free(mem, st);
  if (!r) *index = ((double)h * 100.0) / (double)nnz;
  return r;
}

}  // extern "C"
