"""Seeded synthetic matrices for the workloads this library is measured on.

The reference benchmarks on real Matrix-Market files that it does not ship;
these generators stand in for them with the structures, sizes and value
distributions of the measured workloads.  All return host (numpy) arrays;
CSR columns are ascending within each row unless stated otherwise.
"""
from __future__ import annotations

import numpy as np


def _csr_from_rows(counts: np.ndarray) -> np.ndarray:
    row_ptr = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    if row_ptr[-1] > np.iinfo(np.int32).max:
        raise ValueError("nnz exceeds int32 row_ptr range")
    return row_ptr.astype(np.int32)


def laplacian_2d(n: int, dtype=np.float32):
    """5-point Laplacian on an n x n grid: diagonal 4, neighbours -1, natural
    ordering.  Returns (row_ptr, col, val)."""
    N = n * n
    idx = np.arange(N, dtype=np.int64)
    i, j = idx // n, idx % n
    cols = []
    vals = []
    # ascending column order: (i-1,j), (i,j-1), (i,j), (i,j+1), (i+1,j)
    for di, dj, v in ((-1, 0, -1.0), (0, -1, -1.0), (0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0)):
        ok = (i + di >= 0) & (i + di < n) & (j + dj >= 0) & (j + dj < n)
        c = np.where(ok, idx + di * n + dj, -1)
        cols.append(c)
        vals.append(np.full(N, v))
    C_ = np.stack(cols, axis=1)
    V_ = np.stack(vals, axis=1)
    mask = C_ >= 0
    counts = mask.sum(axis=1)
    return _csr_from_rows(counts), C_[mask].astype(np.int32), V_[mask].astype(dtype)


def banded(N: int, half: int = 5, seed: int = 1, dtype=np.float64):
    """Banded matrix with diagonals at offsets -half..half, values N(0,1).
    Returns (row_ptr, col, val) with ascending columns."""
    rng = np.random.default_rng(seed)
    offs = np.arange(-half, half + 1, dtype=np.int64)
    rows = np.arange(N, dtype=np.int64)[:, None]
    C_ = rows + offs[None, :]
    mask = (C_ >= 0) & (C_ < N)
    counts = mask.sum(axis=1)
    col = C_[mask].astype(np.int32)
    val = rng.standard_normal(col.size).astype(dtype)
    return _csr_from_rows(counts), col, val


def _distinct_uniform_cols(rng, counts, lo, hi):
    """For each row r draw counts[r] distinct integers uniformly in
    [lo[r], hi[r]); returned row by row, ascending within each row."""
    total = int(counts.sum())
    nrows = counts.size
    row_of = np.repeat(np.arange(nrows, dtype=np.int64), counts)
    span = (hi - lo).astype(np.int64)
    width = int(max(1, span.max())) if nrows else 1
    cols = lo[row_of] + (rng.random(total) * span[row_of]).astype(np.int64)
    for _ in range(64):
        key = row_of * width + (cols - lo[row_of])
        key.sort()
        cols = lo[row_of] + key % width
        dup = np.zeros(total, dtype=bool)
        dup[1:] = key[1:] == key[:-1]
        nd = int(dup.sum())
        if nd == 0:
            return cols
        cols[dup] = lo[row_of[dup]] + (rng.random(nd) * span[row_of[dup]]).astype(np.int64)
    raise RuntimeError("could not draw distinct columns")


def power_law(N: int = 2_000_000, s: float = 2.0, cap: int = 2000, shift: int = 15, seed: int = 2,
              dtype=np.float64, sort_cols: bool = True):
    """Power-law rows: L_i = min(cap, Zipf(s) + shift) distinct uniform columns
    in [0, N), values U[-1, 1].  With sort_cols=False the columns of each row
    are left in random order (exercises the stable per-row sort of coo_csr)."""
    rng = np.random.default_rng(seed)
    L = np.minimum(cap, rng.zipf(s, size=N) + shift).astype(np.int64)
    L = np.minimum(L, N)
    cols = _distinct_uniform_cols(rng, L, np.zeros(N, np.int64), np.full(N, N, np.int64))
    val = rng.uniform(-1.0, 1.0, cols.size).astype(dtype)
    row_ptr = _csr_from_rows(L)
    if not sort_cols:
        key = rng.random(cols.size)
        row_of = np.repeat(np.arange(N), L)
        perm = np.lexsort((key, row_of))
        cols = cols[perm]
    return row_ptr, cols.astype(np.int32), val


def laplacian_3d_lower(n: int = 64, dtype=np.float64):
    """Lower triangle (diagonal included, stored last in each row) of the 3-D
    7-point Laplacian on an n^3 grid: diagonal 6, neighbours -1."""
    N = n ** 3
    idx = np.arange(N, dtype=np.int64)
    i, j, k = idx // (n * n), (idx // n) % n, idx % n
    cols = []
    vals = []
    for ok, off in (((i > 0), -n * n), ((j > 0), -n), ((k > 0), -1)):
        cols.append(np.where(ok, idx + off, -1))
        vals.append(np.full(N, -1.0))
    cols.append(idx)
    vals.append(np.full(N, 6.0))
    C_ = np.stack(cols, axis=1)
    V_ = np.stack(vals, axis=1)
    mask = C_ >= 0
    return _csr_from_rows(mask.sum(axis=1)), C_[mask].astype(np.int32), V_[mask].astype(dtype)


def random_lower(N: int = 1_000_000, per_row: int = 7, band: int = 5000, seed: int = 3,
                 dtype=np.float64):
    """Random lower-triangular matrix: row i holds min(per_row, i) distinct
    off-diagonal columns uniform in [max(0, i-band), i), ascending, values
    U[-0.5, 0.5], then its diagonal U[2, 4] stored last."""
    rng = np.random.default_rng(seed)
    rows = np.arange(N, dtype=np.int64)
    lo = np.maximum(0, rows - band)
    cnt = np.minimum(per_row, rows - lo)
    off_cols = _distinct_uniform_cols(rng, cnt, lo, rows)
    off_vals = rng.uniform(-0.5, 0.5, off_cols.size)
    diag = rng.uniform(2.0, 4.0, N)
    counts = cnt + 1
    row_ptr = _csr_from_rows(counts)
    nnz = int(row_ptr[-1])
    col = np.empty(nnz, dtype=np.int64)
    val = np.empty(nnz, dtype=np.float64)
    diag_pos = row_ptr[1:].astype(np.int64) - 1
    is_diag = np.zeros(nnz, dtype=bool)
    is_diag[diag_pos] = True
    col[is_diag] = rows
    val[is_diag] = diag
    col[~is_diag] = off_cols
    val[~is_diag] = off_vals
    return row_ptr, col.astype(np.int32), val.astype(dtype)


def csr_to_coo_rows(row_ptr: np.ndarray) -> np.ndarray:
    N = row_ptr.size - 1
    return np.repeat(np.arange(N, dtype=np.int32), np.diff(row_ptr).astype(np.int64))


def uniform_vec(N: int, seed: int, lo=-1.0, hi=1.0, dtype=np.float64):
    return np.random.default_rng(seed).uniform(lo, hi, N).astype(dtype)


def csr_to_ell_host(row_ptr, col, val, nc=None):
    """Column-major ELL arrays (indices, data, nc) of a CSR matrix, zero padded
    (host-side input preparation; the library's conversion runs on the GPU)."""
    N = row_ptr.size - 1
    lens = np.diff(row_ptr).astype(np.int64)
    if nc is None:
        nc = int(lens.max()) if N else 0
    row_of = np.repeat(np.arange(N, dtype=np.int64), lens)
    pos = np.arange(col.size, dtype=np.int64) - row_ptr[:-1].astype(np.int64)[row_of]
    ind = np.zeros(nc * N, np.int32)
    dat = np.zeros(nc * N, val.dtype)
    ind[pos * N + row_of] = col
    dat[pos * N + row_of] = val
    return ind, dat, nc


def csr_to_dia_host(row_ptr, col, val):
    """Diagonal-major DIA arrays (offset, data) with stride N for a CSR matrix
    without duplicate entries (host-side input preparation)."""
    N = row_ptr.size - 1
    row_of = np.repeat(np.arange(N, dtype=np.int64), np.diff(row_ptr).astype(np.int64))
    d = col.astype(np.int64) - row_of
    offs = np.unique(d)
    slot = np.searchsorted(offs, d)
    data = np.zeros(offs.size * N, val.dtype)
    data[slot * N + row_of] = val
    return offs.astype(np.int32), data
