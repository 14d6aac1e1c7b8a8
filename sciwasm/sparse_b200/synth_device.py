"""Seeded synthetic matrices generated directly in device memory (torch),
for workloads too large to build on the host quickly: banded, 2-D 5-point
Laplacian, power-law rows, and the lower-triangular factors of the SpTS
workloads (3-D 7-point Laplacian lower triangle, band-limited random lower).
The structures follow synth.py; random draws use torch's generator, so the
values differ from the host versions while shapes and distributions match.
Column indices are distinct and sorted within each row (repeated draws are
merged, so a row can come out a little shorter than drawn) and a factor's
diagonal is stored last.  The returned sparse_CSR_t objects view torch tensors (kept alive on
the object as `_torch`)."""
from __future__ import annotations

import numpy as np

from .sparse import DeviceArray, sparse_CSR_t


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("device synthesis needs a CUDA device")
    return torch


def _wrap(rp, col, val) -> sparse_CSR_t:
    torch = _torch()
    npdt = np.float64 if val.dtype == torch.float64 else np.float32
    N = rp.numel() - 1
    nnz = col.numel()
    A = sparse_CSR_t(DeviceArray(N + 1, np.int32, rp.data_ptr()),
                     DeviceArray(nnz, np.int32, col.data_ptr()),
                     DeviceArray(nnz, npdt, val.data_ptr()), N, nnz)
    A._torch = (rp, col, val)
    return A


def _stencil(N, offsets, valid_fn, gen, dev):
    """Rows i with columns i + o (o in ascending `offsets`) where valid."""
    torch = _torch()
    i = torch.arange(N, device=dev, dtype=torch.int64)
    off = torch.tensor(offsets, device=dev, dtype=torch.int64)
    cols = i[:, None] + off[None, :]
    mask = valid_fn(i[:, None], cols, off[None, :])
    counts = mask.sum(1, dtype=torch.int32)
    rp = torch.zeros(N + 1, device=dev, dtype=torch.int32)
    torch.cumsum(counts, 0, out=rp[1:])
    col = cols[mask].to(torch.int32)
    return rp, col, mask


def banded(N: int, half: int = 5, seed: int = 1, dtype="f32"):
    """Offsets -half..half, values ~ N(0, 1)."""
    torch = _torch()
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev).manual_seed(seed)
    rp, col, _ = _stencil(N, list(range(-half, half + 1)),
                          lambda i, c, o: (c >= 0) & (c < N), gen, dev)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    val = torch.randn(col.numel(), generator=gen, device=dev, dtype=tdt)
    return _wrap(rp, col, val)


def laplacian_2d(n: int, dtype="f32"):
    """5-point Laplacian on an n x n grid: 4 on the diagonal, -1 off it."""
    torch = _torch()
    dev = torch.device("cuda")
    N = n * n

    def ok(i, c, o):
        inside = (c >= 0) & (c < N)
        left = (o != -1) | (i % n != 0)
        right = (o != 1) | (i % n != n - 1)
        return inside & left & right

    rp, col, mask = _stencil(N, [-n, -1, 0, 1, n], ok, None, dev)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    diag = torch.tensor([False, False, True, False, False], device=dev).expand(N, 5)[mask]
    val = torch.where(diag, 4.0, -1.0).to(tdt)
    return _wrap(rp, col, val)


def laplacian_3d_lower(n: int, dtype="f32"):
    """Lower triangle of the 7-point Laplacian on an n^3 grid (6 on the
    diagonal, -1 off it; the diagonal last in each row)."""
    torch = _torch()
    dev = torch.device("cuda")
    N = n ** 3

    def ok(i, c, o):
        xm = (o != -1) | (i % n != 0)
        ym = (o != -n) | ((i // n) % n != 0)
        zm = (o != -n * n) | (i >= n * n)
        return xm & ym & zm

    rp, col, mask = _stencil(N, [-n * n, -n, -1, 0], ok, None, dev)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    diag = torch.tensor([False, False, False, True], device=dev).expand(N, 4)[mask]
    val = torch.where(diag, 6.0, -1.0).to(tdt)
    return _wrap(rp, col, val)


def _csr_from_keys(key, N):
    """Sorted, de-duplicated keys row * N + col -> (row_ptr i32, col i32, row i64)."""
    torch = _torch()
    key = torch.unique_consecutive(key)
    row = key // N
    col = (key % N).to(torch.int32)
    counts = torch.bincount(row, minlength=N)
    rp = torch.zeros(N + 1, device=key.device, dtype=torch.int64)
    torch.cumsum(counts, 0, out=rp[1:])
    return rp.to(torch.int32), col, row


def _rows_from_counts(counts):
    torch = _torch()
    N = counts.numel()
    rp = torch.zeros(N + 1, device=counts.device, dtype=torch.int64)
    torch.cumsum(counts.to(torch.int64), 0, out=rp[1:])
    row = torch.repeat_interleave(torch.arange(N, device=counts.device), counts.to(torch.int64))
    return rp, row


def power_law(N: int, s: float = 2.0, cap: int = 2000, shift: int = 15, seed: int = 2,
              dtype="f32"):
    """Row lengths min(cap, Zipf(s) + shift, N), uniform distinct columns,
    values ~ U[-1, 1]."""
    torch = _torch()
    dev = torch.device("cuda")
    rng = np.random.default_rng(seed)
    lens = np.minimum(np.minimum(rng.zipf(s, N) + shift, cap), N).astype(np.int32)
    counts = torch.from_numpy(lens).to(dev)
    rp, row = _rows_from_counts(counts)
    gen = torch.Generator(device=dev).manual_seed(seed)
    c = torch.randint(0, N, (row.numel(),), generator=gen, device=dev, dtype=torch.int64)
    key, _ = torch.sort(row * N + c)
    rp, col, _ = _csr_from_keys(key, N)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    val = (torch.rand(col.numel(), generator=gen, device=dev, dtype=tdt) * 2 - 1)
    return _wrap(rp, col, val)


def random_lower(N: int, per_row: int = 7, band: int = 5000, seed: int = 3, dtype="f32"):
    """Row i: min(per_row, i) distinct columns uniform in [max(0, i - band), i)
    with values ~ U[-0.5, 0.5], then the diagonal ~ U[2, 4]."""
    torch = _torch()
    dev = torch.device("cuda")
    gen = torch.Generator(device=dev).manual_seed(seed)
    i = torch.arange(N, device=dev, dtype=torch.int64)
    k = torch.clamp(i, max=per_row)
    rp, row = _rows_from_counts(k + 1)
    nnz = row.numel()
    lo = torch.clamp(row - band, min=0)
    width = row - lo
    u = torch.rand(nnz, generator=gen, device=dev, dtype=torch.float64)
    c = lo + torch.clamp((u * width).to(torch.int64), max=torch.clamp(width - 1, min=0))
    # the last slot of each row is its diagonal
    last = torch.zeros(nnz, device=dev, dtype=torch.bool)
    last[rp[1:] - 1] = True
    c = torch.where(last, row, c)
    key, _ = torch.sort(row * N + c)
    rp, col, row = _csr_from_keys(key, N)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    off = torch.rand(col.numel(), generator=gen, device=dev, dtype=tdt) - 0.5
    dg = torch.rand(col.numel(), generator=gen, device=dev, dtype=tdt) * 2 + 2
    val = torch.where(col.to(torch.int64) == row, dg, off)
    return _wrap(rp, col, val)


def poisson_rows(N: int, mean: float = 12.0, seed: int = 5, dtype="f32"):
    """Row i: Poisson(mean) distinct columns uniform in [0, N) plus the
    diagonal, values ~ U[-1, 1]."""
    torch = _torch()
    dev = torch.device("cuda")
    rng = np.random.default_rng(seed)
    lens = (rng.poisson(mean, N) + 1).astype(np.int32)
    counts = torch.from_numpy(lens).to(dev)
    rp, row = _rows_from_counts(counts)
    gen = torch.Generator(device=dev).manual_seed(seed)
    c = torch.randint(0, N, (row.numel(),), generator=gen, device=dev, dtype=torch.int64)
    last = torch.zeros(row.numel(), device=dev, dtype=torch.bool)
    last[rp[1:] - 1] = True
    c = torch.where(last, row, c)
    key, _ = torch.sort(row * N + c)
    rp, col, _ = _csr_from_keys(key, N)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    val = torch.rand(col.numel(), generator=gen, device=dev, dtype=tdt) * 2 - 1
    return _wrap(rp, col, val)
