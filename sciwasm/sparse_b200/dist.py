"""Row-sharded SpMV across processes (one per GPU) and the multi-process
timing helper.

SpMV shards by contiguous row blocks balanced by nonzeros, the partition the
reference's worker pool uses (static_nnz, src/parallel/src/sparse32.js:2769-2821):
every rank keeps its block of rows resident and the whole x, computes its own
y rows with the library's kernels, and the y blocks are disjoint, so the
data path needs no reduction; `ShardedY` (in place, padded blocks) or
`gather_rows` assembles the full y where a caller needs it (one
all-gather).  `max_over_ranks` is the timing rule of multi-GPU
measurements: the slowest rank's time.

The torch.distributed calls run on whatever backend the process group has
(NCCL on GPUs, gloo for host-side tests).
"""
from __future__ import annotations

import numpy as np

from .sparse import DeviceArray, sparse_CSR_t, spmv, static_nnz


def shard_rows(row_ptr, world: int):
    """(row_start, row_end) of every rank: static_nnz over `world` parts."""
    return static_nnz(row_ptr, world)


def local_block(row_ptr, col, val, r0: int, r1: int):
    """Host arrays of rows [r0, r1) as a CSR of r1 - r0 rows (columns keep
    their global numbering, so the block multiplies the full x)."""
    row_ptr = np.asarray(row_ptr, np.int64)
    s, e = int(row_ptr[r0]), int(row_ptr[r1])
    rp = (row_ptr[r0:r1 + 1] - s).astype(np.int32)
    return rp, np.asarray(col)[s:e], np.asarray(val)[s:e]


class RowShardedCSR:
    """This rank's row block of a CSR matrix, resident on its device.  The
    block is a CSR of r1 - r0 rows whose columns keep their global numbers;
    the kernels index x by column, so x holds all N entries and y only this
    rank's rows."""

    def __init__(self, row_ptr, col, val, rank: int, world: int):
        starts, ends = shard_rows(row_ptr, world)
        self.rank, self.world = int(rank), int(world)
        self.starts, self.ends = starts, ends
        self.r0, self.r1 = int(starts[rank]), int(ends[rank])
        self.N = int(np.asarray(row_ptr).size - 1)
        self.rows = self.r1 - self.r0
        rp, c, v = local_block(row_ptr, col, val, self.r0, self.r1)
        if c.size and (int(np.min(c)) < 0 or int(np.max(c)) >= self.N):
            raise ValueError("column outside the matrix")
        self.A = sparse_CSR_t(DeviceArray.from_host(rp), DeviceArray.from_host(c),
                              DeviceArray.from_host(np.ascontiguousarray(v)), self.rows,
                              c.size) if self.rows > 0 else None

    def spmv(self, x_view, y_view, inner_max=1, stream=None):
        """y_view (this rank's rows) += A[r0:r1, :] x_view (all N entries)."""
        if self.A is not None:
            spmv(self.A, x_view, y_view, inner_max, stream)

    def spmv_allgather(self, x_ptr: int, y_in_ptr: int, dst_dev_ptr: int, ndst: int,
                       opts=None, stream=None):
        """The all-gather fused into the SpMV (sb_spmv_csr_allgather): this
        rank's rows t = y_in + A[r0:r1, :] x are stored at rows r0.. of every
        one of ndst full-length y buffers, whose device pointers are in the
        device array at dst_dev_ptr (this GPU's own buffers, or peers'
        buffers mapped for peer access, e.g. the buffer_ptrs of a torch
        symmetric-memory rendezvous; see PeerY).  Once every rank has run and
        the ranks have synchronised, each buffer holds the whole y.  y_in_ptr
        points at this rank's `rows` values."""
        import ctypes as C
        from . import _lib
        from .sparse import _dtcode, _sp
        if self.A is None:
            return
        o = opts if opts is not None else getattr(self.A, "opts", None)
        _lib.call("sb_spmv_csr_allgather", _dtcode(self.A.dtype), self.A.row_index.ptr,
                  self.A.col_index.ptr, self.A.val_index.ptr, int(x_ptr), int(y_in_ptr),
                  self.rows, self.A.nnz, self.r0, C.c_void_p(int(dst_dev_ptr)), int(ndst),
                  C.byref(o) if o is not None else None, _sp(stream))


def gather_rows(y_local, starts, ends, group=None):
    """All-gather of the ranks' y blocks (torch tensors, 1-D) into the full y
    on every rank; blocks may differ in length."""
    import torch
    import torch.distributed as dist
    world = len(starts)
    counts = [int(e - s) for s, e in zip(starts, ends)]
    top = max(counts) if counts else 0
    buf = torch.zeros(top, dtype=y_local.dtype, device=y_local.device)
    buf[:y_local.numel()] = y_local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)])


class ShardedY:
    """y of a row-sharded SpMV as `world` blocks of `maxrows` entries, rank
    r's rows at r * maxrows: each rank's kernel writes its own block
    (local()), and one in-place all-gather (NCCL over NVLink on GPUs, gloo
    on the host) gives every rank the whole y, e.g. as the x of the next
    iteration.  The padding keeps the blocks equal-sized, which the
    collective needs; full() drops it."""

    def __init__(self, starts, ends, rank: int, dtype, device):
        import torch
        self.counts = [int(e - s) for s, e in zip(starts, ends)]
        self.world = len(self.counts)
        self.rank = int(rank)
        self.maxrows = max(self.counts) if self.counts else 0
        self.buf = torch.zeros(self.world * self.maxrows, dtype=dtype, device=device)

    def local(self):
        """This rank's rows (a view into the gathered buffer)."""
        return self.buf.narrow(0, self.rank * self.maxrows, self.counts[self.rank])

    def allgather(self, group=None) -> None:
        import torch.distributed as dist
        if self.world > 1 and self.maxrows > 0:
            dist.all_gather_into_tensor(
                self.buf, self.buf.narrow(0, self.rank * self.maxrows, self.maxrows), group=group)

    def full(self):
        """All N entries in row order (a new tensor)."""
        import torch
        return torch.cat([self.buf.narrow(0, r * self.maxrows, c)
                          for r, c in enumerate(self.counts)])

    def gather_bytes(self) -> int:
        """Bytes one rank receives per all-gather (the other ranks' blocks)."""
        return (self.world - 1) * self.maxrows * self.buf.element_size()


class PeerY:
    """y of a row-sharded SpMV exchanged by the SpMV's own stores
    (RowShardedCSR.spmv_allgather): every rank holds a full-length y buffer,
    and each rank's kernel stores its rows into all ranks' buffers -- peers'
    buffers mapped through a torch symmetric-memory rendezvous when the
    world has more than one rank (stores over NVLink, no multicast), this
    GPU's own buffer alone otherwise -- followed by the rendezvous' barrier.
    Every run of this build has one GPU, so the world > 1 branch has not run
    on GPUs."""

    def __init__(self, N: int, dtype, device, group=None):
        import torch
        import torch.distributed as dist
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.hdl = None
        if self.world > 1:
            if self.world > 8:
                raise ValueError("the fused exchange stores to at most 8 buffers")
            import torch.distributed._symmetric_memory as symm
            self.buf = symm.empty(N, dtype=dtype, device=device)
            self.hdl = symm.rendezvous(self.buf, group or dist.group.WORLD)
            self.ptrs = [int(q) for q in self.hdl.buffer_ptrs]
        else:
            self.buf = torch.zeros(N, dtype=dtype, device=device)
            self.ptrs = [self.buf.data_ptr()]
        # the destination addresses in device memory, as the kernel reads them
        self.ptrs_dev = torch.tensor(self.ptrs, dtype=torch.int64, device=device)

    def rows_ptr(self, r0: int) -> int:
        """Device address of row r0 of this rank's buffer."""
        return self.buf.data_ptr() + int(r0) * self.buf.element_size()

    def barrier(self) -> None:
        """After every rank's stores: all buffers complete (stream-ordered)."""
        if self.hdl is not None:
            self.hdl.barrier(channel=0)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The largest `value` over all ranks (the time of the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
