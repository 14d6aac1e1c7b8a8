"""Row-sharded SpMV on one device: the blocks of every rank of a world of 3,
each multiplied by the library's kernel, concatenate to the unsharded SpMV
(the rows of a block are the same rows, summed by the same kernel shape)."""
import numpy as np
import pytest

from conftest import TOL, rel_err
from sciwasm.sparse_b200 import dist, synth

pytestmark = pytest.mark.gpu


def test_row_shards_concatenate(gpu, oracle):
    rp, col, val = synth.power_law(30_000, seed=5, cap=500, dtype=np.float64)
    x = synth.uniform_vec(30_000, 6)
    xv = gpu.vec_from_host(x)
    parts = []
    for rank in range(3):
        sh = dist.RowShardedCSR(rp, col, val, rank, 3)
        y = gpu.create_vec(max(sh.rows, 1), 0, np.float64)
        sh.spmv(xv, y)
        parts.append(y.array()[:sh.rows])
    y = np.concatenate(parts)
    truth = oracle.truth_csr(rp, col, val, x)
    assert rel_err(y, truth) <= TOL[np.dtype(np.float64)]


def _drop_rows(rp, col, val, every):
    """The matrix with the entries of every `every`-th row removed (empty rows)."""
    lens = np.diff(rp).copy()
    keep = np.ones(col.size, bool)
    for i in range(0, rp.size - 1, every):
        keep[rp[i]:rp[i + 1]] = False
        lens[i] = 0
    nrp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    return nrp, col[keep], val[keep]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_allgather_fused_emulated_ranks(gpu, dt):
    """sb_spmv_csr_allgather with a world of 3 emulated on one device: each
    rank's launch stores its rows into all three full-length y buffers (the
    stand-ins for the peers' buffers).  Every buffer then equals the unsharded
    sb_spmv_csr_ex bit for bit (same options, same per-row arithmetic; short
    rows, whole-warp long rows, and rows without entries, whose y passes on
    unchanged); a world of 1 with one buffer does too."""
    import ctypes as C
    from sciwasm.sparse_b200 import _lib
    N = 30_000
    rp, col, val = _drop_rows(*synth.power_law(N, seed=5, cap=500, dtype=dt), every=97)
    x = synth.uniform_vec(N, 6, dtype=dt)
    y0 = synth.uniform_vec(N, 7, dtype=dt)
    opts = _lib.CsrOpts(0, 4, 4, 0)
    xv = gpu.DeviceArray.from_host(x)
    A = gpu.csr_from_host(rp, col, val)
    yw = gpu.DeviceArray.from_host(y0)
    code = _lib.SB_F64 if dt == np.float64 else _lib.SB_F32
    _lib.call("sb_spmv_csr_ex", code, A.row_index.ptr, A.col_index.ptr, A.val_index.ptr,
              xv.ptr, yw.ptr, N, A.nnz, 1, C.byref(opts), None)
    gpu.synchronize()
    want = yw.to_host()
    bits = np.uint64 if dt == np.float64 else np.uint32
    for world in (3, 1):
        bufs = [gpu.DeviceArray.from_host(np.full(N, np.nan, dt)) for _ in range(world)]
        dsts = gpu.DeviceArray.from_host(np.array([b.ptr for b in bufs], np.uint64))
        keep = []
        for rank in range(world):
            sh = dist.RowShardedCSR(rp, col, val, rank, world)
            yin = gpu.DeviceArray.from_host(np.ascontiguousarray(y0[sh.r0:sh.r1]))
            keep.append((sh, yin))
            sh.spmv_allgather(xv.ptr, yin.ptr, dsts.ptr, world, opts=opts)
        gpu.synchronize()
        for b in bufs:
            assert np.array_equal(b.to_host().view(bits), want.view(bits)), world
