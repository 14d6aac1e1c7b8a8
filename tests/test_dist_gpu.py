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
