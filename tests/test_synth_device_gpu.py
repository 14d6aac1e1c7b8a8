"""Device-side synthetic generators: the structure each one promises (sorted
distinct columns, in range, the diagonal last in each factor row), so that
workloads built on the device match the host generators' shapes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check_csr(A, lower=False):
    rp, col = A.row_array(), A.col_array()
    N = A.N
    assert rp[0] == 0 and rp[-1] == col.size == A.nnz
    assert np.all(np.diff(rp) >= 0)
    assert col.size == 0 or (col.min() >= 0 and col.max() < N)
    rows = np.repeat(np.arange(N), np.diff(rp))
    key = rows.astype(np.int64) * N + col
    assert np.all(np.diff(key) > 0)  # sorted and distinct within each row
    if lower:
        assert np.all(np.diff(rp) >= 1)
        assert np.array_equal(col[rp[1:] - 1], np.arange(N))  # diagonal last
        assert np.all(col <= rows)
    return rp, col


def test_stencils(gpu):
    from sciwasm.sparse_b200 import synth, synth_device as sd
    A = sd.laplacian_2d(37)
    rp, col = _check_csr(A)
    hrp, hcol, hval = synth.laplacian_2d(37, dtype=np.float32)
    assert np.array_equal(rp, hrp) and np.array_equal(col, hcol)
    assert np.array_equal(A.val_array(), hval)
    L = sd.laplacian_3d_lower(9)
    rp, col = _check_csr(L, lower=True)
    hrp, hcol, hval = synth.laplacian_3d_lower(9, dtype=np.float32)
    assert np.array_equal(rp, hrp) and np.array_equal(col, hcol)
    assert np.array_equal(L.val_array(), hval)
    B = sd.banded(1000, half=5)
    rp, col = _check_csr(B)
    assert A.nnz > 0 and B.nnz == 11 * 1000 - 30


@pytest.mark.parametrize("N", [1, 50, 20_000])
def test_random_structures(gpu, N):
    from sciwasm.sparse_b200 import synth_device as sd
    L = sd.random_lower(N, per_row=7, band=300, seed=3)
    rp, col = _check_csr(L, lower=True)
    lens = np.diff(rp)
    assert lens.max() <= 8
    rows = np.repeat(np.arange(N), lens)
    assert np.all(rows - col <= 300)
    v = L.val_array()
    diag = v[rp[1:] - 1]
    assert np.all((diag >= 2) & (diag <= 4))
    P = sd.power_law(N, cap=50, seed=2)
    rp, _ = _check_csr(P)
    assert np.diff(rp).max() <= min(50, N)
    Q = sd.poisson_rows(N, 12.0, seed=4)
    rp, col = _check_csr(Q)
    rows = np.repeat(np.arange(N), np.diff(rp))
    assert np.all(np.isin(np.arange(N), rows[col == rows]))  # every diagonal present
