"""Row reordering on the device: sort_rows_by_nnz, sort_y_rows_by_nnz and the
locality index are bit-exact with the oracle; SpMV on the reordered matrix,
unpermuted, equals SpMV on the original."""
import numpy as np
import pytest

from conftest import TOL, rel_err
from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu


def _mats():
    rp, col, val = synth.power_law(3000, seed=3, cap=200, dtype=np.float64)
    yield rp, col, val
    rp, col, val = synth.banded(2000, half=3, seed=4, dtype=np.float32)
    yield rp, col, val
    # empty rows and rows of 1-3 entries
    rng = np.random.default_rng(5)
    lens = rng.integers(0, 5, 1500)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(rng.choice(1500, l, replace=False)) for l in lens]).astype(np.int32)
    yield rp, col, rng.standard_normal(col.size).astype(np.float32)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_sort_rows_matches_oracle(gpu, oracle, k):
    rp, col, val = list(_mats())[k]
    A = gpu.csr_from_host(rp, col, val)
    B = gpu.sort_rows_by_nnz(A)
    r = oracle.sort_rows_by_nnz(rp, col, val)
    assert np.array_equal(B.row_array(), r["row_ptr"])
    assert np.array_equal(B.col_array(), r["col"])
    assert np.array_equal(B.val_array(), r["val"])
    assert np.array_equal(B.permutation_index.to_host(), r["permutation"])
    assert np.array_equal(B.nnz_row_index.to_host(), r["nnz_per_row"])
    assert [B.num_zero_rows, B.num_one_rows, B.num_two_rows, B.num_three_rows] == \
        r["small_rows"].tolist()
    # y of the reordered matrix, scattered back, equals y of the original
    x = synth.uniform_vec(A.N, 7, dtype=val.dtype)
    xv = gpu.vec_from_host(x)
    y0 = gpu.create_vec(A.N, 0, val.dtype)
    gpu.spmv(A, xv, y0)
    y1 = gpu.create_vec(A.N, 0, val.dtype)
    gpu.spmv(B, xv, y1)
    yb = y1.array()
    gpu.sort_y_rows_by_nnz(y1, B)
    assert np.array_equal(y1.array(), oracle.unpermute_rows(r["permutation"], yb))
    assert rel_err(y1.array(), y0.array()) <= TOL[np.dtype(val.dtype)]


@pytest.mark.parametrize("k", [0, 1, 2])
def test_locality_index_matches_oracle(gpu, oracle, k):
    rp, col, val = list(_mats())[k]
    A = gpu.csr_from_host(rp, col, val)
    assert gpu.calculate_csr_locality_index(A) == oracle.csr_locality_index(rp, col)


def _nn_cases():
    rng = np.random.default_rng(8)
    out = {"powerlaw": synth.power_law(30_000, seed=6, cap=300, shift=0),
           "banded": synth.banded(5_000, half=4, seed=2),
           "lap2d": synth.laplacian_2d(60, dtype=np.float64)}
    # a few rows long enough (20,000 entries) for the hash sets in global memory
    lens = np.concatenate([rng.integers(1, 30, 3000), [20_000, 20_000, 25_000]])
    N = 50_000
    lens = np.concatenate([lens, np.zeros(N - lens.size, np.int64)])
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(rng.choice(N, int(n), replace=False)) for n in lens]
                         ).astype(np.int32)
    out["long_rows"] = (rp, col, rng.standard_normal(col.size))
    return out


@pytest.mark.parametrize("name", ["powerlaw", "banded", "lap2d", "long_rows"])
def test_reorder_nn_bitexact(gpu, oracle, name):
    """reorder_NN on the output of sort_rows_by_nnz, as the reference calls it:
    walk, composed permutation and the reordered CSR bit-identical to the
    oracle's restatement; and on an unsorted matrix (ranges then mix row
    lengths), the same."""
    rp, col, val = _nn_cases()[name]
    A = gpu.csr_from_host(rp, col, val)
    S = gpu.sort_rows_by_nnz(A)
    srp, scol, sval = S.row_array(), S.col_array(), S.val_array()
    sperm = S.permutation_index.to_host()
    want = oracle.reorder_nn(srp, scol, sval, 16, sperm)
    R = gpu.reorder_NN(S, 16)
    assert np.array_equal(R.walk_index.to_host(), want["walk"])
    assert np.array_equal(R.permutation_index.to_host(), want["permutation"])
    assert np.array_equal(R.row_array(), want["row_ptr"])
    assert np.array_equal(R.col_array(), want["col"])
    assert np.array_equal(R.val_array().view(np.uint8), want["val"].view(np.uint8))
    assert np.array_equal(R.nnz_row_index.to_host(), np.diff(want["row_ptr"]))
    # unsorted input, another window
    want = oracle.reorder_nn(rp, col, val, 8, None)
    R = gpu.reorder_NN(A, 8)
    assert np.array_equal(R.walk_index.to_host(), want["walk"])
    assert np.array_equal(R.permutation_index.to_host(), want["permutation"])
    assert np.array_equal(R.col_array(), want["col"])
