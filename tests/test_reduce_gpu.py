"""COO reductions on the device, bit-exact with the oracle's restatement of
the reference's walks (NaN payloads aside: the device returns its canonical
NaN), on sorted COO matrices with empty rows, negative, zero and NaN values
and duplicate coordinates."""
import numpy as np
import pytest

from sciwasm.sparse_b200 import _lib

pytestmark = pytest.mark.gpu


def _sorted_coo(rng, N, nnz, dtype, empty_frac=0.3):
    rows = rng.integers(0, N, nnz)
    keep = rng.random(N) > empty_frac  # rows allowed to hold entries
    rows = rows[keep[rows]]
    cols = rng.integers(0, N, rows.size)
    order = np.lexsort((cols, rows))
    rows, cols = rows[order].astype(np.int32), cols[order].astype(np.int32)
    val = rng.integers(-4, 5, rows.size).astype(dtype)  # zeros and ties included
    if val.size > 3:
        val[1] = np.nan
    return rows, cols, val


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _same(a, b):
    """Bit-identical except for NaN payloads (arithmetic on a NaN gives the
    device's canonical NaN; wasm leaves NaN bits unspecified)."""
    a, b = np.asarray(a), np.asarray(b)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(_bits(a[~na]), _bits(b[~nb]))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_reductions_match_oracle(gpu, oracle, dtype, seed):
    rng = np.random.default_rng(seed)
    N = int(rng.integers(5, 400))
    rows, cols, val = _sorted_coo(rng, N, int(rng.integers(1, 6 * N)), dtype)
    A = gpu.coo_from_host(rows, cols, val, N)
    for k in sorted({0, 1, -1, 2, -3, N - 1, -(N - 1), N // 2}):
        d = A.diagonal(k).array()
        assert np.array_equal(_bits(d), _bits(oracle.diagonal_coo(k, rows, cols, val, N))), k
    assert A.diagonal(N) is None
    m = A.min(1).array()
    assert _same(m, oracle.min_coo(1, rows, val, N))
    assert not np.any(A.min(0).array())
    s = gpu.sum_coo(A, 1).array()
    assert _same(s, oracle.sum_coo_rows(1, rows, val, N))


def test_min_walk_cases(gpu, oracle):
    cases = [([0, 0, 2, 3, 3], [3, -1, 5, 2, 7], 4), ([0, 0, 2], [3, -1, -5], 4),
             ([0, 0, 2, 2], [4, 2, -3, 1], 3), ([3], [-2], 5), ([1, 1], [-2, -7], 2)]
    for rows, vals, N in cases:
        rows = np.array(rows, np.int32)
        vals = np.array(vals, np.float32)
        A = gpu.coo_from_host(rows, np.zeros_like(rows), vals, N)
        assert A.min(1).array().tolist() == oracle.min_coo(1, rows, vals, N).tolist()


def test_unsorted_rows_refused(gpu):
    A = gpu.coo_from_host(np.array([1, 0], np.int32), np.array([0, 0], np.int32),
                          np.array([1.0, 2.0], np.float32), 2)
    with pytest.raises(_lib.SparseError):
        A.min(1)
    with pytest.raises(_lib.SparseError):
        A.diagonal(0)
