"""COO reductions: the oracle's restatement of diagonal_coo / min_coo against
answers derived by hand from src/sequential/src/sparse_opt_32.wat:1707-1946
(CPU only)."""
import numpy as np


def test_min_coo_walk_kat(oracle):
    # rows: 0 -> [3, -1]; 1 empty (repeats the carried -1); 2 -> [5] (5 > 0
    # with fewer than N entries -> 0); 3 -> [2, 7] (last row, two entries -> 0)
    row = np.array([0, 0, 2, 3, 3])
    val = np.array([3, -1, 5, 2, 7], np.float32)
    assert oracle.min_coo(1, row, val, 4).tolist() == [-1, -1, 0, 0]
    # the last entry is the only entry of row 2: returned before storing (0),
    # and row 3 is never reached (0)
    row = np.array([0, 0, 2])
    val = np.array([3, -1, -5], np.float32)
    assert oracle.min_coo(1, row, val, 4).tolist() == [-1, -1, 0, 0]
    # a full row (N entries) keeps a positive minimum; rows after the last
    # entry's row stay 0
    row = np.array([0, 0])
    val = np.array([4, 2], np.float32)
    assert oracle.min_coo(1, row, val, 2).tolist() == [2, 0]
    # axis 0 is not handled by the reference: the vector stays 0
    assert oracle.min_coo(0, row, val, 3).tolist() == [0, 0, 0]


def test_diagonal_coo_kat(oracle):
    row, col = np.array([0, 0, 1, 2]), np.array([0, 1, 0, 2])
    val = np.array([1, 2, 3, 4], np.float64)
    assert oracle.diagonal_coo(0, row, col, val, 3).tolist() == [1, 0, 4]
    assert oracle.diagonal_coo(-1, row, col, val, 3).tolist() == [3, 0]
    assert oracle.diagonal_coo(1, row, col, val, 3).tolist() == [2, 0]
    assert oracle.diagonal_coo(2, row, col, val, 3).tolist() == [0]


def test_sum_rows(oracle):
    row = np.array([0, 0, 2, 2, 2])
    val = np.array([1, 2, 3, 4, 5], np.float32)
    assert oracle.sum_coo_rows(1, row, val, 4).tolist() == [3, 0, 12, 0]
