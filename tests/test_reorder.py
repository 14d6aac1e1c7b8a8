"""Row reordering on the CPU: the oracle's sort_rows_by_nnz,
sort_y_rows_by_nnz and calculate_csr_locality_index against answers derived
by hand from src/parallel/src/sparse32.js:2148-2269."""
import numpy as np


def test_sort_rows_by_nnz_kat(oracle):
    # row lengths 3, 0, 1, 2 -> stable order by length: rows 1, 2, 3, 0
    rp = np.array([0, 3, 3, 4, 6])
    col = np.array([0, 2, 3, 1, 0, 3])
    val = np.arange(6, dtype=np.float32)
    r = oracle.sort_rows_by_nnz(rp, col, val)
    assert r["permutation"].tolist() == [1, 2, 3, 0]
    assert r["row_ptr"].tolist() == [0, 0, 1, 3, 6]
    assert r["col"].tolist() == [1, 0, 3, 0, 2, 3]
    assert r["val"].tolist() == [3, 4, 5, 0, 1, 2]
    assert r["nnz_per_row"].tolist() == [0, 1, 2, 3]
    assert r["small_rows"].tolist() == [1, 2, 3, 4]  # rows with <= 0, 1, 2, 3 nonzeros
    y = np.array([10, 11, 12, 13], np.float32)
    assert oracle.unpermute_rows(r["permutation"], y).tolist() == [13, 10, 11, 12]


def test_locality_index_kat(oracle):
    # N = 20 (two 16-column lines).  Accesses (row, line): (0,0) first touch,
    # (0,0) distance 0, (1,1) first, (5,0) distance 5, (19,1) distance 18:
    # two of five accesses reuse within 16 rows -> 40%.
    rp = np.zeros(21, np.int64)
    rows = {0: [0, 3], 1: [17], 5: [2], 19: [18]}
    for r in range(20):
        rp[r + 1] = rp[r] + len(rows.get(r, []))
    col = np.concatenate([rows[r] for r in sorted(rows)])
    assert oracle.csr_locality_index(rp, col) == 40.0
