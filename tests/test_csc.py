"""CSC triangular solve on the CPU: the oracle's column sweep (spts_csc)
gives the same bits as its sync-free row kernel on the same matrix in CSR,
which is what the device runs; and a hand-derived 3x3 case."""
import numpy as np
import pytest

from sciwasm.sparse_b200 import synth


def _csc_of_csr(oracle, rp, col, val):
    row = synth.csr_to_coo_rows(rp)
    return oracle.coo_csc(row, col, val, rp.size - 1)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_csc_sweep_equals_syncfree_rows(oracle, dt):
    for rp, col, val in (synth.random_lower(3000, per_row=7, band=400, seed=2, dtype=dt),
                         synth.laplacian_3d_lower(10, dtype=dt)):
        b = synth.uniform_vec(rp.size - 1, 9, dtype=dt)
        cp, r, v = _csc_of_csr(oracle, rp, col, val)
        y_csc = oracle.spts_csc(cp, r, v, b)
        y_sf = oracle.spts_syncfree(rp, col, val, b)
        assert np.array_equal(y_csc.view(np.uint8), y_sf.view(np.uint8))


def test_csc_kat(oracle):
    # L = [[2, 0, 0], [1, 4, 0], [0, 3, 5]], x = [2, 9, 16]
    # y0 = 1; y1 = (9 - 1*1)/4 = 2; y2 = (16 - 3*2)/5 = 2
    cp = np.array([0, 2, 4, 5])
    row = np.array([0, 1, 1, 2, 2])
    val = np.array([2, 1, 4, 3, 5], np.float32)
    y = oracle.spts_csc(cp, row, val, np.array([2, 9, 16], np.float32))
    assert y.tolist() == [1, 2, 2]
