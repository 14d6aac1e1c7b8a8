"""coo_csc and the CSC triangular solve on the device, bit-exact with the
oracle's coo_csc and column sweep."""
import numpy as np
import pytest

from sciwasm.sparse_b200 import _lib, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_coo_csc_and_spts_csc(gpu, oracle, dt):
    for rp, col, val in (synth.random_lower(20_000, per_row=7, band=2000, seed=4, dtype=dt),
                         synth.laplacian_3d_lower(16, dtype=dt)):
        row = synth.csr_to_coo_rows(rp)
        rng = np.random.default_rng(1)
        perm = rng.permutation(row.size)  # an unsorted COO
        A = gpu.coo_from_host(row[perm], col[perm], val[perm], rp.size - 1)
        S = gpu.coo_csc(A)
        cp, r, v = oracle.coo_csc(row[perm], col[perm], val[perm], rp.size - 1)
        assert np.array_equal(S.col_array(), cp) and np.array_equal(S.row_array(), r)
        assert np.array_equal(S.val_array(), v)
        b = synth.uniform_vec(rp.size - 1, 3, dtype=dt)
        y = gpu.create_vec(rp.size - 1, 0, dt)
        gpu.spts_csc(S, gpu.vec_from_host(b), y)
        assert np.array_equal(y.array().view(np.uint8), oracle.spts_csc(cp, r, v, b).view(np.uint8))


def test_spts_csc_rejects_bad_structure(gpu):
    # column 0 starts with row 1 (diagonal missing)
    S = gpu.sparse_CSC_t(gpu.DeviceArray.from_host(np.array([0, 1, 2], np.int32)),
                         gpu.DeviceArray.from_host(np.array([1, 1], np.int32)),
                         gpu.DeviceArray.from_host(np.array([1.0, 2.0], np.float32)), 2, 2)
    with pytest.raises(_lib.SparseError):
        gpu.spts_csc(S, gpu.vec_from_host(np.ones(2, np.float32)), gpu.create_vec(2))
