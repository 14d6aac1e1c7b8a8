"""Bit-exact parity at the measured workload sizes, where size-dependent bugs
live (radix-sort digit passes over 2^22+ keys, scan carries across thousands
of blocks, the 2^27 admission edge, thousands of levels):

* format sweep, FP64: the banded matrix (4,000,000 rows, offsets -5..5,
  43,999,970 nonzeros) from a shuffled COO through the device coo_csr, then
  csr_dia and csr_ell; every output array bit-identical to the oracle's
  restatement of the reference (src/sequential/src/sparse32.js:1436-1720).
  Then SpMV in all four formats on the converted objects: DIA and ELL
  bit-identical to the oracle's serial loops, CSR and COO within 1e-12 of
  the extended-precision product.
* the power-law matrix (2,000,000 rows, row lengths min(2000, Zipf(2)+15),
  ~41M nonzeros) from a shuffled COO through coo_csr, bit-exact, and its
  DIA and ELL forms refused exactly as the reference refuses them;
* SpTS, FP64 and FP32: the lower 3-D Laplacian on a 64^3 grid (262,144 rows,
  190 levels) and the 1,000,000-row random lower factor (7 off-diagonals
  within a band of 5000, seed 3): level, level_ptr, permutation, order and
  the reordered CSR bit-identical to the oracle's level-set construction
  (src/parallel/src/sparse32.js:2942-3181), and the level-set, hybrid and
  sync-free solves bit-identical to the oracle's row kernel
  (src/parallel/src/sparse_opt_32.wat:11679-11757) and sync-free kernel
  (src/parallel/src/spts_opt_32.wat:8-117).
"""
import numpy as np
import pytest

from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu


def _ub(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(_ub(a), _ub(b))


def _shuffled_coo(rp, col, val, seed):
    row = synth.csr_to_coo_rows(rp)
    perm = np.random.default_rng(seed).permutation(row.size)
    return row[perm], col[perm], val[perm]


@pytest.fixture(scope="module")
def banded():
    rp, col, val = synth.banded(4_000_000, half=5, seed=1, dtype=np.float64)
    assert col.size == 43_999_970
    return rp, col, val


def test_banded_4m_conversions_bitexact(gpu, oracle, banded):
    rp, col, val = banded
    N = rp.size - 1
    row, c, v = _shuffled_coo(rp, col, val, seed=21)
    want_csr = oracle.coo_csr(row, c, v, N)
    A = gpu.coo_csr(gpu.coo_from_host(row, c, v, N))
    assert _same(A.row_array(), want_csr[0])
    assert _same(A.col_array(), want_csr[1])
    assert _same(A.val_array(), want_csr[2])
    # the generator's CSR is the sorted form: the stable sort must rebuild it
    assert _same(want_csr[0], rp) and _same(want_csr[1], col) and _same(want_csr[2], val)
    del row, c, v, want_csr

    want = oracle.csr_dia(rp, col, val)
    D = gpu.csr_dia(A)
    assert want is not None and D is not None
    assert (D.ndiags, D.stride) == (want[2], want[3]) == (11, N)
    assert _same(D.offset_array(), want[0])
    assert _same(D.data_array(), want[1])
    del want

    want = oracle.csr_ell(rp, col, val)
    E = gpu.csr_ell(A)
    assert want is not None and E is not None
    assert E.ncols == want[2] == 11
    assert _same(E.indices_array(), want[0])
    assert _same(E.data_array(), want[1])
    del want

    # SpMV in all four formats on the device-converted objects
    x = synth.uniform_vec(N, 0)
    y0 = np.zeros(N)
    truth = oracle.truth_csr(rp, col, val, x, y0)
    den = np.max(np.abs(truth))
    xv = gpu.vec_from_host(x)
    C = gpu.coo_from_host(synth.csr_to_coo_rows(rp), col, val, N)
    got = {}
    for name, M in (("coo", C), ("csr", A), ("dia", D), ("ell", E)):
        yv = gpu.vec_from_host(y0)
        gpu.spmv(M, xv, yv)
        got[name] = yv.array()
    for name in ("coo", "csr"):
        assert np.max(np.abs(got[name] - truth)) / den <= 1e-12, name
    off, dat = synth.csr_to_dia_host(rp, col, val)
    assert _same(got["dia"], oracle.spmv_dia(off, dat, N, x, y0))
    del off, dat
    ind, edat, nc = synth.csr_to_ell_host(rp, col, val)
    assert _same(got["ell"], oracle.spmv_ell(ind, edat, N, nc, x, y0))


def test_powerlaw_2m_coo_csr_bitexact_and_refusals(gpu, oracle):
    rp, col, val = synth.power_law(2_000_000, seed=2, dtype=np.float64, sort_cols=False)
    N = rp.size - 1
    assert col.size > 40_000_000 and int(np.diff(rp).max()) == 2000
    row, c, v = _shuffled_coo(rp, col, val, seed=22)
    want = oracle.coo_csr(row, c, v, N)
    A = gpu.coo_csr(gpu.coo_from_host(row, c, v, N))
    del row, c, v
    assert _same(A.row_array(), want[0])
    assert _same(A.col_array(), want[1])
    assert _same(A.val_array(), want[2])
    # 2000 slots x 2M rows >= 2^27: both formats are refused, as by the reference
    assert gpu.num_cols(A) == 2000
    assert oracle.csr_ell(*want) is None and gpu.csr_ell(A) is None
    assert oracle.csr_dia(*want) is None and gpu.csr_dia(A) is None


_FACTORS = {}


def _factor(name, dt):
    key = (name, np.dtype(dt))
    if key not in _FACTORS:
        _FACTORS.clear()
        if name == "lap3d64":
            _FACTORS[key] = synth.laplacian_3d_lower(64, dtype=dt)
        else:
            _FACTORS[key] = synth.random_lower(1_000_000, per_row=7, band=5000, seed=3, dtype=dt)
    return _FACTORS[key]


@pytest.mark.parametrize("name", ["lap3d64", "random_lower_1m"])
def test_level_sets_fullsize_bitexact(gpu, oracle, name):
    rp, col, val = _factor(name, np.float64)
    want = oracle.level_sets(rp, col, val)
    if name == "lap3d64":
        assert rp.size - 1 == 262_144 and col.size == 1_036_288 and want["nlevels"] == 190
    A = gpu.csr_from_host(rp, col, val)
    R = gpu.CSR_create_level_sets_with_reorder(A)
    assert R.nlevels == want["nlevels"]
    assert _same(R.level_per_row.to_host(), want["level"])
    assert _same(R.level_index.to_host(), want["level_ptr"])
    assert _same(R.permutation_index.to_host(), want["permutation"])
    assert _same(R.order_index.to_host(), want["order"])
    assert _same(R.row_array(), want["row_ptr"])
    assert _same(R.col_array(), want["col"])
    assert _same(R.val_array(), want["val"])


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("name", ["lap3d64", "random_lower_1m"])
def test_solves_fullsize_bitexact(gpu, oracle, name, dt):
    rp, col, val = _factor(name, dt)
    N = rp.size - 1
    b = synth.uniform_vec(N, 4, dtype=dt)
    A = gpu.csr_from_host(rp, col, val)
    bv = gpu.vec_from_host(b)
    row_kernel = oracle.spts_csr(rp, col, val, b)
    syncfree = oracle.spts_syncfree(rp, col, val, b)
    for algo, want in (("level", row_kernel), ("hybrid", row_kernel), ("syncfree", syncfree)):
        yv = gpu.create_vec(N, 0, dt)
        gpu.spts(A, bv, yv, algo=algo)
        assert _same(yv.array(), want), algo
    # the sync-free export on caller arrays (no plan) runs the same arithmetic
    yv = gpu.create_vec(N, 0, dt)
    gpu.spts_csr_sync_free(A, bv, yv)
    assert _same(yv.array(), syncfree)
