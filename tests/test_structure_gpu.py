"""transpose, eliminate_zeros and element-wise maps on the GPU against the
oracle: integer arrays and values bit-exact; transcendental maps within 1 ulp
(f32, after rounding the double result) / 2 ulp (f64) of the host libm."""
import numpy as np
import pytest

from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu
DT = [np.float32, np.float64]


def _ub(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _same(a, b):
    return np.array_equal(_ub(a), _ub(b))


def _with_zeros(rng, val, frac=0.2):
    v = val.copy()
    n = v.size
    idx = rng.choice(n, int(n * frac), replace=False)
    k = idx.size // 3
    v[idx[:k]] = 0.0
    v[idx[k:2 * k]] = -0.0
    v[idx[2 * k:]] = np.nan
    return v


def _mats(dt):
    rng = np.random.default_rng(0)
    out = {}
    rp, col, val = synth.banded(20_000, half=4, seed=2, dtype=dt)
    out["banded_zeros"] = (rp, col, _with_zeros(rng, val))
    rp, col, val = synth.power_law(8_000, seed=3, dtype=dt, cap=200)
    out["powerlaw_zeros"] = (rp, col, _with_zeros(rng, val, 0.05))
    out["clean"] = synth.laplacian_2d(40, dtype=dt)
    return out


@pytest.mark.parametrize("dt", DT)
def test_transpose_csr_coo(gpu, oracle, dt):
    for name, (rp, col, val) in _mats(dt).items():
        A = gpu.csr_from_host(rp, col, val)
        T = gpu.transpose(A)
        want = oracle.transpose_csr(rp, col, val)
        assert _same(T.row_array(), want[0]) and _same(T.col_array(), want[1]), name
        assert _same(T.val_array(), want[2]), name
        row = synth.csr_to_coo_rows(rp)
        TC = gpu.transpose(gpu.coo_from_host(row, col, val, rp.size - 1))
        assert _same(TC.row_array(), col) and _same(TC.col_array(), row)


@pytest.mark.parametrize("dt", DT)
def test_transpose_dia_ell(gpu, oracle, dt):
    rp, col, val = synth.banded(5_000, half=3, seed=1, dtype=dt)
    N = rp.size - 1
    off, dat, nd, stride = oracle.csr_dia(rp, col, val)
    D = gpu.dia_from_host(off, dat, N)
    TD = gpu.transpose(D)
    woff, wdat = oracle.transpose_dia(off, dat, N)
    assert _same(TD.offset_array(), woff) and _same(TD.data_array(), wdat)
    rng = np.random.default_rng(5)
    ind, edat, nc = oracle.csr_ell(rp, col, _with_zeros(rng, val, 0.1))
    E = gpu.ell_from_host(ind, edat, nc, N)
    TE = gpu.transpose(E)
    onc, wd, wi = oracle.transpose_ell(edat, ind, nc, N)
    assert TE.ncols == onc
    assert _same(TE.data_array(), wd) and _same(TE.indices_array(), wi)


@pytest.mark.parametrize("dt", DT)
def test_eliminate_zeros_coo_csr(gpu, oracle, dt):
    for name, (rp, col, val) in _mats(dt).items():
        N = rp.size - 1
        A = gpu.csr_from_host(rp, col, val)
        Z = gpu.eliminate_zeros(A)
        want = oracle.copy_nonzeros_csr(rp, col, val)
        assert Z.nnz == want[1].size, name
        assert _same(Z.row_array(), want[0]) and _same(Z.col_array(), want[1]), name
        assert _same(Z.val_array(), want[2]), name
        row = synth.csr_to_coo_rows(rp)
        ZC = gpu.eliminate_zeros(gpu.coo_from_host(row, col, val, N))
        w = oracle.copy_nonzeros_coo(row, col, val)
        assert _same(ZC.row_array(), w[0]) and _same(ZC.col_array(), w[1])
        assert _same(ZC.val_array(), w[2])


@pytest.mark.parametrize("dt", DT)
def test_eliminate_zeros_dia_ell(gpu, oracle, dt):
    rng = np.random.default_rng(7)
    rp, col, val = synth.banded(6_000, half=4, seed=3, dtype=dt)
    N = rp.size - 1
    val = _with_zeros(rng, val, 0.15)
    # make one whole diagonal zero so it is dropped
    off_all = col.astype(np.int64) - np.repeat(np.arange(N), np.diff(rp))
    val[off_all == 2] = 0.0
    off, dat, nd, stride = oracle.csr_dia(rp, col, val)
    D = gpu.dia_from_host(off, dat, N, nnz=col.size)
    ZD = gpu.eliminate_zeros(D)
    cd, cnt, woff, wdat = oracle.nonzeros_dia(off, dat, N)
    assert (ZD.ndiags, ZD.nnz) == (cd, cnt)
    assert _same(ZD.offset_array(), woff) and _same(ZD.data_array(), wdat)
    ind, edat, nc = oracle.csr_ell(rp, col, val)
    E = gpu.ell_from_host(ind, edat, nc, N, nnz=col.size)
    ZE = gpu.eliminate_zeros(E)
    onc, cnt, wd, wi = oracle.nonzeros_ell(edat, ind, nc, N)
    assert (ZE.ncols, ZE.nnz) == (onc, cnt)
    assert _same(ZE.data_array(), wd) and _same(ZE.indices_array(), wi)


def test_eliminate_zeros_unchanged_copy(gpu):
    rp, col, val = synth.laplacian_2d(16, dtype=np.float32)
    A = gpu.csr_from_host(rp, col, val)
    Z = gpu.eliminate_zeros(A)
    assert Z is not A and Z.nnz == A.nnz
    assert _same(Z.val_array(), val) and _same(Z.col_array(), col)


EXACT = ["deg2rad", "rad2deg", "sign", "abs", "neg", "sqrt", "ceil", "floor", "trunc", "nearest",
         "multiply"]
TRANS = ["expm1", "log1p", "sin", "tan", "pow"]
OPS = {n: i for i, n in enumerate(["expm1", "log1p", "sin", "tan", "pow", "deg2rad", "rad2deg",
                                   "sign", "abs", "neg", "sqrt", "ceil", "floor", "trunc",
                                   "nearest", "multiply"])}


def _ulps(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    it = np.int32 if a.dtype == np.float32 else np.int64
    ia, ib = a.view(it).astype(np.int64), b.view(it).astype(np.int64)
    ia = np.where(ia < 0, np.iinfo(it).min - ia, ia)
    ib = np.where(ib < 0, np.iinfo(it).min - ib, ib)
    d = np.abs(ia - ib)
    both_nan = np.isnan(a) & np.isnan(b)
    return np.where(both_nan, 0, d)


def _param(op):
    return {"pow": 2.5, "deg2rad": np.pi, "rad2deg": np.pi, "multiply": -1.75}.get(op, 0.0)


@pytest.mark.parametrize("dt", DT)
@pytest.mark.parametrize("op", EXACT + TRANS)
def test_maps_coo_csr_ell(gpu, oracle, dt, op):
    rng = np.random.default_rng(OPS[op])
    rp, col, val = synth.power_law(3_000, seed=4, dtype=dt, cap=100)
    val = (val * 7).astype(dt)
    if op in ("log1p", "sqrt", "pow"):
        val = np.abs(val)
    val[:5] = np.array([0.0, -0.0, 2.5, -2.5, 0.5], dt) if op not in ("log1p", "sqrt", "pow") \
        else np.array([0.0, 2.5, 3.5, 0.5, 1.0], dt)
    p = _param(op)
    A = gpu.csr_from_host(rp, col, val)
    B = gpu.map_copy(A, op, p)
    want = oracle.map_values(val, 0, OPS[op], p)
    got = B.val_array()
    if op in EXACT:
        assert _same(got, want), op
    else:
        assert _ulps(got, want).max() <= (1 if dt == np.float32 else 2), op
    gpu.map_inplace(A, op, p)
    assert _same(A.val_array(), got)
    ind, edat, nc = synth.csr_to_ell_host(rp, col, val)
    E = gpu.ell_from_host(ind, edat, nc, rp.size - 1)
    EB = gpu.map_copy(E, op, p)
    want = oracle.map_values(edat, 1, OPS[op], p)
    got = EB.data_array()
    if op in EXACT:
        assert _same(got, want), op
    else:
        assert _ulps(got, want).max() <= (1 if dt == np.float32 else 2), op


@pytest.mark.parametrize("dt", DT)
def test_sign_semantics_differ_by_format(gpu, dt):
    vals = np.array([0.0, -0.0, 3.0, -3.0, np.nan], dt)
    A = gpu.coo_from_host(np.arange(5), np.arange(5), vals, 5)
    assert gpu.sign(A).val_array().tolist() == [-1.0, -1.0, 1.0, -1.0, -1.0]
    E = gpu.ell_from_host(np.arange(5), vals, 1, 5)
    assert gpu.sign(E).data_array().tolist() == [0.0, 0.0, 1.0, -1.0, -1.0]


@pytest.mark.parametrize("dt", DT)
@pytest.mark.parametrize("op", ["abs", "sqrt", "sign", "expm1", "multiply"])
def test_maps_dia_in_band_only(gpu, oracle, dt, op):
    rp, col, val = synth.banded(3_000, half=3, seed=6, dtype=dt)
    N = rp.size - 1
    off, dat, nd, stride = oracle.csr_dia(rp, col, val)
    if op == "sqrt":
        dat = np.abs(dat)
    D = gpu.dia_from_host(off, dat, N)
    p = _param(op)
    out = gpu.map_copy(D, op, p)
    want = oracle.map_dia(off, dat, N, OPS[op], p)
    if op == "expm1":
        assert _ulps(out.data_array(), want).max() <= (1 if dt == np.float32 else 2)
    else:
        assert _same(out.data_array(), want)
    gpu.map_inplace(D, op, p)
    want_inplace = oracle.map_dia(off, dat, N, OPS[op], p, out=dat)
    if op != "expm1":
        assert _same(D.data_array(), want_inplace)
