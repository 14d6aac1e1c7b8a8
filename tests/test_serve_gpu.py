"""Batched triangular solves and the serving loop on the device.

* SptsBatch: every system of a batch is bit-identical to the single hybrid
  solve (same arithmetic), across repeated runs and interleaved single solves
  on the same plan (ready-flag epochs), for f32, f32 with f64 accumulation
  and f64.
* Serving: each result is the same alone and in the mix (bit-identical: a
  row's arithmetic depends only on its own matrix), the per-call path agrees
  within the stated tolerance, and every result is within 1e-5 of the FP64
  oracle on the stored values.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from sciwasm.sparse_b200 import _lib, serve, synth
from sciwasm.sparse_b200.sparse import PinnedBuffer, _STORAGE

pytestmark = pytest.mark.gpu

SERVE_TOL = 1e-5  # relative (max-norm) error against the FP64 oracle


def _factors(dt):
    out = [synth.laplacian_3d_lower(12, dtype=dt),
           synth.random_lower(20_000, per_row=7, band=500, seed=5, dtype=dt),
           synth.random_lower(3_000, per_row=3, band=40, seed=6, dtype=dt),
           (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.0], dt))]
    return out


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


@pytest.mark.parametrize("grid", [0, 1, 3])
@pytest.mark.parametrize("dt,policy", [(np.float32, "native"), (np.float32, "f64"),
                                       (np.float64, "native")])
def test_spts_batch_bit_identical_to_hybrid(gpu, oracle, dt, policy, grid):
    facs = _factors(dt)
    Ls = [gpu.csr_from_host(rp, col, val) for rp, col, val in facs]
    plans = [gpu.SptsPlan(L) for L in Ls]
    bs = [gpu.DeviceArray.from_host(synth.uniform_vec(L.N, 40 + i, dtype=dt))
          for i, L in enumerate(Ls)]
    ys = [gpu.DeviceArray(L.N, dt) for L in Ls]
    want = []
    for L, b in zip(Ls, bs):
        bv = gpu.sparse_vec_t(b, L.N)
        yv = gpu.create_vec(L.N, 0, dt)
        gpu.spts(L, bv, yv, algo="hybrid", policy=policy)
        want.append(yv.array())
    # grid 0: one warp per chunk; 1 or 3: a capped grid whose warps loop
    ex = gpu.SptsBatch(dt, policy, capacity=8, blocks_per_sm=grid)
    pol = _lib.SB_SPTS_ACC_F64 if policy == "f64" else _lib.SB_SPTS_ACC_NATIVE
    for rep in range(3):
        for y in ys:
            y.fill_zero()
        ex.run(zip(plans, bs, ys))
        gpu.synchronize()
        for i, (y, w) in enumerate(zip(ys, want)):
            assert np.array_equal(_bits(y.to_host()), _bits(w)), (rep, i)
        # a single solve on the same plan between batched runs
        _lib.call("sb_spts_solve", plans[0].ptr, _lib.SB_SPTS_HYBRID, pol, bs[0].ptr, ys[0].ptr,
                  None)
        gpu.synchronize()
    code = C.c_int(0)
    _lib.call("sb_device_status", C.byref(code))
    assert code.value == 0
    rp, col, val = facs[1]
    truth = oracle.truth_spts(rp, col, val, synth.uniform_vec(Ls[1].N, 41, dtype=dt))
    assert rel_err(want[1], truth) <= (1e-5 if dt == np.float32 else 1e-12)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_spts_batch_own_work_vectors(gpu, dt):
    """Solves with their own work vectors: one plan three times in a run (with
    different right-hand sides) while a second executor, on another stream,
    solves the same plan on its work vector and a third solve uses the plan's
    own; every result equals the single hybrid solve's bits."""
    rp, col, val = synth.random_lower(20_000, per_row=7, band=500, seed=5, dtype=dt)
    L = gpu.csr_from_host(rp, col, val)
    plan = gpu.SptsPlan(L)
    bs = [gpu.DeviceArray.from_host(synth.uniform_vec(L.N, 70 + i, dtype=dt)) for i in range(5)]
    want = []
    for b in bs:
        yv = gpu.create_vec(L.N, 0, dt)
        gpu.spts(L, gpu.sparse_vec_t(b, L.N), yv, algo="hybrid")
        want.append(yv.array())
    ys = [gpu.DeviceArray(L.N, dt) for _ in bs]
    ws = [gpu.DeviceArray(L.N, dt) for _ in bs]
    s1, s2 = C.c_void_p(), C.c_void_p()
    _lib.call("sb_stream_create", C.byref(s1))
    _lib.call("sb_stream_create", C.byref(s2))
    ex1 = gpu.SptsBatch(dt, "native", capacity=4, blocks_per_sm=1)
    ex2 = gpu.SptsBatch(dt, "native", capacity=4, blocks_per_sm=1)
    for rep in range(2):
        for y in ys:
            y.fill_zero()
        gpu.synchronize()
        ex1.run([(plan, bs[0], ys[0], ws[0]), (plan, bs[1], ys[1], ws[1]),
                 (plan, bs[2], ys[2]), (plan, bs[3], ys[3], ws[3])], stream=s1.value)
        ex2.run([(plan, bs[4], ys[4], ws[4])], stream=s2.value)
        # non-blocking streams: the legacy stream's synchronize does not cover them
        gpu.synchronize(s1.value)
        gpu.synchronize(s2.value)
        for i, (y, w) in enumerate(zip(ys, want)):
            assert np.array_equal(_bits(y.to_host()), _bits(w)), (rep, i)
    code = C.c_int(0)
    _lib.call("sb_device_status", C.byref(code))
    assert code.value == 0
    _lib.call("sb_stream_destroy", s1)
    _lib.call("sb_stream_destroy", s2)


def test_spts_batch_rejects_bad_items(gpu):
    L32 = gpu.csr_from_host(*synth.laplacian_3d_lower(6, dtype=np.float32))
    L64 = gpu.csr_from_host(*synth.laplacian_3d_lower(6, dtype=np.float64))
    p32, p64 = gpu.SptsPlan(L32), gpu.SptsPlan(L64)
    b = gpu.DeviceArray(L32.N, np.float64)
    y = gpu.DeviceArray(L32.N, np.float64)
    ex = gpu.SptsBatch(np.float32, "native", capacity=4)
    with pytest.raises(_lib.SparseError):
        ex.run([(p64, b, y)])                       # plan dtype differs
    with pytest.raises(_lib.SparseError):
        ex.run([(p32, b, y), (p32, b, y)])          # one plan twice on its own vector
    w_odd = gpu.DeviceArray(L32.N + 1, np.float32)
    with pytest.raises(_lib.SparseError):           # work vector not 4-byte aligned
        ex.run([(p32, b, y, gpu.DeviceArray(L32.N, np.float32, w_odd.ptr + 2))])
    with pytest.raises(ValueError):
        ex.run([(p32, b, y)] * 5)                   # above capacity
    upper = gpu.csr_from_host(np.array([0, 2, 3], np.int32), np.array([0, 1, 1], np.int32),
                              np.array([1.0, 2.0, 3.0], np.float32))
    pu = gpu.SptsPlan(upper)
    assert not pu.solvable
    with pytest.raises(_lib.SparseError):
        ex.run([(pu, b, y)])
    ex.run([])  # an empty batch is a no-op
    gpu.synchronize()


def test_growth_estimate(gpu):
    for rp, col, val in _factors(np.float64):
        plan = gpu.SptsPlan(gpu.csr_from_host(rp, col, val))
        want = 0.0
        for i in range(rp.size - 1):
            s, e = rp[i], rp[i + 1]
            want = max(want, np.sum(np.abs(val[s:e - 1])) / abs(val[e - 1]))
        assert plan.growth() == pytest.approx(want, rel=1e-12)


# ------------------------------------------------------------ serving


def _serving_pool(gpu):
    pool = serve.ResidentPool(budget_bytes=4 << 30, reserve_bytes=0)
    host = {}

    def add(name, rp, col, val, spmv=("f32",), spts=()):
        pool.add(name, rp, col, val, spmv, spts)
        host[name] = (rp, col, np.asarray(val, np.float64))

    add("lap2d", *synth.laplacian_2d(70, dtype=np.float64), spmv=("f32", "bf16"))
    add("band", *synth.banded(30_000, half=5, seed=2), spmv=("f32", "bf16"))
    add("power", *synth.power_law(20_000, seed=4, cap=600, dtype=np.float64),
        spmv=("f32", "bf16"))
    add("tiny", *synth.laplacian_2d(3, dtype=np.float64), spmv=("f32",))
    add("lap3d_L", *synth.laplacian_3d_lower(14), spmv=("f32",), spts=("f32", "f64"))
    add("rand_L", *synth.random_lower(8_000, per_row=7, band=300, seed=9), spts=("f32",))
    return pool, host


def _requests(pool, nreq, seed, rate_hz):
    rng = np.random.default_rng(seed)
    kinds = [("lap2d", "spmv", "f32"), ("lap2d", "spmv", "bf16"), ("band", "spmv", "f32"),
             ("band", "spmv", "bf16"), ("power", "spmv", "f32"), ("power", "spmv", "bf16"),
             ("tiny", "spmv", "f32"), ("lap3d_L", "spmv", "f32"), ("lap3d_L", "spts", "f32"),
             ("lap3d_L", "spts", "f64"), ("rand_L", "spts", "f32")]
    picks = rng.integers(0, len(kinds), nreq)
    t = serve.poisson_arrivals(rate_hz, 10.0, seed=seed)[:nreq]
    sizes = [pool.mats[kinds[k][0]].N * (8 if kinds[k][2] == "f64" else 4) for k in picks]
    buf = PinnedBuffer(2 * sum(serve._al(s) for s in sizes))
    reqs, off = [], 0
    for i, k in enumerate(picks):
        name, op, st = kinds[k]
        N = pool.mats[name].N
        vt = np.float64 if st == "f64" else np.float32
        x = buf.view(off, N, vt)
        x[:] = synth.uniform_vec(N, 1000 + i, dtype=vt)
        off += serve._al(x.nbytes)
        reqs.append(serve.Request(i, float(t[i]), name, op, st, x, None))
    for r in reqs:  # outputs after all inputs: inputs stay contiguous
        N = r.x.size
        r.y = buf.view(off, N, r.x.dtype)
        r.y[:] = np.nan
        off += serve._al(r.y.nbytes)
    return reqs, buf


def _truth(oracle, pool, host, r):
    rp, col, val = host[r.matrix]
    if r.op == "spts":
        v = val.astype(_STORAGE[r.storage])
        return oracle.truth_spts(rp, col, v, r.x.astype(v.dtype))
    vals = pool.mats[r.matrix].csr[r.storage].val_array()
    if r.storage == "bf16":
        vals = (vals.astype(np.uint32) << 16).view(np.float32)
    return oracle.truth_csr(rp, col, vals.astype(np.float64), r.x.astype(np.float64))


def test_serving_alone_equals_mix_and_oracle(gpu, oracle):
    pool, host = _serving_pool(gpu)
    reqs, buf = _requests(pool, 160, seed=3, rate_hz=20_000.0)
    srv = serve.Server(pool, max_batch=32, slots=3)
    st = srv.serve(reqs, "batched")
    assert st["requests"] == 160 and st["batches"] < 160
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    mix = [r.y.copy() for r in reqs]
    for r, y in zip(reqs, mix):
        assert np.all(np.isfinite(y)), r.rid
        assert rel_err(y, _truth(oracle, pool, host, r)) <= SERVE_TOL, (r.rid, r.matrix, r.op)
    # alone: the same request served by itself gives the same bits
    for r, y in list(zip(reqs, mix))[::9]:
        one = serve.Request(r.rid, 0.0, r.matrix, r.op, r.storage, r.x, np.full_like(y, np.nan))
        srv.serve([one], "batched")
        assert np.array_equal(_bits(one.y), _bits(y)), (r.rid, r.matrix, r.op, r.storage)
    # the per-call path: solves are the same arithmetic (same bits), SpMV sums
    # in another order (within the tolerance)
    for r in reqs:
        r.y[:] = np.nan
    sp = srv.serve(reqs, "plain")
    assert sp["batches"] == 160
    for r, y in zip(reqs, mix):
        if r.op == "spts":
            assert np.array_equal(_bits(r.y), _bits(y)), r.rid
        else:
            assert rel_err(r.y, y) <= SERVE_TOL, r.rid
    pool.close()


def test_serving_flags_growth_for_f64_accumulation(gpu):
    pool = serve.ResidentPool(budget_bytes=1 << 30, reserve_bytes=0, growth_threshold=1.0)
    rp, col, val = synth.laplacian_3d_lower(8)
    m = pool.add("dominant", rp, col, val, ("f32",), ("f32",))
    assert m.growth == pytest.approx(0.5) and m.policy["f32"] == "native"
    val2 = val.copy()
    val2[rp[1:] - 1] = 0.25   # small diagonal: growth 12 > 1
    m2 = pool.add("weak", rp, col, val2, ("f32",), ("f32",))
    assert m2.growth == pytest.approx(12.0) and m2.policy["f32"] == "f64"
    pool.close()


def test_pool_admission_evicts_lru_and_refuses_pinned(gpu):
    rp, col, val = synth.banded(50_000, half=5, seed=1)
    one = serve.matrix_bytes(rp.size - 1, col.size, ("f32",))
    # CSR only: these sizes count the CSR bytes (the DIA form a pool adds by
    # default is charged on top, see test_pool_charges_the_chosen_format)
    pool = serve.ResidentPool(budget_bytes=2 * one + 100, reserve_bytes=0, spmv_format="csr")
    pool.add("a", rp, col, val)
    pool.add("b", rp, col, val)
    pool.get("a")                       # b is now the least recently used
    pool.add("c", rp, col, val)
    assert set(pool.mats) == {"a", "c"} and pool.admission.used == 2 * one
    pool.close()
    pool = serve.ResidentPool(budget_bytes=2 * one + 100, reserve_bytes=0, spmv_format="csr")
    pool.add("a", rp, col, val, pinned=True)
    pool.add("b", rp, col, val, pinned=True)
    with pytest.raises(serve.AdmissionError):
        pool.add("c", rp, col, val)
    assert set(pool.mats) == {"a", "b"}
    pool.close()


def test_serving_cancelled_requests_are_dropped(gpu, oracle):
    """Requests withdrawn before they join a batch are not run (y keeps its
    NaN fill, status "cancelled"); the others are served as usual, in both
    modes, and a cancel from another thread while the loop runs is safe."""
    import threading
    pool, host = _serving_pool(gpu)
    for mode in ("batched", "plain"):
        reqs, buf = _requests(pool, 60, seed=7, rate_hz=2_000.0)
        srv = serve.Server(pool, max_batch=16, slots=2)
        drop = {r.rid for r in reqs if r.rid % 5 == 2}
        for rid in sorted(drop)[:4]:
            srv.cancel(rid)            # before the loop starts
        # the rest arrive 0.3 s into the trace and are cancelled from another
        # thread 0.05 s into it, while the loop runs
        late = sorted(drop)[4:]
        for r in reqs:
            if r.rid in late:
                r.t_arrival = 0.3 + 1e-4 * r.rid

        def cancel_late():
            import time
            time.sleep(0.05)
            for rid in late:
                srv.cancel(rid)
        th = threading.Thread(target=cancel_late)
        th.start()
        st = srv.serve(reqs, mode)
        th.join()
        assert st["cancelled"] == len(drop) and st["requests"] == 60 - len(drop)
        for r in reqs:
            if r.rid in drop:
                assert r.status == "cancelled" and np.all(np.isnan(r.y)), r.rid
            else:
                assert r.status == "done", r.rid
                assert rel_err(r.y, _truth(oracle, pool, host, r)) <= SERVE_TOL, r.rid
    pool.close()


def test_pool_charges_the_chosen_format(gpu, oracle):
    """With the default format choice a banded matrix is kept in DIA beside its
    CSR; the DIA bytes (offsets once, data per storage) are charged to its
    entry, and when the budget has no room for them the matrix stays CSR."""
    rp, col, val = synth.banded(50_000, half=5, seed=1)
    N = rp.size - 1
    csr_b = serve.matrix_bytes(N, col.size, ("f32", "bf16"))
    dia_b = 4 * 11 + 11 * N * (4 + 2)
    pool = serve.ResidentPool(budget_bytes=10 * csr_b, reserve_bytes=0)
    m = pool.add("band", rp, col, val, spmv_storages=("f32", "bf16"))
    assert m.format == "dia" and pool.admission.used == csr_b + dia_b
    assert isinstance(m.fmt["f32"], gpu.sparse_DIA_t) and m.fmt["bf16"].dtype == np.uint16
    pool.close()
    pool = serve.ResidentPool(budget_bytes=csr_b + 100, reserve_bytes=0)
    m = pool.add("band", rp, col, val, spmv_storages=("f32", "bf16"))
    assert m.format == "csr" and pool.admission.used == csr_b
    assert m.fmt["f32"] is m.csr["f32"]
    pool.close()
