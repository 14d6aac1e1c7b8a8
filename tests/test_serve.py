"""Host logic of the serving loop (CPU only): admission with LRU eviction,
copy-run merging, batch formation and the arrival process."""
import collections

import numpy as np
import pytest

from sciwasm.sparse_b200 import serve


def test_admission_budget_and_lru_order():
    a = serve.AdmissionController(100)
    a.commit("a", 40)
    a.commit("b", 30)
    a.commit("c", 20)
    a.touch("a")  # order now b, c, a
    assert a.plan_admit(10) == []
    assert a.plan_admit(20) == ["b"]          # 90 + 20 - 100 = 10 needed
    assert a.plan_admit(45) == ["b", "c"]     # 35 needed
    a.release("b")
    assert a.used == 60 and list(a.entries) == ["c", "a"]


def test_admission_pinned_busy_and_refusal():
    a = serve.AdmissionController(100)
    a.commit("p", 50, pinned=True)
    a.commit("q", 30)
    a.commit("r", 10)
    assert a.plan_admit(20, busy={"q"}) == ["r"]          # 10 needed
    with pytest.raises(serve.AdmissionError):
        a.plan_admit(45, busy={"q"})          # only r (10) may go, 35 needed
    with pytest.raises(serve.AdmissionError):
        a.plan_admit(101)                     # larger than the budget
    with pytest.raises(serve.AdmissionError):
        a.plan_admit(20, evict=False)         # no eviction allowed
    with pytest.raises(ValueError):
        a.commit("q", 1)


def test_admission_free_memory_bound():
    a = serve.AdmissionController(1000)
    a.commit("a", 100)
    a.commit("b", 100)
    # the budget has room, the device does not: evict until the bytes are free
    assert a.plan_admit(150, free_bytes=60) == ["a"]
    assert a.plan_admit(150, free_bytes=-40) == ["a", "b"]
    with pytest.raises(serve.AdmissionError):
        a.plan_admit(150, free_bytes=-100)


def test_matrix_bytes_counts_storages_and_plans():
    N, nnz = 1000, 5000
    base = 4 * (N + 1) + 4 * nnz
    assert serve.matrix_bytes(N, nnz, ("f32",)) == base + 4 * nnz
    assert serve.matrix_bytes(N, nnz, ("f32", "bf16")) == base + 6 * nnz
    assert serve.matrix_bytes(N, nnz, ("f32",), ("f64",), "f64") == \
        base + 12 * nnz + serve.plan_bytes(N, nnz, np.float64)


def test_merge_runs():
    pairs = [(0, 100, 8), (8, 108, 8), (16, 200, 8), (24, 208, 8), (40, 216, 8)]
    assert serve.merge_runs(pairs) == [[0, 100, 16], [16, 200, 16], [40, 216, 8]]
    assert serve.merge_runs([]) == []


class _FakePool:
    def __init__(self, sizes):
        M = collections.namedtuple("M", "N")
        self.mats = {k: M(v) for k, v in sizes.items()}
        self.max_rows = max(sizes.values())


def _req(rid, mat, op="spmv", storage="f32"):
    return serve.Request(rid, 0.0, mat, op, storage, None, None)


def test_take_respects_batch_arena():
    pool = _FakePool({"A": 1000, "L": 2000, "B": 100_000})
    srv = serve.Server(pool, max_batch=4, slots=2, arena_bytes=1 << 20)
    pend = collections.deque([_req(0, "A"), _req(1, "L", "spts"), _req(2, "L", "spts"),
                              _req(3, "A", "spmv", "bf16"), _req(4, "A"), _req(5, "A")])
    take = srv._take(pend, srv.arena_bytes)
    # solves carry their own work vectors: two solves of L share a batch
    assert [r.rid for r in take] == [0, 1, 2, 3]
    assert [r.rid for r in pend] == [4, 5]
    # arena: sized for the largest request (two B); a third B waits and so
    # does everything behind it
    assert srv.arena_bytes == 2 * 2 * 400_128
    pend = collections.deque([_req(10, "B"), _req(11, "B"), _req(12, "B"), _req(13, "A")])
    take = srv._take(pend, srv.arena_bytes)
    assert [r.rid for r in take] == [10, 11] and [r.rid for r in pend] == [12, 13]
    # a solve takes x, y and its work vector in the arena
    pend = collections.deque([_req(20, "B", "spts"), _req(21, "B", "spts")])
    take = srv._take(pend, 5 * 400_128)
    assert [r.rid for r in take] == [20] and [r.rid for r in pend] == [21]


def test_server_arena_holds_largest_request():
    pool = _FakePool({"big": 30_000_000})
    srv = serve.Server(pool, arena_bytes=1 << 20)
    assert srv.arena_bytes >= 2 * 8 * 30_000_000
    assert srv.spts_arena_bytes >= 3 * 8 * 30_000_000


def test_poisson_arrivals():
    t = serve.poisson_arrivals(1000.0, 2.0, seed=3)
    assert np.all(np.diff(t) > 0) and t[-1] < 2.0
    assert 1800 < t.size < 2200
    assert np.array_equal(t, serve.poisson_arrivals(1000.0, 2.0, seed=3))


def test_take_drops_cancelled_requests():
    pool = _FakePool({"A": 1000, "L": 2000})
    srv = serve.Server(pool, max_batch=4, slots=2, arena_bytes=1 << 20)
    reqs = [_req(0, "A"), _req(1, "L", "spts"), _req(2, "A"), _req(3, "A")]
    srv.cancel(1)
    srv.cancel(3)
    pend = collections.deque(reqs)
    take = srv._take(pend, srv.arena_bytes)
    assert [r.rid for r in take] == [0, 2] and not pend
    assert [r.status for r in reqs] == ["pending", "cancelled", "pending", "cancelled"]


class _Refused(Exception):
    pass


def test_pool_rolls_back_after_an_injected_allocation_failure(monkeypatch):
    """A failed device allocation while a matrix is admitted leaves the pool's
    accounting as it was (the reference's parallel calls resolve to -1 and
    keep their state, src/parallel/src/sparse32.js:2640-2651)."""
    from sciwasm.sparse_b200 import _lib
    monkeypatch.setattr(serve, "device_free_bytes", lambda: 1 << 40)

    def no_memory(*a, **k):
        raise _lib.SparseError("sb_malloc", _lib.SB_ENOMEM, "injected allocation failure")
    monkeypatch.setattr(serve, "csr_from_host", no_memory)
    pool = serve.ResidentPool(budget_bytes=10**9)
    rp = np.array([0, 1, 2], np.int32)
    with pytest.raises(_lib.SparseError) as ei:
        pool.add("m", rp, np.array([0, 1], np.int32), np.ones(2))
    assert ei.value.status == _lib.SB_ENOMEM
    assert pool.admission.used == 0 and not pool.admission.entries and not pool.mats
    # the failure inside the attach step (e.g. a plan that cannot be built)
    # is rolled back the same way, and a later admission still works
    monkeypatch.setattr(serve, "csr_from_host", lambda *a, **k: object())

    def attach_fails(*a, **k):
        raise _Refused("plan allocation failed")
    monkeypatch.setattr(pool, "_attach", attach_fails)
    with pytest.raises(_Refused):
        pool.add("m", rp, np.array([0, 1], np.int32), np.ones(2))
    assert pool.admission.used == 0 and "m" not in pool.admission.entries


def test_slot_creation_failure_closes_the_slots_already_made(monkeypatch):
    made, closed = [], []

    class FakeSlot:
        def __init__(self, index, *a, **k):
            if len(made) == 2:
                raise _Refused("injected arena allocation failure")
            self.index, self.busy = index, False
            made.append(index)

        def close(self):
            closed.append(self.index)

    monkeypatch.setattr(serve, "_Slot", FakeSlot)
    srv = serve.Server(_FakePool({"A": 10}), slots=2, spts_slots=1, priorities=False)
    with pytest.raises(_Refused):
        srv._serve_batched([])
    assert made == [0, 1] and sorted(closed) == [0, 1]
