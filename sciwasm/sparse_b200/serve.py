"""Serving SpMV / SpTS requests on resident matrices with continuous batching.

No counterpart in the reference (a browser library with a single caller).
The pieces:

* `AdmissionController`: HBM accounting for resident matrices.  It keeps a
  byte budget, evicts unpinned entries least recently used first, and
  refuses a matrix that cannot fit.
* `ResidentPool`: matrices uploaded once and kept in device memory.  Each
  holds its CSR index arrays, one value array per requested SpMV storage
  (f32, bf16, f64) and, for triangular factors, a level-set plan per solve
  dtype.  The analysis is paid once and amortised over every solve.  A
  factor whose growth estimate exceeds a threshold is flagged for f64
  accumulation.
* `Server.serve(requests, mode)`: a host loop over requests whose vectors
  live in host memory (pinned, so that copies overlap with device work).
  - "batched": continuous batching.  Requests are released as their arrival
    times pass into one queue per kind.  Whenever a slot of that kind is
    free, the oldest pending requests that fit its device arena (x, y and,
    for a solve, its own work vector, so that solves of one factor can share
    a batch and overlap each other across slots) are packed into one batch:
    their inputs go up with one copy per contiguous host range, all SpMVs of
    a value storage run as one graph-replayed persistent launch (all solves
    of a dtype and accumulation policy as one graph-replayed launch), and
    the outputs come back the same way.  Slots retire as their completion
    events fire, so batches in different slots overlap on the device and
    requests that arrive meanwhile join the next batch.  SpMV and SpTS have
    their own slots, so a short SpMV never waits behind a deep solve.
  - "plain": the per-call path.  Each request runs alone, in arrival order:
    copy in, one library call, copy out, synchronise.
  A request's latency is the time from its arrival until the host sees its
  result.
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import call
from .sparse import (BatchExecutor, DeviceArray, SptsBatch, SptsPlan, _STORAGE, _dtcode,
                     csr_from_host, csr_with_storage, sparse_CSR_t, sparse_DIA_t, sparse_ELL_t,
                     spmv_autotune, with_storage)

_ALIGN = 256
_VEC = {"f32": np.float32, "bf16": np.float32, "f64": np.float64}


def _al(n: int) -> int:
    return (n + _ALIGN - 1) // _ALIGN * _ALIGN


class AdmissionError(RuntimeError):
    """A matrix does not fit the resident-memory budget."""


class AdmissionController:
    """Byte budget for resident objects with LRU eviction of unpinned ones."""

    def __init__(self, budget_bytes: int):
        self.budget = int(budget_bytes)
        self.used = 0
        self.entries: "collections.OrderedDict[str, tuple]" = collections.OrderedDict()

    def touch(self, name: str) -> None:
        if name in self.entries:
            self.entries.move_to_end(name)

    def plan_admit(self, nbytes: int, evict: bool = True, free_bytes: Optional[int] = None,
                   busy=()) -> list:
        """Names to evict (least recently used first) so that nbytes fit both
        the budget and, when given, the device's free memory; raises
        AdmissionError when that is impossible.  Entries in `busy` stay."""
        nbytes = int(nbytes)
        if nbytes > self.budget:
            raise AdmissionError(f"{nbytes} bytes exceed the budget of {self.budget}")
        need_budget = self.used + nbytes - self.budget
        need_free = nbytes - free_bytes if free_bytes is not None else 0
        need = max(need_budget, need_free)
        victims = []
        if need > 0:
            if not evict:
                raise AdmissionError(f"{nbytes} bytes do not fit ({self.used}/{self.budget} "
                                     f"used, {free_bytes} free on the device)")
            got = 0
            for name, (sz, pinned) in self.entries.items():
                if got >= need:
                    break
                if pinned or name in busy:
                    continue
                victims.append(name)
                got += sz
            if got < need:
                raise AdmissionError(f"{nbytes} bytes do not fit even after evicting every "
                                     f"unpinned entry")
        return victims

    def commit(self, name: str, nbytes: int, pinned: bool = False) -> None:
        if name in self.entries:
            raise ValueError(f"{name} is already resident")
        self.entries[name] = (int(nbytes), bool(pinned))
        self.used += int(nbytes)

    def release(self, name: str) -> None:
        sz, _ = self.entries.pop(name)
        self.used -= sz

    def grow(self, name: str, extra: int) -> None:
        """Charge `extra` more bytes to a resident entry (after plan_admit of
        those bytes has made room)."""
        sz, pinned = self.entries[name]
        self.entries[name] = (sz + int(extra), pinned)
        self.used += int(extra)


def device_free_bytes() -> int:
    free = C.c_size_t(0)
    total = C.c_size_t(0)
    call("sb_mem_info", C.byref(free), C.byref(total))
    return int(free.value)


def plan_bytes(N: int, nnz: int, dtype) -> int:
    """Device bytes of one level-set plan: level, perm, order (4 N each),
    reordered row_ptr / col / values, work vector, level_ptr bound."""
    vb = np.dtype(dtype).itemsize
    return 12 * N + 4 * (N + 1) + (4 + vb) * nnz + vb * N + 4 * (N + 1) + 64


def matrix_bytes(N: int, nnz: int, spmv_storages=("f32",), spts_dtypes=(),
                 base_storage: str = "f32") -> int:
    b = 4 * (N + 1) + 4 * nnz
    for s in set(spmv_storages) | set(spts_dtypes) | {base_storage}:
        b += np.dtype(_STORAGE[s]).itemsize * nnz
    for s in spts_dtypes:
        b += plan_bytes(N, nnz, _STORAGE[s])
    return b


def format_bytes(M, storages) -> int:
    """Device bytes of a DIA or ELL form kept beside the CSR: its index array
    once, its values once per storage."""
    if isinstance(M, sparse_DIA_t):
        idx, slots = 4 * M.ndiags, M.ndiags * M.N
    elif isinstance(M, sparse_ELL_t):
        idx, slots = 4 * M.ncols * M.N, M.ncols * M.N
    else:
        return 0
    return idx + sum(np.dtype(_STORAGE[s]).itemsize * slots for s in set(storages))


@dataclass
class ResidentMatrix:
    name: str
    N: int
    nnz: int
    csr: dict                                   # storage -> sparse_CSR_t (shared index arrays)
    plans: dict = field(default_factory=dict)   # "f32" / "f64" -> SptsPlan
    policy: dict = field(default_factory=dict)  # "f32" / "f64" -> "native" | "f64"
    growth: float = 0.0
    nbytes: int = 0
    fmt: dict = field(default_factory=dict)     # storage -> SpMV object (CSR, DIA or ELL)
    format: str = "csr"                         # the SpMV format chosen at admission


class ResidentPool:
    """Resident matrices under an HBM budget (default: 150 GB, or 90% of the
    device's free memory when that is less)."""

    def __init__(self, budget_bytes: Optional[int] = None, evict: bool = True,
                 growth_threshold: float = 1.0, reserve_bytes: int = 1 << 30,
                 spmv_format: str = "auto"):
        if budget_bytes is None:
            budget_bytes = min(150 * 10**9, int(device_free_bytes() * 0.9))
        if spmv_format not in ("auto", "csr"):
            raise ValueError(f"spmv_format must be 'auto' or 'csr', not {spmv_format!r}")
        self.admission = AdmissionController(budget_bytes)
        self.spmv_format = spmv_format
        self.evict = evict
        self.growth_threshold = float(growth_threshold)
        self.reserve = int(reserve_bytes)  # kept free for slot arenas and scratch
        self.mats: dict = {}
        self.busy: set = set()  # names with requests in flight (never evicted)
        self.max_rows = 0

    def add(self, name, row_ptr, col, val, spmv_storages=("f32",), spts_dtypes=(),
            pinned=False):
        """Upload a host CSR (values in any float type) and keep it resident."""
        if name in self.mats:
            raise ValueError(f"{name} is already resident")
        row_ptr = np.asarray(row_ptr, np.int32)
        N, nnz = row_ptr.size - 1, int(np.asarray(col).size)
        base = "f64" if ("f64" in spmv_storages or "f64" in spts_dtypes) else "f32"
        nb = matrix_bytes(N, nnz, spmv_storages, spts_dtypes, base)
        free = device_free_bytes() - self.reserve
        for victim in self.admission.plan_admit(nb, self.evict, free, self.busy):
            self.drop(victim)
        self.admission.commit(name, nb, pinned)
        try:
            A = csr_from_host(row_ptr, col, np.asarray(val, dtype=_STORAGE[base]))
            return self._attach(name, A, spmv_storages, spts_dtypes)
        except Exception:
            self.drop(name)
            raise

    def add_csr(self, name, A: sparse_CSR_t, spmv_storages=("f32",), spts_dtypes=(),
                pinned=False):
        """Keep an already uploaded CSR (f32 or f64 values) resident; the pool
        takes it over.  Its own arrays are already allocated, so it is
        admitted against the budget only."""
        if name in self.mats:
            raise ValueError(f"{name} is already resident")
        base = "f64" if A.dtype == np.float64 else "f32"
        nb = matrix_bytes(A.N, A.nnz, spmv_storages, spts_dtypes, base)
        for victim in self.admission.plan_admit(nb, self.evict, None, self.busy):
            self.drop(victim)
        self.admission.commit(name, nb, pinned)
        try:
            return self._attach(name, A, spmv_storages, spts_dtypes)
        except Exception:
            self.drop(name)
            raise

    def _attach(self, name, A, spmv_storages, spts_dtypes):
        base = "f64" if A.dtype == np.float64 else "f32"
        csr = {base: A}
        for s in sorted(set(spmv_storages) | set(spts_dtypes)):
            if s not in csr:
                csr[s] = csr_with_storage(A, s)
        m = ResidentMatrix(name, A.N, A.nnz, csr, nbytes=self.admission.entries[name][0])
        self.mats[name] = m
        m.fmt = {s: csr[s] for s in spmv_storages}
        if spmv_storages and self.spmv_format == "auto":
            self._choose_format(m, A, spmv_storages)
        for s in spts_dtypes:
            plan = SptsPlan(csr[s])
            m.plans[s] = plan
            if not plan.solvable:
                raise ValueError(f"{name}: not lower triangular with its diagonal stored last")
        if m.plans:
            m.growth = next(iter(m.plans.values())).growth()
            for s in m.plans:
                m.policy[s] = ("f64" if s == "f32" and m.growth > self.growth_threshold
                               else "native")
        self.max_rows = max(self.max_rows, A.N)
        return m

    def _choose_format(self, m, A, storages) -> None:
        """The SpMV format from the matrix's statistics (the admitted format
        with the fewest compulsory bytes, sb_spmv_autotune's statistics mode).
        A DIA or ELL form is kept beside the CSR (the per-call path of BF16
        values and the solves use the CSR) when the budget has room for it;
        otherwise the matrix stays CSR."""
        M, info = spmv_autotune(A, timed=False)
        if M is A:
            return
        extra = format_bytes(M, storages)
        try:
            free = device_free_bytes() - self.reserve
            victims = self.admission.plan_admit(extra, self.evict, free,
                                                self.busy | {m.name})
        except AdmissionError:
            return
        for victim in victims:
            self.drop(victim)
        self.admission.grow(m.name, extra)
        m.nbytes += extra
        base = "f64" if A.dtype == np.float64 else "f32"
        m.fmt = {s: (M if s == base else with_storage(M, s)) for s in storages}
        m.format = info["format"]

    def drop(self, name) -> None:
        m = self.mats.pop(name, None)
        if m is not None:
            for p in m.plans.values():
                p.close()
            m.plans.clear()
            m.csr.clear()
            m.fmt.clear()
        if name in self.admission.entries:
            self.admission.release(name)

    def get(self, name) -> ResidentMatrix:
        self.admission.touch(name)
        return self.mats[name]

    def close(self) -> None:
        for name in list(self.mats):
            self.drop(name)


@dataclass
class Request:
    rid: int
    t_arrival: float     # seconds after the start of the trace
    matrix: str
    op: str              # "spmv" (y = A x) or "spts" (solve L y = x)
    storage: str         # spmv: "f32" | "bf16" | "f64"; spts: "f32" | "f64"
    x: np.ndarray        # host input (pinned memory lets the copy overlap)
    y: np.ndarray        # host output, same length
    t_done: float = -1.0
    slot: int = -1
    status: str = "pending"  # "done" or "cancelled" once served


class _Event:
    def __init__(self):
        p = C.c_void_p()
        call("sb_event_create", C.byref(p))
        self.ptr = p.value

    def record(self, stream):
        call("sb_event_record", self.ptr, stream)

    def done(self) -> bool:
        return call("sb_event_query", self.ptr) == 1

    def wait(self):
        call("sb_event_synchronize", self.ptr)

    def close(self):
        if self.ptr:
            _lib.load().sb_event_destroy(self.ptr)
            self.ptr = None


def _stream(priority: Optional[int] = None):
    s = C.c_void_p()
    if priority is None:
        call("sb_stream_create", C.byref(s))
    else:
        call("sb_stream_create_priority", C.byref(s), int(priority))
    return s.value


def _priority_range():
    least, greatest = C.c_int(0), C.c_int(0)
    call("sb_stream_priority_range", C.byref(least), C.byref(greatest))
    return least.value, greatest.value


def merge_runs(pairs) -> list:
    """Maximal runs of (dst, src, nbytes) copies that are contiguous on both
    sides, as [dst, src, nbytes] lists in order."""
    runs = []
    for dst, src, nb in pairs:
        if runs and runs[-1][0] + runs[-1][2] == dst and runs[-1][1] + runs[-1][2] == src:
            runs[-1][2] += nb
        else:
            runs.append([dst, src, nb])
    return runs


def _copies(pairs, kind, stream) -> int:
    """One cudaMemcpyAsync per contiguous run; returns the copies issued."""
    fn = "sb_memcpy_htod" if kind == "h2d" else "sb_memcpy_dtoh"
    runs = merge_runs(pairs)
    for dst, src, nb in runs:
        call(fn, dst, src, nb, stream)
    return len(runs)


class _Slot:
    """One stream with its device arena and executors; serves batches of one
    kind ("spmv" or "spts")."""

    def __init__(self, index, kind, arena_bytes, max_batch, priority=None, spts_grid=0):
        self.index = index
        self.spts_grid = spts_grid
        self.kind = kind
        self.stream = _stream(priority)
        self.ev_done = _Event()
        self.arena = DeviceArray(arena_bytes, np.uint8)
        self.arena_bytes = arena_bytes
        self.max_batch = max_batch
        self.execs = {}
        self.busy = False
        self.reqs = []
        self.plans = []
        self.copies = 0
        self.launches = 0

    def executor(self, key):
        if key not in self.execs:
            if self.kind == "spmv":
                self.execs[key] = BatchExecutor(key, capacity=self.max_batch)
            else:
                dtype, policy = key
                self.execs[key] = SptsBatch(_STORAGE[dtype], policy, capacity=self.max_batch,
                                            blocks_per_sm=self.spts_grid)
        return self.execs[key]

    def close(self):
        for e in self.execs.values():
            e.close()
        self.ev_done.close()
        call("sb_stream_destroy", self.stream)
        self.arena.free()


def _vec_bytes(m: ResidentMatrix, r: Request) -> int:
    return m.N * np.dtype(_VEC[r.storage]).itemsize


class Server:
    """Continuous-batching request loop over a ResidentPool.

    SpMV and SpTS requests are batched separately, into `slots` SpMV slots
    (at most `max_batch` requests each) and `spts_slots` SpTS slots (at most
    `spts_batch` solves each), so that short SpMVs never wait behind a deep
    solve.  One launch advances all solves of its batch together.  SpTS
    launches run `spts_grid` persistent blocks per SM (0 = one warp per chunk,
    all resident at once), so a few SpTS slots run side by side without
    filling the SMs with polling warps (at 20k req/s: 3 slots of 32 solves on
    1 block per SM gave p99 22 ms, 1 slot of 256 on the full grid 69 ms).
    SpMV streams have the higher priority so that their blocks go before
    pending solve blocks."""

    def __init__(self, pool: ResidentPool, max_batch: int = 64, slots: int = 4,
                 arena_bytes: Optional[int] = None, spts_slots: int = 3, spts_batch: int = 32,
                 priorities: bool = True, spts_arena_bytes: Optional[int] = None,
                 spts_grid: int = 1):
        self.pool = pool
        self.spts_grid = int(spts_grid)  # SpTS launches: blocks per SM (0 = one warp per chunk)
        self.priorities = bool(priorities)
        self.max_batch = int(max_batch)
        self.nslots = int(slots)
        self.spts_slots = int(spts_slots)
        self.spts_batch = int(spts_batch)
        # the largest single request: x and y (and a solve's work vector)
        need = 2 * 8 * max(pool.max_rows, 1) + 2 * _ALIGN
        need_spts = 3 * 8 * max(pool.max_rows, 1) + 3 * _ALIGN
        self.arena_bytes = _al(max(int(arena_bytes or (256 << 20)), need))
        self.spts_arena_bytes = _al(max(int(spts_arena_bytes or (1 << 30)), need_spts))
        self._cancel_lock = threading.Lock()
        self._cancelled: set = set()

    def cancel(self, rid: int) -> None:
        """Withdraw request `rid` (callable from any thread, also while serve()
        runs).  A request that has not yet been put into a batch is dropped:
        its y is not written and its status becomes "cancelled".  One already
        on the device completes normally (its work cannot be recalled)."""
        with self._cancel_lock:
            self._cancelled.add(int(rid))

    def _is_cancelled(self, r: Request) -> bool:
        with self._cancel_lock:
            return r.rid in self._cancelled

    def _check(self, r: Request, m: ResidentMatrix):
        if r.op == "spmv":
            if r.storage not in m.csr:
                raise KeyError(f"request {r.rid}: {r.matrix} holds no {r.storage} values")
        elif r.op == "spts":
            if r.storage not in m.plans:
                raise KeyError(f"request {r.rid}: {r.matrix} has no {r.storage} level-set plan")
        else:
            raise ValueError(f"request {r.rid}: unknown op {r.op!r}")
        dt = np.dtype(_VEC[r.storage])
        if r.x.dtype != dt or r.y.dtype != dt or r.x.size != m.N or r.y.size != m.N:
            raise ValueError(f"request {r.rid}: x and y must be {dt} vectors of {m.N} values")
        if not (r.x.flags.c_contiguous and r.y.flags.c_contiguous):
            raise ValueError(f"request {r.rid}: x and y must be contiguous")

    # ------------------------------------------------------------ batched
    def _launch(self, slot: _Slot, reqs: list, busy_plans: frozenset = frozenset()) -> None:
        mats = [self.pool.get(r.matrix) for r in reqs]
        base = slot.arena.ptr
        off = 0
        xo, yo, wo = [], [], []
        for m, r in zip(mats, reqs):
            xo.append(off)
            off += _al(_vec_bytes(m, r))
        for m, r in zip(mats, reqs):
            yo.append(off)
            off += _al(_vec_bytes(m, r))
        for m, r in zip(mats, reqs):  # a solve's own work vector (N values)
            wo.append(off if r.op == "spts" else -1)
            off += _al(_vec_bytes(m, r)) if r.op == "spts" else 0
        h2d = [(base + o, r.x.ctypes.data, _vec_bytes(m, r)) for m, r, o in zip(mats, reqs, xo)]
        slot.copies = _copies(h2d, "h2d", slot.stream)
        groups = collections.defaultdict(list)
        for m, r, a, b, w in zip(mats, reqs, xo, yo, wo):
            vt = _VEC[r.storage]
            xd = DeviceArray(m.N, vt, base + a)
            yd = DeviceArray(m.N, vt, base + b)
            if r.op == "spmv":
                groups[r.storage].append((m.fmt.get(r.storage, m.csr[r.storage]), xd, yd, 1))
            else:
                groups[(r.storage, m.policy[r.storage])].append(
                    (m.plans[r.storage], xd, yd, DeviceArray(m.N, vt, base + w),
                     (r.matrix, r.storage)))
        slot.plans = []
        for key, jobs in groups.items():
            if slot.kind == "spmv":
                slot.executor(key).run(jobs, stream=slot.stream, overwrite=True)
            elif len(jobs) == 1 and jobs[0][4] not in busy_plans:
                # one solve whose plan is idle: the single hybrid solve on the
                # plan's own work vector and tickets, whose launch suits one
                # system (the batch kernel gives the same bits)
                plan, xd, yd, _, pk = jobs[0]
                pol = _lib.SB_SPTS_ACC_F64 if key[1] == "f64" else _lib.SB_SPTS_ACC_NATIVE
                call("sb_spts_solve", plan.ptr, _lib.SB_SPTS_HYBRID, pol, xd.ptr, yd.ptr,
                     slot.stream)
                slot.plans.append(pk)
            else:
                # every solve on its own work vector: a plan may repeat in the
                # batch and run beside other slots' solves of it
                slot.executor(key).run([j[:4] for j in jobs], stream=slot.stream)
        d2h = [(r.y.ctypes.data, base + o, _vec_bytes(m, r)) for m, r, o in zip(mats, reqs, yo)]
        slot.copies += _copies(d2h, "d2h", slot.stream)
        slot.ev_done.record(slot.stream)
        slot.launches = len(groups)
        slot.busy = True
        slot.reqs = reqs
        self.pool.busy.update(r.matrix for r in reqs)

    def _take(self, pending: collections.deque, arena: int,
              max_batch: Optional[int] = None) -> list:
        """Pending requests for one batch, oldest first: at most max_batch,
        within the arena (x and y, and a work vector for a solve, which
        then needs nothing of its plan's own: solves of a plan may share a
        batch and overlap the plan's solves in other slots)."""
        max_batch = self.max_batch if max_batch is None else max_batch
        take, keep = [], []
        used = 0
        while pending and len(take) < max_batch:
            r = pending.popleft()
            if self._is_cancelled(r):
                r.status = "cancelled"
                continue
            m = self.pool.mats[r.matrix]
            need = (3 if r.op == "spts" else 2) * _al(_vec_bytes(m, r))
            if used + need > arena:
                keep.append(r)
                break
            used += need
            take.append(r)
        pending.extendleft(reversed(keep))
        return take

    def _serve_batched(self, reqs: list) -> dict:
        # SpMV streams are the more urgent: their blocks are dispatched before
        # pending blocks of solves, whose waiting warps would otherwise hold
        # the SMs
        least, greatest = _priority_range() if self.priorities else (None, None)
        all_slots: list = []
        busy_plans: set = set()
        n = len(reqs)
        i = done = batches = copies = launches = 0
        try:
            # slots are created inside the try: if one of them cannot get its
            # stream or arena, the ones already made are closed below
            spmv_slots, spts_slots = [], []
            for k in range(self.nslots):
                spmv_slots.append(_Slot(k, "spmv", self.arena_bytes, self.max_batch, greatest))
                all_slots.append(spmv_slots[-1])
            for k in range(self.spts_slots):
                spts_slots.append(_Slot(self.nslots + k, "spts", self.spts_arena_bytes,
                                        self.spts_batch, least, self.spts_grid))
                all_slots.append(spts_slots[-1])
            kinds = {"spmv": (spmv_slots, collections.deque(), self.max_batch),
                     "spts": (spts_slots, collections.deque(), self.spts_batch)}
            t0 = time.perf_counter()
            while done < n:
                now = time.perf_counter() - t0
                while i < n and reqs[i].t_arrival <= now:
                    kinds[reqs[i].op][1].append(reqs[i])
                    i += 1
                retired = False
                for sl in all_slots:
                    if sl.busy and sl.ev_done.done():
                        t = time.perf_counter() - t0
                        for r in sl.reqs:
                            r.t_done = t
                            r.status = "done"
                        done += len(sl.reqs)
                        busy_plans.difference_update(sl.plans)
                        sl.busy = False
                        sl.reqs = []
                        retired = True
                if retired:
                    self.pool.busy = {r.matrix for s in all_slots for r in s.reqs}
                for slots, pending, mb in kinds.values():
                    while pending:
                        free = next((sl for sl in slots if not sl.busy), None)
                        if free is None:
                            break
                        before = len(pending)
                        take = self._take(pending, free.arena_bytes, mb)
                        # cancelled requests left the queue without a batch
                        done += before - len(pending) - len(take)
                        if not take:
                            break
                        self._launch(free, take, frozenset(busy_plans))
                        for r in take:
                            r.slot = free.index
                        busy_plans.update(free.plans)
                        batches += 1
                        copies += free.copies
                        launches += free.launches
        finally:
            for sl in all_slots:
                if sl.busy:
                    sl.ev_done.wait()
            for sl in all_slots:
                sl.close()
            self.pool.busy = set()
        st = _stats([r for r in reqs if r.status == "done"], batches)
        st["cancelled"] = sum(1 for r in reqs if r.status == "cancelled")
        st.update(copies=copies, gpu_launches=launches)
        return st

    # ------------------------------------------------------------ plain
    def _serve_plain(self, reqs: list) -> dict:
        stream = _stream()
        dev = DeviceArray(self.arena_bytes, np.uint8)
        ev = _Event()
        t0 = time.perf_counter()
        launches = 0
        try:
            for r in reqs:
                while time.perf_counter() - t0 < r.t_arrival:
                    pass
                if self._is_cancelled(r):
                    r.status = "cancelled"
                    continue
                m = self.pool.get(r.matrix)
                nb = _vec_bytes(m, r)
                xp, yp = dev.ptr, dev.ptr + _al(nb)
                call("sb_memcpy_htod", xp, r.x.ctypes.data, nb, stream)
                if r.op == "spmv":
                    call("sb_memset", yp, 0, nb, stream)
                    _spmv_call(m, r.storage, xp, yp, stream)
                else:
                    pol = _lib.SB_SPTS_ACC_F64 if m.policy[r.storage] == "f64" else \
                        _lib.SB_SPTS_ACC_NATIVE
                    call("sb_spts_solve", m.plans[r.storage].ptr, _lib.SB_SPTS_HYBRID, pol, xp, yp,
                         stream)
                launches += 1
                call("sb_memcpy_dtoh", r.y.ctypes.data, yp, nb, stream)
                ev.record(stream)
                ev.wait()
                r.t_done = time.perf_counter() - t0
                r.status = "done"
        finally:
            ev.close()
            call("sb_stream_synchronize", stream)
            call("sb_stream_destroy", stream)
            dev.free()
        served = [r for r in reqs if r.status == "done"]
        st = _stats(served, len(served))
        st.update(copies=2 * len(served), gpu_launches=launches,
                  cancelled=sum(1 for r in reqs if r.status == "cancelled"))
        return st

    def serve(self, requests: list, mode: str = "batched") -> dict:
        """Serve the requests in arrival order; fills each request's y and
        t_done and returns throughput and latency statistics."""
        reqs = sorted(requests, key=lambda r: r.t_arrival)
        for r in reqs:
            self._check(r, self.pool.get(r.matrix))
            r.status = "pending"
        if mode == "plain":
            st = self._serve_plain(reqs)
        elif mode == "batched":
            st = self._serve_batched(reqs)
        else:
            raise ValueError(f"unknown mode {mode!r}")
        code = C.c_int(0)
        call("sb_device_status", C.byref(code))
        if code.value:
            raise _lib.SparseError("serve", _lib.SB_ETIMEOUT,
                                   f"device status {code.value}: a dependency wait ran out")
        st["mode"] = mode
        return st


def _spmv_call(m: ResidentMatrix, storage: str, xp: int, yp: int, stream) -> None:
    """The per-call path's y += A x: the matrix's chosen format where a
    single-call kernel takes its values (DIA: f32, f64 and BF16; ELL: f32 and
    f64), else the CSR."""
    M = m.fmt.get(storage, m.csr[storage])
    if isinstance(M, sparse_DIA_t):
        call("sb_spmv_dia", _dtcode(M.dtype), M.offset_index.ptr, M.data_index.ptr, M.N,
             M.ndiags, M.stride, xp, yp, 1, stream)
    elif isinstance(M, sparse_ELL_t) and storage != "bf16":
        call("sb_spmv_ell", _dtcode(M.dtype), M.indices_index.ptr, M.data_index.ptr, M.N,
             M.ncols, xp, yp, 1, stream)
    else:
        A = m.csr[storage]
        opts = getattr(A, "opts", None)
        call("sb_spmv_csr_ex", _dtcode(A.dtype), A.row_index.ptr, A.col_index.ptr,
             A.val_index.ptr, xp, yp, A.N, A.nnz, 1, C.byref(opts) if opts is not None else None,
             stream)


def _stats(reqs, batches) -> dict:
    if not reqs:
        return {"requests": 0, "batches": 0, "req_per_s": 0.0, "p50_ms": 0.0, "p99_ms": 0.0,
                "mean_batch": 0.0, "span_s": 0.0}
    lat = np.array([r.t_done - r.t_arrival for r in reqs])
    span = max(r.t_done for r in reqs) - min(r.t_arrival for r in reqs)
    out = {"requests": len(reqs), "batches": int(batches),
           "req_per_s": len(reqs) / span if span > 0 else 0.0,
           "p50_ms": float(np.percentile(lat, 50) * 1e3),
           "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "mean_batch": len(reqs) / max(batches, 1), "span_s": float(span)}
    for op in ("spmv", "spts"):
        lo = np.array([r.t_done - r.t_arrival for r in reqs if r.op == op])
        if lo.size:
            out[f"{op}_p50_ms"] = float(np.percentile(lo, 50) * 1e3)
            out[f"{op}_p99_ms"] = float(np.percentile(lo, 99) * 1e3)
    return out


def poisson_arrivals(rate_hz: float, duration_s: float, seed: int = 6) -> np.ndarray:
    """Arrival times (seconds) of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    n = int(rate_hz * duration_s * 1.2) + 16
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    return t[t < duration_s]
