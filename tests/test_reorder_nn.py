"""reorder_NN (src/parallel/src/sparse32.js:2271-2622) on the CPU: the C
oracle against an independent pure-Python restatement of the reference's
loops on small matrices, and the properties of its output (the walk is a
permutation that keeps every row inside its length group, the new CSR holds
the walked rows, the permutation composes with the input's)."""
import numpy as np
import pytest

from sciwasm.sparse_b200 import synth


def _py_reorder_nn(rp, col, w=16):
    """The reference's reorder_NN / reorder_subset / find_next_row /
    assign_w_min_elems, line by line (Float32Array lists, double compares)."""
    N = rp.size - 1
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    walk = list(range(N))
    visited = [0] * N
    freq = [0] * (N + 1)
    nlines = [0] * N
    for i in range(N):
        ln = rp[i + 1] - rp[i]
        freq[ln] += 1
        if ln == 0:
            visited[i] = 2
    for i in range(N):
        if visited[i]:
            continue
        j = rp[i]
        while j < rp[i + 1]:
            nlines[i] += 1
            j += 1
            while j < rp[i + 1] and col[j - 1] // 16 == col[j] // 16:
                j += 1

    def assign(jac, nidx, nxt, v):
        i = 0
        while i < w and jac[i] >= 0 and jac[i] >= v:
            i += 1
        if i == w:
            return
        if jac[i] == -1:
            jac[i], nidx[i] = f32(v), nxt
            return
        j = w - 1
        while jac[j] == -1:
            j -= 1
        while j != i:
            jac[j], nidx[j] = jac[j - 1], nidx[j - 1]
            j -= 1
        jac[i], nidx[i] = f32(v), nxt

    def find_next(index, jac, nidx, last_used, start, end):
        if visited[index] == 3:
            visited[index] = 1
            jac[:] = [-1.0] * w
            nidx[:] = [N] * w
            for j in range(rp[index], rp[index + 1]):
                last_used[col[j] // 16] = index
            for i in range(start, end):
                if visited[i]:
                    continue
                j, al = rp[i], 0
                while j < rp[i + 1]:
                    if last_used[col[j] // 16] == index:
                        al += 1
                    j += 1
                    while j < rp[i + 1] and col[j - 1] // 16 == col[j] // 16:
                        j += 1
                assign(jac, nidx, i, al / (nlines[index] + nlines[i] - al))
        for i in range(w):
            if jac[i] >= 0 and visited[nidx[i]] == 0:
                return nidx[i], jac[i]
        return N, 0.0

    def subset(start, end):
        win = [0] * w
        last_used = [-1] * (N // 16 + 1)
        jacs = [[0.0] * w for _ in range(w)]
        nids = [[0] * w for _ in range(w)]
        index, pos, nnb, count = start, start, 0, 0
        while index != N:
            visited[index] = 3
            win[count] = index
            count += 1
            nnb = min(nnb + 1, w)
            if count == w:
                count = 0
            walk[pos] = index
            pos += 1
            nxt, mx = N, 0.0
            for i in range(nnb):
                c, v = find_next(win[i], jacs[i], nids[i], last_used, start, end)
                if mx <= v and c != N:
                    mx, nxt = v, c
            index = nxt

    start = 0
    while start < N and visited[start]:
        start += 1
    if start < N:
        for ln in range(1, N + 1):
            while freq[ln] >= 1024:
                freq[ln] -= 1024
                subset(start, start + 1024)
                start += 1024
            if freq[ln] > 0:
                subset(start, start + freq[ln])
                start += freq[ln]
                freq[ln] = 0
    return np.array(walk, np.int32)


def _sorted_by_length(oracle, rp, col, val):
    s = oracle.sort_rows_by_nnz(rp, col, val)
    return s["row_ptr"], s["col"], s["val"], s["permutation"]


@pytest.mark.parametrize("case", ["banded", "powerlaw", "ragged", "lap2d"])
def test_oracle_matches_python_restatement(oracle, case):
    rng = np.random.default_rng(4)
    if case == "banded":
        rp, col, val = synth.banded(900, half=3, seed=2)
    elif case == "powerlaw":
        rp, col, val = synth.power_law(1500, seed=5, cap=60, shift=0)
    elif case == "lap2d":
        rp, col, val = synth.laplacian_2d(30, dtype=np.float64)
    else:
        lens = rng.integers(0, 7, 1300)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        col = np.concatenate([np.sort(rng.choice(1300, n, replace=False)) for n in lens]
                             ).astype(np.int32)
        val = rng.standard_normal(col.size)
    srp, scol, sval, sperm = _sorted_by_length(oracle, rp, col, val)
    got = oracle.reorder_nn(srp, scol, sval, 16, sperm)
    want = _py_reorder_nn(srp, scol, 16)
    assert np.array_equal(got["walk"], want)
    # a permutation that keeps rows inside their length group
    N = srp.size - 1
    assert np.array_equal(np.sort(got["walk"]), np.arange(N))
    lens = np.diff(srp)
    assert np.array_equal(lens[got["walk"]], lens)
    # the new CSR holds the walked rows; the permutation composes
    assert np.array_equal(np.diff(got["row_ptr"]), lens[got["walk"]])
    for i in range(0, N, max(1, N // 50)):
        s = got["walk"][i]
        assert np.array_equal(got["col"][got["row_ptr"][i]:got["row_ptr"][i + 1]],
                              scol[srp[s]:srp[s + 1]])
    assert np.array_equal(got["permutation"], sperm[got["walk"]])


def test_window_and_chunking(oracle):
    """A 2500-row length group is walked in chunks of 1024, 1024 and 452 rows,
    and window sizes other than 16 follow the same loops."""
    rp, col, val = synth.banded(2500, half=2, seed=3)
    rp = rp.copy()
    # make every row 5 long so that one length group spans all chunks
    keep = np.diff(rp) == 5
    assert keep.sum() == 2496
    srp, scol, sval, sperm = _sorted_by_length(oracle, rp, col, val)
    for w in (4, 16):
        got = oracle.reorder_nn(srp, scol, sval, w, sperm)
        assert np.array_equal(got["walk"], _py_reorder_nn(srp, scol, w))
    first = 4  # the four shorter edge rows come first after sorting by length
    chunks = [(first, first + 1024), (first + 1024, first + 2048), (first + 2048, 2500)]
    for a, b in chunks:
        assert sorted(got["walk"][a:b]) == list(range(a, b))
