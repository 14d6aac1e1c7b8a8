"""Make tests/golden/js_vectors.npz: outputs of the reference's JavaScript functions.

Runs SciWasm.Sparse's host-side functions -- the format conversions, the
level-set analysis and the static_nnz partitioner -- through js_machine.py (a
JavaScript interpreter in Python) on small seeded inputs and stores every
input and output array.  tests/test_js_vectors.py checks the oracle against
them bit for bit, so the restatements of these functions are pinned to the
reference's code as it ships.

Usage (where the reference sources are available; the vectors are committed
and nothing reads the reference at test time):

    python tests/golden/make_js_vectors.py /path/to/SciWasm.Sparse

Functions run (paths relative to the reference's project root):
  src/sequential/src/sparse32.js (Float32Array values) and sparse64.js
  (Float64Array values): coo_csr with its per-row sort, num_cols, csr_ell,
  num_diags, csr_dia (admitted and refused), coo_csc, quick_sort_COO;
  sparse32.js: fletcher_sum_y; read_matrix_MM_files (with read_MM_header and
  calculate_actual_nnz) on the lines load_file produces, then
  create_COO_from_MM or create_LCOO_from_MM
  src/parallel/src/sparse32.js: static_nnz, CSR_create_level_sets,
  CSR_create_level_sets_with_reorder (and its copy in spts32.js)
  (its sswasm_CSR_t constructor is not defined in the shipped sources; it is
  supplied here storing its arguments as row_index, col_index, val_index,
  nnz_row_index, nrows, nnz -- the fields the function reads),
  sort_rows_by_nnz, sort_y_rows_by_nnz, calculate_csr_locality_index,
  reorder_NN
The host objects these functions touch (linear memory, _malloc, the
allocate_* helpers and matrix constructors, console.log) are supplied here.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from js_machine import UNDEF, JSArray, JSMachine, JSObject  # noqa: E402
from make_wat_vectors import banded_csr, coo_of, lower_csr, ragged_csr  # noqa: E402

OUT = os.path.join(HERE, "js_vectors.npz")


def machine(src, names, val_kind):
    m = JSMachine(mem_bytes=16 << 20)
    vb = 4 if val_kind == "Float32Array" else 8
    I4 = 4.0

    def obj(**kw):
        return JSObject({k: (float(v) if isinstance(v, (int, np.integer)) else v)
                         for k, v in kw.items()})

    def allocate_CSR(nrows, nnz):
        return obj(row_index=m.malloc(I4 * (nrows + 1)), nnz_row_index=m.malloc(I4 * nrows),
                   col_index=m.malloc(I4 * nnz), val_index=m.malloc(vb * nnz), N=nrows, nnz=nnz)

    def allocate_DIA(N, nnz, ndiags, stride):
        return obj(offset_index=m.malloc(I4 * ndiags), data_index=m.malloc(vb * ndiags * stride),
                   ndiags=ndiags, stride=stride, N=N, nnz=nnz)

    def allocate_ELL(N, nnz, ncols):
        return obj(indices_index=m.malloc(I4 * ncols * N), data_index=m.malloc(vb * ncols * N),
                   ncols=ncols, N=N, nnz=nnz)

    class Ctor:
        def construct(self, row_index, col_index, val_index, nnz_row_index, N, nnz):
            return obj(row_index=row_index, col_index=col_index, val_index=val_index,
                       nnz_row_index=nnz_row_index, nrows=N, nnz=nnz)

    m.define("allocate_CSR", allocate_CSR)
    m.define("allocate_DIA", allocate_DIA)
    m.define("allocate_ELL", allocate_ELL)
    m.define("sswasm_CSR_t", Ctor())
    m.define("num_workers", 4.0)   # read by the level-set function's statistics only
    m.load(src, names)
    return m, obj


def put(m, arr):
    a = m.malloc(arr.nbytes)
    m.mem[int(a):int(a) + arr.nbytes] = np.ascontiguousarray(arr).tobytes()
    return a


def get(m, addr, dtype, n):
    n = int(n)
    dt = np.dtype(dtype)
    return np.frombuffer(bytes(m.mem[int(addr):int(addr) + dt.itemsize * n]), dt).copy()


def shuffled_coo(N, seed, dt, dup=0.1):
    rng = np.random.default_rng(seed)
    rp, col, val = ragged_csr(N, seed, dt)
    row, col, val = coo_of(rp, col, val)
    nd = int(row.size * dup)
    src, dst = rng.integers(0, row.size, nd), rng.integers(0, row.size, nd)
    row[dst], col[dst] = row[src], col[src]          # repeated (row, col) keys
    p = rng.permutation(row.size)
    return row[p].copy(), col[p].copy(), val[p].copy()


def mm_texts():
    """The Matrix Market known-answer files, and two seeded ones (general real
    with explicit zeros and repeated coordinates; symmetric real)."""
    out = []
    for f in sorted(os.listdir(os.path.join(HERE, "mm"))):
        with open(os.path.join(HERE, "mm", f)) as fh:
            out.append((f.split(".")[0], fh.read()))
    rng = np.random.default_rng(40)
    n, ne = 60, 400
    r, c = rng.integers(1, n + 1, ne), rng.integers(1, n + 1, ne)
    r[-20:], c[-20:] = r[:20], c[:20]
    v = np.round(rng.standard_normal(ne), 6)
    v[rng.random(ne) < 0.05] = 0.0
    lines = ["%%MatrixMarket matrix coordinate real general", "% seeded", f"{n} {n} {ne}"]
    lines += [f"{a} {b} {float(x)!r}" for a, b, x in zip(r, c, v)]
    out.append(("gen_real_seeded", "\n".join(lines) + "\n"))
    keep = r >= c
    lines = ["%%MatrixMarket matrix coordinate real symmetric", f"{n} {n} {int(keep.sum())}"]
    lines += [f"{a} {b} {float(x)!r}" for a, b, x in zip(r[keep], c[keep], v[keep])]
    out.append(("sym_real_seeded", "\n".join(lines) + "\n"))
    return out


def main(ref):
    out = {}

    def rec(case, **arrs):
        for k, v in arrs.items():
            out[f"{case}/{k}"] = np.asarray(v)

    conv = ["coo_csr", "sort", "num_cols", "csr_ell", "num_diags", "csr_dia", "coo_csc",
            "quick_sort_COO"]
    for tag, fname, dt, kind in (("f32", "sparse32.js", np.float32, "Float32Array"),
                                 ("f64", "sparse64.js", np.float64, "Float64Array")):
        src = open(os.path.join(ref, "src/sequential/src", fname)).read()
        N = 150
        # coo_csr on a shuffled COO with repeated keys
        m, obj = machine(src, conv, kind)
        row, col, val = shuffled_coo(N, 31, dt)
        A = obj(row_index=put(m, row), col_index=put(m, col), val_index=put(m, val), N=N,
                nnz=row.size)
        C = m.call("coo_csr", A)
        crp = get(m, C.get("row_index"), np.int32, N + 1)
        ccol = get(m, C.get("col_index"), np.int32, row.size)
        cval = get(m, C.get("val_index"), dt, row.size)
        rec(f"coo_csr_{tag}", row=row, col=col, val=val, N=N, row_ptr=crp, ccol=ccol, cval=cval)
        # coo_csc on the same COO
        m, obj = machine(src, conv, kind)
        A = obj(row_index=put(m, row), col_index=put(m, col), val_index=put(m, val), N=N,
                nnz=row.size)
        S = obj(col_index=m.malloc(4 * (N + 1)), row_index=m.malloc(4 * row.size),
                val_index=m.malloc(dt().itemsize * row.size), ncols=N, nnz=row.size)
        m.call("coo_csc", A, S)
        rec(f"coo_csc_{tag}", row=row, col=col, val=val, N=N,
            col_ptr=get(m, S.get("col_index"), np.int32, N + 1),
            srow=get(m, S.get("row_index"), np.int32, row.size),
            sval=get(m, S.get("val_index"), dt, row.size))
        # quick_sort_COO (unstable; repeated keys included)
        m, obj = machine(src, conv, kind)
        A = obj(row_index=put(m, row), col_index=put(m, col), val_index=put(m, val), N=N,
                nnz=row.size)
        m.call("quick_sort_COO", A, 0.0, float(row.size - 1))
        rec(f"qsort_{tag}", row=row, col=col, val=val,
            srow=get(m, A.get("row_index"), np.int32, row.size),
            scol=get(m, A.get("col_index"), np.int32, row.size),
            sval=get(m, A.get("val_index"), dt, row.size))

        # csr_ell / csr_dia on a band with a repeated entry, and refused forms
        cases = {"band": banded_csr(N, (-4, -1, 0, 2, 6), 32, dt),
                 "ragged": ragged_csr(N, 33, dt)}
        brp, bcol, bval = cases["band"]
        # a repeated (row, col) entry: csr_dia keeps the later one
        bcol = bcol.copy()
        bcol[brp[10] + 1] = bcol[brp[10]]
        cases["band"] = (brp, bcol, bval)
        for cname, (rp, ccol_, cval_) in cases.items():
            m, obj = machine(src, conv, kind)
            nnz = ccol_.size
            A = obj(row_index=put(m, rp), col_index=put(m, ccol_), val_index=put(m, cval_), N=N,
                    nnz=nnz)
            nc = m.call("num_cols", A)
            E = m.call("csr_ell", A)
            nd = m.call("num_diags", A)
            D = m.call("csr_dia", A)
            arrs = dict(row_ptr=rp, col=ccol_, val=cval_, nc=nc, nd=nd.get(0.0),
                        stride=nd.get(1.0), ell=E is not UNDEF, dia=D is not UNDEF)
            if E is not UNDEF:
                w = int(E.get("ncols"))
                arrs["indices"] = get(m, E.get("indices_index"), np.int32, w * N)
                arrs["edata"] = get(m, E.get("data_index"), dt, w * N)
            if D is not UNDEF:
                w, st = int(D.get("ndiags")), int(D.get("stride"))
                arrs["offset"] = get(m, D.get("offset_index"), np.int32, w)
                arrs["ddata"] = get(m, D.get("data_index"), dt, w * st)
            rec(f"fmt_{cname}_{tag}", **arrs)

    # ---- fletcher_sum_y, the reference benchmark's checksum of y (FP32) ----
    src = open(os.path.join(ref, "src/sequential/src/sparse32.js")).read()
    rng = np.random.default_rng(44)
    for i, y in enumerate((rng.standard_normal(1000).astype(np.float32),
                           (rng.standard_normal(777) * 1e4).astype(np.float32),
                           np.array([0.0, -0.0, 254.99, 255.0, -1.5, 3e7], np.float32))):
        m, obj = machine(src, ["matlab_modulo", "fletcher_sum", "fletcher_sum_y"], "Float32Array")
        yv = obj(vec_index=put(m, y), vec_nelem=y.size)
        rec(f"fletcher_{i}", y=y, sum=m.call("fletcher_sum_y", yv))

    # ---- Matrix Market input: read_matrix_MM_files on the lines load_file
    # hands over (text up to its last newline, split at newlines), then
    # create_COO_from_MM or create_LCOO_from_MM, each ending in quick_sort_COO
    src = open(os.path.join(ref, "src/sequential/src/sparse32.js")).read()
    mm_names = ["read_MM_header", "calculate_actual_nnz", "read_matrix_MM_files",
                "create_COO_from_MM", "create_LCOO_from_MM", "quick_sort_COO"]
    for fname, text in mm_texts():
        for lower in (False, True):
            m, obj = machine(src, mm_names, "Float32Array")

            def allocate_COO_from_MM(info, m=m, obj=obj):
                nnz = int(info.get("nnz"))
                return obj(row_index=m.malloc(4 * nnz), col_index=m.malloc(4 * nnz),
                           val_index=m.malloc(4 * nnz), N=info.get("nrows"), nnz=nnz)

            m.define("allocate_COO_from_MM", allocate_COO_from_MM)
            portion = text[:text.rfind("\n")]
            files = JSArray([JSArray(portion.split("\n"))])
            info = obj(field="", symmetry="", nrows=0, ncols=0, nentries=0, nnz=0)
            m.call("read_matrix_MM_files", files, 1.0, info)
            nnz_read = int(info.get("nnz"))
            if lower:
                A = m.call("create_LCOO_from_MM", info)
            else:
                A = allocate_COO_from_MM(info)
                m.call("create_COO_from_MM", info, A)
            nnz = int(A.get("nnz"))
            rec(f"mm_{fname}_{'lower' if lower else 'full'}",
                text=np.frombuffer(text.encode(), np.uint8), nnz=nnz_read,
                row=get(m, A.get("row_index"), np.int32, nnz),
                col=get(m, A.get("col_index"), np.int32, nnz),
                val=get(m, A.get("val_index"), np.float32, nnz))

    # ---- the parallel build's partitioner and level sets (Float32Array) ----
    src = open(os.path.join(ref, "src/parallel/src/sparse32.js")).read()
    dt = np.float32
    tiny = np.array([0, 3, 3, 8, 9, 11, 15], np.int32)   # 6 rows for 8 workers
    for nw, (rp, col, val) in ((3, ragged_csr(200, 34, dt)), (5, ragged_csr(97, 35, dt)),
                               (8, (tiny, np.zeros(15, np.int32), np.ones(15, dt)))):
        m, obj = machine(src, ["static_nnz"], "Float32Array")
        N = rp.size - 1
        A = obj(row_index=put(m, rp), nnz_row_index=m.malloc(4 * N), N=N, nnz=col.size)
        # the callers pass fresh Int32Array(num_workers) (tests/main32.js:176-187)
        rs = m.builtins["Int32Array"].construct(float(nw))
        re_ = m.builtins["Int32Array"].construct(float(nw))
        m.call("static_nnz", A, float(nw), rs, re_)
        rec(f"static_nnz_{N}_{nw}", row_ptr=rp, nw=nw, row_start=rs.a.copy(), row_end=re_.a.copy())
    spts_src = open(os.path.join(ref, "src/parallel/src/spts32.js")).read()
    # a lower factor whose rows 5 and 40 are empty (the level rule puts an
    # empty row on level 1, since only a row of exactly one entry is level 0)
    erp, ecol, evl = lower_csr(120, 39, dt)
    keep = np.ones(ecol.size, bool)
    for r in (5, 40):
        keep[erp[r]:erp[r + 1]] = False
    elens = np.diff(erp)
    elens[[5, 40]] = 0
    erp = np.concatenate([[0], np.cumsum(elens)]).astype(np.int32)
    ecol, evl = ecol[keep], evl[keep]
    for name, (rp, col, val) in (("lower", lower_csr(300, 37, dt)),
                                 ("narrow", lower_csr(200, 38, dt, band=3)),
                                 ("empty_rows", (erp, ecol, evl))):
        m, obj = machine(src, ["CSR_create_level_sets"], "Float32Array")
        N, nnz = rp.size - 1, col.size
        A = obj(row_index=put(m, rp), col_index=put(m, col), val_index=put(m, val), nrows=N,
                nnz=nnz)
        m.call("CSR_create_level_sets", A)
        nl = int(A.get("nlevels"))
        rec(f"levels_plain_{name}", row_ptr=rp, col=col, val=val, nlevels=nl,
            level_ptr=get(m, A.get("level_index"), np.int32, nl + 1),
            permutation=get(m, A.get("permutation_index"), np.int32, N))
        # the same function as the SpTS module (src/parallel/src/spts32.js)
        # ships it, which the SpTS benchmark calls
        m, obj = machine(spts_src, ["CSR_create_level_sets_with_reorder"], "Float32Array")
        N, nnz = rp.size - 1, col.size
        A = obj(row_index=put(m, rp), col_index=put(m, col), val_index=put(m, val), nrows=N,
                nnz=nnz)
        L = m.call("CSR_create_level_sets_with_reorder", A)
        nl = int(L.get("nlevels"))
        rec(f"levels_spts_{name}", row_ptr=rp, col=col, val=val, nlevels=nl,
            level_ptr=get(m, L.get("level_index"), np.int32, nl + 1),
            permutation=get(m, L.get("permutation_index"), np.int32, N),
            nrow_ptr=get(m, L.get("row_index"), np.int32, N + 1),
            ncol=get(m, L.get("col_index"), np.int32, nnz),
            nval=get(m, L.get("val_index"), dt, nnz))
        m, obj = machine(src, ["CSR_create_level_sets_with_reorder"], "Float32Array")
        N, nnz = rp.size - 1, col.size
        A = obj(row_index=put(m, rp), col_index=put(m, col), val_index=put(m, val), nrows=N,
                nnz=nnz)
        L = m.call("CSR_create_level_sets_with_reorder", A)
        nl = int(L.get("nlevels"))
        rec(f"levels_{name}", row_ptr=rp, col=col, val=val, nlevels=nl,
            level_ptr=get(m, L.get("level_index"), np.int32, nl + 1),
            permutation=get(m, L.get("permutation_index"), np.int32, N),
            nrow_ptr=get(m, L.get("row_index"), np.int32, N + 1),
            ncol=get(m, L.get("col_index"), np.int32, nnz),
            nval=get(m, L.get("val_index"), dt, nnz))

    # ---- row reordering (src/parallel/src/sparse32.js): sort_rows_by_nnz,
    # sort_y_rows_by_nnz, calculate_csr_locality_index, and reorder_NN on the
    # row-sorted matrix with w = 16 as tests/main32.js:339 calls it.  The new
    # matrices come from the file's sparse_CSR_t, which stores N and nnz but
    # no `nrows`; both functions size their new row-pointer view by
    # `A_csr_new.nrows + 1`, so that view is empty and the reference writes no
    # row pointers (recorded here as what the memory held: zeros).
    reo = ["sort_rows_by_nnz", "sort_y_rows_by_nnz", "calculate_csr_locality_index",
           "reorder_subset", "find_next_row", "assign_w_min_elems", "reorder_NN"]
    reo_jobs = []
    for tag, fname, dtr, kind in (("", "sparse32.js", np.float32, "Float32Array"),
                                  ("_f64", "sparse64.js", np.float64, "Float64Array")):
        srcr = open(os.path.join(ref, "src/parallel/src", fname)).read()
        reo_jobs += [(f"ragged{tag}", srcr, kind, ragged_csr(300, 41, dtr)),
                     (f"band{tag}", srcr, kind, banded_csr(200, (-9, -3, 0, 1, 17), 42, dtr))]
    for name, src_r, kind, (rp, col, val) in reo_jobs:
        dt = val.dtype.type
        m, obj = machine(src_r, reo, kind)

        class CSRCtor:
            def construct(self, row_index, col_index, val_index, nnz_row_index, N, nnz, obj=obj):
                return obj(row_index=row_index, col_index=col_index, val_index=val_index,
                           nnz_row_index=nnz_row_index, N=N, nnz=nnz, num_zero_rows=0,
                           num_one_rows=0, num_two_rows=0, num_three_rows=0)

        m.define("sparse_CSR_t", CSRCtor())
        m.define("pretty_print_CSR_permutation", lambda *a: UNDEF)
        m.define("free_memory_y", lambda *a: UNDEF)
        N, nnz = rp.size - 1, col.size
        A = obj(row_index=put(m, rp), col_index=put(m, col), val_index=put(m, val), N=N, nnz=nnz)
        loc = m.call("calculate_csr_locality_index", A)
        S = m.call("sort_rows_by_nnz", A)
        y = np.random.default_rng(43).standard_normal(N).astype(dt)
        yv = obj(y_index=put(m, y), y_nelem=N)
        m.call("sort_y_rows_by_nnz", yv, S)
        rec(f"sortrows_{name}", row_ptr=rp, col=col, val=val, locality=loc,
            permutation=get(m, S.get("permutation_index"), np.int32, N),
            nnz_per_row=get(m, S.get("nnz_row_index"), np.int32, N),
            nrow_ptr=get(m, S.get("row_index"), np.int32, N + 1),
            ncol=get(m, S.get("col_index"), np.int32, nnz),
            nval=get(m, S.get("val_index"), dt, nnz),
            small_rows=np.array([S.get(k) for k in ("num_zero_rows", "num_one_rows",
                                                     "num_two_rows", "num_three_rows")], np.int32),
            y=y, y_new=get(m, yv.get("y_index"), dt, N))
        # reorder_NN on the sorted matrix; its row pointers are the sorted
        # matrix's own (a correct CSR, written here since the reference's
        # view of them was empty)
        # (the reference's nnz_per_row holds the original order's lengths)
        lens = get(m, S.get("nnz_row_index"), np.int32, N)[get(m, S.get("permutation_index"),
                                                               np.int32, N)]
        srp = np.concatenate([[0], np.cumsum(lens)])
        m.mem[int(S.get("row_index")):int(S.get("row_index")) + 4 * (N + 1)] = \
            srp.astype(np.int32).tobytes()
        R = m.call("reorder_NN", S, 16.0)
        rec(f"reorder_nn_{name}", srow_ptr=srp.astype(np.int32),
            scol=get(m, S.get("col_index"), np.int32, nnz), sval=get(m, S.get("val_index"), dt, nnz),
            sperm=get(m, S.get("permutation_index"), np.int32, N),
            permutation=get(m, R.get("permutation_index"), np.int32, N),
            ncol=get(m, R.get("col_index"), np.int32, nnz),
            nval=get(m, R.get("val_index"), dt, nnz))

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SCIWASM_SPARSE_SRC", "."))
