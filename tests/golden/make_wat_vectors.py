"""Make tests/golden/wat_vectors.npz: outputs of the reference's own kernels.

Runs SciWasm.Sparse's hand-written WebAssembly text through wat_machine.py
(a WebAssembly interpreter in Python) on small seeded inputs and stores every
input and output array.  The tests compare the oracle and the CUDA path with
these arrays, so parity is pinned to the reference's code as it ships, not
only to a restatement of it.

Usage (where the reference sources are available; the vectors are committed
and nothing reads the reference at test time):

    python tests/golden/make_wat_vectors.py /path/to/SciWasm.Sparse

Kernels run, by file of the reference (paths relative to its project root):
  src/sequential/src/sparse_opt_32.wat, sparse_opt_64.wat:
      spmv_coo, spmv_csr, spmv_dia, spmv_ell and their _wrapper forms
      (inner_max), sum_coo (as shipped),
      count/copy_nonzeros_{coo,csr,dia,ell}, transpose_{csr,dia,ell},
      count_transpose_cols_ell, diagonal_coo, min_coo, spts_csc and the exact
      element-wise maps (abs, neg, sqrt, ceil, floor, trunc, nearest, sign,
      multiply_scalar, deg2rad, rad2deg; COO/CSR, DIA and ELL forms)
  src/parallel/src/sparse_opt_32.wat: spts_level_csr and the hybrid
      metadata + spts_csr_opt_level_sync_free_wrapper (one worker), and the
      worker SpMV kernels spmv_csr/coo/dia/ell_wrapper, sum,
      spmv_dia_col_basic_wrapper and spmv_ell_col_wrapper (three workers run
      in turn)
  src/parallel/src/spts_opt_32.wat:   spts_csr_sync_free_wrapper and
      spts_csr_level_sync_free_wrapper (one worker)
The transcendental maps call imported JavaScript Math functions, which are
not part of the reference, so they are not pinned here.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

from wat_machine import WatModule  # noqa: E402

OUT = os.path.join(HERE, "wat_vectors.npz")
PI32 = np.float32(np.pi)
PI64 = np.pi


class Mem:
    """Bump allocator over one module's linear memory."""

    def __init__(self, mod):
        self.m, self.top = mod, 64
        mod.mem[:] = bytes(len(mod.mem))      # every case starts from zeroed memory

    def put(self, arr):
        a = self.top
        end = self.m.write(a, arr)
        self.top = (end + 63) // 64 * 64
        return a

    def zeros(self, n, dtype):
        return self.put(np.zeros(max(n, 1), dtype))

    def get(self, addr, dtype, n):
        return self.m.read(addr, dtype, n)


def ragged_csr(N, seed, dt, zeros=False):
    """Rows of 0-24 entries (first and last rows empty), sorted columns."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 25, N)
    lens[rng.random(N) < 0.1] = 0
    lens[0] = lens[-1] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(rng.choice(N, l, replace=False)) for l in lens]).astype(np.int32)
    val = rng.standard_normal(col.size).astype(dt)
    if zeros:
        k = col.size
        val[rng.choice(k, k // 8, replace=False)] = 0.0
        val[rng.choice(k, k // 16, replace=False)] = -0.0
        val[rng.choice(k, k // 32, replace=False)] = np.nan
    return rp, col, val


def banded_csr(N, offsets, seed, dt):
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(N):
        for k in offsets:
            if 0 <= i + k < N:
                rows.append(i)
                cols.append(i + k)
    rows, cols = np.array(rows, np.int32), np.array(cols, np.int32)
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=N))]).astype(np.int32)
    return rp, cols, rng.standard_normal(cols.size).astype(dt)


def lower_csr(N, seed, dt, band=40):
    """Lower triangular, diagonal stored last, dominant diagonal."""
    rng = np.random.default_rng(seed)
    rp, col = [0], []
    for i in range(N):
        lo = max(0, i - band)
        k = min(i - lo, int(rng.integers(0, 6)))
        c = np.sort(rng.choice(np.arange(lo, i), k, replace=False)) if k else np.zeros(0, int)
        col.extend(c.tolist() + [i])
        rp.append(len(col))
    rp, col = np.array(rp, np.int32), np.array(col, np.int32)
    val = rng.uniform(-0.5, 0.5, col.size).astype(dt)
    val[rp[1:] - 1] = rng.uniform(2.0, 4.0, N).astype(dt)
    return rp, col, val


def csc_lower_mult4(N, seed, dt):
    """Lower-triangular CSC, diagonal first in each column, and 0, 4 or 8
    entries below it."""
    rng = np.random.default_rng(seed)
    cp, rows, vals = [0], [], []
    for j in range(N):
        k = int(rng.choice([0, 4, 8]))
        k = min(k, (N - 1 - j) // 4 * 4)
        below = np.sort(rng.choice(np.arange(j + 1, N), k, replace=False)) if k else np.zeros(0, int)
        rows.extend([j] + below.tolist())
        vals.extend([rng.uniform(2.0, 4.0)] + rng.uniform(-0.5, 0.5, k).tolist())
        cp.append(len(rows))
    return np.array(cp, np.int32), np.array(rows, np.int32), np.array(vals, dt)


def coo_of(rp, col, val):
    row = np.repeat(np.arange(rp.size - 1, dtype=np.int32), np.diff(rp))
    return row, col.copy(), val.copy()


def load_case(z, case):
    """The arrays of one case from the loaded npz, references resolved."""
    pre = case + "/"
    res = {}
    for k in z.files:
        if k.startswith(pre):
            v = z[k]
            if v.dtype.kind == "U" and str(v).startswith("@"):
                v = z[str(v)[1:]]
            res[k[len(pre):]] = v
    return res


def main(ref):
    from oracle import binding as ob
    seq = {4: os.path.join(ref, "src/sequential/src/sparse_opt_32.wat"),
           8: os.path.join(ref, "src/sequential/src/sparse_opt_64.wat")}
    out, seen = {}, {}

    def rec(case, **arrs):
        """Store a case's arrays; an array equal to one stored before is kept
        as a reference "@<key>" to it (load_case resolves these)."""
        for k, v in arrs.items():
            v = np.asarray(v)
            sig = (v.dtype.str, v.shape, v.tobytes())
            if v.size > 1 and sig in seen:
                out[f"{case}/{k}"] = np.array("@" + seen[sig])
            else:
                seen.setdefault(sig, f"{case}/{k}")
                out[f"{case}/{k}"] = v

    for vb, dt in ((4, np.float32), (8, np.float64)):
        tag = "f32" if vb == 4 else "f64"
        mod = WatModule(seq[vb], mem_bytes=8 << 20)
        rng = np.random.default_rng(100 + vb)

        # ---- SpMV, y += A x -------------------------------------------
        N = 300
        rp, col, val = ragged_csr(N, 1, dt)
        x = rng.standard_normal(N).astype(dt)
        y0 = rng.standard_normal(N).astype(dt)
        M = Mem(mod)
        a = [M.put(rp), M.put(col), M.put(val), M.put(x), M.put(y0)]
        mod.call("spmv_csr", *a, N)
        rec(f"spmv_csr_{tag}", row_ptr=rp, col=col, val=val, x=x, y0=y0, y=M.get(a[4], dt, N))
        M = Mem(mod)
        a = [M.put(rp), M.put(col), M.put(val), M.put(x), M.put(y0)]
        mod.call("spmv_csr_wrapper", *a, N, 3)
        rec(f"spmv_csr3_{tag}", row_ptr=rp, col=col, val=val, x=x, y0=y0, y=M.get(a[4], dt, N))

        row, ccol, cval = coo_of(rp, col, val)
        p = rng.permutation(row.size)
        row, ccol, cval = row[p], ccol[p], cval[p]
        M = Mem(mod)
        a = [M.put(row), M.put(ccol), M.put(cval), M.put(x), M.put(y0)]
        mod.call("spmv_coo", *a, row.size)
        rec(f"spmv_coo_{tag}", row=row, col=ccol, val=cval, N=N, x=x, y0=y0, y=M.get(a[4], dt, N))

        brp, bcol, bval = banded_csr(N, (-7, -2, 0, 1, 5), 2, dt)
        off, dat, nd, stride = ob.csr_dia(brp, bcol, bval)
        M = Mem(mod)
        po, pd, px, py = M.put(off), M.put(dat), M.put(x), M.put(y0)
        mod.call("spmv_dia", po, pd, N, nd, stride, px, py)
        rec(f"spmv_dia_{tag}", offset=off, data=dat, N=N, stride=stride, x=x, y0=y0,
            y=M.get(py, dt, N))

        ind, edat, nc = ob.csr_ell(rp, col, val)
        M = Mem(mod)
        pi_, pd, px, py = M.put(ind), M.put(edat), M.put(x), M.put(y0)
        mod.call("spmv_ell", pi_, pd, N, nc, px, py)
        rec(f"spmv_ell_{tag}", indices=ind, data=edat, N=N, nc=nc, x=x, y0=y0, y=M.get(py, dt, N))

        # the inner_max wrappers of the other formats (y += A x, three times)
        M = Mem(mod)
        a = [M.put(row), M.put(ccol), M.put(cval), M.put(x), M.put(y0)]
        mod.call("spmv_coo_wrapper", *a, row.size, 3)
        rec(f"spmv_coo3_{tag}", row=row, col=ccol, val=cval, N=N, x=x, y0=y0, y=M.get(a[4], dt, N))
        M = Mem(mod)
        po, pd, px, py = M.put(off), M.put(dat), M.put(x), M.put(y0)
        mod.call("spmv_dia_wrapper", po, pd, N, nd, stride, px, py, 3)
        rec(f"spmv_dia3_{tag}", offset=off, data=dat, N=N, stride=stride, x=x, y0=y0,
            y=M.get(py, dt, N))
        M = Mem(mod)
        pi_, pd, px, py = M.put(ind), M.put(edat), M.put(x), M.put(y0)
        mod.call("spmv_ell_wrapper", pi_, pd, N, nc, px, py, 3)
        rec(f"spmv_ell3_{tag}", indices=ind, data=edat, N=N, nc=nc, x=x, y0=y0, y=M.get(py, dt, N))

        # sum_coo (axis 1) as shipped: its row counter also advances per entry
        srow, scol, sval = coo_of(rp, col, val)
        M = Mem(mod)
        a = [M.put(srow), M.put(scol), M.put(sval), M.zeros(N, dt)]
        mod.call("sum_coo", 1, *a, N, srow.size)
        rec(f"sum_coo_{tag}", row=srow, col=scol, val=sval, N=N, out=M.get(a[3], dt, N))

        # ---- eliminate_zeros and transpose (the FP32 module exports them) --
        if "count_nonzeros_coo" in mod.exports:
            zrp, zcol, zval = ragged_csr(200, 3, dt, zeros=True)
            zrow = np.repeat(np.arange(200, dtype=np.int32), np.diff(zrp))
            M = Mem(mod)
            pv = M.put(zval)
            cnt = mod.call("count_nonzeros_coo", pv, zval.size)[0]
            a = [M.put(zrow), M.put(zcol), pv, M.zeros(cnt, np.int32), M.zeros(cnt, np.int32),
                 M.zeros(cnt, dt)]
            mod.call("copy_nonzeros_coo", *a, zval.size)
            rec(f"nz_coo_{tag}", row=zrow, col=zcol, val=zval, count=cnt,
                orow=M.get(a[3], np.int32, cnt), ocol=M.get(a[4], np.int32, cnt), oval=M.get(a[5], dt, cnt))
            M = Mem(mod)
            a = [M.put(zrp), M.put(zcol), M.put(zval), M.zeros(201, np.int32), M.zeros(cnt, np.int32),
                 M.zeros(cnt, dt)]
            mod.call("copy_nonzeros_csr", *a, 200)
            rec(f"nz_csr_{tag}", row_ptr=zrp, col=zcol, val=zval, orow_ptr=M.get(a[3], np.int32, 201),
                ocol=M.get(a[4], np.int32, cnt), oval=M.get(a[5], dt, cnt))

            zb = banded_csr(200, (-3, 0, 2, 9), 4, dt)
            zoff, zdat, znd, zstride = ob.csr_dia(*zb)
            zdat = zdat.copy()
            r = np.random.default_rng(5)
            zdat[r.random(zdat.size) < 0.3] = 0.0
            zdat[np.arange(zstride) + 2 * zstride] = 0.0          # one diagonal all zero
            M = Mem(mod)
            po, pd = M.put(zoff), M.put(zdat)
            cdiags, cnnz = mod.call("count_nonzeros_dia", po, pd, znd, zstride, 200)
            oo, od = M.zeros(cdiags, np.int32), M.zeros(cdiags * zstride, dt)
            mod.call("copy_nonzeros_dia", po, pd, oo, od, znd, zstride, 200)
            rec(f"nz_dia_{tag}", offset=zoff, data=zdat, N=200, stride=zstride, count_diags=cdiags,
                count=cnnz, ooffset=M.get(oo, np.int32, cdiags), odata=M.get(od, dt, cdiags * zstride))

            erp, ecol, evl = ragged_csr(200, 6, dt, zeros=True)
            eind, edat2, enc = ob.csr_ell(erp, ecol, np.nan_to_num(evl, nan=0.0).astype(dt))
            edat2 = edat2.copy()
            edat2[np.random.default_rng(7).random(edat2.size) < 0.05] = np.nan
            M = Mem(mod)
            pd, pi_, pn = M.put(edat2), M.put(eind), M.zeros(200, np.int32)
            ccols, ccount = mod.call("count_nonzeros_ell", pd, pn, enc, 200)
            mod.write(pn, np.zeros(200, np.int32))
            od, oi = M.zeros(ccols * 200, dt), M.zeros(ccols * 200, np.int32)
            mod.call("copy_nonzeros_ell", pd, pi_, od, oi, pn, enc, 200)
            rec(f"nz_ell_{tag}", indices=eind, data=edat2, nc=enc, N=200, count_cols=ccols, count=ccount,
                odata=M.get(od, dt, ccols * 200), oindices=M.get(oi, np.int32, ccols * 200))

            # ---- transpose -------------------------------------------------
            M = Mem(mod)
            a = [M.put(rp), M.put(col), M.put(val), M.zeros(N + 1, np.int32), M.zeros(col.size, np.int32),
                 M.zeros(col.size, dt)]
            mod.call("transpose_csr", *a, N, col.size)
            rec(f"tr_csr_{tag}", row_ptr=rp, col=col, val=val, orow_ptr=M.get(a[3], np.int32, N + 1),
                ocol=M.get(a[4], np.int32, col.size), oval=M.get(a[5], dt, col.size))
            M = Mem(mod)
            po, pd = M.put(off), M.put(dat)
            oo, od = M.zeros(nd, np.int32), M.zeros(nd * stride, dt)
            mod.call("transpose_dia", po, pd, oo, od, nd, stride, N)
            rec(f"tr_dia_{tag}", offset=off, data=dat, N=N, stride=stride,
                ooffset=M.get(oo, np.int32, nd), odata=M.get(od, dt, nd * stride))
            M = Mem(mod)
            pd, pi_, pn = M.put(edat), M.put(ind), M.zeros(N, np.int32)
            tcols = mod.call("count_transpose_cols_ell", pd, pi_, pn, nc, N)[0]
            mod.write(pn, np.zeros(N, np.int32))
            od, oi = M.zeros(tcols * N, dt), M.zeros(tcols * N, np.int32)
            mod.call("transpose_ell", pd, pi_, od, oi, pn, nc, N)
            rec(f"tr_ell_{tag}", indices=ind, data=edat, nc=nc, N=N, ncols=tcols,
                odata=M.get(od, dt, tcols * N), oindices=M.get(oi, np.int32, tcols * N))

        # ---- COO reductions (row-sorted COO) ---------------------------
        srow, scol, sval = coo_of(rp, col, val)
        for k in (0, 3, -4):
            M = Mem(mod)
            nk = N - abs(k)
            a = [M.put(srow), M.put(scol), M.put(sval), M.zeros(nk, dt)]
            mod.call("diagonal_coo", k, *a, N, srow.size)
            rec(f"diag{k}_{tag}", row=srow, col=scol, val=sval, N=N, diag=M.get(a[3], dt, nk))
        M = Mem(mod)
        a = [M.put(srow), M.put(scol), M.put(sval), M.zeros(N, dt)]
        mod.call("min_coo", 1, *a, N, srow.size)
        rec(f"min_{tag}", row=srow, col=scol, val=sval, N=N, out=M.get(a[3], dt, N))

        # ---- CSC triangular solve (column sweep) -----------------------
        lrp, lcol, lval = lower_csr(250, 8, dt)
        lrow = np.repeat(np.arange(250, dtype=np.int32), np.diff(lrp))
        order = np.lexsort((lrow, lcol))                      # column-major, rows ascending
        ccol_ptr = np.concatenate([[0], np.cumsum(np.bincount(lcol, minlength=250))]).astype(np.int32)
        crow, cval2 = lrow[order].astype(np.int32), lval[order]
        b = rng.uniform(-1, 1, 250).astype(dt)
        M = Mem(mod)
        a = [M.put(ccol_ptr), M.put(crow), M.put(cval2), M.put(b), M.zeros(250, dt)]
        mod.call("spts_csc", *a, 250)
        rec(f"spts_csc_{tag}", col_ptr=ccol_ptr, row=crow, val=cval2, x=b, y=M.get(a[4], dt, 250))
        # columns of 0, 4 or 8 off-diagonal entries: only the 4-wide SIMD body runs
        cp4, row4, val4 = csc_lower_mult4(250, 12, dt)
        M = Mem(mod)
        a = [M.put(cp4), M.put(row4), M.put(val4), M.put(b), M.zeros(250, dt)]
        mod.call("spts_csc", *a, 250)
        rec(f"spts_csc4_{tag}", col_ptr=cp4, row=row4, val=val4, x=b, y=M.get(a[4], dt, 250))

        # ---- exact element-wise maps -----------------------------------
        mv = np.concatenate([rng.standard_normal(45) * 4, [0.0, -0.0, 2.5, -2.5, 0.5, -0.5, 1.5, np.inf,
                                                            -np.inf, np.nan, 1e30, -3.0, 3.5]]).astype(dt)
        nnzm = mv.size
        pi_val = PI32 if vb == 4 else PI64
        for op, extra in (("abs", ()), ("neg", ()), ("sqrt", ()), ("ceil", ()), ("floor", ()),
                          ("trunc", ()), ("nearest", ()), ("sign", ()), ("deg2rad", (pi_val,)),
                          ("rad2deg", (pi_val,))):
            M = Mem(mod)
            pin, pout = M.put(mv), M.zeros(nnzm, dt)
            mod.call(f"{op}_coo", *extra, pin, pout, nnzm)
            f_out = M.get(pout, dt, nnzm)
            M = Mem(mod)
            pin = M.put(mv)
            mod.call(f"self_{op}_coo", *extra, pin, nnzm)
            rec(f"map_{op}_coo_{tag}", val=mv, out=f_out, self_out=M.get(pin, dt, nnzm))
            # ELL: every slot of a 2-column, nnzm/2-row layout; DIA: in-band slots
            if nnzm % 2 == 0:
                M = Mem(mod)
                pin, pout = M.put(mv), M.zeros(nnzm, dt)
                if f"{op}_ell" in mod.exports:
                    mod.call(f"{op}_ell", *extra, pin, pout, 2, nnzm // 2)
                else:
                    mod.call(f"self_{op}_ell", *extra, pin, 2, nnzm // 2)
                    pout = pin
                rec(f"map_{op}_ell_{tag}", val=mv, out=M.get(pout, dt, nnzm))
            dv = dat.copy()
            dv[: min(dv.size, nnzm)] = mv[: min(dv.size, nnzm)]
            M = Mem(mod)
            po, pin, pout = M.put(off), M.put(dv), M.zeros(dv.size, dt)
            if f"{op}_dia" in mod.exports:
                mod.call(f"{op}_dia", *extra, po, pin, pout, nd, stride, N)
            else:
                mod.call(f"self_{op}_dia", *extra, po, pin, nd, stride, N)
                pout = pin
            rec(f"map_{op}_dia_{tag}", offset=off, data=dv, N=N, stride=stride,
                out=M.get(pout, dt, dv.size))
        M = Mem(mod)
        pin = M.put(mv)
        mod.call("self_multiply_scalar_coo", dt(-1.75), pin, nnzm)
        rec(f"map_multiply_coo_{tag}", val=mv, p=dt(-1.75), self_out=M.get(pin, dt, nnzm))

    # ---- SpTS, one worker (FP32: the parallel modules are FP32 only) -----
    dt = np.float32
    par = WatModule(os.path.join(ref, "src/parallel/src/sparse_opt_32.wat"), mem_bytes=8 << 20)
    spts = WatModule(os.path.join(ref, "src/parallel/src/spts_opt_32.wat"), mem_bytes=8 << 20)
    for name, (lrp, lcol, lval) in (("lower", lower_csr(400, 9, dt)),
                                    ("lower_narrow", lower_csr(300, 10, dt, band=3))):
        Nl = lrp.size - 1
        b = np.random.default_rng(11).uniform(-1, 1, Nl).astype(dt)
        # sync-free: y starts as b (x = y in the wrapper's call), flags per row
        M = Mem(spts)
        a = [M.put(lrp), M.put(lcol), M.put(lval), M.put(b), M.zeros(Nl, dt)]
        bar, gfl, fl = M.zeros(1, np.int32), M.zeros(1, np.int32), M.zeros(Nl, np.int32)
        spts.call("spts_csr_sync_free_wrapper", 0, *a, Nl, bar, gfl, fl, 1, 1)
        rec(f"spts_syncfree_{name}", row_ptr=lrp, col=lcol, val=lval, b=b, y=M.get(a[4], dt, Nl))
        # level-set solve on the level-ordered matrix
        L = ob.level_sets(lrp, lcol, lval)
        bp = b.copy()
        M = Mem(par)
        lp = M.put(L["level_ptr"].astype(np.int32))
        a = [M.put(L["row_ptr"]), M.put(L["col"]), M.put(L["val"]), M.put(bp), M.zeros(Nl, dt)]
        perm = M.put(L["permutation"])
        bar, gfl = M.zeros(1, np.int32), M.zeros(1, np.int32)
        par.call("spts_level_csr", 0, lp, *a, perm, L["nlevels"], bar, gfl, 1, Nl, 1)
        rec(f"spts_level_{name}", row_ptr=lrp, col=lcol, val=lval, level_ptr=L["level_ptr"],
            lrow_ptr=L["row_ptr"], lcol=L["col"], lval=L["val"], permutation=L["permutation"],
            b=bp, y=M.get(a[4], dt, Nl))
        # the hybrid level/sync-free solve (tests/main32.js "spts_metadata" then
        # "spts_csr_opt_level_sync_free", one worker): y starts at 1.0 as
        # spts_init_y leaves it, the level flag at -1, the worker level at -1
        nl = L["nlevels"]
        M = Mem(par)
        lp = M.put(L["level_ptr"].astype(np.int32))
        a = [M.put(L["row_ptr"]), M.put(L["col"]), M.put(L["val"]), M.put(bp),
             M.put(np.ones(Nl, dt))]
        perm = M.put(L["permutation"])
        bar, gfl = M.zeros(1, np.int32), M.zeros(1, np.int32)
        glevel, grows = M.put(np.array([-1], np.int32)), M.zeros(1, np.int32)
        alevel = M.zeros(nl + 1, np.int32)
        rli, rwi = M.zeros(Nl, np.int32), M.zeros(Nl, np.int32)
        wlev = M.put(np.array([-1], np.int32))
        par.call("metadata", 0, lp, nl, 1, Nl, rli, rwi)
        par.call("spts_csr_opt_level_sync_free_wrapper", 0, lp, *a, perm, nl, bar, gfl, glevel,
                 grows, alevel, rli, rwi, wlev, 1, Nl, 1)
        # the SpTS module's own level/sync-free hybrid (spts_opt_32.wat
        # spts_csr_level_sync_free_wrapper, one worker): the sync-free row
        # arithmetic on the level-ordered matrix
        M2 = Mem(spts)
        lp2 = M2.put(L["level_ptr"].astype(np.int32))
        a2 = [M2.put(L["row_ptr"]), M2.put(L["col"]), M2.put(L["val"]), M2.put(bp),
              M2.zeros(Nl, dt)]
        perm2 = M2.put(L["permutation"])
        bar2, gfl2, fl2 = M2.zeros(1, np.int32), M2.zeros(1, np.int32), M2.zeros(Nl, np.int32)
        spts.call("spts_csr_level_sync_free_wrapper", 0, lp2, *a2, perm2, nl, bar2, gfl2, fl2, 1,
                  Nl, 1)
        rec(f"spts_lsf_{name}", lrow_ptr=L["row_ptr"], lcol=L["col"], lval=L["val"], b=bp,
            y=M2.get(a2[4], dt, Nl))
        rec(f"spts_hybrid_{name}", lrow_ptr=L["row_ptr"], lcol=L["col"], lval=L["val"],
            permutation=L["permutation"], row_ptr=lrp, col=lcol, val=lval, b=bp,
            y=M.get(a[4], dt, Nl))

    # ---- the parallel build's worker kernels, three workers run in turn --
    # (src/parallel/src/worker32.js "csr", "spmv_coo"/"sum", "dia_row",
    # "ell_row"; the CPU baseline restates this partitioning).  Workers write
    # disjoint rows of y (CSR, DIA, ELL) or their own private y (COO), so
    # running them one after another gives the threaded result.
    nw = 3
    N = 300
    rp, col, val = ragged_csr(N, 21, dt)
    r3 = np.random.default_rng(22)
    x = r3.standard_normal(N).astype(dt)
    y0 = r3.standard_normal(N).astype(dt)
    rs, re = ob.static_nnz(rp, nw)
    M = Mem(par)
    a = [M.put(rp), M.put(col), M.put(val), M.put(x), M.put(y0)]
    for w in range(nw):
        par.call("spmv_csr_wrapper", w, a[0] + 4 * int(rs[w]), a[1], a[2], a[3],
                 a[4] + 4 * int(rs[w]), int(re[w] - rs[w]), 1)
    rec("par_csr", row_ptr=rp, col=col, val=val, x=x, y0=y0, nw=nw, y=M.get(a[4], dt, N))

    row, ccol, cval = coo_of(rp, col, val)
    p = r3.permutation(row.size)
    row, ccol, cval = row[p], ccol[p], cval[p]
    nnz = row.size
    per, rem = nnz // nw, nnz - (nnz // nw) * nw
    nper, nrem = N // nw, N - (N // nw) * nw
    M = Mem(par)
    a = [M.put(row), M.put(ccol), M.put(cval), M.put(x), M.put(y0)]
    wy = [M.zeros(N, dt) for _ in range(nw)]
    for w in range(nw):
        s, e = w * per, (w + 1) * per + (rem if w == nw - 1 else 0)
        par.call("spmv_coo_wrapper", w, a[0] + 4 * s, a[1] + 4 * s, a[2] + 4 * s, a[3], wy[w],
                 e - s, 1)
    for d in range(nw):
        for w in range(nw):
            s, e = w * nper, (w + 1) * nper + (nrem if w == nw - 1 else 0)
            par.call("sum", a[4], wy[d], s, e)
    rec("par_coo", row=row, col=ccol, val=cval, N=N, x=x, y0=y0, nw=nw, y=M.get(a[4], dt, N))

    brp, bcol, bval = banded_csr(N, (-7, -2, 0, 1, 5), 23, dt)
    off, dat, nd, stride = ob.csr_dia(brp, bcol, bval)
    # the parallel build stores DIA and ELL data row by row (data[i*nd + k],
    # src/parallel/src/sparse32.js csr_dia / csr_ell), the sequential build
    # and the oracle column by column: the vectors keep the column layout
    dat_rows = dat.reshape(nd, stride)[:, :N].T.copy()
    M = Mem(par)
    po, pd, px, py = M.put(off), M.put(dat_rows), M.put(x), M.put(y0)
    for w in range(nw):
        s, e = w * nper, (w + 1) * nper + (nrem if w == nw - 1 else 0)
        par.call("spmv_dia_wrapper", w, po, pd, s, e, nd, N, px, py, 1)
    rec("par_dia", offset=off, data=dat, N=N, x=x, y0=y0, nw=nw, y=M.get(py, dt, N))
    # the column-layout worker kernel (tests/main32.js "dia_col_basic": end row inclusive)
    M = Mem(par)
    po, pd, px, py = M.put(off), M.put(dat), M.put(x), M.put(y0)
    for w in range(nw):
        s, e = w * nper, (w + 1) * nper - 1 + (nrem if w == nw - 1 else 0)
        par.call("spmv_dia_col_basic_wrapper", w, po, pd, s, e, nd, N, stride, px, py, 1)
    rec("par_dia_col", offset=off, data=dat, N=N, x=x, y0=y0, nw=nw, y=M.get(py, dt, N))

    ind, edat, nc = ob.csr_ell(rp, col, val)
    M = Mem(par)
    pi_, pd = M.put(ind.reshape(nc, N).T.copy()), M.put(edat.reshape(nc, N).T.copy())
    px, py = M.put(x), M.put(y0)
    for w in range(nw):
        s, e = w * nper, (w + 1) * nper + (nrem if w == nw - 1 else 0)
        par.call("spmv_ell_wrapper", w, pi_, pd, s, e, nc, N, px, py, 1)
    rec("par_ell", indices=ind, data=edat, N=N, nc=nc, x=x, y0=y0, nw=nw, y=M.get(py, dt, N))
    # the column-layout worker kernel (tests/main32.js "ell_col")
    M = Mem(par)
    pi_, pd, px, py = M.put(ind), M.put(edat), M.put(x), M.put(y0)
    for w in range(nw):
        s, e = w * nper, (w + 1) * nper + (nrem if w == nw - 1 else 0)
        par.call("spmv_ell_col_wrapper", w, pi_, pd, s, e, nc, N, px, py, 1)
    rec("par_ell_col", indices=ind, data=edat, N=N, nc=nc, x=x, y0=y0, nw=nw, y=M.get(py, dt, N))

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SCIWASM_SPARSE_SRC", "."))
