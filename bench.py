"""SpMV throughput benchmark of libsparse_b200 on B200.

Workload (default, `format_sweep_fp64`): the FP64 format sweep -- a banded
matrix with 4,000,000 rows and 11 diagonals at offsets -5..5 (values N(0,1),
43,999,970 nonzeros) in COO, CSR, DIA and ELL, and a power-law matrix with
2,000,000 rows (row lengths min(2000, Zipf(2)+15), ~41M nonzeros, uniform
distinct columns, values U[-1,1]) in COO and CSR (its DIA/ELL forms are
refused by the admission test).  One step = one y <- y + A x per (matrix,
format) pair.  The metric is algorithmic HBM GB/s (bytes that must move per
call, x counted once) at <= 1e-5 relative error against an FP64 check.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload format_sweep_fp64|laplacian_fp32] [--small]

With N > 1 (torchrun, one rank per GPU) every rank processes its own copy
of the workload (independent objects, no collective on the data path):
weak scaling, value = bytes of all ranks / max-over-ranks time.
`--impl reference` times the CPU restatement of the reference's parallel
worker kernels (static_nnz CSR split, private-y COO, row-split DIA/ELL) on all
host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SECTIONS = ("batched", "laplacian4096_fp32", "spts", "serving", "powerlaw_csr", "serving_sweep",
            "gather_ceiling", "conversions")
METRIC = "served SpMV/SpTS req/s + p99 vs plain path; SpMV HBM GB/s at \u22641e-5 rel err"
UNIT = "GB/s"


# ------------------------------------------------------------------ workload

def algo_bytes(fmt: str, N: int, nnz: int, s_v: int, width: int = 0) -> int:
    """Compulsory bytes of one y <- y + A x call (x read once, y read+written)."""
    vec = N * s_v + 2 * N * s_v
    if fmt == "csr":
        return nnz * (s_v + 4) + 4 * (N + 1) + vec
    if fmt == "coo":
        return nnz * (8 + s_v) + vec
    if fmt == "dia":
        return width * N * s_v + 4 * width + vec
    if fmt == "ell":
        return width * N * (s_v + 4) + vec
    raise ValueError(fmt)


def make_workload(name: str, small: bool):
    """Host arrays of every (label, format, arrays...) job."""
    from sciwasm.sparse_b200 import synth
    jobs = []
    if name == "format_sweep_fp64":
        nb = 1_000_000 if small else 4_000_000
        npl = 500_000 if small else 2_000_000
        rp, col, val = synth.banded(nb, half=5, seed=1, dtype=np.float64)
        jobs.append(dict(label="banded", N=nb, rp=rp, col=col, val=val,
                         formats=["coo", "csr", "dia", "ell"]))
        rp, col, val = synth.power_law(npl, seed=2, dtype=np.float64)
        jobs.append(dict(label="powerlaw", N=npl, rp=rp, col=col, val=val,
                         formats=["coo", "csr"]))
    elif name == "laplacian_fp32":
        n = 1024 if small else 256
        rp, col, val = synth.laplacian_2d(n, dtype=np.float32)
        jobs.append(dict(label=f"laplacian{n}", N=n * n, rp=rp, col=col, val=val,
                         formats=["coo", "csr", "dia", "ell"]))
    else:
        raise SystemExit(f"unknown workload {name}")
    for j in jobs:
        j["x"] = synth.uniform_vec(j["N"], 0, dtype=j["val"].dtype)
    return jobs


def truth_f64(rp, col, val, x):
    prod = val.astype(np.float64) * x.astype(np.float64)[col]
    out = np.zeros(rp.size - 1)
    nz = np.diff(rp) > 0
    out[nz] = np.add.reduceat(prod, rp[:-1][nz])
    return out


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during timing."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


# ------------------------------------------------------------------ CPU arm

def cpu_pass(jobs, nthreads, fmt_data):
    """One pass of every (matrix, format) SpMV on the CPU restatement."""
    from oracle import binding as orc
    for j in jobs:
        for fmt in j["formats"]:
            d = fmt_data[(j["label"], fmt)]
            y = d["y"]
            y[:] = 0
            if fmt == "csr":
                orc.par_spmv_csr(nthreads, j["rp"], j["col"], j["val"], j["x"], y)
            elif fmt == "coo":
                orc.par_spmv_coo(d["nt_coo"], d["row"], j["col"], j["val"], j["x"], y, j["N"],
                                 d["wy"])
            elif fmt == "dia":
                if d["layout"] == "rows":
                    orc.par_spmv_dia_rows(nthreads, d["off"], d["data_rows"], j["N"], j["x"], y)
                else:
                    orc.par_spmv_dia(nthreads, d["off"], d["data"], j["N"], j["x"], y)
            elif fmt == "ell":
                if d["layout"] == "rows":
                    orc.par_spmv_ell_rows(nthreads, d["ind_rows"], d["data_rows"], j["N"], d["nc"],
                                          j["x"], y)
                else:
                    orc.par_spmv_ell(nthreads, d["ind"], d["data"], j["N"], d["nc"], j["x"], y)


def _choose_layout(j, d, fmt, nthreads):
    """The reference benchmarks DIA and ELL with two worker kernels each: over
    column-by-column data ("dia_col_basic", "ell_col") and over row-by-row data
    ("dia_row", "ell_row").  Time both once (after a warm call) and keep the
    faster, so the baseline is the reference's better CPU path."""
    from oracle import binding as orc
    n = j["N"]
    k = d["off"].size if fmt == "dia" else d["nc"]
    if fmt == "dia":
        d["data_rows"] = d["data"].reshape(k, n).T.copy()
    else:
        d["ind_rows"] = d["ind"].reshape(k, n).T.copy()
        d["data_rows"] = d["data"].reshape(k, n).T.copy()
    best = None
    for layout in ("cols", "rows"):
        d["layout"] = layout
        ts = []
        for _ in range(2):
            t0 = time.perf_counter()
            cpu_pass([{**j, "formats": [fmt]}], nthreads, {(j["label"], fmt): d})
            ts.append(time.perf_counter() - t0)
        if best is None or ts[-1] < best[1]:
            best = (layout, ts[-1])
    d["layout"] = best[0]


def prepare_cpu(jobs):
    from sciwasm.sparse_b200 import synth
    nthreads = os.cpu_count() or 1
    fmt_data = {}
    for j in jobs:
        for fmt in j["formats"]:
            d = {"y": np.zeros(j["N"], j["val"].dtype)}
            if fmt == "coo":
                d["row"] = synth.csr_to_coo_rows(j["rp"])
                budget = 2 << 30
                d["nt_coo"] = max(1, min(nthreads, budget // max(1, j["N"] * j["val"].itemsize)))
                d["wy"] = np.zeros(d["nt_coo"] * j["N"], j["val"].dtype)
            elif fmt == "dia":
                d["off"], d["data"] = synth.csr_to_dia_host(j["rp"], j["col"], j["val"])
            elif fmt == "ell":
                d["ind"], d["data"], d["nc"] = synth.csr_to_ell_host(j["rp"], j["col"], j["val"])
            if fmt in ("dia", "ell"):
                _choose_layout(j, d, fmt, nthreads)
            fmt_data[(j["label"], fmt)] = d
    return nthreads, fmt_data


def layouts_note(fmt_data):
    """Which worker-kernel layout the baseline kept for each DIA/ELL object."""
    chosen = [f"{k[0]}/{k[1]}: {v['layout']}" for k, v in fmt_data.items() if "layout" in v]
    return "; DIA/ELL worker kernels (the faster layout of the reference's two): " + \
        ", ".join(chosen) if chosen else ""


def step_bytes(jobs, fmt_data=None):
    tot = 0
    for j in jobs:
        s_v = j["val"].itemsize
        nnz = j["col"].size
        for fmt in j["formats"]:
            w = 0
            if fmt == "dia":
                w = int(np.unique(j["col"].astype(np.int64) -
                                  np.repeat(np.arange(j["N"]), np.diff(j["rp"]))).size) \
                    if fmt_data is None else fmt_data[(j["label"], fmt)]["off"].size
            if fmt == "ell":
                w = int(np.diff(j["rp"]).max())
            tot += algo_bytes(fmt, j["N"], nnz, s_v, w)
    return tot


def run_reference(args, jobs, config):
    nthreads, fmt_data = prepare_cpu(jobs)
    bytes_step = step_bytes(jobs, fmt_data)
    for _ in range(args.warmup):
        cpu_pass(jobs, nthreads, fmt_data)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_pass(jobs, nthreads, fmt_data)
    dt = time.perf_counter() - t0
    value = bytes_step * args.steps / dt / 1e9
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": config["dtype"], "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": nthreads,
                         "kind": "port",
                         "sample": f"full workload, {args.steps} passes of every "
                                   "(matrix, format) SpMV, pthreads over all host cores "
                                   "(reference worker kernels restated in C, not V8/wasm)"
                                   + layouts_note(fmt_data)},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(jobs, budget_s=12.0):
    nthreads, fmt_data = prepare_cpu(jobs)
    bytes_step = step_bytes(jobs, fmt_data)
    cpu_pass(jobs, nthreads, fmt_data)  # warm
    t0 = time.perf_counter()
    cpu_pass(jobs, nthreads, fmt_data)
    one = time.perf_counter() - t0
    reps = max(1, min(50, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(reps):
        cpu_pass(jobs, nthreads, fmt_data)
    dt = time.perf_counter() - t0
    return {"value": round(bytes_step * reps / dt / 1e9, 3), "unit": UNIT, "cores": nthreads,
            "kind": "port",
            "sample": f"{reps} full passes of the workload's SpMVs on {nthreads} threads "
                      "(C restatement of the reference's worker kernels, pthreads)"
                      + layouts_note(fmt_data)}


# ------------------------------------------------------------------ GPU arm

def conversion_bytes(kind, N, nnz, s_v, width=0):
    """Algorithmic bytes of one conversion: its input read plus its output
    written (zero fill included)."""
    csr = nnz * (4 + s_v) + 4 * (N + 1)
    if kind == "coo_csr":
        return nnz * (8 + s_v) + csr
    if kind == "csr_dia":
        return csr + width * N * s_v + 4 * width
    if kind == "csr_ell":
        return csr + width * N * (4 + s_v)
    raise ValueError(kind)


def _timed_call(stream, fn, reps=3):
    """(median device ms over reps calls of fn bracketed by CUDA events on
    `stream`, result of the last call); fn's own host synchronisations fall
    inside the bracket."""
    import torch
    times, out = [], None
    for _ in range(reps):
        out = None
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.median(times)), out


def device_conversions(jobs, stream):
    """Objects of the format sweep built on the device.  For each matrix: a
    COO sorted by (row, col) is uploaded (the "coo" object), coo_csr runs on
    it (the copy-speed path) and on a shuffled copy (the row-bucket sort,
    whose output becomes the "csr" object), then csr_dia and csr_ell
    run on the CSR (refused for the power-law matrix, as in the reference).
    Returns (objects, timings, host copies of inputs and outputs for the
    bit-exact check)."""
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib, synth
    from sciwasm.sparse_b200 import sparse as sbs
    sp = stream.cuda_stream
    objs, conv, check = [], {}, {}

    def coo_csr_into(Acoo, out):
        # the conversion alone: its output is allocated outside the timing
        # (cudaMalloc of a few hundred MB varied from 1 to 90 ms between runs)
        _lib.call("sb_coo_csr", sbs._dtcode(Acoo.dtype), Acoo.row_index.ptr,
                  Acoo.col_index.ptr, Acoo.val_index.ptr, Acoo.N, Acoo.nnz,
                  out.row_index.ptr, out.col_index.ptr, out.val_index.ptr, sp)
        return out

    for j in jobs:
        N, rp, col, val = j["N"], j["rp"], j["col"], j["val"]
        s_v, nnz = val.itemsize, col.size
        x = sb.vec_from_host(j["x"])
        row = synth.csr_to_coo_rows(rp)
        Acoo = sb.coo_from_host(row, col, val, N)
        c = {}
        Asorted = sbs.allocate_CSR(N, nnz, val.dtype)
        ms, _ = _timed_call(stream, lambda: coo_csr_into(Acoo, Asorted))
        b = conversion_bytes("coo_csr", N, nnz, s_v)
        c["coo_csr_sorted_input"] = {"ms": round(ms, 3), "GB_s": round(b / ms / 1e6, 1),
                                     "algorithmic_bytes": b}
        del Asorted
        perm = np.random.default_rng(20 + len(conv)).permutation(nnz)
        shuf = (row[perm], col[perm], val[perm])
        del perm
        Ashuf = sb.coo_from_host(*shuf, N)
        Acsr = sbs.allocate_CSR(N, nnz, val.dtype)
        ms, _ = _timed_call(stream, lambda: coo_csr_into(Ashuf, Acsr))
        c["coo_csr_shuffled_input"] = {"ms": round(ms, 3), "GB_s": round(b / ms / 1e6, 1),
                                       "algorithmic_bytes": b}
        del Ashuf
        chk = {"N": N, "shuffled": shuf, "csr": (Acsr.row_array(), Acsr.col_array(),
                                                 Acsr.val_array())}
        made = {"coo": (Acoo, 0), "csr": (Acsr, 0)}
        for kind, fmt in (("csr_dia", "dia"), ("csr_ell", "ell")):
            # the counting pass (num_diags / num_cols) and the fill are timed;
            # the output is allocated outside the timing, as for coo_csr
            if fmt == "dia":
                nd, stride = sb.num_diags(Acsr, stream=sp)
                ok = _lib.load().sb_dia_admitted(nd, stride, nnz)
                M = sbs.allocate_DIA(N, nnz, nd, stride, val.dtype) if ok else None

                def conv_fn(M=M):
                    nd2, stride2 = sb.num_diags(Acsr, stream=sp)
                    if M is not None:
                        _lib.call("sb_csr_dia", sbs._dtcode(Acsr.dtype), Acsr.row_index.ptr,
                                  Acsr.col_index.ptr, Acsr.val_index.ptr, N, nnz, nd2, stride2,
                                  M.offset_index.ptr, M.data_index.ptr, sp)
                    return M
            else:
                nc = sb.num_cols(Acsr, stream=sp)
                ok = _lib.load().sb_ell_admitted(nc, N, nnz)
                M = sbs.allocate_ELL(N, nnz, nc, val.dtype) if ok else None

                def conv_fn(M=M):
                    nc2 = sb.num_cols(Acsr, stream=sp)
                    if M is not None:
                        _lib.call("sb_csr_ell", sbs._dtcode(Acsr.dtype), Acsr.row_index.ptr,
                                  Acsr.col_index.ptr, Acsr.val_index.ptr, N, nnz, nc2,
                                  M.indices_index.ptr, M.data_index.ptr, sp)
                    return M
            ms, M = _timed_call(stream, conv_fn)
            if M is None:
                c[kind] = {"refused": True, "ms": round(ms, 3)}
                chk[fmt] = None
                continue
            w = M.ndiags if fmt == "dia" else M.ncols
            b2 = conversion_bytes(kind, N, nnz, s_v, w)
            c[kind] = {"ms": round(ms, 3), "GB_s": round(b2 / ms / 1e6, 1),
                       "algorithmic_bytes": b2, "width": w}
            chk[fmt] = ((M.offset_array(), M.data_array()) if fmt == "dia"
                        else (M.indices_array(), M.data_array()))
            made[fmt] = (M, w)
        for fmt in j["formats"]:
            if fmt not in made:
                raise SystemExit(f"{j['label']}: {fmt} form was refused by the conversion")
            A, w = made[fmt]
            y = sb.create_vec(N, 0, val.dtype)
            objs.append(dict(label=f"{j['label']}/{fmt}", fmt=fmt, A=A, x=x, y=y, job=j,
                             bytes=algo_bytes(fmt, N, nnz, s_v, w)))
        conv[j["label"]] = c
        check[j["label"]] = chk
    return objs, conv, check


def run_conversions(stream, small):
    """The format sweep's device conversions alone (coo_csr on sorted and
    shuffled input, csr_dia, csr_ell), timed as in the bench line; for
    profiling the conversion kernels.  The oracle check is left to the full
    run."""
    jobs = make_workload("format_sweep_fp64", small)
    _, conv, _ = device_conversions(jobs, stream)
    return conv


def conversions_cpu_check(conv, check):
    """CPU-baseline leg of the conversions: the oracle's serial coo_csr,
    csr_dia and csr_ell (the reference's conversions are serial JavaScript),
    timed on the same inputs, and the device outputs compared with them bit
    for bit."""
    from oracle import binding as orc

    def same(a, b):
        a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
        return a.dtype == b.dtype and a.shape == b.shape and \
            np.array_equal(a.view(np.uint8), b.view(np.uint8))

    for label, chk in check.items():
        c = conv[label]
        t0 = time.perf_counter()
        want = orc.coo_csr(*chk["shuffled"], chk["N"])
        t_csr = time.perf_counter() - t0
        ok = all(same(a, b) for a, b in zip(chk["csr"], want))
        cpu = {"coo_csr_shuffled_input_ms": round(t_csr * 1e3, 1)}
        for fmt, fn in (("dia", orc.csr_dia), ("ell", orc.csr_ell)):
            t0 = time.perf_counter()
            w = fn(*want)
            cpu[f"csr_{fmt}_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
            if w is None or chk[fmt] is None:
                ok = ok and (w is None) and (chk[fmt] is None)
            else:
                ok = ok and same(chk[fmt][0], w[0]) and same(chk[fmt][1], w[1])
        c["cpu_baseline"] = {**cpu, "cores": 1, "kind": "port",
                             "sample": "one call each, serial C restatement of the "
                                       "reference's conversions (JavaScript, serial)"}
        c["bit_exact"] = bool(ok)



def run_ours(args, jobs, config, rank, world, local_rank):
    import torch
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib, synth
    from sciwasm.sparse_b200.dist import max_over_ranks

    sb.load_library()
    torch.cuda.set_device(local_rank)
    _lib.call("sb_set_device", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_

    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    # every (matrix, format) object comes from the device conversions:
    # COO (rows sorted, as the reference's reader leaves it) uploaded, then
    # coo_csr -> csr_dia / csr_ell on the device, each timed
    objs, conversions, conv_check = device_conversions(jobs, stream)
    bytes_step = sum(o["bytes"] for o in objs)

    # the autotuner picks each CSR matrix's kernel options (setup, untimed),
    # unless --csr-fixed pins them (e.g. to profile the kernels a plain run
    # chose: the tuning trials are not representative under a profiler)
    fixed = {}
    for item in (args.csr_fixed or "").split(";"):
        if item.strip():
            label, vals = item.split(":")
            fixed[label.strip()] = [int(v) for v in vals.split(",")]
    for o in objs:
        if o["fmt"] == "csr":
            label = o["label"].split("/")[0]
            if label in fixed:
                o["A"].opts = _lib.CsrOpts(*fixed[label])
                o["tuned"] = dict(zip(("kernel", "lanes_per_row", "unroll", "grid"), fixed[label]))
            else:
                o["tuned"] = sb.csr_autotune(o["A"], o["x"], stream=sptr)
    torch.cuda.synchronize()

    # correctness gate: one call from y = 0 against an FP64 check
    max_err = 0.0
    truths = {}
    for o in objs:
        j = o["job"]
        if j["label"] not in truths:
            truths[j["label"]] = truth_f64(j["rp"], j["col"], j["val"], j["x"])
        o["y"].vec_index.fill_zero(sptr)
        sb.spmv(o["A"], o["x"], o["y"], stream=sptr)
        stream.synchronize()
        t = truths[j["label"]]
        err = float(np.max(np.abs(o["y"].array() - t)) / max(np.max(np.abs(t)), 1e-300))
        o["rel_err"] = err
        max_err = max(max_err, err)
    if max_err > 1e-5:
        raise SystemExit(f"correctness gate failed: max rel err {max_err:.3e}")

    def step(ev=None):
        for k, o in enumerate(objs):
            if ev is not None:
                ev[k][0].record(stream)
            sb.spmv(o["A"], o["x"], o["y"], stream=sptr)
            if ev is not None:
                ev[k][1].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    # pad the sampled window so the clock record has samples under load
    pad_until = time.perf_counter() + 0.5
    with torch.cuda.stream(stream):
        while time.perf_counter() < pad_until:
            step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in objs] for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        t_start.record(stream)
        for s in range(args.steps):
            step(evs[s])
        t_end.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    pad_until = time.perf_counter() + 0.3
    with torch.cuda.stream(stream):
        while time.perf_counter() < pad_until:
            step()
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed_ms = t_start.elapsed_time(t_end)
    per_obj_ms = [float(np.mean([evs[s][k][0].elapsed_time(evs[s][k][1])
                                 for s in range(args.steps)])) for k in range(len(objs))]
    elapsed_ms = max_over_ranks(elapsed_ms, device="cuda")
    value = bytes_step * args.steps * world / (elapsed_ms / 1e3) / 1e9

    # ---------------- e2e through the public API with host buffers
    # Every call does what the reference's benchmark does around spmv
    # (src/sequential/tests/main32.js:123-124): clear_vec(y), then
    # spmv(A, x, y) -- here with x uploaded from pinned host memory first and
    # y read back after.  clear_vec zeroes y on the device.  Calls rotate over
    # --e2e-streams streams, each call with its own device x and y, so one
    # call's copies overlap another's kernel and the two copy directions
    # overlap each other.
    h2d = 0
    d2h = 0
    host = []
    e2e_streams = [stream] + [torch.cuda.Stream() for _ in range(max(1, args.e2e_streams) - 1)]
    for k, o in enumerate(objs):
        N = o["job"]["N"]
        dt = o["job"]["val"].dtype
        nb = N * dt.itemsize
        xp, yo = _pinned(nb), _pinned(nb)
        _host_view(xp, N, dt)[:] = o["job"]["x"]
        xd, yd = sb.create_vec(N, 0, dt), sb.create_vec(N, 0, dt)
        host.append((xp, yo, nb, xd, yd, e2e_streams[k % len(e2e_streams)].cuda_stream))
        h2d += nb
        d2h += nb

    def e2e_step():
        for o, (xp, yo, nb, xd, yd, sp_k) in zip(objs, host):
            _lib.call("sb_memcpy_htod", xd.vec_index.ptr, xp, nb, sp_k)
            sb.clear_vec(yd, stream=sp_k)
            sb.spmv(o["A"], xd, yd, stream=sp_k)
            _lib.call("sb_memcpy_dtoh", yo, yd.vec_index.ptr, nb, sp_k)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for sd in e2e_streams[1:]:
        sd.wait_event(e0)
    for _ in range(args.steps):
        e2e_step()
    for sd in e2e_streams[1:]:
        side_done = torch.cuda.Event()
        side_done.record(sd)
        stream.wait_event(side_done)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, device="cuda")
    e2e_value = bytes_step * args.steps * world / (e2e_ms / 1e3) / 1e9

    # the same step's copies alone (same buffers and streams, no kernels):
    # the host link's floor under the e2e time
    def copy_step():
        for o, (xp, yo, nb, xd, yd, sp_k) in zip(objs, host):
            _lib.call("sb_memcpy_htod", xd.vec_index.ptr, xp, nb, sp_k)
            _lib.call("sb_memcpy_dtoh", yo, yd.vec_index.ptr, nb, sp_k)
    copy_step()
    torch.cuda.synchronize()
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    for sd in e2e_streams[1:]:
        sd.wait_event(c0)
    for _ in range(args.steps):
        copy_step()
    for sd in e2e_streams[1:]:
        side_done = torch.cuda.Event()
        side_done.record(sd)
        stream.wait_event(side_done)
    c1.record(stream)
    torch.cuda.synchronize()
    copy_ms = max_over_ranks(c0.elapsed_time(c1), device="cuda")
    # the read-back results meet the same check as the device results
    for o, (xp, yo, nb, xd, yd, sp_k) in zip(objs, host):
        t = truths[o["job"]["label"]]
        got = _host_view(yo, o["job"]["N"], o["job"]["val"].dtype)
        err = float(np.max(np.abs(got - t)) / max(np.max(np.abs(t)), 1e-300))
        if not err <= 1e-5:
            raise SystemExit(f"e2e read-back of {o['label']}: rel err {err:.3e}")
    for xp, yo, *_ in host:
        for p_ in (xp, yo):
            _lib.call("sb_host_free", p_)

    # ---------------- roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    tot = [per_obj_ms[k] for k in range(len(objs))]
    dom = int(np.argmax(tot))
    achieved = objs[dom]["bytes"] / (per_obj_ms[dom] / 1e3) / 1e9
    traffic = profiled_traffic().get(objs[dom]["label"] + ("/small" if args.small else ""))
    # the gather floor of each matrix: its col/val streams and x gathers with
    # no row structure (sb_gather_dot), timed the same way
    floors = {}
    for o in objs:
        label = o["job"]["label"]
        if o["fmt"] == "csr" and label not in floors:
            floors[label] = gather_floor_ms(stream, o["A"], o["x"])
    detail = {o["label"]: {"ms": round(per_obj_ms[k], 4),
                           "GB_s": round(o["bytes"] / (per_obj_ms[k] / 1e3) / 1e9, 1),
                           "frac": round(o["bytes"] / (per_obj_ms[k] / 1e3) / 1e9 / peak, 3),
                           "rel_err": o["rel_err"],
                           "gather_floor_ms": round(floors[o["job"]["label"]], 4),
                           "frac_of_gather_floor": round(floors[o["job"]["label"]] /
                                                         per_obj_ms[k], 3),
                           **({"tuned": {k2: v for k2, v in o["tuned"].items() if k2 != "ms"}}
                              if "tuned" in o else {})}
              for k, o in enumerate(objs)}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(elapsed_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": config["dtype"], "data": "synthetic",
        "config": config,
        "roofline": {"bound": "hbm", "kernel": objs[dom]["label"],
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic,
                     "algorithmic_bytes": objs[dom]["bytes"],
                     "gather_floor_ms": round(floors[objs[dom]["job"]["label"]], 4),
                     "frac_of_gather_floor": round(floors[objs[dom]["job"]["label"]] /
                                                   per_obj_ms[dom], 3)},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "ms_per_step": round(e2e_ms / args.steps, 4),
                "copies_only_ms_per_step": round(copy_ms / args.steps, 4),
                "frac_of_copy_floor": round(copy_ms / e2e_ms, 3),
                "host_link_GB_s": round((h2d + d2h) / (copy_ms / args.steps / 1e3) / 1e9, 1),
                "path": "sciwasm.sparse_b200 via the C ABI, per call the reference "
                        "benchmark's sequence clear_vec(y); spmv(A, x, y) with x uploaded "
                        "from pinned host memory before it and y read back after it "
                        "(clear_vec zeroes y on the device); matrices resident; calls "
                        f"rotate over {len(e2e_streams)} streams"},
        "gpu_launches": len(objs) * args.steps,
        "clocks": clk,
        "max_rel_err": max_err,
        "per_call": detail,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(jobs)
        conversions_cpu_check(conversions, conv_check)
    del conv_check
    line["conversions"] = conversions
    if world == 1 and not args.no_sections:
        line["laplacian4096_fp32"] = run_laplacian_large(stream, peak)
        line["batched"] = run_batched(stream, peak)
        line["spts"] = run_spts_section(stream, cpu=not args.no_cpu_baseline)
        torch.cuda.empty_cache()
    if world == 1 and not args.no_serving:
        line["serving"] = run_serving(args)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ serving

SERVE_STRUCT_MV = ("banded", "powerlaw", "laplacian2d")
SERVE_STRUCT_TS = ("laplacian3d_lower", "random_lower")


def build_serving_pool(n_mats, min_rows, max_rows, seed=11):
    """Resident pool of the serving workload, generated on the device: rows
    log-uniform in [min_rows, max_rows]; two thirds SpMV matrices (banded /
    power-law / 2-D Laplacian, f32 and bf16 values), one third triangular
    factors (3-D Laplacian lower / random lower, f32 values with a level-set
    plan; f64 accumulation where the growth estimate exceeds 1)."""
    from sciwasm.sparse_b200 import serve, synth_device as sd
    rng = np.random.default_rng(seed)
    pool = serve.ResidentPool(budget_bytes=150 * 10**9)
    mv, ts = [], []
    nrows = np.exp(rng.uniform(np.log(min_rows), np.log(max_rows), n_mats)).astype(np.int64)
    for i, N in enumerate(nrows):
        N = int(N)
        name = f"m{i}"
        if i % 3 == 2:
            kind = SERVE_STRUCT_TS[(i // 3) % 2]
            if kind == "laplacian3d_lower":
                A = sd.laplacian_3d_lower(max(2, int(round(N ** (1 / 3)))))
            else:
                A = sd.random_lower(N, per_row=7, band=5000, seed=seed + i)
            pool.add_csr(name, A, spmv_storages=(), spts_dtypes=("f32",))
            ts.append(name)
        else:
            kind = SERVE_STRUCT_MV[(i // 3 * 2 + i % 3) % 3]
            if kind == "banded":
                A = sd.banded(N, half=5, seed=seed + i)
            elif kind == "powerlaw":
                A = sd.power_law(N, seed=seed + i)
            else:
                A = sd.laplacian_2d(max(2, int(round(N ** 0.5))))
            pool.add_csr(name, A, spmv_storages=("f32", "bf16"))
            mv.append(name)
    return pool, mv, ts


def serving_requests(pool, mv, ts, rate, seconds, in_ring, out_ring, seed=12, spmv_frac=0.7):
    """Poisson arrivals; 70% SpMV (f32 or bf16 values, even odds) on a
    uniformly drawn SpMV matrix, 30% SpTS on a uniformly drawn factor.
    Inputs and outputs are consecutive slices of pinned rings (wrapping)."""
    from sciwasm.sparse_b200 import serve
    rng = np.random.default_rng(seed)
    t = serve.poisson_arrivals(rate, seconds, seed=seed)
    is_mv = rng.random(t.size) < spmv_frac
    pick_mv = rng.integers(0, len(mv), t.size)
    pick_ts = rng.integers(0, len(ts), t.size)
    bf = rng.random(t.size) < 0.5
    reqs = []
    io = oo = 0
    for k in range(t.size):
        if is_mv[k]:
            name, op, st = mv[pick_mv[k]], "spmv", ("bf16" if bf[k] else "f32")
        else:
            name, op, st = ts[pick_ts[k]], "spts", "f32"
        N = pool.mats[name].N
        nb = serve._al(4 * N)
        if io + nb > in_ring.nbytes:
            io = 0
        if oo + nb > out_ring.nbytes:
            oo = 0
        x = in_ring.view(io, N, np.float32)
        y = out_ring.view(oo, N, np.float32)
        io += nb
        oo += nb
        reqs.append(serve.Request(k, float(t[k]), name, op, st, x, y))
    return reqs


def serving_errors(pool, srv, mv, ts, n_check=24, seed=13):
    """Max relative error (max norm) against an FP64 host computation (scipy)
    of a sample of requests served in one batched mix: SpMV on the stored
    values (f32, or bf16 widened), SpTS on the f32 factor."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sl
    from sciwasm.sparse_b200 import serve
    rng = np.random.default_rng(seed)
    small_mv = [n for n in mv if pool.mats[n].N <= 400_000] or mv
    small_ts = [n for n in ts if pool.mats[n].N <= 400_000] or ts
    reqs = []
    for k in range(n_check):
        if k % 3 == 2:
            name, op, st = small_ts[rng.integers(len(small_ts))], "spts", "f32"
        else:
            name, op, st = small_mv[rng.integers(len(small_mv))], "spmv", ("f32", "bf16")[k % 2]
        N = pool.mats[name].N
        x = rng.uniform(-1, 1, N).astype(np.float32)
        reqs.append(serve.Request(k, 0.0, name, op, st, x, np.zeros(N, np.float32)))
    srv.serve(reqs, "batched")
    errs = {"spmv_f32": 0.0, "spmv_bf16": 0.0, "spts_f32": 0.0}
    for r in reqs:
        A = pool.mats[r.matrix].csr[r.storage]
        rp, col = A.row_array(), A.col_array()
        v = A.val_array()
        if r.storage == "bf16":
            v = (v.astype(np.uint32) << 16).view(np.float32)
        M = sp.csr_matrix((v.astype(np.float64), col, rp), shape=(A.N, A.N))
        if r.op == "spmv":
            t = M @ r.x.astype(np.float64)
        else:
            t = sl.spsolve_triangular(M, r.x.astype(np.float64), lower=True)
        e = float(np.max(np.abs(r.y - t)) / max(np.max(np.abs(t)), 1e-300))
        key = f"{r.op}_{r.storage}"
        errs[key] = max(errs[key], e)
    return errs


# ------------------------------------------------------------------ other configs

def _time_each_ms(stream, fn, reps):
    """Mean device time of fn() over reps runs, each bracketed by CUDA events
    on `stream` (host gaps between runs are not counted)."""
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(reps)]
    with torch.cuda.stream(stream):
        for e0, e1 in evs:
            e0.record(stream)
            fn()
            e1.record(stream)
    torch.cuda.synchronize()
    return float(np.mean([e0.elapsed_time(e1) for e0, e1 in evs]))


def _vec(t):
    import sciwasm.sparse_b200 as sb
    n = t.numel()
    dt = np.float64 if str(t.dtype) == "torch.float64" else np.float32
    return sb.sparse_vec_t(sb.DeviceArray(n, dt, t.data_ptr()), n)


def gather_floor_ms(stream, A, x, reps=20):
    """Mean device time of sb_gather_dot on A's col/val and x: the column and
    value streams an SpMV must read and its x gathers, with no row
    structure -- the floor of any SpMV kernel on this matrix."""
    import torch
    from sciwasm.sparse_b200 import _lib
    from sciwasm.sparse_b200.sparse import DeviceArray
    out = DeviceArray.from_host(np.zeros(1))
    code = _lib.SB_F64 if A.dtype == np.float64 else _lib.SB_F32
    sp = stream.cuda_stream

    def fn():
        _lib.call("sb_gather_dot", code, A.col_index.ptr, A.val_index.ptr, x.vec_index.ptr,
                  A.nnz, out.ptr, sp)
    for _ in range(3):
        with torch.cuda.stream(stream):
            fn()
    return _time_each_ms(stream, fn, reps)


def run_gather_ceiling(stream, peak, small=False):
    """The power-law matrix of the format sweep (2M rows, ~41M nonzeros, FP64;
    1M rows with small, ~250 MB of col/val, still above L2): the gather floor
    (sb_gather_dot) beside CSR (row blocks with tuned options, block stream)
    and COO, each as a fraction of the HBM peak and of the floor."""
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib, synth
    n = 1_000_000 if small else 2_000_000
    rp, col, val = synth.power_law(n, seed=2, dtype=np.float64)
    A = sb.csr_from_host(rp, col, val)
    x = sb.vec_from_host(synth.uniform_vec(n, 0))
    y = sb.create_vec(n, 0, np.float64)
    sp = stream.cuda_stream
    floor = gather_floor_ms(stream, A, x)
    nnz = col.size
    out = {"N": n, "nnz": int(nnz), "gather_floor_ms": round(floor, 4),
           "gather_floor_GB_s": round(nnz * 12 / floor / 1e6, 1)}
    tuned = sb.csr_autotune(A, x, stream=sp)
    cands = [("csr_tuned", tuple(tuned[k] for k in ("kernel", "lanes_per_row", "unroll", "grid"))),
             ("csr_block_stream", (3, 0, 0, 0)), ("csr_row_blocks_8_4_1", (0, 8, 4, 1))]
    for label, opts in cands:
        A.opts = _lib.CsrOpts(*opts)
        for _ in range(3):
            sb.spmv(A, x, y, stream=sp)
        ms = _time_each_ms(stream, lambda: sb.spmv(A, x, y, stream=sp), 20)
        b = algo_bytes("csr", n, nnz, 8)
        out[label] = {"opts": list(opts), "ms": round(ms, 4), "frac": round(b / ms / 1e6 / peak, 3),
                      "frac_of_gather_floor": round(floor / ms, 3)}
    C = sb.coo_from_host(synth.csr_to_coo_rows(rp), col, val, n)
    for _ in range(3):
        sb.spmv(C, x, y, stream=sp)
    ms = _time_each_ms(stream, lambda: sb.spmv(C, x, y, stream=sp), 20)
    b = algo_bytes("coo", n, nnz, 8)
    out["coo"] = {"ms": round(ms, 4), "frac": round(b / ms / 1e6 / peak, 3),
                  "frac_of_gather_floor": round(floor / ms, 3)}
    return out


def run_laplacian_large(stream, peak):
    """CSR SpMV, FP32 and BF16 values, on the 5-point Laplacian of a 4096 x 4096
    grid (16,777,216 rows, 83,869,696 nonzeros; 0.94 GB in FP32, above L2)."""
    import torch
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import synth_device as sd
    n = 4096
    A = sd.laplacian_2d(n)
    N, nnz = A.N, A.nnz
    g = torch.Generator(device="cuda").manual_seed(0)
    xt = torch.rand(N, generator=g, device="cuda") * 2 - 1
    yt = torch.zeros(N, device="cuda")
    x, y = _vec(xt), _vec(yt)
    sp = stream.cuda_stream
    X = xt.double().reshape(n, n)
    T = 4 * X
    T[1:, :] -= X[:-1, :]
    T[:-1, :] -= X[1:, :]
    T[:, 1:] -= X[:, :-1]
    T[:, :-1] -= X[:, 1:]
    out = {"workload": "5-point Laplacian 4096^2, x ~ U[-1,1] seed 0, y <- y + A x",
           "N": N, "nnz": nnz}
    for storage in ("f32", "bf16"):
        B = A if storage == "f32" else sb.csr_with_storage(A, "bf16")
        tuned = sb.csr_autotune(B, x, stream=sp)
        torch.cuda.synchronize()
        yt.zero_()
        with torch.cuda.stream(stream):
            sb.spmv(B, x, y, stream=sp)
        torch.cuda.synchronize()
        err = float((yt.double().reshape(n, n) - T).abs().max() / T.abs().max())
        for _ in range(3):
            with torch.cuda.stream(stream):
                sb.spmv(B, x, y, stream=sp)
        ms = _time_each_ms(stream, lambda: sb.spmv(B, x, y, stream=sp), 20)
        nbytes = algo_bytes("csr", N, nnz, 2 if storage == "bf16" else 4) + \
            (3 * N * 4 - 3 * N * (2 if storage == "bf16" else 4))  # x, y stay f32
        gbs = nbytes / (ms / 1e3) / 1e9
        out[storage] = {"ms": round(ms, 4), "GB_s": round(gbs, 1), "frac": round(gbs / peak, 3),
                        "algorithmic_bytes": nbytes, "rel_err_vs_fp64": err,
                        "tuned": {k: v for k, v in tuned.items() if k != "ms"}}
    # the format the statistics choose for a 5-point stencil (DIA, no index
    # arrays), with FP32 and BF16 data
    D, info = sb.spmv_autotune(A, timed=False)
    out["format_choice"] = info["format"]
    if info["format"] == "dia":
        for storage in ("f32", "bf16"):
            Ds = D if storage == "f32" else sb.with_storage(D, "bf16")
            yt.zero_()
            with torch.cuda.stream(stream):
                sb.spmv(Ds, x, y, stream=sp)
            torch.cuda.synchronize()
            err = float((yt.double().reshape(n, n) - T).abs().max() / T.abs().max())
            for _ in range(3):
                with torch.cuda.stream(stream):
                    sb.spmv(Ds, x, y, stream=sp)
            ms = _time_each_ms(stream, lambda: sb.spmv(Ds, x, y, stream=sp), 20)
            s_v = 2 if storage == "bf16" else 4
            nbytes = D.ndiags * N * s_v + 4 * D.ndiags + 3 * N * 4
            gbs = nbytes / (ms / 1e3) / 1e9
            out[f"dia_{storage}"] = {"ms": round(ms, 4), "GB_s": round(gbs, 1),
                                     "frac": round(gbs / peak, 3), "algorithmic_bytes": nbytes,
                                     "rel_err_vs_fp64": err}
    return out


def run_powerlaw_csr(stream, peak, opts=None, small=False):
    """CSR SpMV, FP64, on the power-law matrix of the format sweep (2M rows,
    ~41M nonzeros; 500k rows with small), autotuned or with fixed options
    "lanes,unroll,grid"."""
    import torch
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib, synth
    n = 500_000 if small else 2_000_000
    rp, col, val = synth.power_law(n, seed=2, dtype=np.float64)
    A = sb.csr_from_host(rp, col, val)
    x = sb.vec_from_host(synth.uniform_vec(n, 0))
    y = sb.create_vec(n, 0, np.float64)
    sp = stream.cuda_stream
    if opts:
        lanes, unroll, grid = (int(v) for v in opts.split(","))
        A.opts = _lib.CsrOpts(0, lanes, unroll, grid)
        tuned = {"kernel": 0, "lanes_per_row": lanes, "unroll": unroll, "grid": grid}
    else:
        tuned = sb.csr_autotune(A, x, stream=sp)
    for _ in range(3):
        with torch.cuda.stream(stream):
            sb.spmv(A, x, y, stream=sp)
    ms = _time_each_ms(stream, lambda: sb.spmv(A, x, y, stream=sp), 20)
    nbytes = algo_bytes("csr", n, col.size, 8)
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"N": n, "nnz": int(col.size), "ms": round(ms, 4), "GB_s": round(gbs, 1),
            "frac": round(gbs / peak, 3), "opts": tuned}


def run_batched(stream, peak, n_mats=512, seed=5):
    """Batched CSR SpMV: n_mats matrices with rows log-uniform in [1e3, 2e5],
    Poisson(12) off-diagonals plus the diagonal per row, values U[-1,1] stored
    FP32 and BF16 (FP32 accumulation), 1-8 right-hand sides each; one
    graph-replayed persistent launch for the whole batch against one
    sb_spmv_csr call per (matrix, right-hand side)."""
    import torch
    import scipy.sparse as sps
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib, synth_device as sd
    rng = np.random.default_rng(seed)
    Ns = np.floor(np.exp(rng.uniform(np.log(1e3), np.log(2e5), n_mats))).astype(np.int64)
    ks = rng.integers(1, 9, n_mats)
    sp = stream.cuda_stream
    mats = [sd.poisson_rows(int(N), 12.0, seed=seed * 1000 + i) for i, N in enumerate(Ns)]
    g = torch.Generator(device="cuda").manual_seed(seed)
    xs = [torch.rand(int(N) * int(k), generator=g, device="cuda") * 2 - 1 for N, k in zip(Ns, ks)]
    ys = [torch.zeros(int(N) * int(k), device="cuda") for N, k in zip(Ns, ks)]
    xcols = [[x.reshape(int(N), int(k))[:, j].contiguous() for j in range(int(k))]
             for x, N, k in zip(xs, Ns, ks)]
    ycols = [[torch.zeros(int(N), device="cuda") for _ in range(int(k))] for N, k in zip(Ns, ks)]
    nnz_tot = int(sum(A.nnz for A in mats))
    out = {"workload": f"{n_mats} CSR matrices, rows log-uniform in [1e3, 2e5] "
                       f"({int(Ns.sum())} rows), Poisson(12)+diagonal per row "
                       f"({nnz_tot} nonzeros), 1-8 right-hand sides, y <- y + A x",
           "matrices": n_mats, "rows": int(Ns.sum()), "nnz": nnz_tot,
           "rhs": int(ks.sum())}
    sample = list(range(0, n_mats, max(1, n_mats // 8)))
    for storage in ("f32", "bf16"):
        As = mats if storage == "f32" else [sb.csr_with_storage(A, "bf16") for A in mats]
        s_v = 2 if storage == "bf16" else 4
        ex = sb.BatchExecutor(storage, capacity=n_mats)
        jobs = [(A, sb.DeviceArray(x.numel(), np.float32, x.data_ptr()),
                 sb.DeviceArray(y.numel(), np.float32, y.data_ptr()), int(k))
                for A, x, y, k in zip(As, xs, ys, ks)]
        for y in ys:
            y.zero_()
        ex.run(jobs, stream=sp)
        torch.cuda.synchronize()
        err = 0.0
        for i in sample:
            A = As[i]
            v = A.val_array()
            if storage == "bf16":
                v = (v.astype(np.uint32) << 16).view(np.float32)
            M = sps.csr_matrix((v.astype(np.float64), A.col_array(), A.row_array()),
                               shape=(A.N, A.N))
            X = xs[i].double().cpu().numpy().reshape(A.N, int(ks[i]))
            Y = ys[i].double().cpu().numpy().reshape(A.N, int(ks[i]))
            T = M @ X
            err = max(err, float(np.max(np.abs(Y - T)) / max(np.max(np.abs(T)), 1e-300)))
        nbytes = sum(A.nnz * (s_v + 4) + 4 * (A.N + 1) + int(k) * A.N * 12
                     for A, k in zip(As, ks))
        # descriptors filled once; each timed launch uploads them and runs
        # the kernel (the graph), so no host-side Python is inside the events
        n_items = ex.prepare(jobs)
        for _ in range(3):
            ex.launch(n_items, stream=sp)
        ms = _time_each_ms(stream, lambda: ex.launch(n_items, stream=sp), 10)
        dt = _lib.SB_BF16 if storage == "bf16" else _lib.SB_F32

        def per_call():
            for A, xc, yc in zip(As, xcols, ycols):
                for xj, yj in zip(xc, yc):
                    _lib.call("sb_spmv_csr", dt, A.row_index.ptr, A.col_index.ptr,
                              A.val_index.ptr, xj.data_ptr(), yj.data_ptr(), A.N, A.nnz, 1, sp)
        per_call()
        ms_pc = _time_each_ms(stream, per_call, 3)
        gbs = nbytes / (ms / 1e3) / 1e9
        out[storage] = {"ms": round(ms, 4), "GB_s": round(gbs, 1), "frac": round(gbs / peak, 3),
                        "per_call_ms": round(ms_pc, 4),
                        "speedup_vs_per_call": round(ms_pc / ms, 2),
                        "algorithmic_bytes": nbytes, "launches": 1,
                        "per_call_launches": int(ks.sum()),
                        "max_rel_err_vs_fp64": err, "error_sample_matrices": len(sample)}
        ex.close()
    # the batch's gather floor: one sb_gather_dot over all matrices' col/val
    # (FP32 values) with the columns offset into one concatenated x -- the
    # streams and one x gather per nonzero, no rows, one right-hand side
    from sciwasm.sparse_b200.sparse import DeviceArray
    offs = np.concatenate([[0], np.cumsum(Ns)[:-1]])
    cat_col = torch.cat([A._torch[1] + int(o) for A, o in zip(mats, offs)])
    cat_val = torch.cat([A._torch[2] for A in mats])
    cat_x = torch.cat([xc[0] for xc in xcols])
    dot = DeviceArray.from_host(np.zeros(1))

    def floor_fn():
        _lib.call("sb_gather_dot", _lib.SB_F32, cat_col.data_ptr(), cat_val.data_ptr(),
                  cat_x.data_ptr(), nnz_tot, dot.ptr, sp)
    for _ in range(3):
        floor_fn()
    floor = _time_each_ms(stream, floor_fn, 10)
    out["gather_floor_ms"] = round(floor, 4)
    out["gather_floor"] = ("sb_gather_dot over the concatenated col/val (FP32) with one "
                           "x gather per nonzero from the concatenated x: no row structure, "
                           "no y, one right-hand side -- a lower bound on the batch's time")
    for storage in ("f32", "bf16"):
        out[storage]["of_gather_floor"] = round(floor / out[storage]["ms"], 3)
    del cat_col, cat_val, cat_x
    # the floor with each matrix's right-hand sides: per K, one
    # sb_gather_dot_rows over the matrices with K right-hand sides, which
    # gathers a K-value x row per nonzero with the batch kernel's loads
    rows_floor, by_k = 0.0, {}
    for K in sorted(set(int(k) for k in ks)):
        idx = [i for i in range(n_mats) if int(ks[i]) == K]
        offs_k = np.concatenate([[0], np.cumsum([int(Ns[i]) for i in idx])[:-1]])
        cc = torch.cat([mats[i]._torch[1] + int(o) for i, o in zip(idx, offs_k)])
        vv = torch.cat([mats[i]._torch[2] for i in idx])
        xx = torch.cat([xs[i] for i in idx])
        nnz_k = int(cc.numel())
        rows_k = int(sum(int(Ns[i]) for i in idx))

        def rows_fn():
            _lib.call("sb_gather_dot_rows", _lib.SB_F32, cc.data_ptr(), vv.data_ptr(),
                      xx.data_ptr(), rows_k, K, nnz_k, dot.ptr, sp)
        for _ in range(3):
            rows_fn()
        t = _time_each_ms(stream, rows_fn, 10)
        by_k[str(K)] = round(t, 4)
        rows_floor += t
        del cc, vv, xx
    out["gather_floor_rows_ms"] = round(rows_floor, 4)
    out["gather_floor_rows_by_k_ms"] = by_k
    out["gather_floor_rows"] = ("per number of right-hand sides K, sb_gather_dot_rows over those "
                                "matrices' col/val (FP32) gathering one K-value x row per nonzero "
                                "with the batch kernel's loads; no rows, no y; the sum over K")
    for storage in ("f32", "bf16"):
        out[storage]["of_gather_floor_rows"] = round(rows_floor / out[storage]["ms"], 3)
    return out


def run_rowshard(args, rank, world, local_rank):
    """Row-sharded SpMV (strong scaling): the format sweep's CSR matrices
    (4M-row banded, 2M-row power-law, FP64) split into static_nnz row blocks,
    one per rank, the whole x on every rank; a step is, per matrix, the
    rank's block SpMV into its part of y and one in-place all-gather of y
    (NCCL), so that every rank ends the step with the whole y (the x of an
    iterative method's next step).  One rank runs the unsplit SpMV with no
    collective.  Returns rank 0's result (None elsewhere)."""
    import torch
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib
    from sciwasm.sparse_b200.dist import PeerY, RowShardedCSR, ShardedY, max_over_ranks
    peer = args.exchange == "peer"
    sb.load_library()
    torch.cuda.set_device(local_rank)
    _lib.call("sb_set_device", local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    jobs = make_workload("format_sweep_fp64", args.small)
    parts = []
    for j in jobs:
        sh = RowShardedCSR(j["rp"], j["col"], j["val"], rank, world)
        x = torch.from_numpy(j["x"]).to(dev)
        y = PeerY(j["N"], torch.float64, dev) if peer else \
            ShardedY(sh.starts, sh.ends, rank, torch.float64, dev)
        xv = _vec(x)
        yv = None if peer else _vec(y.local())
        tuned = sb.csr_autotune(sh.A, xv, stream=sptr) if sh.A is not None else None
        parts.append(dict(job=j, sh=sh, x=x, y=y, xv=xv, yv=yv, tuned=tuned,
                          bytes=algo_bytes("csr", j["N"], int(j["rp"][-1]), 8)))

    def exchange_step(p):
        """This rank's block SpMV and the exchange that completes y."""
        if peer:
            # the rows go straight into every rank's buffer, then a barrier
            p["sh"].spmv_allgather(p["x"].data_ptr(), p["y"].rows_ptr(p["sh"].r0),
                                   p["y"].ptrs_dev.data_ptr(), len(p["y"].ptrs), stream=sptr)
            return
        if p["sh"].A is not None:
            sb.spmv(p["sh"].A, p["xv"], p["yv"], stream=sptr)

    def exchange_finish(p):
        if peer:
            p["y"].barrier()
        else:
            p["y"].allgather()
    torch.cuda.synchronize()
    # correctness: one step from y = 0, the gathered y against an FP64 check
    errs = {}
    with torch.cuda.stream(stream):
        for p in parts:
            p["y"].buf.zero_()
            if peer:
                p["y"].barrier()  # every buffer zeroed before any rank stores
            exchange_step(p)
            exchange_finish(p)
    torch.cuda.synchronize()
    for p in parts:
        j = p["job"]
        t = truth_f64(j["rp"], j["col"], j["val"], j["x"])
        got = (p["y"].buf if peer else p["y"].full()).cpu().numpy()
        errs[j["label"]] = float(np.max(np.abs(got - t)) / max(np.max(np.abs(t)), 1e-300))
    if max(errs.values()) > 1e-5:
        raise SystemExit(f"row-shard correctness gate failed: {errs}")

    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in parts] for _ in range(args.steps)]

    def step(k=None):
        for i, p in enumerate(parts):
            if k is not None:
                ev[k][i][0].record(stream)
            exchange_step(p)
            if k is not None:
                ev[k][i][1].record(stream)
            exchange_finish(p)
            if k is not None:
                ev[k][i][2].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        t0.record(stream)
        for k in range(args.steps):
            step(k)
        t1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = t0.elapsed_time(t1) / args.steps
    ms_max = max_over_ranks(ms, device=dev)
    total = sum(p["bytes"] for p in parts)
    per = {}
    for i, p in enumerate(parts):
        sp = float(np.mean([ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(args.steps)]))
        ag = float(np.mean([ev[k][i][1].elapsed_time(ev[k][i][2]) for k in range(args.steps)]))
        per[p["job"]["label"]] = {
            "rows_local": p["sh"].rows, "nnz_local": int(p["sh"].A.nnz) if p["sh"].A else 0,
            "spmv_ms_max": round(max_over_ranks(sp, device=dev), 4),
            "exchange_ms_max": round(max_over_ranks(ag, device=dev), 4),
            "exchange_bytes_in": (p["sh"].N - p["sh"].rows) * 8 if peer else p["y"].gather_bytes(),
            "csr_opts": p["tuned"], "max_rel_err": errs[p["job"]["label"]]}
    if rank != 0:
        return None
    return {"world": world, "scaling": "strong",
            "workload": "format_sweep_fp64 CSR matrices (4M-row banded, 2M-row power-law, FP64) "
                        "in static_nnz row blocks, x on every rank, y all-gathered each step",
            "exchange": ("peer: each rank's SpMV stores its rows into every rank's y buffer "
                         "(sb_spmv_csr_allgather; symmetric memory when world > 1), then a "
                         "barrier" if peer else "allgather: NCCL in-place all-gather of y"),
            "value_GB_s": round(total / (ms_max / 1e3) / 1e9, 1), "unit": UNIT,
            "ms_per_step": round(ms_max, 4), "algorithmic_bytes": total,
            "steps": args.steps, "warmup": args.warmup, "per_matrix": per,
            "timing": "CUDA events on the SpMV stream around the steps, max over ranks; "
                      "the exchange is stream-ordered after the SpMV (NCCL's stream is waited "
                      "for; the peer barrier runs on the SpMV stream)"}


def _spts_cpu_baseline(rp, col, val, b, plan_levels, gpu_y, reps=3):
    """CPU-baseline leg of one SpTS case: the oracle's serial analysis and row
    kernel, and its pthread ports of the reference's parallel level-set and
    sync-free solves on 5 threads (the published setting) and on every host
    core, best of `reps` runs each.  The GPU's levels (level, level_ptr,
    permutation, order) and its three solves are compared with the oracle's
    bit for bit."""
    from oracle import binding as orc
    cores = os.cpu_count() or 1
    N = rp.size - 1

    def best(fn):
        t = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            t.append((time.perf_counter() - t0) * 1e3)
        return round(min(t), 3)

    ls = {}

    def analysis():
        ls.update(orc.level_sets(rp, col, val))
    out = {"analysis_ms_serial": best(analysis)}
    out["row_kernel_ms_serial"] = best(lambda: orc.spts_csr(rp, col, val, b))
    bp = np.ascontiguousarray(b[ls["permutation"]])
    yl = np.zeros(N, val.dtype)
    flag = np.zeros(N, np.int32)
    ysf = np.zeros(N, val.dtype)
    for nt in sorted({5, cores}):
        out[f"level_ms_{nt}t"] = best(lambda: orc.par_spts_level(
            nt, ls["level_ptr"], ls["row_ptr"], ls["col"], ls["val"], bp, yl))
        out[f"syncfree_ms_{nt}t"] = best(lambda: orc.par_spts_syncfree(
            nt, rp, col, val, b, ysf, flag))
    out.update(cores=cores, kind="port",
               sample="whole factor per run, best of 3: serial analysis and row kernel; "
                      "pthread level-set (barrier per level) and sync-free (ready flags) "
                      "solves on 5 threads and on all cores (C restatement of the "
                      "reference's worker kernels, not V8/wasm)")

    def same(a, c):
        return np.array_equal(np.ascontiguousarray(a).view(np.uint8),
                              np.ascontiguousarray(c).view(np.uint8))
    lv, lp, perm, order = plan_levels
    ok_levels = same(lv, ls["level"]) and same(lp, ls["level_ptr"]) and \
        same(perm, ls["permutation"]) and same(order, ls["order"])
    row_kernel = orc.spts_csr(rp, col, val, b)
    syncfree = orc.spts_syncfree(rp, col, val, b)
    ok_solves = {an: same(y, syncfree if an == "syncfree" else row_kernel)
                 for an, y in gpu_y.items()}
    ok_solves["syncfree_cpu_threads"] = same(ysf, syncfree)
    return out, {"levels": ok_levels, **ok_solves}


def run_spts_section(stream, cpu=True):
    """SpTS: lower triangle of the 3-D 7-point Laplacian on a 64^3 grid and a
    random lower-triangular matrix (1M rows, 7 off-diagonals per row within
    5,000 of the diagonal, diagonal U[2,4]), FP64 and FP32, b ~ U[-1,1];
    analysis (device time from events around its kernels, and the host time
    of the whole call) and the three solves, errors against an FP64 host
    solve (scipy); with cpu, the CPU baselines and bit-exact checks."""
    import torch
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    import sciwasm.sparse_b200 as sb
    from sciwasm.sparse_b200 import _lib, synth
    sp = stream.cuda_stream
    npdt = {"f64": np.float64, "f32": np.float32}
    cases = [("laplacian3d_64", lambda dt: synth.laplacian_3d_lower(64, dtype=npdt[dt])),
             ("random_lower_1M", lambda dt: synth.random_lower(1_000_000, 7, 5000, seed=3,
                                                                dtype=npdt[dt]))]
    algos = {"level": _lib.SB_SPTS_LEVEL, "syncfree": _lib.SB_SPTS_SYNCFREE,
             "hybrid": _lib.SB_SPTS_HYBRID}
    out = {}
    for name, gen in cases:
        for dt in ("f64", "f32"):
            rp, col, val = gen(dt)
            L = sb.csr_from_host(rp, col, val)
            torch.cuda.synchronize()
            # five analyses: device time of the analysis kernels (events on
            # the stream) and host time of the whole call; the first build
            # also pays one-time module-load costs
            dev_ms, host_ms = [], []
            plan = None
            for rep in range(5):
                if plan is not None:
                    plan.close()
                t0 = time.perf_counter()
                plan = sb.SptsPlan(L, stream=sp)
                torch.cuda.synchronize()
                host_ms.append((time.perf_counter() - t0) * 1e3)
                dev_ms.append(plan.analysis_ms)
            b_host = synth.uniform_vec(L.N, 4, dtype=npdt[dt])
            bt = torch.from_numpy(b_host).cuda()
            yt = torch.zeros(L.N, device="cuda", dtype=bt.dtype)
            M = sps.csr_matrix((val.astype(np.float64), col, rp), shape=(L.N, L.N))
            truth = spl.spsolve_triangular(M, b_host.astype(np.float64), lower=True)
            s_v = 8 if dt == "f64" else 4
            nbytes = L.nnz * (s_v + 4) + 4 * (L.N + 1) + 2 * L.N * s_v
            row = {"N": L.N, "nnz": L.nnz, "levels": plan.nlevels,
                   "analysis_device_ms": round(float(np.median(dev_ms)), 3),
                   "analysis_device_ms_all": [round(v, 3) for v in dev_ms],
                   "analysis_host_ms": round(float(np.median(host_ms)), 3),
                   "analysis_host_ms_first": round(host_ms[0], 2),
                   "algorithmic_bytes": nbytes}
            runs = [(an, code, _lib.SB_SPTS_ACC_NATIVE) for an, code in algos.items()]
            if dt == "f32":
                runs.append(("hybrid_acc_f64", _lib.SB_SPTS_HYBRID, _lib.SB_SPTS_ACC_F64))
            gpu_y = {}
            for an, code, pol in runs:
                def solve():
                    _lib.call("sb_spts_solve", plan.ptr, code, pol, bt.data_ptr(), yt.data_ptr(),
                              sp)
                yt.zero_()
                with torch.cuda.stream(stream):
                    solve()
                torch.cuda.synchronize()
                y = yt.cpu().numpy()
                if an in algos:
                    gpu_y[an] = y.copy()
                err = float(np.max(np.abs(y.astype(np.float64) - truth)) /
                            max(np.max(np.abs(truth)), 1e-300))
                with torch.cuda.stream(stream):
                    solve()
                ms = _time_each_ms(stream, solve, 5)
                row[an] = {"ms": round(ms, 4), "us_per_level": round(ms * 1e3 / plan.nlevels, 3),
                           "rows_per_s": round(L.N / (ms / 1e3), 1), "rel_err_vs_fp64": err}
            code = __import__("ctypes").c_int(0)
            _lib.call("sb_device_status", __import__("ctypes").byref(code))
            row["device_status"] = code.value
            if cpu:
                levels = tuple(a.to_host() for a in plan.levels())
                row["cpu_baseline"], row["bit_exact"] = _spts_cpu_baseline(
                    rp, col, val, b_host, levels, gpu_y)
            out[f"{name}/{dt}"] = row
            plan.close()
    return out


def run_serving(args):
    """Batched (continuous batching) and plain per-call serving of the same
    request stream; returns the statistics of both and the sampled errors."""
    from sciwasm.sparse_b200 import serve
    from sciwasm.sparse_b200.sparse import PinnedBuffer
    t0 = time.perf_counter()
    pool, mv, ts = build_serving_pool(args.serve_pool, 1000, args.serve_max_rows)
    build_s = time.perf_counter() - t0
    in_ring = PinnedBuffer(1 << 30)
    out_ring = PinnedBuffer(1 << 30)
    xs = in_ring.view(0, in_ring.nbytes // 4, np.float32)
    np.random.default_rng(5).random(out=xs, dtype=np.float32)
    xs *= 2
    xs -= 1
    reqs = serving_requests(pool, mv, ts, args.serve_rate, args.serve_seconds, in_ring,
                            out_ring)
    srv = serve.Server(pool, max_batch=args.serve_batch, slots=args.serve_slots,
                       spts_slots=args.serve_spts_slots, spts_batch=args.serve_spts_batch,
                       spts_grid=args.serve_spts_grid)
    # warm-up: executors, graphs and first-touch costs
    srv.serve([serve.Request(r.rid, 0.0, r.matrix, r.op, r.storage, r.x, r.y)
               for r in reqs[:200]], "batched")
    srv.serve([serve.Request(r.rid, 0.0, r.matrix, r.op, r.storage, r.x, r.y)
               for r in reqs[:50]], "plain")
    batched = srv.serve(reqs, "batched")
    for r in reqs:
        r.t_done = -1.0
    plain = srv.serve(reqs, "plain")
    # capacity: the same kind of requests all present at t = 0 (a backlog),
    # so that the rate is the server's, not the arrival process's
    burst = [serve.Request(r.rid, 0.0, r.matrix, r.op, r.storage, r.x, r.y) for r in reqs]
    cap_b = srv.serve(burst, "batched")
    cap_p = srv.serve(burst[:max(1, len(burst) // 10)], "plain")
    capacity = {"batched_req_per_s": round(cap_b["req_per_s"], 1),
                "plain_req_per_s": round(cap_p["req_per_s"], 1),
                "batched_requests": cap_b["requests"], "plain_requests": cap_p["requests"]}
    errs = serving_errors(pool, srv, mv, ts)
    rows = np.array([pool.mats[r.matrix].N for r in reqs])
    bytes_io = int(np.sum(rows) * 8)
    out = {
        "workload": (f"{args.serve_pool} resident matrices, rows log-uniform in "
                     f"[1000, {args.serve_max_rows}] (2/3 banded / power-law / 2-D Laplacian "
                     "with f32 and bf16 values, 1/3 triangular factors: 3-D Laplacian lower / "
                     "random lower, f32 with f64 accumulation where growth > 1); "
                     f"Poisson arrivals at {args.serve_rate:g} req/s for "
                     f"{args.serve_seconds:g} s, 70% SpMV (f32 or bf16 by request), 30% SpTS; "
                     "vectors in pinned host memory, copies inside the measured latency"),
        "requests": len(reqs), "mean_rows": float(rows.mean()),
        "h2d_plus_d2h_bytes": bytes_io,
        "pool_bytes": pool.admission.used, "pool_build_s": round(build_s, 2),
        "flagged_f64_factors": sum(1 for n in ts if pool.mats[n].policy["f32"] == "f64"),
        "batched": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in batched.items()},
        "plain": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in plain.items()},
        "capacity_backlog": capacity,
        "max_rel_err_vs_fp64": errs,
        "slots": {"spmv": args.serve_slots, "spts": args.serve_spts_slots},
        "max_batch": {"spmv": args.serve_batch, "spts": args.serve_spts_batch},
        "spts_blocks_per_sm": args.serve_spts_grid,
        "timing": "host wall clock from each request's arrival to the host seeing its result",
    }
    pool.close()
    in_ring.free()
    out_ring.free()
    return out


def run_serving_sweep(args):
    """Serving at several arrival rates on one resident pool: for each rate
    the same Poisson trace (args.sweep_seconds long) is served batched and
    per call (the per-call path on at most its first args.plain_seconds,
    since above its capacity its queue only grows); then one long batched
    trace (args.serve_seconds) at args.serve_rate.  Per-op p50/p99 for both."""
    from sciwasm.sparse_b200 import serve
    from sciwasm.sparse_b200.sparse import PinnedBuffer
    t0 = time.perf_counter()
    pool, mv, ts = build_serving_pool(args.serve_pool, 1000, args.serve_max_rows)
    build_s = time.perf_counter() - t0
    in_ring = PinnedBuffer(1 << 30)
    out_ring = PinnedBuffer(1 << 30)
    xs = in_ring.view(0, in_ring.nbytes // 4, np.float32)
    np.random.default_rng(5).random(out=xs, dtype=np.float32)
    xs *= 2
    xs -= 1
    srv = serve.Server(pool, max_batch=args.serve_batch, slots=args.serve_slots,
                       spts_slots=args.serve_spts_slots, spts_batch=args.serve_spts_batch,
                       spts_grid=args.serve_spts_grid)
    warm = serving_requests(pool, mv, ts, 2000.0, 0.2, in_ring, out_ring, seed=99)
    for mode in ("batched", "plain"):
        srv.serve([serve.Request(r.rid, 0.0, r.matrix, r.op, r.storage, r.x, r.y)
                   for r in warm], mode)
    keys = ("requests", "req_per_s", "p50_ms", "p99_ms", "spmv_p50_ms", "spmv_p99_ms",
            "spts_p50_ms", "spts_p99_ms", "mean_batch", "span_s")

    def pick(st):
        return {k: (round(st[k], 3) if isinstance(st[k], float) else st[k])
                for k in keys if k in st}
    sweep = {}
    for rate in [float(v) for v in args.serve_rates.split(",")]:
        reqs = serving_requests(pool, mv, ts, rate, args.sweep_seconds, in_ring, out_ring,
                                seed=int(rate) % 1000 + 17)
        b = srv.serve(reqs, "batched")
        n_plain = max(1, min(len(reqs), int(rate * args.plain_seconds)))
        prefix = reqs[:n_plain]
        for r in prefix:
            r.t_done = -1.0
        p = srv.serve(prefix, "plain")
        sweep[f"{int(rate)}"] = {"batched": pick(b), "plain": pick(p),
                                 "plain_prefix_s": round(prefix[-1].t_arrival, 3)}
        print(json.dumps({"rate": rate, **sweep[f"{int(rate)}"]}), file=sys.stderr, flush=True)
    reqs = serving_requests(pool, mv, ts, args.serve_rate, args.serve_seconds, in_ring, out_ring)
    long_b = srv.serve(reqs, "batched")
    deep = max(ts, key=lambda n: pool.mats[n].plans["f32"].nlevels)
    deepest = pool.mats[deep].plans["f32"].nlevels
    single = deepest_single_solve(pool, srv, deep, in_ring, out_ring)
    out = {"pool": f"{args.serve_pool} matrices, rows log-uniform in [1000, "
                   f"{args.serve_max_rows}], 70% SpMV / 30% SpTS requests",
           "pool_build_s": round(build_s, 2), "deepest_factor_levels": deepest,
           "deepest_single_solve": single,
           "formats": dict(collections_counter(pool.mats[n].format for n in mv)),
           "sweep_seconds": args.sweep_seconds, "plain_seconds": args.plain_seconds,
           "server": {"spmv_slots": args.serve_slots, "spmv_batch": args.serve_batch,
                      "spts_slots": args.serve_spts_slots, "spts_batch": args.serve_spts_batch,
                      "spts_blocks_per_sm": args.serve_spts_grid},
           "sweep": sweep,
           "long_trace": {"rate": args.serve_rate, "seconds": args.serve_seconds,
                          "batched": pick(long_b)}}
    pool.close()
    in_ring.free()
    out_ring.free()
    return out


def deepest_single_solve(pool, srv, name, in_ring, out_ring, reps=10):
    """The pool's deepest factor solved alone: the device time of one hybrid
    sb_spts_solve (CUDA events, mean of reps) and the per-call path's latency
    for one request of it (copies in and out included, median of reps)."""
    import torch
    from sciwasm.sparse_b200 import _lib, serve
    m = pool.get(name)
    stream = torch.cuda.Stream()
    x = torch.rand(m.N, device="cuda") * 2 - 1
    y = torch.empty_like(x)
    pol = _lib.SB_SPTS_ACC_F64 if m.policy["f32"] == "f64" else _lib.SB_SPTS_ACC_NATIVE

    def fn():
        _lib.call("sb_spts_solve", m.plans["f32"].ptr, _lib.SB_SPTS_HYBRID, pol, x.data_ptr(),
                  y.data_ptr(), stream.cuda_stream)
    for _ in range(3):
        fn()
    dev_ms = _time_each_ms(stream, fn, reps)
    lat = []
    for k in range(reps):
        r = serve.Request(k, 0.0, name, "spts", "f32", in_ring.view(0, m.N, np.float32),
                          out_ring.view(0, m.N, np.float32))
        lat.append(srv.serve([r], "plain")["p50_ms"])
    return {"matrix": name, "rows": m.N, "levels": pool.mats[name].plans["f32"].nlevels,
            "accumulation": m.policy["f32"], "device_ms": round(dev_ms, 3),
            "plain_request_ms": round(float(np.median(lat)), 3)}


def collections_counter(it):
    import collections
    return collections.Counter(it)


def _pinned(nbytes):
    import ctypes
    from sciwasm.sparse_b200 import _lib
    p = ctypes.c_void_p()
    _lib.call("sb_host_alloc", ctypes.byref(p), nbytes)
    return p.value


def _host_view(ptr, n, dtype):
    import ctypes
    raw = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)),
                                shape=(n * np.dtype(dtype).itemsize,))
    return raw.view(dtype)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="format_sweep_fp64",
                    help="format_sweep_fp64 (the bench line), laplacian_fp32, rowshard_fp64 "
                         "(row-sharded CSR with an all-gather of y, strong scaling), or one "
                         "section alone: " + ", ".join(SECTIONS))
    ap.add_argument("--csr-fixed", default=None,
                    help="pinned CSR options of the default workload instead of the autotuner, "
                         "e.g. 'banded:0,2,8,0;powerlaw:0,8,4,1' (kernel,lanes,unroll,grid)")
    ap.add_argument("--csr-opts", default=None,
                    help="powerlaw_csr: fixed CSR options lanes,unroll,grid (else autotuned)")
    ap.add_argument("--batch-mats", type=int, default=512,
                    help="matrices of the batched section when run alone")
    ap.add_argument("--small", action="store_true",
                    help="quarter-size matrices (profiling captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-sections", action="store_true",
                    help="skip the 4096^2 Laplacian, batched and SpTS sections")
    ap.add_argument("--exchange", default="allgather", choices=["allgather", "peer"],
                    help="rowshard_fp64: how y is completed on every rank")
    ap.add_argument("--e2e-streams", type=int, default=3,
                    help="streams the e2e calls rotate over")
    ap.add_argument("--serve-pool", type=int, default=2000)
    ap.add_argument("--serve-max-rows", type=int, default=2_000_000)
    ap.add_argument("--serve-rate", type=float, default=20_000.0)
    ap.add_argument("--serve-seconds", type=float, default=5.0)
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--serve-batch", type=int, default=64)
    ap.add_argument("--serve-spts-slots", type=int, default=3)
    ap.add_argument("--serve-spts-batch", type=int, default=32)
    ap.add_argument("--serve-spts-grid", type=int, default=1,
                    help="SpTS launches: persistent blocks per SM (0 = one warp per chunk)")
    ap.add_argument("--serve-rates", default="1000,2000,3000,10000,20000",
                    help="serving_sweep: arrival rates (req/s)")
    ap.add_argument("--sweep-seconds", type=float, default=3.0,
                    help="serving_sweep: trace length per rate")
    ap.add_argument("--plain-seconds", type=float, default=2.0,
                    help="serving_sweep: trace prefix served by the per-call path")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    config = {"workload": args.workload + ("_small" if args.small else ""),
              "dtype": "f64" if "fp64" in args.workload else "f32",
              "l2": "inputs larger than L2 (126 MB); no flush between steps",
              "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
    if args.workload == "laplacian_fp32":
        config["l2"] = "3.7 MB working set stays L2-resident (reported, not a roofline claim)"
    dtype = config["dtype"]

    if args.workload == "rowshard_fp64":
        if args.impl == "reference":
            if rank == 0:
                jobs = make_workload("format_sweep_fp64", args.small)
                for j in jobs:
                    j["formats"] = ["csr"]
                run_reference(args, jobs, {**config, "dtype": "f64",
                                           "parallelism": "host threads"})
            return
        import datetime
        import torch
        if world > 1:
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local_rank))
        try:
            out = run_rowshard(args, rank, world, local_rank)
            if rank == 0:
                print(json.dumps({"workload": args.workload, "result": out}), flush=True)
        finally:
            if world > 1:
                import torch.distributed as dist
                dist.destroy_process_group()
        return

    if args.workload in SECTIONS:
        # one configuration alone, one GPU (profiling and focused runs)
        if args.impl == "reference" or rank != 0:
            return
        import torch
        import sciwasm.sparse_b200 as sb
        sb.load_library()
        torch.cuda.set_device(local_rank)
        stream = torch.cuda.Stream()
        peak, _ = measured_peak()
        if args.workload == "batched":
            out = run_batched(stream, peak, n_mats=args.batch_mats)
        elif args.workload == "laplacian4096_fp32":
            out = run_laplacian_large(stream, peak)
        elif args.workload == "spts":
            out = run_spts_section(stream)
        elif args.workload == "powerlaw_csr":
            out = run_powerlaw_csr(stream, peak, args.csr_opts, args.small)
        elif args.workload == "serving_sweep":
            out = run_serving_sweep(args)
        elif args.workload == "gather_ceiling":
            out = run_gather_ceiling(stream, peak, args.small)
        elif args.workload == "conversions":
            out = run_conversions(stream, args.small)
        else:
            out = run_serving(args)
        print(json.dumps({"workload": args.workload, "result": out}), flush=True)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        jobs = make_workload(args.workload, args.small)
        run_reference(args, jobs, {**config, "dtype": dtype})
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        jobs = make_workload(args.workload, args.small)
        run_ours(args, jobs, config, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
