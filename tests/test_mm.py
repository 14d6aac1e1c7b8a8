"""Matrix Market input on the CPU: the oracle against the hand-derived known
answers, and the library's host parser (header and entry lines) against the
oracle's reading of the same text, including generated files."""
import ctypes as C
import json
import os
import zlib

import numpy as np
import pytest

from sciwasm.sparse_b200 import _lib

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KAT = json.load(open(os.path.join(GOLD, "mm_kat.json")))
FILES = [k for k in KAT if not k.startswith("_")]


def _text(name):
    return open(os.path.join(GOLD, "mm", name), "rb").read()


def _parse(sb, text, nthreads=0):
    t = np.frombuffer(text, np.uint8)
    h = _lib.MMHeader()
    _lib.call("sb_mm_read_header", t.ctypes.data, t.size, C.byref(h))
    n = int(h.nentries)
    row, col, val = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
    _lib.call("sb_mm_read_entries", t.ctypes.data, t.size, C.byref(h), row.ctypes.data,
              col.ctypes.data, val.ctypes.data, nthreads)
    return h, row, col, val


@pytest.mark.parametrize("name", FILES)
def test_oracle_kat(oracle, name):
    k = KAT[name]
    info = oracle.mm_read(_text(name))
    for key in ("nrows", "ncols", "nentries", "field", "symmetric", "nnz"):
        assert info[key] == k[key], key
    for lower, key in ((False, "coo"), (True, "lcoo")):
        r, c, v = oracle.mm_coo(info, np.float32, lower=lower)
        assert r.tolist() == k[key]["row"] and c.tolist() == k[key]["col"]
        assert np.array_equal(v, np.array(k[key]["val"], np.float32))


@pytest.mark.parametrize("name", FILES)
def test_host_parser_matches_oracle(sb, oracle, name):
    text = _text(name)
    h, row, col, val = _parse(sb, text)
    info = oracle.mm_read(text)
    assert (h.nrows, h.ncols, h.nentries, h.field, h.symmetric) == \
        (info["nrows"], info["ncols"], info["nentries"], info["field"], info["symmetric"])
    assert np.array_equal(row, info["row"]) and np.array_equal(col, info["col"])
    if h.field != _lib.SB_MM_PATTERN:
        assert np.array_equal(val, info["val"])


def make_mm(rng, n, m, nent, field="real", sym="general", comments=2):
    """A Matrix Market text with distinct coordinates (single spaces, as the
    reference's split(" ") expects)."""
    cells = rng.choice(n * m, size=nent, replace=False)
    r, c = cells // m + 1, cells % m + 1
    if sym == "symmetric":  # keep the lower triangle, as symmetric files do
        keep = r >= c
        r, c = r[keep], c[keep]
    lines = [f"%%MatrixMarket matrix coordinate {field} {sym}"]
    lines += ["% generated"] * comments
    lines.append(f"{n} {m} {r.size}")
    for i in range(r.size):
        if field == "pattern":
            lines.append(f"{r[i]} {c[i]}")
        elif field == "integer":
            lines.append(f"{r[i]} {c[i]} {int(rng.integers(-3, 4))}")
        else:
            v = 0.0 if rng.random() < 0.1 else float(rng.standard_normal())
            lines.append(f"{r[i]} {c[i]} {v!r}")
    return ("\n".join(lines) + "\n").encode()


@pytest.mark.parametrize("field,sym", [("real", "general"), ("real", "symmetric"),
                                       ("integer", "general"), ("pattern", "symmetric"),
                                       ("pattern", "general")])
@pytest.mark.parametrize("nthreads", [1, 3, 16])
def test_generated_files(sb, oracle, field, sym, nthreads):
    rng = np.random.default_rng(zlib.crc32(f"{field}/{sym}".encode()))
    text = make_mm(rng, 300, 300, 5000, field, sym)
    h, row, col, val = _parse(sb, text, nthreads)
    info = oracle.mm_read(text)
    assert h.nentries == info["nentries"]
    assert np.array_equal(row, info["row"]) and np.array_equal(col, info["col"])
    if field != "pattern":
        assert np.array_equal(val, info["val"])


def test_whitespace_and_line_endings(sb):
    """Tabs, repeated spaces, CRLF and blank lines parse like the plain file."""
    plain = _text("sym_real.mtx")
    messy = plain.replace(b" ", b" \t ").replace(b"\n", b"\r\n").replace(b"2 1 -1", b"\r\n2 1 -1")
    a = _parse(sb, plain)
    b = _parse(sb, messy)
    assert (a[0].nrows, a[0].nentries, a[0].field, a[0].symmetric) == \
        (b[0].nrows, b[0].nentries, b[0].field, b[0].symmetric)
    for x, y in zip(a[1:], b[1:]):
        assert np.array_equal(x, y)


def test_parser_refusals(sb):
    def bad(text, fn="header"):
        with pytest.raises(_lib.SparseError):
            _parse(sb, text)
    bad(b"not a matrix market file\n1 1 1\n1 1 1\n")
    bad(b"%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    bad(b"%%MatrixMarket matrix coordinate real general\n10 10 200000000\n")  # > 2^27
    bad(b"%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n")  # too few lines
    bad(b"%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n")  # row out of range
    bad(b"%%MatrixMarket matrix coordinate real general\n3 3 1\n1 x 1.0\n")  # malformed
