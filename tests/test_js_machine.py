"""The JavaScript interpreter that made tests/golden/js_vectors.npz, checked
on small functions whose results follow from the language's own rules
(hoisting, implicit globals, typed-array conversions, postfix/prefix
updates, parseInt, floating-point division, statements ended by a line
break)."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

from js_machine import UNDEF, JSMachine  # noqa: E402

SRC = r"""
function hoist(n) {
  for (i = 0; i < n; i++) { s = (s || 0) + i; }
  var i, s
  return [i, s];
}
function globals_made() { leaked = 7; return leaked * 2 }
function typed() {
  var a = new Int32Array(3);
  a[0] = 2147483648;  a[1] = -1.9;  a[2] = 5;
  var f = new Float32Array(2);
  f[0] = 0.1;  f[1] = 16777217;
  var out = a[5];
  return [a[0], a[1], a[2]++, ++a[2], f[0], f[1], out];
}
function counts(x) {
  var ind = new Int32Array(4), n = 0;
  for (var j = 0; j < x.length; j++)
    if (!ind[x[j]]++) n++;
  return [n, ind[1]];
}
function parse(a) { return [parseInt(a / 2), -(parseInt((2*a-1)/2)), 7 / 2, 7 % 3, 1 / 0] }
function strings(line) {
  var f = line.split(" ");
  return [f[0][0] == "%", f[1] == "7", Number(f[1]) == 7, f.length, line[99]];
}
function views(addr) {
  var v = new Int32Array(memory.buffer, addr, 2);
  v[1] = v[0] + 40;
  return v.length;
}
"""


def run(name, *args):
    m = JSMachine(mem_bytes=1 << 16)
    m.load(SRC, ["hoist", "globals_made", "typed", "counts", "parse", "views"])
    return m, m.call(name, *args)


def test_hoisting_and_implicit_globals():
    _, r = run("hoist", 5.0)
    assert r.items == [5.0, 10.0]
    m, r = run("globals_made")
    assert r == 14.0 and m.globals["leaked"] == 7.0


def test_typed_array_conversions():
    _, r = run("typed")
    a0, a1, post, pre, f0, f1, out = r.items
    assert (a0, a1, post, pre) == (-2147483648.0, -1.0, 5.0, 7.0)
    assert f0 == float(np.float32(0.1)) and f1 == 16777216.0
    assert out is UNDEF


def test_postfix_in_condition():
    m = JSMachine(mem_bytes=1 << 16)
    m.load(SRC, ["counts"])
    arr = m.builtins["Int32Array"].construct(5.0)
    arr.a[:] = [1, 2, 1, 3, 1]
    assert m.call("counts", arr).items == [3.0, 3.0]


def test_numbers():
    _, r = run("parse", 7.0)
    assert r.items[:4] == [3.0, -6.0, 3.5, 1.0] and r.items[4] == math.inf


def test_strings():
    m = JSMachine(mem_bytes=1 << 16)
    m.load(SRC, ["strings"])
    r = m.call("strings", "%a 7 x").items
    assert r[:4] == [True, True, True, 3.0] and r[4] is UNDEF


def test_memory_views():
    m = JSMachine(mem_bytes=1 << 16)
    m.load(SRC, ["views"])
    m.mem[128:132] = np.int32(2).tobytes()
    assert m.call("views", 128.0) == 2.0
    assert np.frombuffer(bytes(m.mem[132:136]), np.int32)[0] == 42
