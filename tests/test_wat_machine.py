"""The WebAssembly-text interpreter that made tests/golden/wat_vectors.npz,
checked on small modules whose results follow from the WebAssembly
specification alone (control flow, integer wrap-around and signedness, f32
rounding, SIMD lanes, multi-value returns, the instruction limit)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

from wat_machine import WatModule  # noqa: E402

MOD = r"""
(module
  (import "js" "mem" (memory 1))
  (import "console" "log" (func $log (param i32)))
  ;; sum of 0..n-1 with a block/loop/br_if exit, flat form
  (func (export "sum") (param $n i32) (result i32)
    (local $i i32) (local $s i32)
    block $done
      loop $top
        local.get $i
        local.get $n
        i32.ge_s
        br_if $done
        (local.set $s (i32.add (local.get $s) (local.get $i)))
        (local.set $i (i32.add (local.get $i) (i32.const 1)))
        br $top
      end
    end
    local.get $s)
  ;; folded if/then/else with a result
  (func (export "absdiff") (param $a i32) (param $b i32) (result i32)
    (if (result i32) (i32.gt_s (local.get $a) (local.get $b))
      (then (i32.sub (local.get $a) (local.get $b)))
      (else (i32.sub (local.get $b) (local.get $a)))))
  ;; a branch out of two nested blocks keeps the value
  (func (export "nested") (result i32)
    (block $outer (result i32)
      (block $inner
        (br $outer (i32.const 7)))
      (i32.const 3)))
  (func (export "wrap") (param $a i32) (result i32)
    (i32.add (local.get $a) (i32.const 1)))
  (func (export "shr") (param $a i32) (result i32 i32)
    (i32.shr_s (local.get $a) (i32.const 1))
    (i32.shr_u (local.get $a) (i32.const 1)))
  (func (export "f32add") (param $a f32) (param $b f32) (result f32)
    (f32.add (local.get $a) (local.get $b)))
  (func (export "lanes") (param $p i32) (result f32)
    (f32x4.extract_lane 3
      (f32x4.mul (v128.load (local.get $p)) (f32x4.splat (f32.const 2)))))
  (func (export "store_load") (param $p i32) (param $v f64) (result f64)
    (f64.store (local.get $p) (local.get $v))
    (call $log (i32.const 1))
    (f64.load (local.get $p)))
  (func (export "spin") (param $p i32)
    (loop $w (br_if $w (i32.eqz (i32.load (local.get $p))))))
  (func (export "two") (result i32 i32)
    (i32.const 4) (i32.const 9))
  (func (export "sum2") (result i32)
    (call $two_internal) (i32.add))
  (func $two_internal (result i32 i32) (i32.const 40) (i32.const 2))
  (func (export "divrem") (param $a i32) (param $b i32) (result i32 i32)
    (i32.div_s (local.get $a) (local.get $b)) (i32.rem_s (local.get $a) (local.get $b)))
  (func (export "nearest") (param $a f64) (result f64) (f64.nearest (local.get $a)))
  (func (export "nearest32") (param $a f32) (result f32) (f32.nearest (local.get $a)))
  (func (export "pick") (param $c i32) (result i32)
    (select (i32.const 11) (i32.const 22) (local.get $c)))
  (func (export "copy") (param $d i32) (param $s i32) (param $n i32)
    (memory.copy (local.get $d) (local.get $s) (local.get $n)))
  (func (export "early") (param $a i32) (result i32)
    (block $out (result i32)
      (loop $l
        (br_if $out (i32.const 5) (i32.gt_s (local.get $a) (i32.const 3)))
        (local.set $a (i32.add (local.get $a) (i32.const 1)))
        (br $l))
      (i32.const 0)))
)
"""


@pytest.fixture(scope="module")
def m():
    return WatModule(text=MOD, max_steps=2_000_000)


def test_control_flow(m):
    assert m.call("sum", 10) == [45]
    assert m.call("sum", 0) == [0]
    assert m.call("absdiff", 3, 10) == [7] and m.call("absdiff", 10, 3) == [7]
    assert m.call("nested") == [7]


def test_integers(m):
    assert m.call("wrap", 0x7FFFFFFF) == [0x80000000]
    assert m.call("wrap", -1) == [0]
    assert m.call("shr", -4) == [(-2) & 0xFFFFFFFF, 0x7FFFFFFE]


def test_f32_rounding(m):
    (r,) = m.call("f32add", 1.0, 2.0 ** -24)          # ties to even: stays 1.0
    assert r == np.float32(1.0) and isinstance(r, np.float32)
    (r,) = m.call("f32add", 1.0, 2.0 ** -23)
    assert r == np.float32(1.0 + 2.0 ** -23)


def test_simd_and_memory(m):
    m.write(64, np.array([1, 2, 3, 4.5], np.float32))
    assert m.call("lanes", 64) == [np.float32(9.0)]
    assert m.call("store_load", 128, -0.1) == [-0.1]


def test_wait_that_cannot_end_is_an_error(m):
    m.write(256, np.zeros(1, np.int32))
    with pytest.raises(RuntimeError, match="instruction limit"):
        m.call("spin", 256)


def test_multi_value_and_calls(m):
    assert m.call("two") == [4, 9]
    assert m.call("sum2") == [42]


def test_signed_division_truncates(m):
    q, r = m.call("divrem", -7, 2)
    assert (q, r) == ((-3) & 0xFFFFFFFF, (-1) & 0xFFFFFFFF)


def test_nearest_ties_to_even(m):
    assert [m.call("nearest", v)[0] for v in (0.5, 1.5, 2.5, -0.5, -2.5)] == [0.0, 2.0, 2.0, -0.0, -2.0]
    assert np.signbit(m.call("nearest", -0.5)[0])
    assert [float(m.call("nearest32", v)[0]) for v in (0.5, 1.5, 2.5)] == [0.0, 2.0, 2.0]


def test_select_copy_and_branch_values(m):
    assert m.call("pick", 1) == [11] and m.call("pick", 0) == [22]
    m.write(512, np.arange(8, dtype=np.uint8))
    m.call("copy", 600, 512, 8)
    assert bytes(m.mem[600:608]) == bytes(range(8))
    assert m.call("early", 0) == [5]
