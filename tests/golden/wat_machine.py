"""A small WebAssembly-text interpreter that runs the reference's own kernels.

TEST INFRASTRUCTURE ONLY.  SciWasm.Sparse writes its sparse kernels by hand in
WebAssembly text (``src/sequential/src/sparse_opt_32.wat``,
``sparse_opt_64.wat``, ``src/parallel/src/spts_opt_32.wat`` ...).  No JS or
wasm engine is installed where the fixtures are made, so this module executes
that text directly: it reads the s-expressions, flattens folded expressions
into the stack-machine instruction sequence the WebAssembly specification
defines for them, and steps through it over a little-endian linear memory.

It implements the part of the instruction set those files use: i32 integer
arithmetic, comparisons and shifts; f32/f64 arithmetic with IEEE single and
double rounding (numpy float32 scalars for f32, Python floats for f64; wasm
has no fused multiply-add, and neither has this); loads and stores; the
structured control instructions (block, loop, if/else, br, br_if, return,
call); the 128-bit SIMD lanes the kernels touch (f32x4, f64x2, i32x4);
memory.copy; and the i32 atomics, which on one thread are plain loads, stores
and adds.  Functions may return several values.  An instruction limit turns a
wait that can never end (a spin on a flag that one thread never sets) into an
error instead of a hang.

The semantics here are the WebAssembly specification's, not the sparse
algorithms': the interpreter knows nothing of CSR or SpTS, so fixtures made by
running the reference's text through it are outputs of the reference itself.
"""
import math
import struct

import numpy as np

M32 = 0xFFFFFFFF
F32 = np.float32


def _s32(v):
    return v - 0x100000000 if v & 0x80000000 else v


# --------------------------------------------------------------------------
# s-expression reader
# --------------------------------------------------------------------------
def _tokenize(text):
    toks, i, n = [], 0, len(text)
    while i < n:
        c = text[i]
        if c in " \t\r\n":
            i += 1
        elif text.startswith(";;", i):
            j = text.find("\n", i)
            i = n if j < 0 else j + 1
        elif text.startswith("(;", i):
            depth, i = 1, i + 2
            while depth:
                if text.startswith("(;", i):
                    depth, i = depth + 1, i + 2
                elif text.startswith(";)", i):
                    depth, i = depth - 1, i + 2
                else:
                    i += 1
        elif c in "()":
            toks.append(c)
            i += 1
        elif c == '"':
            j = i + 1
            while text[j] != '"':
                j += 2 if text[j] == "\\" else 1
            toks.append(text[i:j + 1])
            i = j + 1
        else:
            j = i
            while j < n and text[j] not in " \t\r\n()" and not text.startswith(";;", j):
                j += 1
            toks.append(text[i:j])
            i = j
    return toks


def _parse(toks):
    stack = [[]]
    for t in toks:
        if t == "(":
            stack.append([])
        elif t == ")":
            x = stack.pop()
            stack[-1].append(x)
        else:
            stack[-1].append(t)
    assert len(stack) == 1, "unbalanced parentheses"
    return stack[0]


# --------------------------------------------------------------------------
# instruction flattening
# --------------------------------------------------------------------------
_ONE_IMM = ("local.get", "local.set", "local.tee", "get_local", "set_local", "tee_local",
            "global.get", "global.set", "get_global", "set_global", "br", "br_if", "call")
_RENAME = {"get_local": "local.get", "set_local": "local.set", "tee_local": "local.tee",
           "get_global": "global.get", "set_global": "global.set"}


def _is_mem(op):
    return (".load" in op or ".store" in op or ".atomic.rmw" in op) and not op.startswith("memory.")


def _n_imm(op):
    if op in _ONE_IMM or op.endswith(".const") or op.endswith("_lane"):
        return 1
    return 0


def _block_type(items, k):
    """Optional label and (result ...) after block/loop/if; returns (label, arity, k)."""
    label = None
    if k < len(items) and isinstance(items[k], str) and items[k].startswith("$"):
        label, k = items[k], k + 1
    arity = 0
    while k < len(items) and isinstance(items[k], list) and items[k] and items[k][0] in ("result", "param", "type"):
        if items[k][0] == "result":
            arity += len(items[k]) - 1
        k += 1
    return label, arity, k


def _flatten_seq(items, out):
    """Flatten a sequence of flat and folded instructions into out."""
    k = 0
    while k < len(items):
        it = items[k]
        if isinstance(it, list):
            _flatten_folded(it, out)
            k += 1
            continue
        op = _RENAME.get(it, it)
        k += 1
        if op in ("block", "loop", "if"):
            label, arity, k = _block_type(items, k)
            out.append((op, label, arity))
        elif op in ("else", "end"):
            if k < len(items) and isinstance(items[k], str) and items[k].startswith("$"):
                k += 1
            out.append((op,))
        elif _is_mem(op):
            offset = 0
            while k < len(items) and isinstance(items[k], str) and items[k].split("=")[0] in ("offset", "align"):
                if items[k].startswith("offset="):
                    offset = int(items[k][7:], 0)
                k += 1
            out.append((op, offset))
        else:
            n = _n_imm(op)
            out.append((op,) + tuple(items[k:k + n]))
            k += n


def _flatten_folded(expr, out):
    op = _RENAME.get(expr[0], expr[0])
    if op in ("block", "loop"):
        label, arity, k = _block_type(expr, 1)
        out.append((op, label, arity))
        _flatten_seq(expr[k:], out)
        out.append(("end",))
        return
    if op == "if":
        label, arity, k = _block_type(expr, 1)
        rest = expr[k:]
        then_ = [e for e in rest if isinstance(e, list) and e and e[0] == "then"]
        else_ = [e for e in rest if isinstance(e, list) and e and e[0] == "else"]
        conds = [e for e in rest if not (isinstance(e, list) and e and e[0] in ("then", "else"))]
        _flatten_seq(conds, out)
        out.append(("if", label, arity))
        if then_:
            _flatten_seq(then_[0][1:], out)
        if else_:
            out.append(("else",))
            _flatten_seq(else_[0][1:], out)
        out.append(("end",))
        return
    k = 1
    imms = []
    while k < len(expr) and isinstance(expr[k], str):
        imms.append(expr[k])
        k += 1
    for child in expr[k:]:
        _flatten_folded(child, out)
    if _is_mem(op):
        offset = 0
        for a in imms:
            if a.startswith("offset="):
                offset = int(a[7:], 0)
        out.append((op, offset))
    else:
        out.append((op,) + tuple(imms))


# --------------------------------------------------------------------------
# module
# --------------------------------------------------------------------------
def _zero(t):
    return {"i32": 0, "i64": 0, "f32": F32(0.0), "f64": 0.0, "v128": bytes(16)}[t]


def _const(t, lit):
    if t in ("i32", "i64"):
        v = int(lit.replace("_", ""), 0)
        return v & (M32 if t == "i32" else 0xFFFFFFFFFFFFFFFF)
    s = lit.replace("_", "")
    if "0x" in s.lower() and "p" in s.lower():
        x = float.fromhex(s)
    elif s.lstrip("+-") in ("inf", "nan"):
        x = float(s)
    else:
        x = float(s)
    return F32(x) if t == "f32" else x


class _Func:
    def __init__(self, name, ptypes, results, pyfunc=None):
        self.name, self.ptypes, self.results, self.pyfunc = name, ptypes, results, pyfunc
        self.ltypes, self.code, self.ends, self.elses = [], [], {}, {}


class WatModule:
    """One parsed .wat module over its own linear memory (a bytearray)."""

    def __init__(self, path=None, mem_bytes=1 << 20, max_steps=400_000_000, text=None):
        if text is None:
            with open(path) as f:
                text = f.read()
        tree = _parse(_tokenize(text))
        assert tree and tree[0][0] == "module"
        self.mem = bytearray(mem_bytes)
        self.max_steps = max_steps
        self.steps = 0
        self.funcs, self.exports = {}, {}
        self._pending = []
        order = []
        for field in tree[0][1:]:
            if not isinstance(field, list):
                continue
            if field[0] == "import" and isinstance(field[3], list) and field[3][0] == "func":
                mod, nm = field[1].strip('"'), field[2].strip('"')
                fdecl = field[3]
                fname = fdecl[1] if len(fdecl) > 1 and isinstance(fdecl[1], str) else None
                ptypes, results = self._sig(fdecl)
                fn = _Func(fname, ptypes, results, self._import(mod, nm, results))
                order.append(fn)
                if fname:
                    self.funcs[fname] = fn
            elif field[0] == "func":
                fn = self._declare(field)
                order.append(fn)
        self._order = order
        for fn, field in self._pending:
            self._compile(fn, field)

    # imports: logging is a no-op; the math imports are the host's (V8's
    # Math.* is not part of the reference, and no fixture depends on them)
    @staticmethod
    def _import(mod, nm, results):
        if mod == "console":
            if nm == "time":
                return lambda *a: [0.0]
            return lambda *a: []
        if mod == "math":
            fn = getattr(math, nm)
            f32 = results == ["f32"]
            return lambda *a: [F32(fn(*map(float, a))) if f32 else fn(*map(float, a))]
        raise NotImplementedError(f"import {mod}.{nm}")

    @staticmethod
    def _sig(fdecl):
        ptypes, results = [], []
        for e in fdecl:
            if isinstance(e, list) and e and e[0] == "param":
                ptypes += [t for t in e[1:] if not t.startswith("$")]
            elif isinstance(e, list) and e and e[0] == "result":
                results += e[1:]
        return ptypes, results

    def _declare(self, field):
        k = 1
        fname = None
        if isinstance(field[k], str) and field[k].startswith("$"):
            fname, k = field[k], k + 1
        fn = _Func(fname, [], [])
        names = {}
        exports = []
        while k < len(field) and isinstance(field[k], list) and field[k][0] in ("export", "param", "result", "local", "type"):
            e = field[k]
            if e[0] == "export":
                exports.append(e[1].strip('"'))
            elif e[0] in ("param", "local"):
                lst = fn.ptypes if e[0] == "param" else fn.ltypes
                if len(e) == 3 and e[1].startswith("$"):
                    names[e[1]] = len(fn.ptypes) + len(fn.ltypes)
                    lst.append(e[2])
                else:
                    for t in e[1:]:
                        lst.append(t)
            elif e[0] == "result":
                fn.results += e[1:]
            k += 1
        fn.local_names = names
        if fname:
            self.funcs[fname] = fn
        for x in exports:
            self.exports[x] = fn
        self._pending.append((fn, field[k:]))
        return fn

    def _compile(self, fn, body):
        raw = []
        _flatten_seq(body, raw)
        code, labels = [], []
        for pc, ins in enumerate(raw):
            op = ins[0]
            if op in ("block", "loop", "if"):
                labels.append((ins[1], pc))
                code.append([op, ins[2]])
            elif op == "else":
                fn.elses[labels[-1][1]] = pc
                code.append([op])
            elif op == "end":
                _, start = labels.pop()
                fn.ends[start] = pc
                code.append([op])
            elif op in ("br", "br_if"):
                tgt = ins[1]
                if tgt.startswith("$"):
                    depth = next(d for d, (nm, _) in enumerate(reversed(labels)) if nm == tgt)
                else:
                    depth = int(tgt)
                code.append([op, depth])
            elif op in ("local.get", "local.set", "local.tee"):
                ref = ins[1]
                idx = fn.local_names[ref] if ref.startswith("$") else int(ref)
                code.append([op, idx])
            elif op == "call":
                ref = ins[1]
                tgt = self.funcs[ref] if ref.startswith("$") else self._order[int(ref)]
                code.append([op, tgt])
            elif op.endswith(".const"):
                code.append([op, _const(op.split(".")[0], ins[1])])
            elif op.endswith("_lane"):
                code.append([op, int(ins[1])])
            else:
                code.append(list(ins))
        assert not labels, f"unclosed block in {fn.name}"
        # patch control targets: block/if -> (arity, end, else)
        for pc, ins in enumerate(code):
            if ins[0] in ("block", "loop", "if"):
                ins.append(fn.ends[pc])
                ins.append(fn.elses.get(pc, -1))
            elif ins[0] == "else":
                # the matching if's end
                start = next(s for s, e in fn.elses.items() if e == pc)
                ins.append(fn.ends[start])
        fn.code = [tuple(i) for i in code]

    # ------------------------------------------------------------------
    def call(self, export, *args):
        fn = self.exports[export]
        conv = []
        for t, a in zip(fn.ptypes, args):
            if t == "i32":
                conv.append(int(a) & M32)
            elif t == "f32":
                conv.append(F32(a))
            elif t == "f64":
                conv.append(float(a))
            else:
                conv.append(a)
        assert len(conv) == len(fn.ptypes), (export, len(args), len(fn.ptypes))
        with np.errstate(all="ignore"):
            return self._run(fn, conv)

    def _run(self, fn, args):
        if fn.pyfunc is not None:
            return fn.pyfunc(*args)
        mem = self.mem
        unpack, pack = struct.unpack_from, struct.pack_into
        locs = list(args) + [_zero(t) for t in fn.ltypes]
        st = []
        labels = []          # (height, arity, continuation pc, is_loop)
        code = fn.code
        n = len(code)
        pc = 0
        steps = 0
        nres = len(fn.results)
        while pc < n:
            ins = code[pc]
            op = ins[0]
            steps += 1
            if op == "local.get":
                st.append(locs[ins[1]])
            elif op == "i32.const" or op == "f32.const" or op == "f64.const":
                st.append(ins[1])
            elif op == "local.set":
                locs[ins[1]] = st.pop()
            elif op == "local.tee":
                locs[ins[1]] = st[-1]
            elif op == "i32.add":
                b = st.pop()
                st[-1] = (st[-1] + b) & M32
            elif op == "i32.sub":
                b = st.pop()
                st[-1] = (st[-1] - b) & M32
            elif op == "i32.shl":
                b = st.pop()
                st[-1] = (st[-1] << (b & 31)) & M32
            elif op == "i32.load" or op == "i32.atomic.load":
                st[-1] = unpack("<I", mem, st[-1] + ins[1])[0]
            elif op == "f32.load":
                st[-1] = F32(unpack("<f", mem, st[-1] + ins[1])[0])
            elif op == "f64.load":
                st[-1] = unpack("<d", mem, st[-1] + ins[1])[0]
            elif op == "f32.store":
                v = st.pop()
                pack("<f", mem, st.pop() + ins[1], float(v))
            elif op == "f64.store":
                v = st.pop()
                pack("<d", mem, st.pop() + ins[1], v)
            elif op == "i32.store" or op == "i32.atomic.store":
                v = st.pop()
                pack("<I", mem, st.pop() + ins[1], v)
            elif op == "i32.atomic.rmw.add":
                v = st.pop()
                a = st.pop() + ins[1]
                old = unpack("<I", mem, a)[0]
                pack("<I", mem, a, (old + v) & M32)
                st.append(old)
            elif op == "br_if":
                if st.pop():
                    pc = self._br(ins[1], st, labels)
                    if pc < 0:
                        break
                    continue
            elif op == "br":
                pc = self._br(ins[1], st, labels)
                if pc < 0:
                    break
                continue
            elif op == "loop":
                labels.append((len(st), 0, pc + 1, True))
            elif op == "block":
                labels.append((len(st) , ins[1], ins[2] + 1, False))
            elif op == "if":
                c = st.pop()
                labels.append((len(st), ins[1], ins[2] + 1, False))
                if not c:
                    pc = ins[3] + 1 if ins[3] >= 0 else ins[2]
                    continue
            elif op == "else":
                labels.pop()
                pc = ins[1] + 1
                continue
            elif op == "end":
                labels.pop()
            elif op == "return":
                break
            elif op == "call":
                tgt = ins[1]
                k = len(tgt.ptypes)
                a = st[len(st) - k:] if k else []
                del st[len(st) - k:]
                self.steps += steps
                steps = 0
                st.extend(self._run(tgt, a))
            elif op in _BIN32:
                b = st.pop()
                st[-1] = _BIN32[op](st[-1], b)
            elif op == "i32.eqz":
                st[-1] = int(st[-1] == 0)
            elif op in _FBIN:
                b = st.pop()
                st[-1] = _FBIN[op](st[-1], b)
            elif op in _FUN:
                st[-1] = _FUN[op](st[-1])
            elif op == "v128.load":
                a = st[-1] + ins[1]
                st[-1] = bytes(mem[a:a + 16])
            elif op == "v128.store":
                v = st.pop()
                a = st.pop() + ins[1]
                mem[a:a + 16] = v
            elif op in _SIMD:
                _SIMD[op](st, ins)
            elif op == "memory.copy":
                ln = st.pop()
                src = st.pop()
                dst = st.pop()
                mem[dst:dst + ln] = mem[src:src + ln]
            elif op == "drop":
                st.pop()
            elif op == "nop":
                pass
            elif op == "select":
                c = st.pop()
                b = st.pop()
                if not c:
                    st[-1] = b
            elif op == "unreachable":
                raise RuntimeError(f"unreachable executed in {fn.name}")
            else:
                raise NotImplementedError(op)
            pc += 1
            if steps > 1_000_000:
                self.steps += steps
                steps = 0
                if self.steps > self.max_steps:
                    raise RuntimeError(f"instruction limit reached in {fn.name} (a wait that cannot end?)")
        self.steps += steps
        return st[len(st) - nres:] if nres else []

    @staticmethod
    def _br(depth, st, labels):
        if depth >= len(labels):
            return -1                      # branch to the function body: return
        height, arity, cont, is_loop = labels[len(labels) - 1 - depth]
        if is_loop:
            del st[height:]
            del labels[len(labels) - depth:]
        else:
            vals = st[len(st) - arity:] if arity else []
            del st[height:]
            st.extend(vals)
            del labels[len(labels) - 1 - depth:]
        return cont

    # ------------------------------------------------------------------
    # memory helpers for callers
    def write(self, addr, arr):
        b = np.ascontiguousarray(arr).tobytes()
        self.mem[addr:addr + len(b)] = b
        return addr + len(b)

    def read(self, addr, dtype, count):
        dt = np.dtype(dtype)
        return np.frombuffer(bytes(self.mem[addr:addr + dt.itemsize * count]), dt).copy()


def _cmp_s(f):
    return lambda a, b: int(f(_s32(a), _s32(b)))


def _div_s(a, b):
    a, b = _s32(a), _s32(b)
    q = abs(a) // abs(b)
    return (q if (a < 0) == (b < 0) else -q) & M32


def _rem_s(a, b):
    a, b = _s32(a), _s32(b)
    r = abs(a) % abs(b)
    return (r if a >= 0 else -r) & M32


_BIN32 = {
    "i32.mul": lambda a, b: (a * b) & M32,
    "i32.div_u": lambda a, b: a // b,
    "i32.rem_u": lambda a, b: a % b,
    "i32.div_s": _div_s,
    "i32.rem_s": _rem_s,
    "i32.and": lambda a, b: a & b,
    "i32.or": lambda a, b: a | b,
    "i32.xor": lambda a, b: a ^ b,
    "i32.shr_u": lambda a, b: a >> (b & 31),
    "i32.shr_s": lambda a, b: (_s32(a) >> (b & 31)) & M32,
    "i32.eq": lambda a, b: int(a == b),
    "i32.ne": lambda a, b: int(a != b),
    "i32.lt_u": lambda a, b: int(a < b),
    "i32.gt_u": lambda a, b: int(a > b),
    "i32.le_u": lambda a, b: int(a <= b),
    "i32.ge_u": lambda a, b: int(a >= b),
    "i32.lt_s": _cmp_s(lambda a, b: a < b),
    "i32.gt_s": _cmp_s(lambda a, b: a > b),
    "i32.le_s": _cmp_s(lambda a, b: a <= b),
    "i32.ge_s": _cmp_s(lambda a, b: a >= b),
}


def _fdiv64(a, b):
    if b == 0.0:
        if a != a or a == 0.0:
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def _fbin(name, f32fn, f64fn):
    return {f"f32.{name}": f32fn, f"f64.{name}": f64fn}


_FBIN = {}
_FBIN.update(_fbin("add", lambda a, b: a + b, lambda a, b: a + b))
_FBIN.update(_fbin("sub", lambda a, b: a - b, lambda a, b: a - b))
_FBIN.update(_fbin("mul", lambda a, b: a * b, lambda a, b: a * b))
_FBIN.update(_fbin("div", lambda a, b: a / b, _fdiv64))
for _nm, _f in (("eq", lambda a, b: a == b), ("ne", lambda a, b: a != b), ("lt", lambda a, b: a < b),
                ("gt", lambda a, b: a > b), ("le", lambda a, b: a <= b), ("ge", lambda a, b: a >= b)):
    _FBIN.update(_fbin(_nm, (lambda f: lambda a, b: int(bool(f(a, b))))(_f),
                       (lambda f: lambda a, b: int(bool(f(a, b))))(_f)))


def _wasm_min(a, b):
    if a != a or b != b:
        return a + b
    if a == b == 0:
        return a if math.copysign(1.0, float(a)) < 0 else b
    return a if a < b else b


def _wasm_max(a, b):
    if a != a or b != b:
        return a + b
    if a == b == 0:
        return b if math.copysign(1.0, float(a)) < 0 else a
    return a if a > b else b


_FBIN.update(_fbin("min", _wasm_min, _wasm_min))
_FBIN.update(_fbin("max", _wasm_max, _wasm_max))


def _sqrt64(a):
    if a != a or a < 0:
        return math.nan
    return math.sqrt(a)


def _nearest64(a):
    if a != a or a in (math.inf, -math.inf):
        return a
    r = float(round(a))          # Python rounds half to even
    return math.copysign(r, a) if r == 0.0 else r


def _f64u(fn):
    def g(a):
        if a != a or a in (math.inf, -math.inf):
            return a
        r = float(fn(a))
        return math.copysign(r, a) if r == 0.0 else r
    return g


_FUN = {
    "f32.abs": lambda a: np.abs(a),
    "f32.neg": lambda a: -a,
    "f32.sqrt": lambda a: np.sqrt(a),
    "f32.ceil": lambda a: np.ceil(a),
    "f32.floor": lambda a: np.floor(a),
    "f32.trunc": lambda a: np.trunc(a),
    "f32.nearest": lambda a: np.rint(a),
    "f64.abs": lambda a: abs(a) if a == a else math.copysign(a, 1.0),
    "f64.neg": lambda a: -a,
    "f64.sqrt": _sqrt64,
    "f64.ceil": _f64u(math.ceil),
    "f64.floor": _f64u(math.floor),
    "f64.trunc": _f64u(math.trunc),
    "f64.nearest": _nearest64,
}


def _lanes(v, dt):
    return np.frombuffer(v, dt)


def _simd_table():
    t = {}
    for shape, dt, cast in (("f32x4", np.float32, F32), ("f64x2", np.float64, float),
                            ("i32x4", np.uint32, int)):
        nl = 16 // np.dtype(dt).itemsize

        def splat(st, ins, dt=dt, nl=nl):
            st[-1] = np.full(nl, st[-1], dt).tobytes()

        def extract(st, ins, dt=dt, cast=cast):
            st[-1] = cast(_lanes(st[-1], dt)[ins[1]])

        def replace(st, ins, dt=dt):
            x = st.pop()
            a = _lanes(st[-1], dt).copy()
            a[ins[1]] = x
            st[-1] = a.tobytes()

        t[f"{shape}.splat"] = splat
        t[f"{shape}.extract_lane"] = extract
        t[f"{shape}.replace_lane"] = replace
        for nm, f in (("add", np.add), ("sub", np.subtract), ("mul", np.multiply)):
            def binop(st, ins, dt=dt, f=f):
                b = st.pop()
                st[-1] = f(_lanes(st[-1], dt), _lanes(b, dt)).astype(dt).tobytes()
            t[f"{shape}.{nm}"] = binop
        if shape != "i32x4":
            def div(st, ins, dt=dt):
                b = st.pop()
                st[-1] = np.divide(_lanes(st[-1], dt), _lanes(b, dt)).astype(dt).tobytes()
            t[f"{shape}.div"] = div
            for nm, f in (("abs", np.abs), ("neg", np.negative), ("sqrt", np.sqrt), ("ceil", np.ceil),
                          ("floor", np.floor), ("trunc", np.trunc), ("nearest", np.rint)):
                def un(st, ins, dt=dt, f=f):
                    st[-1] = f(_lanes(st[-1], dt)).astype(dt).tobytes()
                t[f"{shape}.{nm}"] = un
        else:
            def shl(st, ins):
                s = st.pop() & 31
                st[-1] = (_lanes(st[-1], np.uint32) << np.uint32(s)).astype(np.uint32).tobytes()
            t["i32x4.shl"] = shl
    return t


_SIMD = _simd_table()
