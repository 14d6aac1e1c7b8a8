"""A small JavaScript interpreter that runs the reference's own host functions.

TEST INFRASTRUCTURE ONLY.  SciWasm.Sparse writes its format conversions, the
level-set analysis and the row partitioner in plain JavaScript
(``src/sequential/src/sparse32.js``, ``src/parallel/src/sparse32.js``).  No
JavaScript engine is installed where the fixtures are made, so this module
executes the text of those functions: it reads the source of the functions
it is asked for (matched by name, so the rest of the file -- modules,
promises, workers -- is never parsed), parses the ECMAScript subset they use
and evaluates it with the language's own rules:

* numbers are IEEE doubles; ``/`` and ``%`` are floating point, bitwise
  operators go through ToInt32;
* typed arrays (``Int32Array``, ``Float32Array``, ``Float64Array``, over
  ``memory.buffer`` or fresh) convert on store (ToInt32 wraps, Float32
  rounds to nearest) and read ``undefined`` outside their length;
* ``var`` is function scoped and hoisted; assignment to an undeclared name
  creates a global (sloppy mode); statements may end at a line break;
* evaluation order is left to right (a member target before the value
  assigned to it), postfix ``++``/``--`` yield the old value.

The host objects the functions touch -- ``memory.buffer``,
``malloc_instance.exports._malloc``, the ``allocate_*`` helpers and the
matrix constructors, ``console.log`` -- are supplied by the caller as Python
callables.  The interpreter knows nothing of sparse formats, so fixtures made
by running the reference's functions through it are outputs of the
reference itself.
"""
import math
import re

import numpy as np


class _Undefined:
    def __repr__(self):
        return "undefined"


UNDEF = _Undefined()


class JSError(Exception):
    pass


class _Break(Exception):
    pass


class _Continue(Exception):
    pass


class _Return(Exception):
    def __init__(self, value):
        self.value = value


# --------------------------------------------------------------------------
# values
# --------------------------------------------------------------------------
class JSObject:
    def __init__(self, props=None):
        self.props = dict(props or {})

    def get(self, k):
        return self.props.get(k, UNDEF)

    def put(self, k, v):
        self.props[k] = v


class JSArray:
    def __init__(self, items):
        self.items = list(items)

    def get(self, k):
        if k == "length":
            return float(len(self.items))
        if k == "push":
            return lambda *a: (self.items.extend(a), float(len(self.items)))[1]
        i = _as_index(k)
        if i is not None and 0 <= i < len(self.items):
            return self.items[i]
        return UNDEF

    def put(self, k, v):
        i = _as_index(k)
        if i is None:
            raise JSError(f"array property {k!r}")
        while len(self.items) <= i:
            self.items.append(UNDEF)
        self.items[i] = v


def to_int32(v):
    v = to_number(v)
    if v != v or v in (math.inf, -math.inf):
        return 0
    v = int(v) & 0xFFFFFFFF
    return v - 0x100000000 if v & 0x80000000 else v


class TypedArray:
    KINDS = {"Int32Array": np.int32, "Float32Array": np.float32, "Float64Array": np.float64,
             "Uint32Array": np.uint32}

    def __init__(self, kind, arr):
        self.kind, self.a = kind, arr

    def get(self, k):
        if k == "length":
            return float(self.a.size)
        if k == "fill":
            def fill(v, *rest):
                self.a[:] = self._conv(v)
                return self
            return fill
        i = _as_index(k)
        if i is not None and 0 <= i < self.a.size:
            return float(self.a[i])
        return UNDEF

    def _conv(self, v):
        if self.kind == "Int32Array":
            return np.int32(to_int32(v))
        if self.kind == "Uint32Array":
            return np.uint32(to_int32(v) & 0xFFFFFFFF)
        if self.kind == "Float32Array":
            with np.errstate(over="ignore"):
                return np.float32(to_number(v))
        return np.float64(to_number(v))

    def put(self, k, v):
        i = _as_index(k)
        if i is not None and 0 <= i < self.a.size:
            self.a[i] = self._conv(v)


def _as_index(k):
    if isinstance(k, str):
        return int(k) if k.isdigit() else None
    if isinstance(k, bool):
        return None
    if isinstance(k, (int, float)) and k == k and float(k).is_integer():
        return int(k)
    return None


def to_number(v):
    if isinstance(v, bool):
        return 1.0 if v else 0.0
    if isinstance(v, (int, float)):
        return float(v)
    if v is UNDEF:
        return math.nan
    if v is None:
        return 0.0
    if isinstance(v, str):
        t = v.strip(" \t\n\r\v\f")
        if t == "":
            return 0.0
        if re.fullmatch(r"[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?", t):
            return float(t)
        if re.fullmatch(r"0[xX][0-9a-fA-F]+", t):
            return float(int(t, 16))
        if t in ("Infinity", "+Infinity", "-Infinity"):
            return -math.inf if t[0] == "-" else math.inf
        return math.nan
    raise JSError(f"ToNumber of {v!r}")


def truthy(v):
    if isinstance(v, bool):
        return v
    if isinstance(v, (int, float)):
        return not (v == 0 or v != v)
    if v is UNDEF or v is None:
        return False
    if isinstance(v, str):
        return v != ""
    return True


def number_to_string(x):
    if x != x:
        return "NaN"
    if x in (math.inf, -math.inf):
        return "Infinity" if x > 0 else "-Infinity"
    if float(x).is_integer() and abs(x) < 1e21:
        return str(int(x))
    return repr(float(x))


def js_parseint(v, *rest):
    s = v if isinstance(v, str) else number_to_string(to_number(v))
    m = re.match(r"\s*([+-]?\d+)", s)
    return float(int(m.group(1))) if m else math.nan


# --------------------------------------------------------------------------
# tokenizer
# --------------------------------------------------------------------------
_PUNCT = sorted(""">>>= === !== >>> <<= >>= **= && || ++ -- += -= *= /= %= &= |= ^= == != <= >= << >> => **
{ } ( ) [ ] ; , < > + - * / % & | ^ ! ~ ? : = .""".split(), key=len, reverse=True)


def tokenize(src):
    toks, i, n, nl = [], 0, len(src), False
    while i < n:
        c = src[i]
        if c in " \t\r":
            i += 1
        elif c == "\n":
            nl, i = True, i + 1
        elif src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            nl = nl or "\n" in src[i:j]
            i = j + 2
        elif c.isdigit() or (c == "." and i + 1 < n and src[i + 1].isdigit()):
            m = re.compile(r"0[xX][0-9a-fA-F]+|(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?").match(src, i)
            t = m.group(0)
            toks.append(("num", float(int(t, 16)) if t[:2] in ("0x", "0X") else float(t), nl))
            nl, i = False, m.end()
        elif c.isalpha() or c in "_$":
            m = re.compile(r"[A-Za-z_$][A-Za-z0-9_$]*").match(src, i)
            toks.append(("name", m.group(0), nl))
            nl, i = False, m.end()
        elif c in "'\"":
            j = i + 1
            while src[j] != c:
                j += 2 if src[j] == "\\" else 1
            toks.append(("str", src[i + 1:j], nl))
            nl, i = False, j + 1
        else:
            for p in _PUNCT:
                if src.startswith(p, i):
                    toks.append(("punc", p, nl))
                    nl, i = False, i + len(p)
                    break
            else:
                raise JSError(f"unexpected character {c!r}")
    toks.append(("eof", None, True))
    return toks


# --------------------------------------------------------------------------
# parser
# --------------------------------------------------------------------------
_BINARY = [
    ("||",), ("&&",), ("|",), ("^",), ("&",), ("==", "!=", "===", "!=="),
    ("<", ">", "<=", ">=", "instanceof"), ("<<", ">>", ">>>"), ("+", "-"), ("*", "/", "%"),
]
_ASSIGN = ("=", "+=", "-=", "*=", "/=", "%=", "<<=", ">>=", ">>>=", "&=", "|=", "^=")


class Parser:
    def __init__(self, toks):
        self.t, self.p = toks, 0

    def peek(self, k=0):
        return self.t[self.p + k]

    def at(self, v, kind=None):
        tk = self.t[self.p]
        return tk[1] == v and (kind is None or tk[0] == kind) and tk[0] in ("punc", "name")

    def eat(self, v=None):
        tk = self.t[self.p]
        if v is not None and tk[1] != v:
            raise JSError(f"expected {v!r}, found {tk[1]!r} (token {self.p})")
        self.p += 1
        return tk

    def semi(self):
        if self.at(";"):
            self.eat()

    # statements
    def function(self):
        self.eat("function")
        name = self.eat()[1]
        self.eat("(")
        params = []
        while not self.at(")"):
            params.append(self.eat()[1])
            if self.at(","):
                self.eat()
        self.eat(")")
        return ("func", name, params, self.block())

    def block(self):
        self.eat("{")
        body = []
        while not self.at("}"):
            body.append(self.statement())
        self.eat("}")
        return ("block", body)

    def statement(self):
        tk = self.peek()
        v = tk[1]
        if tk[0] == "punc" and v == "{":
            return self.block()
        if tk[0] == "punc" and v == ";":
            self.eat()
            return ("empty",)
        if tk[0] == "name":
            if v in ("var", "let", "const"):
                s = self.vardecl()
                self.semi()
                return s
            if v == "if":
                self.eat()
                self.eat("(")
                c = self.expression()
                self.eat(")")
                th = self.statement()
                el = None
                if self.at("else"):
                    self.eat()
                    el = self.statement()
                return ("if", c, th, el)
            if v == "for":
                self.eat()
                self.eat("(")
                init = None
                if not self.at(";"):
                    init = (self.vardecl() if self.peek()[1] in ("var", "let", "const")
                            else ("expr", self.expression()))
                self.eat(";")
                cond = None if self.at(";") else self.expression()
                self.eat(";")
                upd = None if self.at(")") else self.expression()
                self.eat(")")
                return ("for", init, cond, upd, self.statement())
            if v == "while":
                self.eat()
                self.eat("(")
                c = self.expression()
                self.eat(")")
                return ("while", c, self.statement())
            if v == "do":
                self.eat()
                body = self.statement()
                self.eat("while")
                self.eat("(")
                c = self.expression()
                self.eat(")")
                self.semi()
                return ("dowhile", body, c)
            if v == "return":
                self.eat()
                e = None
                nt = self.peek()
                if not (nt[2] or (nt[0] == "punc" and nt[1] in (";", "}")) or nt[0] == "eof"):
                    e = self.expression()
                self.semi()
                return ("return", e)
            if v in ("break", "continue"):
                self.eat()
                self.semi()
                return (v,)
            if v == "throw":
                self.eat()
                e = self.expression()
                self.semi()
                return ("throw", e)
            if v == "function":
                return self.function()
            if v == "try":
                self.eat()
                body = self.block()
                cname, cbody, fbody = None, None, None
                if self.at("catch"):
                    self.eat()
                    self.eat("(")
                    cname = self.eat()[1]
                    self.eat(")")
                    cbody = self.block()
                if self.at("finally"):
                    self.eat()
                    fbody = self.block()
                return ("try", body, cname, cbody, fbody)
        e = self.expression()
        self.semi()
        return ("expr", e)

    def vardecl(self):
        self.eat()
        decls = []
        while True:
            name = self.eat()[1]
            init = None
            if self.at("="):
                self.eat()
                init = self.assignment()
            decls.append((name, init))
            if not self.at(","):
                break
            self.eat()
        return ("var", decls)

    # expressions
    def expression(self):
        e = self.assignment()
        if self.at(","):
            seq = [e]
            while self.at(","):
                self.eat()
                seq.append(self.assignment())
            return ("seq", seq)
        return e

    def assignment(self):
        left = self.conditional()
        tk = self.peek()
        if tk[0] == "punc" and tk[1] in _ASSIGN:
            self.eat()
            if left[0] not in ("name", "member", "index"):
                raise JSError("invalid assignment target")
            return ("assign", tk[1], left, self.assignment())
        return left

    def conditional(self):
        c = self.binary(0)
        if self.at("?"):
            self.eat()
            a = self.assignment()
            self.eat(":")
            b = self.assignment()
            return ("cond", c, a, b)
        return c

    def binary(self, level):
        if level == len(_BINARY):
            return self.unary()
        left = self.binary(level + 1)
        while True:
            tk = self.peek()
            if tk[0] in ("punc", "name") and tk[1] in _BINARY[level]:
                self.eat()
                right = self.binary(level + 1)
                kind = "logic" if tk[1] in ("||", "&&") else "bin"
                left = (kind, tk[1], left, right)
            else:
                return left

    def unary(self):
        tk = self.peek()
        if tk[0] == "punc" and tk[1] in ("!", "-", "+", "~"):
            self.eat()
            return ("unary", tk[1], self.unary())
        if tk[0] == "punc" and tk[1] in ("++", "--"):
            self.eat()
            return ("preinc", tk[1], self.unary())
        if tk[0] == "name" and tk[1] in ("typeof",):
            self.eat()
            return ("typeof", self.unary())
        e = self.postfix()
        return e

    def postfix(self):
        e = self.call_member()
        tk = self.peek()
        if tk[0] == "punc" and tk[1] in ("++", "--") and not tk[2]:
            self.eat()
            return ("postinc", tk[1], e)
        return e

    def call_member(self):
        if self.at("new", "name"):
            self.eat()
            callee = self.primary()
            while self.at("."):
                self.eat()
                callee = ("member", callee, self.eat()[1])
            args = self.arguments() if self.at("(") else []
            e = ("new", callee, args)
        else:
            e = self.primary()
        while True:
            if self.at("."):
                self.eat()
                e = ("member", e, self.eat()[1])
            elif self.at("["):
                self.eat()
                k = self.expression()
                self.eat("]")
                e = ("index", e, k)
            elif self.at("("):
                e = ("call", e, self.arguments())
            else:
                return e

    def arguments(self):
        self.eat("(")
        args = []
        while not self.at(")"):
            args.append(self.assignment())
            if self.at(","):
                self.eat()
        self.eat(")")
        return args

    def primary(self):
        tk = self.eat()
        if tk[0] == "num":
            return ("num", tk[1])
        if tk[0] == "str":
            return ("str", tk[1])
        if tk[0] == "name":
            if tk[1] == "this":
                return ("this",)
            if tk[1] in ("true", "false"):
                return ("const", tk[1] == "true")
            if tk[1] == "null":
                return ("const", None)
            if tk[1] == "undefined":
                return ("const", UNDEF)
            return ("name", tk[1])
        if tk[0] == "punc" and tk[1] == "(":
            e = self.expression()
            self.eat(")")
            return e
        if tk[0] == "punc" and tk[1] == "[":
            items = []
            while not self.at("]"):
                items.append(self.assignment())
                if self.at(","):
                    self.eat()
            self.eat("]")
            return ("arr", items)
        raise JSError(f"unexpected token {tk[1]!r}")


def extract_function(src, name):
    """The source text of `function name(...) {...}` in src."""
    m = re.search(r"(?:^|\n)\s*(?:export\s+)?function\s+" + re.escape(name) + r"\s*\(", src)
    if not m:
        raise JSError(f"function {name} not found")
    start = src.index("function", m.start())
    i = src.index("{", m.end())
    depth = 0
    j = i
    while True:
        # skip comments and strings while matching braces
        if src.startswith("//", j):
            j = src.index("\n", j)
            continue
        if src.startswith("/*", j):
            j = src.index("*/", j) + 2
            continue
        c = src[j]
        if c in "'\"":
            k = j + 1
            while src[k] != c:
                k += 2 if src[k] == "\\" else 1
            j = k + 1
            continue
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return src[start:j + 1]
        j += 1


# --------------------------------------------------------------------------
# evaluator
# --------------------------------------------------------------------------
class JSFunction:
    def __init__(self, machine, decl):
        self.m, self.name, self.params, self.body = machine, decl[1], decl[2], decl[3]
        self.hoisted = sorted(_var_names(self.body))

    def __call__(self, *args, this=UNDEF):
        scope = {v: UNDEF for v in self.hoisted}
        for i, p in enumerate(self.params):
            scope[p] = args[i] if i < len(args) else UNDEF
        frame = (scope, this)
        try:
            self.m.exec_stmt(self.body, frame)
        except _Return as r:
            return r.value
        return UNDEF


def _var_names(node, out=None):
    out = set() if out is None else out
    if isinstance(node, tuple) and node:
        if node[0] == "var":
            out.update(n for n, _ in node[1])
        if node[0] == "func":
            return out
        for ch in node[1:]:
            if isinstance(ch, tuple):
                _var_names(ch, out)
            elif isinstance(ch, list):
                for c in ch:
                    if isinstance(c, tuple):
                        _var_names(c, out)
    return out


class JSMachine:
    """Parses the named functions from JavaScript source text and runs them
    over one linear memory (a bytearray the typed-array views share)."""

    def __init__(self, mem_bytes=16 << 20, max_steps=200_000_000):
        self.mem = bytearray(mem_bytes)
        self.brk = 64
        self.steps, self.max_steps = 0, max_steps
        self.globals = {}
        self.builtins = self._builtins()

    # host environment -------------------------------------------------
    def malloc(self, nbytes):
        a = self.brk
        self.brk = (a + int(nbytes) + 63) // 64 * 64
        if self.brk > len(self.mem):
            raise JSError("out of linear memory")
        return float(a)

    def view(self, kind, addr, n):
        dt = np.dtype(TypedArray.KINDS[kind])
        a, n = int(addr), int(n)
        return np.frombuffer(self.mem, dt, n, a) if n else np.zeros(0, dt)

    def _typed_ctor(self, kind):
        def make(*args):
            if len(args) >= 2 and args[0] is self.buffer:
                n = args[2] if len(args) > 2 else (len(self.mem) - int(args[1])) // 4
                n = to_number(n)
                n = 0 if n != n else n     # ToIndex: a NaN length is 0
                return TypedArray(kind, self.view(kind, args[1], n))
            if isinstance(args[0], (int, float)):
                return TypedArray(kind, np.zeros(int(args[0]), TypedArray.KINDS[kind]))
            raise JSError(f"new {kind}{args!r}")
        obj = JSObject({"BYTES_PER_ELEMENT": float(np.dtype(TypedArray.KINDS[kind]).itemsize)})
        obj.construct = make
        return obj

    def _builtins(self):
        self.buffer = JSObject()
        math_obj = JSObject({
            "floor": lambda x: float(math.floor(to_number(x))),
            "ceil": lambda x: float(math.ceil(to_number(x))),
            "abs": lambda x: abs(to_number(x)),
            "pow": lambda a, b: float(to_number(a) ** to_number(b)),
            "sqrt": lambda x: math.sqrt(to_number(x)),
            "max": lambda *a: max(map(to_number, a)),
            "min": lambda *a: min(map(to_number, a)),
        })
        console = JSObject({"log": lambda *a: UNDEF})
        malloc = JSObject({"exports": JSObject({"_malloc": self.malloc,
                                                "_free": lambda *a: UNDEF})})
        array = JSObject()
        array.construct = lambda n=0.0, *r: JSArray([UNDEF] * int(to_number(n)))
        error = JSObject()
        error.construct = lambda *a: JSObject({"message": a[0] if a else ""})
        b = {"Math": math_obj, "console": console, "parseInt": js_parseint,
             "Number": lambda *a: to_number(a[0]) if a else 0.0, "Error": error, "Array": array,
             "memory": JSObject({"buffer": self.buffer}), "malloc_instance": malloc}
        for k in TypedArray.KINDS:
            b[k] = self._typed_ctor(k)
        return b

    def define(self, name, value):
        self.globals[name] = value

    def load(self, src, names):
        for nm in names:
            decl = Parser(tokenize(extract_function(src, nm))).function()
            self.globals[nm] = JSFunction(self, decl)

    def call(self, name, *args):
        return self.globals[name](*args)

    # statements ----------------------------------------------------------
    def exec_stmt(self, s, fr):
        self.steps += 1
        if self.steps > self.max_steps:
            raise JSError("step limit reached")
        k = s[0]
        if k == "expr":
            self.ev(s[1], fr)
        elif k == "block":
            for st in s[1]:
                self.exec_stmt(st, fr)
        elif k == "var":
            for name, init in s[1]:
                if init is not None:
                    fr[0][name] = self.ev(init, fr)
        elif k == "if":
            if truthy(self.ev(s[1], fr)):
                self.exec_stmt(s[2], fr)
            elif s[3] is not None:
                self.exec_stmt(s[3], fr)
        elif k == "for":
            if s[1] is not None:
                self.exec_stmt(s[1], fr)
            while s[2] is None or truthy(self.ev(s[2], fr)):
                try:
                    self.exec_stmt(s[4], fr)
                except _Break:
                    break
                except _Continue:
                    pass
                if s[3] is not None:
                    self.ev(s[3], fr)
        elif k == "while":
            while truthy(self.ev(s[1], fr)):
                try:
                    self.exec_stmt(s[2], fr)
                except _Break:
                    break
                except _Continue:
                    pass
        elif k == "dowhile":
            while True:
                try:
                    self.exec_stmt(s[1], fr)
                except _Break:
                    break
                except _Continue:
                    pass
                if not truthy(self.ev(s[2], fr)):
                    break
        elif k == "return":
            raise _Return(UNDEF if s[1] is None else self.ev(s[1], fr))
        elif k == "break":
            raise _Break()
        elif k == "continue":
            raise _Continue()
        elif k == "empty":
            pass
        elif k == "throw":
            v = self.ev(s[1], fr)
            raise JSError(v.get("message") if isinstance(v, JSObject) else v)
        elif k == "func":
            fr[0][s[1]] = JSFunction(self, s)
        elif k == "try":
            try:
                self.exec_stmt(s[1], fr)
            except JSError:
                if s[3] is None:
                    raise
                fr[0][s[2]] = UNDEF
                self.exec_stmt(s[3], fr)
            finally:
                if s[4] is not None:
                    self.exec_stmt(s[4], fr)
        else:
            raise JSError(f"statement {k}")

    # expressions ---------------------------------------------------------
    def lookup(self, name, fr):
        if name in fr[0]:
            return fr[0][name]
        if name in self.globals:
            return self.globals[name]
        if name in self.builtins:
            return self.builtins[name]
        raise JSError(f"ReferenceError: {name} is not defined")

    def assign_name(self, name, v, fr):
        if name in fr[0]:
            fr[0][name] = v
        else:
            self.globals[name] = v      # sloppy mode: implicit global

    def get_prop(self, obj, key):
        if isinstance(obj, (JSObject, JSArray, TypedArray)):
            if isinstance(key, float) and isinstance(obj, JSObject):
                key = number_to_string(key)
            return obj.get(key)
        if isinstance(obj, str):
            if key == "length":
                return float(len(obj))
            if key == "split":
                return lambda sep=UNDEF, *r: JSArray([obj] if sep is UNDEF else obj.split(sep))
            i = _as_index(key)
            if i is not None:
                return obj[i] if 0 <= i < len(obj) else UNDEF
        raise JSError(f"TypeError: cannot read {key!r} of {obj!r}")

    def put_prop(self, obj, key, v):
        if isinstance(obj, (JSObject, JSArray, TypedArray)):
            if isinstance(key, float) and isinstance(obj, JSObject):
                key = number_to_string(key)
            obj.put(key, v)
            return
        raise JSError(f"TypeError: cannot set {key!r} of {obj!r}")

    def reference(self, t, fr):
        """(getter, setter) of an assignment target, its parts evaluated once."""
        if t[0] == "name":
            return (lambda: self.lookup(t[1], fr)), (lambda v: self.assign_name(t[1], v, fr))
        obj = self.ev(t[1], fr)
        key = t[2] if t[0] == "member" else self.ev(t[2], fr)
        return (lambda: self.get_prop(obj, key)), (lambda v: self.put_prop(obj, key, v))

    def ev(self, e, fr):
        k = e[0]
        if k == "num":
            return e[1]
        if k == "name":
            return self.lookup(e[1], fr)
        if k == "index":
            obj = self.ev(e[1], fr)
            return self.get_prop(obj, self.ev(e[2], fr))
        if k == "member":
            return self.get_prop(self.ev(e[1], fr), e[2])
        if k == "bin":
            return self.binop(e[1], self.ev(e[2], fr), self.ev(e[3], fr))
        if k == "assign":
            get, put = self.reference(e[2], fr)
            if e[1] == "=":
                v = self.ev(e[3], fr)
            else:
                old = get()
                v = self.binop(e[1][:-1], old, self.ev(e[3], fr))
            put(v)
            return v
        if k == "postinc" or k == "preinc":
            get, put = self.reference(e[2], fr)
            old = to_number(get())
            new = old + 1 if e[1] == "++" else old - 1
            put(new)
            return old if k == "postinc" else new
        if k == "logic":
            a = self.ev(e[2], fr)
            if e[1] == "&&":
                return self.ev(e[3], fr) if truthy(a) else a
            return a if truthy(a) else self.ev(e[3], fr)
        if k == "unary":
            v = self.ev(e[2], fr)
            if e[1] == "!":
                return not truthy(v)
            if e[1] == "-":
                return -to_number(v)
            if e[1] == "+":
                return to_number(v)
            return float(~to_int32(v))
        if k == "call":
            callee = e[1]
            this = UNDEF
            if callee[0] in ("member", "index"):
                this = self.ev(callee[1], fr)
                key = callee[2] if callee[0] == "member" else self.ev(callee[2], fr)
                fn = self.get_prop(this, key)
            else:
                fn = self.ev(callee, fr)
            args = [self.ev(a, fr) for a in e[2]]
            if isinstance(fn, JSFunction):
                return fn(*args, this=this)
            if callable(fn):
                return fn(*args)
            raise JSError(f"TypeError: {callee!r} is not a function")
        if k == "new":
            ctor = self.ev(e[1], fr)
            args = [self.ev(a, fr) for a in e[2]]
            if isinstance(ctor, JSFunction):
                obj = JSObject()
                ctor(*args, this=obj)
                obj.ctor = ctor
                return obj
            if hasattr(ctor, "construct"):
                return ctor.construct(*args)
            raise JSError(f"TypeError: not a constructor: {e[1]!r}")
        if k == "str":
            return e[1]
        if k == "const":
            return e[1]
        if k == "this":
            return fr[1]
        if k == "arr":
            return JSArray(self.ev(a, fr) for a in e[1])
        if k == "cond":
            return self.ev(e[2], fr) if truthy(self.ev(e[1], fr)) else self.ev(e[3], fr)
        if k == "seq":
            v = UNDEF
            for x in e[1]:
                v = self.ev(x, fr)
            return v
        if k == "typeof":
            v = self.ev(e[1], fr)
            return ("undefined" if v is UNDEF else "number" if isinstance(v, float)
                    else "string" if isinstance(v, str) else "object")
        raise JSError(f"expression {k}")

    @staticmethod
    def binop(op, a, b):
        if op == "+":
            if isinstance(a, str) or isinstance(b, str):
                sa = a if isinstance(a, str) else number_to_string(to_number(a))
                sb = b if isinstance(b, str) else number_to_string(to_number(b))
                return sa + sb
            return to_number(a) + to_number(b)
        if op in ("===", "!=="):
            same = _strict_eq(a, b)
            return same if op == "===" else not same
        if op in ("==", "!="):
            if (a is UNDEF or a is None) and (b is UNDEF or b is None):
                same = True
            elif a is UNDEF or a is None or b is UNDEF or b is None:
                same = False
            elif isinstance(a, (JSObject, JSArray, TypedArray)) or isinstance(
                    b, (JSObject, JSArray, TypedArray)):
                same = a is b
            elif isinstance(a, str) and isinstance(b, str):
                same = a == b
            else:
                same = to_number(a) == to_number(b)
            return same if op == "==" else not same
        if op == "instanceof":
            return isinstance(a, JSObject) and getattr(a, "ctor", None) is b
        x, y = to_number(a), to_number(b)
        if op == "-":
            return x - y
        if op == "*":
            return x * y
        if op == "/":
            if y == 0:
                if x == 0 or x != x:
                    return math.nan
                return math.copysign(math.inf, x) * math.copysign(1.0, y)
            return x / y
        if op == "%":
            if y == 0 or x != x or y != y or x in (math.inf, -math.inf):
                return math.nan
            return math.fmod(x, y)
        if op == "<":
            return x < y
        if op == ">":
            return x > y
        if op == "<=":
            return x <= y
        if op == ">=":
            return x >= y
        ia, ib = to_int32(x), to_int32(y)
        if op == "&":
            return float(to_int32(ia & ib))
        if op == "|":
            return float(to_int32(ia | ib))
        if op == "^":
            return float(to_int32(ia ^ ib))
        if op == "<<":
            return float(to_int32(ia << (ib & 31)))
        if op == ">>":
            return float(ia >> (ib & 31))
        if op == ">>>":
            return float((ia & 0xFFFFFFFF) >> (ib & 31))
        raise JSError(f"operator {op}")


def _strict_eq(a, b):
    if isinstance(a, (int, float)) and not isinstance(a, bool) and isinstance(b, (int, float)) \
            and not isinstance(b, bool):
        return float(a) == float(b)
    if type(a) is not type(b):
        return False
    if isinstance(a, (str, bool)):
        return a == b
    return a is b
