"""A small WGSL interpreter: runs the reference's compute shaders on the CPU.

The reference's GPU solver is a set of WGSL compute kernels
(src/gpu/wgsl.js, the source text produced by makeShaderSource, which
tests/golden/jsmini.py evaluates). No WebGPU implementation exists on this
machine, so this module executes that WGSL text itself, one invocation after
another, for the subset of the language those kernels use:

  - module scope: const declarations, struct types, storage / uniform /
    workgroup variables, functions (entry points marked @compute);
  - statements: let / var / const, assignment and compound assignment,
    ++ / --, if / else, for, loop, while, break, continue, return;
  - expressions: the arithmetic, bit, comparison and logical operators,
    indexing, member and swizzle access, function calls, type constructors
    (vec2/3/4 of f32, i32, u32; scalar conversions; bitcast);
  - built-ins: floor, fract, sqrt, sin, cos, abs, sign, min, max, clamp,
    select, dot, cross, length, distance, normalize, and the atomics
    (load, store, add, sub, min, max, or, and).

Arithmetic follows WGSL's types: f32 operations round to float32 after every
operation (numpy float32 scalars; no fused multiply-add), u32 and i32 wrap
modulo 2^32, integer division and remainder truncate toward zero, float to
integer conversions truncate and saturate. Abstract literals take the type of
the other operand, or f32 / i32 when declared on their own.

Invocations of a dispatch run sequentially in global-id order, so atomics see
a deterministic order (the order a GPU would pick is unspecified). Kernels
that synchronize a workgroup (workgroupBarrier) are not supported: the one
place the reference uses them, the hash-grid prefix scan, is an exclusive
prefix sum that the caller computes directly.

Test infrastructure only (golden-vector generation): nothing in the product
imports it.
"""
from __future__ import annotations

import math
import re
import warnings

import numpy as np

F32, I32, U32, BOOL = np.float32, np.int32, np.uint32, np.bool_

# ---------------------------------------------------------------- lexer

_TOK = re.compile(r"""
  (?P<ws>\s+)|(?P<lc>//[^\n]*)|(?P<bc>/\*.*?\*/)|
  (?P<num>0[xX][0-9a-fA-F]+[iu]?|(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[fhiu]?)|
  (?P<id>[A-Za-z_][A-Za-z0-9_]*)|
  (?P<op><<=|>>=|->|\+\+|--|\+=|-=|\*=|/=|%=|&=|\|=|\^=|<<|>>|<=|>=|==|!=|&&|\|\||[{}()\[\];,.:<>+\-*/%&|^!~=@])
""", re.S | re.X)


def lex(src: str) -> list[tuple[str, object]]:
    out = []
    i = 0
    while i < len(src):
        m = _TOK.match(src, i)
        if not m:
            raise SyntaxError(f"WGSL: bad character {src[i]!r} at {i}")
        i = m.end()
        k, v = m.lastgroup, m.group()
        if k in ("ws", "lc", "bc"):
            continue
        if k == "num":
            out.append(("num", _literal(v)))
        else:
            out.append((k, v))
    out.append(("eof", None))
    return out


def _literal(t: str):
    """A WGSL numeric literal: ('u32'|'i32'|'f32'|'aint'|'afloat', value)."""
    if t[:2] in ("0x", "0X"):
        suf = t[-1] if t[-1] in "iu" else ""
        v = int(t[2:-1] if suf else t[2:], 16)
        return ({"u": "u32", "i": "i32"}.get(suf, "aint"), v)
    suf = t[-1] if t[-1] in "fhiu" else ""
    body = t[:-1] if suf else t
    if suf in ("i", "u"):
        return ({"u": "u32", "i": "i32"}[suf], int(body))
    if suf in ("f", "h"):
        return ("f32", float(body))
    if "." in body or "e" in body or "E" in body:
        return ("afloat", float(body))
    return ("aint", int(body))


# ---------------------------------------------------------------- parser
# AST nodes are tuples (kind, ...). Types are strings ("f32", "vec3f",
# "array<u32,256>", struct names).

_BIN_PREC = [("||",), ("&&",), ("|",), ("^",), ("&",), ("==", "!="), ("<", ">", "<=", ">="), ("<<", ">>"),
             ("+", "-"), ("*", "/", "%")]
_ASSIGN_OPS = {"=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>="}
_VEC_ALIAS = {f"vec{n}{s}": (n, {"f": "f32", "i": "i32", "u": "u32"}[s]) for n in (2, 3, 4) for s in "fiu"}


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def accept(self, v):
        if self.t[self.i][1] == v and self.t[self.i][0] != "num":
            self.i += 1
            return True
        return False

    def expect(self, v):
        tok = self.next()
        if tok[1] != v:
            raise SyntaxError(f"WGSL: expected {v!r}, got {tok[1]!r} (token {self.i})")
        return tok

    def close_angle(self):
        """A '>' that ends a template list; '>>' closes two."""
        tok = self.peek()
        if tok == ("op", ">>"):
            self.t[self.i] = ("op", ">")
            return
        self.expect(">")

    def ident(self):
        tok = self.next()
        if tok[0] != "id":
            raise SyntaxError(f"WGSL: expected a name, got {tok[1]!r}")
        return tok[1]

    # ---- types
    def type_(self) -> str:
        name = self.ident()
        if self.peek()[1] == "<" and name in ("array", "atomic", "vec2", "vec3", "vec4", "ptr"):
            self.next()
            args = [self.type_or_expr()]
            while self.accept(","):
                args.append(self.type_or_expr())
            self.close_angle()
            if name in ("vec2", "vec3", "vec4"):
                return f"{name}{args[0][0]}"  # vec3<f32> -> vec3f
            return f"{name}<{','.join(str(a) for a in args)}>"
        return name

    def type_or_expr(self):
        tok = self.peek()
        if tok[0] == "num":
            self.next()
            return str(tok[1][1])
        if tok[0] == "id" and tok[1] in ("read_write", "read", "storage", "function", "workgroup", "uniform"):
            self.next()
            return tok[1]
        return self.type_()

    def attrs(self):
        out = {}
        while self.accept("@"):
            name = self.ident()
            args = []
            if self.accept("("):
                while not self.accept(")"):
                    tok = self.next()
                    if tok[1] != ",":
                        args.append(tok[1][1] if tok[0] == "num" else tok[1])
            out[name] = args
        return out

    # ---- module
    def module(self):
        items = []
        while self.peek()[0] != "eof":
            at = self.attrs()
            kw = self.ident()
            if kw == "const":
                name = self.ident()
                ty = self.type_() if self.accept(":") else None
                self.expect("=")
                e = self.expr()
                self.expect(";")
                items.append(("const", name, ty, e))
            elif kw == "struct":
                name = self.ident()
                self.expect("{")
                fields = []
                while not self.accept("}"):
                    self.attrs()
                    fname = self.ident()
                    self.expect(":")
                    fields.append((fname, self.type_()))
                    self.accept(",")
                items.append(("struct", name, fields))
            elif kw == "var":
                space = []
                if self.accept("<"):
                    space.append(self.ident())
                    while self.accept(","):
                        space.append(self.ident())
                    self.expect(">")
                name = self.ident()
                self.expect(":")
                ty = self.type_()
                self.expect(";")
                items.append(("gvar", name, tuple(space), ty, at))
            elif kw == "fn":
                name = self.ident()
                self.expect("(")
                params = []
                while not self.accept(")"):
                    pat = self.attrs()
                    pname = self.ident()
                    self.expect(":")
                    params.append((pname, self.type_(), pat))
                    self.accept(",")
                ret = self.type_() if self.accept("->") else None
                body = self.block()
                items.append(("fn", name, params, ret, body, at))
            else:
                raise SyntaxError(f"WGSL: unexpected {kw!r} at module scope")
        return items

    # ---- statements
    def block(self):
        self.expect("{")
        out = []
        while not self.accept("}"):
            out.append(self.stmt())
        return ("block", out)

    def stmt(self):
        tok = self.peek()
        v = tok[1]
        if tok[0] == "op" and v == "{":
            return self.block()
        if tok[0] == "op" and v == ";":
            self.next()
            return ("block", [])
        if tok[0] == "id":
            if v in ("let", "var", "const"):
                s = self.decl()
                self.expect(";")
                return s
            if v == "if":
                return self.if_()
            if v == "for":
                self.next()
                self.expect("(")
                init = None if self.peek()[1] == ";" else self.simple()
                self.expect(";")
                cond = None if self.peek()[1] == ";" else self.expr()
                self.expect(";")
                upd = None if self.peek()[1] == ")" else self.simple()
                self.expect(")")
                return ("for", init, cond, upd, self.block())
            if v == "while":
                self.next()
                cond = self.expr()
                return ("for", None, cond, None, self.block())
            if v == "loop":
                self.next()
                return ("for", None, None, None, self.block())
            if v in ("break", "continue"):
                self.next()
                self.expect(";")
                return (v,)
            if v == "return":
                self.next()
                e = None if self.peek()[1] == ";" else self.expr()
                self.expect(";")
                return ("return", e)
        s = self.simple()
        self.expect(";")
        return s

    def decl(self):
        kw = self.ident()
        name = self.ident()
        ty = self.type_() if self.accept(":") else None
        e = self.expr() if self.accept("=") else None
        return ("decl", name, ty, e, kw)

    def if_(self):
        self.expect("if")
        cond = self.expr()
        then = self.block()
        els = None
        if self.accept("else"):
            els = self.if_() if self.peek()[1] == "if" else self.block()
        return ("if", cond, then, els)

    def simple(self):
        if self.peek()[0] == "id" and self.peek()[1] in ("let", "var", "const"):
            return self.decl()
        e = self.expr()
        tok = self.peek()
        if tok[0] == "op" and tok[1] in _ASSIGN_OPS:
            self.next()
            return ("assign", tok[1], e, self.expr())
        if tok[0] == "op" and tok[1] in ("++", "--"):
            self.next()
            return ("assign", "+=" if tok[1] == "++" else "-=", e, ("num", ("aint", 1)))
        return ("expr", e)

    # ---- expressions
    def expr(self, level=0):
        if level == len(_BIN_PREC):
            return self.unary()
        e = self.expr(level + 1)
        while True:
            tok = self.peek()
            if tok[0] == "op" and tok[1] in _BIN_PREC[level]:
                self.next()
                e = ("bin", tok[1], e, self.expr(level + 1))
            else:
                return e

    def unary(self):
        tok = self.peek()
        if tok[0] == "op" and tok[1] in ("-", "!", "~", "&", "*"):
            self.next()
            return ("unary", tok[1], self.unary())
        return self.postfix(self.primary())

    def postfix(self, e):
        while True:
            if self.accept("["):
                k = self.expr()
                self.expect("]")
                e = ("index", e, k)
            elif self.peek()[1] == "." and self.peek()[0] == "op":
                self.next()
                e = ("member", e, self.ident())
            else:
                return e

    def primary(self):
        tok = self.next()
        if tok[0] == "num":
            return ("num", tok[1])
        if tok[1] == "(":
            e = self.expr()
            self.expect(")")
            return e
        if tok[0] != "id":
            raise SyntaxError(f"WGSL: unexpected {tok[1]!r}")
        name = tok[1]
        if name in ("true", "false"):
            return ("bool", name == "true")
        targs = None
        if self.peek()[1] == "<" and name in ("bitcast", "vec2", "vec3", "vec4", "array"):
            self.next()
            targs = [self.type_()]
            while self.accept(","):
                targs.append(self.type_or_expr())
            self.expect(">")
        if self.accept("("):
            args = []
            while not self.accept(")"):
                args.append(self.expr())
                self.accept(",")
            if name in ("vec2", "vec3", "vec4") and targs:
                name = f"{name}{targs[0][0]}"
                targs = None
            return ("call", name, targs, args)
        return ("name", name)


# ---------------------------------------------------------------- values
# Scalars: np.float32 (f32), np.uint32 (u32), np.int32 (i32), bool; Python
# int / float are abstract literals not yet given a type. Vectors: Vec.

class Vec:
    __slots__ = ("c", "t")

    def __init__(self, comps, t):
        self.c = tuple(comps)
        self.t = t

    def __repr__(self):
        return f"vec{len(self.c)}<{self.t}>{self.c}"


_NP = {"f32": F32, "u32": U32, "i32": I32}
_SWZ = {"x": 0, "y": 1, "z": 2, "w": 3, "r": 0, "g": 1, "b": 2, "a": 3}


def tname(x) -> str:
    if isinstance(x, Vec):
        return x.t
    if isinstance(x, np.float32):
        return "f32"
    if isinstance(x, np.uint32):
        return "u32"
    if isinstance(x, np.int32):
        return "i32"
    if isinstance(x, (bool, np.bool_)):
        return "bool"
    if isinstance(x, int):
        return "aint"
    return "afloat"


def conv(x, t: str):
    """Value conversion to scalar type t (WGSL's f32(), u32(), i32(), bool())."""
    if isinstance(x, Vec):
        return Vec([conv(c, t) for c in x.c], t)
    if t == "f32":
        if isinstance(x, (bool, np.bool_)):
            return F32(1.0 if x else 0.0)
        return F32(x) if not isinstance(x, np.floating) else F32(x)
    if t in ("u32", "i32"):
        lo, hi = (0, 2 ** 32 - 1) if t == "u32" else (-2 ** 31, 2 ** 31 - 1)
        if isinstance(x, (bool, np.bool_)):
            return _NP[t](1 if x else 0)
        if isinstance(x, (np.floating, float)):
            f = float(x)
            if math.isnan(f):
                return _NP[t](0)
            v = int(math.trunc(max(min(f, hi), lo))) if math.isfinite(f) else (hi if f > 0 else lo)
            return _NP[t](v)
        v = int(x) & 0xFFFFFFFF
        if t == "i32" and v >= 2 ** 31:
            v -= 2 ** 32
        return _NP[t](v)
    if t == "bool":
        return bool(x)
    raise TypeError(f"WGSL: no conversion to {t}")


def concrete(x):
    """An abstract literal takes its default type: int -> i32, float -> f32."""
    if isinstance(x, bool):
        return x
    if isinstance(x, int):
        return conv(x, "i32")
    if isinstance(x, float):
        return F32(x)
    if isinstance(x, Vec) and x.t in ("aint", "afloat"):
        return conv(x, "i32" if x.t == "aint" else "f32")
    return x


def _unify(a, b):
    ta, tb = tname(a), tname(b)
    if ta == tb:
        return a, b, ta
    if ta in ("aint", "afloat") and tb not in ("aint", "afloat"):
        return conv(a, tb), b, tb
    if tb in ("aint", "afloat") and ta not in ("aint", "afloat"):
        return a, conv(b, ta), ta
    if {ta, tb} == {"aint", "afloat"}:
        return float(a), float(b), "afloat"
    raise TypeError(f"WGSL: operands of types {ta} and {tb}")


def _idiv(a, b, t):
    a, b = int(a), int(b)
    if b == 0:
        return conv(a, t)
    q = abs(a) // abs(b)
    if (a < 0) != (b < 0):
        q = -q
    return conv(q, t)


def _imod(a, b, t):
    a, b = int(a), int(b)
    if b == 0:
        return conv(0, t)
    q = abs(a) // abs(b)
    if (a < 0) != (b < 0):
        q = -q
    return conv(a - b * q, t)


def _scalar_bin(op, a, b):
    if op in ("==", "!=", "<", ">", "<=", ">="):
        a, b, _ = _unify(a, b)
        if op == "==":
            return bool(a == b)
        if op == "!=":
            return bool(a != b)
        if op == "<":
            return bool(a < b)
        if op == ">":
            return bool(a > b)
        if op == "<=":
            return bool(a <= b)
        return bool(a >= b)
    if op in ("<<", ">>"):
        t = tname(a)
        if t == "aint":
            a, t = conv(a, "i32"), "i32"
        s = int(b) & 31
        if op == "<<":
            return conv(int(a) << s, t)
        return conv(int(a) >> s, t)  # arithmetic for i32 (Python ints), logical for u32 (non-negative)
    a, b, t = _unify(a, b)
    if t == "bool":
        if op == "&":
            return bool(a and b)
        if op == "|":
            return bool(a or b)
        if op == "^":
            return bool(a) != bool(b)
    if t in ("aint", "afloat"):
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if op == "/":
            return a / b if t == "afloat" else int(a / b)
        if op == "%":
            return math.fmod(a, b) if t == "afloat" else int(math.fmod(a, b))
        if op == "&":
            return a & b
        if op == "|":
            return a | b
        if op == "^":
            return a ^ b
    if t == "f32":
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if op == "/":
            return a / b
        if op == "%":
            return F32(a - b * F32(math.trunc(float(a) / float(b)))) if b != 0 else F32(math.nan)
    if op == "+":
        return conv(int(a) + int(b), t)
    if op == "-":
        return conv(int(a) - int(b), t)
    if op == "*":
        return conv(int(a) * int(b), t)
    if op == "/":
        return _idiv(a, b, t)
    if op == "%":
        return _imod(a, b, t)
    if op == "&":
        return conv(int(a) & int(b), t)
    if op == "|":
        return conv(int(a) | int(b), t)
    if op == "^":
        return conv(int(a) ^ int(b), t)
    raise TypeError(f"WGSL: operator {op} on {t}")


def binop(op, a, b):
    va, vb = isinstance(a, Vec), isinstance(b, Vec)
    if not va and not vb:
        return _scalar_bin(op, a, b)
    n = len(a.c) if va else len(b.c)
    ca = a.c if va else (a,) * n
    cb = b.c if vb else (b,) * n
    comps = [_scalar_bin(op, x, y) for x, y in zip(ca, cb)]
    if op in ("==", "!=", "<", ">", "<=", ">="):
        return Vec(comps, "bool")
    return Vec(comps, tname(comps[0]))


def unop(op, a):
    if isinstance(a, Vec):
        comps = [unop(op, c) for c in a.c]
        return Vec(comps, tname(comps[0]))
    if op == "-":
        t = tname(a)
        if t in ("aint", "afloat", "f32"):
            return -a
        return conv(-int(a), t)
    if op == "!":
        return not a
    if op == "~":
        t = tname(a)
        if t == "aint":
            a, t = conv(a, "i32"), "i32"
        return conv(~int(a), t)
    raise TypeError(f"WGSL: unary {op}")


def swizzle(v: Vec, s: str):
    if len(s) == 1:
        return v.c[_SWZ[s]]
    return Vec([v.c[_SWZ[ch]] for ch in s], v.t)


def with_comp(v: Vec, s: str, val):
    comps = list(v.c)
    if len(s) == 1:
        comps[_SWZ[s]] = conv(val, v.t) if v.t != "bool" else bool(val)
    else:
        for k, ch in enumerate(s):
            comps[_SWZ[ch]] = conv(val.c[k], v.t)
    return Vec(comps, v.t)


def make_vec(n: int, t: str, args: list):
    comps = []
    for a in args:
        if isinstance(a, Vec):
            comps.extend(a.c)
        else:
            comps.append(a)
    if len(comps) == 1 and n > 1:
        comps = comps * n
    if len(comps) != n:
        raise TypeError(f"WGSL: vec{n} from {len(comps)} components")
    return Vec([conv(c, t) for c in comps], t)


def zero_of(ty: str):
    if ty in _VEC_ALIAS:
        n, t = _VEC_ALIAS[ty]
        return Vec([conv(0, t)] * n, t)
    if ty in _NP:
        return conv(0, ty)
    if ty == "bool":
        return False
    m = re.match(r"array<(\w+),(\d+)>", ty)
    if m:
        return np.zeros(int(m.group(2)), dtype=_NP[m.group(1)])
    raise TypeError(f"WGSL: no zero value for {ty}")


def to_type(x, ty):
    """A value stored into a declaration of type ty (None: the default type)."""
    if ty is None:
        return concrete(x)
    if ty in _VEC_ALIAS:
        n, t = _VEC_ALIAS[ty]
        return make_vec(n, t, [x]) if not isinstance(x, Vec) else conv(x, t)
    if ty in _NP or ty == "bool":
        return conv(x, ty)
    return x


# ---------------------------------------------------------------- built-ins

def _map1(f, x):
    if isinstance(x, Vec):
        return Vec([f(c) for c in x.c], x.t)
    return f(x)


def _f32un(npf):
    return lambda x: _map1(lambda c: F32(npf(F32(c))), x)


def _min(a, b):
    a, b, _ = _unify(a, b) if not (isinstance(a, Vec) or isinstance(b, Vec)) else (a, b, None)
    if isinstance(a, Vec):
        return Vec([_min(x, y) for x, y in zip(a.c, b.c)], a.t)
    return b if b < a else a


def _max(a, b):
    a, b, _ = _unify(a, b) if not (isinstance(a, Vec) or isinstance(b, Vec)) else (a, b, None)
    if isinstance(a, Vec):
        return Vec([_max(x, y) for x, y in zip(a.c, b.c)], a.t)
    return b if a < b else a


def _dot(a: Vec, b: Vec):
    s = binop("*", a.c[0], b.c[0])
    for x, y in zip(a.c[1:], b.c[1:]):
        s = binop("+", s, binop("*", x, y))
    return s


def _cross(a: Vec, b: Vec):
    ax, ay, az = a.c
    bx, by, bz = b.c
    m = lambda x, y: binop("*", x, y)  # noqa: E731
    return Vec([binop("-", m(ay, bz), m(az, by)), binop("-", m(az, bx), m(ax, bz)),
                binop("-", m(ax, by), m(ay, bx))], a.t)


def _length(v):
    if not isinstance(v, Vec):
        return _map1(lambda c: F32(np.abs(F32(c))), v)
    return F32(np.sqrt(_dot(v, v)))


def _abs(x):
    def one(c):
        t = tname(c)
        if t == "f32":
            return F32(np.abs(c))
        if t == "i32":
            return conv(abs(int(c)), "i32")
        return c
    return _map1(one, x)


def _sign(x):
    return _map1(lambda c: F32(np.sign(F32(c))) if tname(c) in ("f32", "afloat") else conv(np.sign(int(c)), tname(c)), x)


def _fract(x):
    return _map1(lambda c: F32(F32(c) - np.floor(F32(c))), x)


def _bitcast(x, t):
    if isinstance(x, Vec):
        return Vec([_bitcast(c, t) for c in x.c], t)
    src = {"f32": np.float32, "u32": np.uint32, "i32": np.int32}[tname(concrete(x))]
    return np.array([concrete(x)], dtype=src).view(_NP[t])[0]


class Ref:
    """&array[index]: the operand of an atomic built-in."""
    __slots__ = ("a", "i")

    def __init__(self, a, i):
        self.a, self.i = a, int(i)


def _atomic(op):
    def f(r, v=None):
        old = U32(r.a[r.i]) if r.a.dtype == np.uint32 else I32(r.a[r.i])
        if op == "load":
            return old
        t = tname(old)
        v = conv(v, t)
        if op == "store":
            r.a[r.i] = v
            return None
        new = {"add": lambda: conv(int(old) + int(v), t), "sub": lambda: conv(int(old) - int(v), t),
               "min": lambda: min(old, v), "max": lambda: max(old, v),
               "or": lambda: conv(int(old) | int(v), t), "and": lambda: conv(int(old) & int(v), t),
               "exchange": lambda: v}[op]()
        r.a[r.i] = new
        return old
    return f


BUILTINS = {
    "floor": _f32un(np.floor), "sqrt": _f32un(np.sqrt), "sin": _f32un(np.sin), "cos": _f32un(np.cos),
    "fract": _fract, "abs": _abs, "sign": _sign, "min": _min, "max": _max,
    "clamp": lambda e, lo, hi: _min(_max(e, lo), hi),
    "select": lambda f, t, c: (Vec([y if k else x for x, y, k in zip(f.c, t.c, c.c)], f.t)
                               if isinstance(c, Vec) else (t if c else f)),
    "dot": _dot, "cross": _cross, "length": _length,
    "distance": lambda a, b: _length(binop("-", a, b)),
    "normalize": lambda v: binop("/", v, _length(v)),
    "atomicLoad": _atomic("load"), "atomicStore": _atomic("store"), "atomicAdd": _atomic("add"),
    "atomicSub": _atomic("sub"), "atomicMin": _atomic("min"), "atomicMax": _atomic("max"),
    "atomicOr": _atomic("or"), "atomicAnd": _atomic("and"), "atomicExchange": _atomic("exchange"),
}


# ---------------------------------------------------------------- compiler
# Statements compile to closures env -> signal (None, "break", "continue",
# "return"); expressions to closures env -> value. env is a dict of the
# invocation's locals ("$ret" holds a returned value).

class _Return(Exception):
    pass


class Module:
    """A parsed WGSL module with its storage bindings. Buffers are numpy
    arrays (uint32 / int32 / float32; rows of vectors as 2-D arrays) bound by
    variable name; the uniform struct is a dict of field values."""

    def __init__(self, src: str):
        self.items = Parser(lex(src)).module()
        self.consts = {}
        self.structs = {}
        self.gvars = {}
        self.fns = {}
        self.buffers = {}
        self.uniforms = {}
        self._compiled = {}
        for it in self.items:
            if it[0] == "struct":
                self.structs[it[1]] = it[2]
            elif it[0] == "gvar":
                self.gvars[it[1]] = it
            elif it[0] == "fn":
                self.fns[it[1]] = it
        for it in self.items:
            if it[0] == "const":
                v = self._expr(it[3], set())({})
                self.consts[it[1]] = to_type(v, it[2])

    # ---- bindings
    def bind(self, name: str, array: np.ndarray) -> None:
        if name not in self.gvars:
            raise KeyError(f"WGSL: no module variable {name}")
        self.buffers[name] = array

    def set_uniform(self, name: str, values: dict) -> None:
        ty = self.gvars[name][3]
        out = {}
        for fname, fty in self.structs[ty]:
            v = values[fname]
            if fty in _VEC_ALIAS:
                n, t = _VEC_ALIAS[fty]
                out[fname] = make_vec(n, t, list(v))
            else:
                out[fname] = conv(v, fty)
        self.uniforms[name] = out

    # ---- execution
    def dispatch(self, entry: str, workgroups: int) -> None:
        """dispatchWorkgroups(workgroups) of an entry point: invocations in
        global-id order."""
        with warnings.catch_warnings(), np.errstate(all="ignore"):
            # u32 / i32 arithmetic wraps and f32 may overflow to inf, as in WGSL
            warnings.simplefilter("ignore", RuntimeWarning)
            self._dispatch(entry, workgroups)

    def _dispatch(self, entry: str, workgroups: int) -> None:
        fn = self.fns[entry]
        size = int(fn[5]["workgroup_size"][0])
        body = self._function(entry)
        params = fn[2]
        for wg in range(workgroups):
            for lid in range(size):
                gid = wg * size + lid
                env = {}
                for pname, pty, pat in params:
                    b = pat.get("builtin", [None])[0]
                    if b == "global_invocation_id":
                        env[pname] = Vec([U32(gid), U32(0), U32(0)], "u32")
                    elif b == "local_invocation_id":
                        env[pname] = Vec([U32(lid), U32(0), U32(0)], "u32")
                    elif b == "workgroup_id":
                        env[pname] = Vec([U32(wg), U32(0), U32(0)], "u32")
                    elif b == "num_workgroups":
                        env[pname] = Vec([U32(workgroups), U32(1), U32(1)], "u32")
                    elif b == "local_invocation_index":
                        env[pname] = U32(lid)
                    else:
                        raise TypeError(f"WGSL: entry parameter {pname}")
                body(env)

    def _function(self, name):
        if name in self._compiled:
            return self._compiled[name]
        fn = self.fns[name]
        params, body = fn[2], fn[4]
        local = {p[0] for p in params} | _declared(body)
        run = self._stmt(body, local)
        self._compiled[name] = run
        return run

    def call(self, name, args):
        fn = self.fns[name]
        env = {p[0]: to_type(a, p[1]) for p, a in zip(fn[2], args)}
        self._function(name)(env)
        return env.get("$ret")

    # ---- statements
    def _stmt(self, s, local):
        k = s[0]
        if k == "block":
            parts = [self._stmt(x, local) for x in s[1]]

            def block(env):
                for p in parts:
                    r = p(env)
                    if r is not None:
                        return r
                return None
            return block
        if k == "decl":
            name, ty, e = s[1], s[2], s[3]
            if e is None:
                z = zero_of(ty)

                def decl0(env):
                    env[name] = z.copy() if isinstance(z, np.ndarray) else z
                return decl0
            f = self._expr(e, local)

            def decl(env):
                env[name] = to_type(f(env), ty)
            return decl
        if k == "assign":
            return self._assign(s[1], s[2], s[3], local)
        if k == "expr":
            f = self._expr(s[1], local)

            def ex(env):
                f(env)
            return ex
        if k == "if":
            c = self._expr(s[1], local)
            t = self._stmt(s[2], local)
            e = self._stmt(s[3], local) if s[3] is not None else None

            def if_(env):
                if c(env):
                    return t(env)
                if e is not None:
                    return e(env)
                return None
            return if_
        if k == "for":
            init = self._stmt(s[1], local) if s[1] is not None else None
            cond = self._expr(s[2], local) if s[2] is not None else None
            upd = self._stmt(s[3], local) if s[3] is not None else None
            body = self._stmt(s[4], local)

            def for_(env):
                if init is not None:
                    init(env)
                while cond is None or cond(env):
                    r = body(env)
                    if r == "break":
                        break
                    if r == "return":
                        return r
                    if upd is not None:
                        upd(env)
                return None
            return for_
        if k == "break":
            return lambda env: "break"
        if k == "continue":
            return lambda env: "continue"
        if k == "return":
            if s[1] is None:
                return lambda env: "return"
            f = self._expr(s[1], local)

            def ret(env):
                env["$ret"] = f(env)
                return "return"
            return ret
        raise SyntaxError(f"WGSL: statement {k}")

    def _assign(self, op, lhs, rhs, local):
        r = self._expr(rhs, local)
        bop = None if op == "=" else op[:-1]

        def combine(old, new):
            return new if bop is None else binop(bop, old, new)

        if lhs[0] == "name":
            name = lhs[1]
            if name in local:
                def set_local(env):
                    old = env.get(name)
                    v = combine(old, r(env))
                    env[name] = conv(v, tname(old)) if old is not None and not isinstance(old, np.ndarray) \
                        and tname(old) in _NP else (concrete(v) if old is None else v)
                return set_local
            raise SyntaxError(f"WGSL: assignment to {name}")
        if lhs[0] == "index":
            getarr = self._array(lhs[1], local)
            idx = self._expr(lhs[2], local)

            def set_elem(env):
                a = getarr(env)
                i = int(idx(env))
                old = _load(a, i)
                _store(a, i, combine(old, r(env)))
            return set_elem
        if lhs[0] == "member":
            base, comp = lhs[1], lhs[2]
            if base[0] == "name" and base[1] in local:
                name = base[1]

                def set_comp(env):
                    v = env[name]
                    old = swizzle(v, comp)
                    env[name] = with_comp(v, comp, combine(old, r(env)))
                return set_comp
            if base[0] == "index":
                getarr = self._array(base[1], local)
                idx = self._expr(base[2], local)

                def set_elem_comp(env):
                    a = getarr(env)
                    i = int(idx(env))
                    v = _load(a, i)
                    _store(a, i, with_comp(v, comp, combine(swizzle(v, comp), r(env))))
                return set_elem_comp
        raise SyntaxError(f"WGSL: assignment target {lhs[0]}")

    def _array(self, e, local):
        """The numpy array an index expression's base names."""
        if e[0] != "name":
            raise SyntaxError("WGSL: indexing supports named arrays only")
        name = e[1]
        if name in local:
            return lambda env: env[name]
        bufs = self.buffers

        def get(env):
            return bufs[name]
        return get

    # ---- expressions
    def _expr(self, e, local):
        k = e[0]
        if k == "num":
            t, v = e[1]
            val = conv(v, t) if t in _NP else v
            return lambda env: val
        if k == "bool":
            b = e[1]
            return lambda env: b
        if k == "name":
            name = e[1]
            if name in local:
                return lambda env: env[name]
            if name in self.consts:
                c = self.consts[name]
                return lambda env: c
            if name in self.gvars:
                gv = self.gvars[name]
                if "uniform" in gv[2]:
                    u = self.uniforms
                    return lambda env: u[name]
                bufs = self.buffers
                return lambda env: bufs[name]
            raise NameError(f"WGSL: unknown name {name}")
        if k == "bin":
            op = e[1]
            a, b = self._expr(e[2], local), self._expr(e[3], local)
            if op == "&&":
                return lambda env: bool(a(env)) and bool(b(env))
            if op == "||":
                return lambda env: bool(a(env)) or bool(b(env))
            return lambda env: binop(op, a(env), b(env))
        if k == "unary":
            op = e[1]
            if op == "&":
                inner = e[2]
                if inner[0] != "index":
                    raise SyntaxError("WGSL: & of a non-element")
                getarr = self._array(inner[1], local)
                idx = self._expr(inner[2], local)
                return lambda env: Ref(getarr(env), idx(env))
            a = self._expr(e[2], local)
            return lambda env: unop(op, a(env))
        if k == "index":
            getarr = self._array(e[1], local)
            idx = self._expr(e[2], local)
            return lambda env: _load(getarr(env), int(idx(env)))
        if k == "member":
            base = self._expr(e[1], local)
            m = e[2]

            def member(env):
                v = base(env)
                if isinstance(v, Vec):
                    return swizzle(v, m)
                return v[m]
            return member
        if k == "call":
            return self._call(e[1], e[2], [self._expr(a, local) for a in e[3]])
        raise SyntaxError(f"WGSL: expression {k}")

    def _call(self, name, targs, args):
        if name in _VEC_ALIAS:
            n, t = _VEC_ALIAS[name]
            return lambda env: make_vec(n, t, [a(env) for a in args])
        if name in ("f32", "u32", "i32", "bool"):
            a0 = args[0]
            return lambda env: conv(a0(env), name)
        if name == "bitcast":
            t = targs[0]
            a0 = args[0]
            return lambda env: _bitcast(a0(env), t)
        if name == "workgroupBarrier":
            raise NotImplementedError("WGSL: workgroupBarrier is not supported by this interpreter")
        if name in BUILTINS:
            f = BUILTINS[name]
            return lambda env: f(*[a(env) for a in args])
        if name in self.fns:
            mod = self
            return lambda env: mod.call(name, [a(env) for a in args])
        raise NameError(f"WGSL: unknown function {name}")


def _declared(s) -> set:
    """Names a function body declares (let / var / const), for resolution."""
    out = set()
    if isinstance(s, tuple):
        if s and s[0] == "decl":
            out.add(s[1])
        for x in s:
            out |= _declared(x)
    elif isinstance(s, list):
        for x in s:
            out |= _declared(x)
    return out


def _load(a: np.ndarray, i: int):
    if a.ndim == 2:
        t = {np.dtype(np.float32): "f32", np.dtype(np.uint32): "u32", np.dtype(np.int32): "i32"}[a.dtype]
        return Vec(a[i], t)
    return a.dtype.type(a[i])


def _store(a: np.ndarray, i: int, v) -> None:
    if a.ndim == 2:
        a[i] = [c for c in v.c]
    else:
        a[i] = v
