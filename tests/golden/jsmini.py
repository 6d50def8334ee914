"""jsmini — a small JavaScript interpreter (test infrastructure only).

No JavaScript engine exists on this machine, so the reference's CPU solver
(src/solver.js) and the host-side scene builder of src/gpu/sim.js cannot be
run as shipped. This interpreter executes those unmodified source files to
produce golden vectors that pin the C++ restatement (oracle O1) and the
scene builder of the CUDA library.

Semantics implemented (the subset those files use):
  - numbers are IEEE doubles (Python float); `^ & | << >>` apply ToInt32,
    `>>>` ToUint32; `/` and `%` follow IEEE (x/0 = +-Infinity or NaN);
  - Float32Array / Int32Array / Uint32Array / Uint8Array are views of an
    ArrayBuffer (memoryview casts, so views alias like in JS); stores round
    to float32 or wrap to the integer width exactly as a JS engine does;
  - classes, methods (async methods parse, run synchronously), arrow and
    nested functions, object/array literals with spread, destructuring
    (object patterns with defaults and renames, array patterns), for / for-of
    / while, `??`, `**`, ternaries, Set, Array.from, Math, Object.entries,
    Function.prototype.apply / call, String.fromCharCode and btoa.
Statements signal break/continue/return by return value (no exceptions in
hot loops). Performance: roughly 1-3 million AST nodes per second.
"""
from __future__ import annotations

import base64
import math
import re
import struct

# ---------------------------------------------------------------- values


class _Undef:
    def __repr__(self):
        return "undefined"


UNDEF = _Undef()


def to_number(v):
    if isinstance(v, float):
        return v
    if isinstance(v, bool):
        return 1.0 if v else 0.0
    if isinstance(v, int):
        return float(v)
    if v is None:
        return 0.0
    if v is UNDEF:
        return math.nan
    if isinstance(v, str):
        try:
            return float(v)
        except ValueError:
            return math.nan
    return math.nan


def js_to_string(v) -> str:
    """ToString of a primitive (template substitutions)."""
    if v is True:
        return "true"
    if v is False:
        return "false"
    if v is None:
        return "null"
    if v is UNDEF:
        return "undefined"
    if isinstance(v, (int, float)) and not isinstance(v, bool):
        f = float(v)
        if math.isnan(f):
            return "NaN"
        if math.isinf(f):
            return "Infinity" if f > 0 else "-Infinity"
        if f == int(f) and abs(f) < 1e21:
            return str(int(f))
        return repr(f)
    return str(v)


def to_int32(v) -> int:
    x = to_number(v)
    if not math.isfinite(x):
        return 0
    i = int(x) & 0xFFFFFFFF
    return i - 0x100000000 if i >= 0x80000000 else i


def to_uint32(v) -> int:
    x = to_number(v)
    if not math.isfinite(x):
        return 0
    return int(x) & 0xFFFFFFFF


def truthy(v) -> bool:
    if isinstance(v, bool):
        return v
    if isinstance(v, float):
        return not (v == 0.0 or v != v)
    if isinstance(v, int):
        return v != 0
    if v is None or v is UNDEF:
        return False
    if isinstance(v, str):
        return v != ""
    return True


def js_div(a, b):
    a, b = to_number(a), to_number(b)
    try:
        return a / b
    except ZeroDivisionError:
        if a != a or a == 0:
            return math.nan
        neg = (a < 0) != (math.copysign(1.0, b) < 0)
        return -math.inf if neg else math.inf


def js_mod(a, b):
    a, b = to_number(a), to_number(b)
    if b == 0 or a != a or b != b or math.isinf(a):
        return math.nan
    if math.isinf(b):
        return a
    return math.fmod(a, b)


def strict_eq(a, b):
    if isinstance(a, bool) or isinstance(b, bool):
        return type(a) is type(b) and a == b
    if isinstance(a, (float, int)) and isinstance(b, (float, int)):
        return float(a) == float(b)
    return a is b if not isinstance(a, str) else a == b


class JSObject:
    __slots__ = ("props", "proto")

    def __init__(self, props=None, proto=None):
        self.props = props if props is not None else {}
        self.proto = proto

    def get(self, k):
        o = self
        while o is not None:
            if k in o.props:
                return o.props[k]
            o = o.proto
        return UNDEF

    def set(self, k, v):
        self.props[k] = v


class JSArray:
    __slots__ = ("items",)

    def __init__(self, items=None):
        self.items = items if items is not None else []


class ArrayBuffer:
    __slots__ = ("buf",)

    def __init__(self, nbytes):
        self.buf = bytearray(int(nbytes))


class TypedArray:
    FMT = {"Float32Array": ("f", 4), "Float64Array": ("d", 8), "Int32Array": ("i", 4),
           "Uint32Array": ("I", 4), "Uint8Array": ("B", 1), "Int8Array": ("b", 1),
           "Uint16Array": ("H", 2), "Int16Array": ("h", 2)}
    __slots__ = ("kind", "fmt", "size", "buffer", "mv", "offset", "length", "_conv")

    def __init__(self, kind, buffer: ArrayBuffer, offset=0, length=None):
        self.kind = kind
        self.fmt, self.size = self.FMT[kind]
        self.buffer = buffer
        self.offset = int(offset)
        n = (len(buffer.buf) - self.offset) // self.size if length is None else int(length)
        self.length = n
        self.mv = memoryview(buffer.buf)[self.offset:self.offset + n * self.size].cast(self.fmt)
        f = self.fmt
        if f in "fd":
            self._conv = to_number
        elif f == "i":
            self._conv = to_int32
        elif f == "I":
            self._conv = to_uint32
        else:
            bits = self.size * 8
            signed = f.islower()
            mask = (1 << bits) - 1

            def conv(v, bits=bits, signed=signed, mask=mask):
                x = to_number(v)
                if not math.isfinite(x):
                    return 0
                i = int(x) & mask
                return i - (1 << bits) if signed and i >= (1 << (bits - 1)) else i
            self._conv = conv

    def getitem(self, i):
        i = int(i)
        if 0 <= i < self.length:
            return float(self.mv[i])
        return UNDEF

    def setitem(self, i, v):
        i = int(i)
        if 0 <= i < self.length:
            self.mv[i] = self._conv(v)


class Fn:
    """A callable value: native (py(this, args)) or compiled JS."""
    __slots__ = ("call", "props", "name")

    def __init__(self, call, name=""):
        self.call = call
        self.props = {}
        self.name = name


class JSClass(Fn):
    __slots__ = ("proto", "ctor", "parent", "native")

    def __init__(self, name, ctor, proto, parent=None, native=None):
        super().__init__(None, name)
        self.ctor = ctor
        self.proto = proto
        self.parent = parent
        self.native = native

    def construct(self, args):
        if self.native is not None:
            return self.native(args)
        obj = JSObject(proto=self.proto)
        if self.ctor is not None:
            self.ctor.call(obj, args)
        return obj


class JSSet:
    __slots__ = ("s",)

    def __init__(self):
        self.s = set()


def _key(v):
    if isinstance(v, float) and v == int(v) and math.isfinite(v):
        return int(v)
    return v


# ---------------------------------------------------------------- lexer

TOKEN_RE = re.compile(r"""
  (?P<ws>[ \t\r]+)|(?P<nl>\n)|(?P<lc>//[^\n]*)|(?P<bc>/\*.*?\*/)|
  (?P<num>0[xX][0-9a-fA-F]+|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)|
  (?P<str>'(?:[^'\\\n]|\\.)*'|"(?:[^"\\\n]|\\.)*")|
  (?P<id>[A-Za-z_$][A-Za-z0-9_$]*)|
  (?P<op>>>>=|>>>|\.\.\.|===|!==|\*\*=|<<=|>>=|\?\?=|\?\?|\?\.|=>|==|!=|<=|>=|&&|\|\||\+\+|--|
        \+=|-=|\*=|/=|%=|&=|\|=|\^=|\*\*|<<|>>|[{}()\[\];,.<>+\-*/%&|^!~?:=])
""", re.S | re.X)


class Tok:
    __slots__ = ("kind", "val", "nl", "pos")

    def __init__(self, kind, val, nl, pos):
        self.kind, self.val, self.nl, self.pos = kind, val, nl, pos

    def __repr__(self):
        return f"{self.kind}:{self.val}"


_TPL_ESC = {"n": "\n", "t": "\t", "r": "\r", "\\": "\\", "`": "`", "$": "$", "'": "'", '"': '"', "0": "\0"}


def _lex_template(src: str, i: int):
    """A template literal starting at the backtick src[i]: returns (cooked
    text parts, substitution sources, index after the closing backtick)."""
    j = i + 1
    parts, subs, buf = [], [], []
    while True:
        if j >= len(src):
            raise SyntaxError("unterminated template literal")
        c = src[j]
        if c == "\\":
            nxt = src[j + 1]
            buf.append(_TPL_ESC.get(nxt, nxt))
            j += 2
            continue
        if c == "`":
            break
        if c == "$" and src[j + 1:j + 2] == "{":
            parts.append("".join(buf))
            buf = []
            depth, k = 1, j + 2
            while depth:
                ch = src[k]
                if ch in "'\"":  # a quoted string inside the substitution
                    k += 1
                    while src[k] != ch:
                        k += 2 if src[k] == "\\" else 1
                elif ch == "{":
                    depth += 1
                elif ch == "}":
                    depth -= 1
                k += 1
            subs.append(src[j + 2:k - 1])
            j = k
            continue
        buf.append(c)
        j += 1
    parts.append("".join(buf))
    return parts, subs, j + 1


def lex(src: str) -> list[Tok]:
    out = []
    nl = False
    i = 0
    while i < len(src):
        if src[i] == "`":
            parts, subs, i2 = _lex_template(src, i)
            out.append(Tok("tpl", (parts, [lex(x) for x in subs]), nl, i))
            nl = False
            i = i2
            continue
        m = TOKEN_RE.match(src, i)
        if not m:
            raise SyntaxError(f"bad char {src[i]!r} at {i}")
        i = m.end()
        k = m.lastgroup
        v = m.group()
        if k in ("ws", "lc"):
            continue
        if k == "nl" or (k == "bc" and "\n" in v):
            nl = True
            continue
        if k == "bc":
            continue
        if k == "num":
            v = float(int(v, 16)) if v[:2] in ("0x", "0X") else float(v)
        elif k == "str":
            v = bytes(v[1:-1], "utf-8").decode("unicode_escape")
        out.append(Tok(k, v, nl, m.start()))
        nl = False
    out.append(Tok("eof", None, True, len(src)))
    return out


# ---------------------------------------------------------------- parser
# AST nodes are tuples: (type, ...).

KEYWORDS = {"const", "let", "var", "if", "else", "for", "while", "do", "return", "break", "continue",
            "function", "class", "new", "this", "true", "false", "null", "undefined", "of", "in",
            "export", "import", "from", "async", "await", "extends", "super", "typeof"}

BINARY_PREC = {
    "??": 1, "||": 2, "&&": 3, "|": 4, "^": 5, "&": 6,
    "==": 7, "!=": 7, "===": 7, "!==": 7,
    "<": 8, ">": 8, "<=": 8, ">=": 8, "instanceof": 8, "in": 8,
    "<<": 9, ">>": 9, ">>>": 9,
    "+": 10, "-": 10, "*": 11, "/": 11, "%": 11, "**": 12,
}
ASSIGN_OPS = {"=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>=", ">>>=", "**=", "??="}


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

    def at(self, val, k=0):
        tok = self.t[self.i + k]
        return tok.kind in ("op", "id") and tok.val == val

    def eat(self, val):
        if self.at(val):
            self.i += 1
            return True
        return False

    def expect(self, val):
        tok = self.next()
        if tok.val != val:
            raise SyntaxError(f"expected {val!r}, got {tok.val!r} at {tok.pos}")
        return tok

    def semi(self):
        if self.eat(";"):
            return
        tok = self.peek()
        if tok.val == "}" or tok.kind == "eof" or tok.nl:
            return
        raise SyntaxError(f"expected ';' at {tok.pos}, got {tok.val!r}")

    # -- program / statements
    def program(self):
        body = []
        while self.peek().kind != "eof":
            body.append(self.statement())
        return ("block", body)

    def statement(self):
        tok = self.peek()
        if tok.kind == "op" and tok.val == "{":
            return self.block()
        if tok.kind == "op" and tok.val == ";":
            self.next()
            return ("empty",)
        if tok.kind == "id":
            v = tok.val
            if v == "import":
                while not self.eat(";"):
                    self.next()
                return ("empty",)
            if v == "export":
                self.next()
                if self.eat("default"):
                    pass
                return self.statement()
            if v in ("const", "let", "var"):
                s = self.vardecl()
                self.semi()
                return s
            if v == "if":
                self.next()
                self.expect("(")
                c = self.expression()
                self.expect(")")
                a = self.statement()
                b = self.statement() if self.eat("else") else None
                return ("if", c, a, b)
            if v == "for":
                return self.for_stmt()
            if v == "while":
                self.next()
                self.expect("(")
                c = self.expression()
                self.expect(")")
                return ("while", c, self.statement())
            if v == "return":
                self.next()
                tok2 = self.peek()
                if tok2.val in (";", "}") or tok2.nl or tok2.kind == "eof":
                    self.semi()
                    return ("return", None)
                e = self.expression()
                self.semi()
                return ("return", e)
            if v == "break":
                self.next()
                self.semi()
                return ("break",)
            if v == "continue":
                self.next()
                self.semi()
                return ("continue",)
            if v == "class":
                return self.class_decl()
            if v == "function" or (v == "async" and self.at("function", 1)):
                if v == "async":
                    self.next()
                return self.function_decl()
        e = self.expression()
        self.semi()
        return ("expr", e)

    def block(self):
        self.expect("{")
        body = []
        while not self.eat("}"):
            body.append(self.statement())
        return ("block", body)

    def vardecl(self):
        kind = self.next().val
        decls = []
        while True:
            target = self.binding_target()
            init = self.assign() if self.eat("=") else None
            decls.append((target, init))
            if not self.eat(","):
                break
        return ("var", kind, decls)

    def binding_target(self):
        if self.at("{"):
            return self.object_pattern()
        if self.at("["):
            return self.array_pattern()
        tok = self.next()
        if tok.kind != "id":
            raise SyntaxError(f"binding name expected at {tok.pos}")
        return ("id", tok.val)

    def object_pattern(self):
        self.expect("{")
        props = []
        while not self.eat("}"):
            key = self.next().val
            if self.eat(":"):
                target = self.binding_target()
            else:
                target = ("id", key)
            default = self.assign() if self.eat("=") else None
            props.append((key, target, default))
            if not self.eat(","):
                self.expect("}")
                break
        return ("opat", props)

    def array_pattern(self):
        self.expect("[")
        elems = []
        while not self.eat("]"):
            target = self.binding_target()
            default = self.assign() if self.eat("=") else None
            elems.append((target, default))
            if not self.eat(","):
                self.expect("]")
                break
        return ("apat", elems)

    def for_stmt(self):
        self.expect("for")
        self.expect("(")
        if self.peek().val in ("const", "let", "var"):
            save = self.i
            kind = self.next().val
            target = self.binding_target()
            if self.eat("of"):
                it = self.assign()
                self.expect(")")
                return ("forof", kind, target, it, self.statement())
            self.i = save
            init = self.vardecl()
        elif self.at(";"):
            init = None
        else:
            init = ("expr", self.expression())
        self.expect(";")
        cond = None if self.at(";") else self.expression()
        self.expect(";")
        upd = None if self.at(")") else self.expression()
        self.expect(")")
        return ("for", init, cond, upd, self.statement())

    def params(self):
        self.expect("(")
        ps = []
        while not self.eat(")"):
            if self.eat("..."):
                ps.append(("rest", self.binding_target(), None))
            else:
                target = self.binding_target()
                default = self.assign() if self.eat("=") else None
                ps.append(("p", target, default))
            if not self.eat(","):
                self.expect(")")
                break
        return ps

    def function_decl(self):
        self.expect("function")
        name = self.next().val
        ps = self.params()
        body = self.block()
        return ("var", "let", [(("id", name), ("func", name, ps, body, False))])

    def class_decl(self):
        self.expect("class")
        name = self.next().val
        parent = None
        if self.eat("extends"):
            parent = self.lhs()
        self.expect("{")
        methods = []
        while not self.eat("}"):
            if self.eat(";"):
                continue
            is_static = False
            if self.at("static") and not self.at("(", 1):
                self.next()
                is_static = True
            if self.at("async") and not self.at("(", 1):
                self.next()
            mname = self.next().val
            ps = self.params()
            body = self.block()
            methods.append((mname, ps, body, is_static))
        return ("class", name, parent, methods)

    # -- expressions
    def expression(self):
        e = self.assign()
        if self.at(","):
            seq = [e]
            while self.eat(","):
                seq.append(self.assign())
            return ("seq", seq)
        return e

    def is_arrow(self):
        # ( ... ) =>   or   id =>
        tok = self.peek()
        if tok.kind == "id" and self.at("=>", 1):
            return True
        if not self.at("("):
            return False
        depth = 0
        j = self.i
        while True:
            t = self.t[j]
            if t.kind == "eof":
                return False
            if t.kind == "op" and t.val in "([{":
                depth += 1
            elif t.kind == "op" and t.val in ")]}":
                depth -= 1
                if depth == 0:
                    nx = self.t[j + 1]
                    return nx.kind == "op" and nx.val == "=>"
            j += 1

    def arrow(self):
        if self.peek().kind == "id" and not self.at("("):
            ps = [("p", ("id", self.next().val), None)]
        else:
            ps = self.params()
        self.expect("=>")
        if self.at("{"):
            body = self.block()
        else:
            body = ("block", [("return", self.assign())])
        return ("func", "", ps, body, True)

    def assign(self):
        if self.at("async") and (self.at("(", 1) or (self.peek(1).kind == "id" and self.at("=>", 2))):
            self.next()
        if self.is_arrow():
            return self.arrow()
        left = self.conditional()
        tok = self.peek()
        if tok.kind == "op" and tok.val in ASSIGN_OPS:
            self.next()
            right = self.assign()
            return ("assign", tok.val, left, right)
        return left

    def conditional(self):
        c = self.binary(1)
        if self.eat("?"):
            a = self.assign()
            self.expect(":")
            b = self.assign()
            return ("cond", c, a, b)
        return c

    def binary(self, min_prec):
        left = self.unary()
        while True:
            tok = self.peek()
            op = tok.val if tok.kind in ("op", "id") else None
            prec = BINARY_PREC.get(op)
            if prec is None or prec < min_prec:
                return left
            self.next()
            right = self.binary(prec if op == "**" else prec + 1)
            left = ("logic", op, left, right) if op in ("&&", "||", "??") else ("bin", op, left, right)

    def unary(self):
        tok = self.peek()
        if tok.kind == "op" and tok.val in ("!", "-", "+", "~"):
            self.next()
            return ("unary", tok.val, self.unary())
        if tok.kind == "op" and tok.val in ("++", "--"):
            self.next()
            return ("update", tok.val, True, self.unary())
        if tok.kind == "id" and tok.val in ("typeof", "await"):
            self.next()
            e = self.unary()
            return ("typeof", e) if tok.val == "typeof" else e
        e = self.postfix()
        return e

    def postfix(self):
        e = self.lhs()
        tok = self.peek()
        if tok.kind == "op" and tok.val in ("++", "--") and not tok.nl:
            self.next()
            return ("update", tok.val, False, e)
        return e

    def args(self):
        self.expect("(")
        out = []
        while not self.eat(")"):
            if self.eat("..."):
                out.append(("spread", self.assign()))
            else:
                out.append(self.assign())
            if not self.eat(","):
                self.expect(")")
                break
        return out

    def lhs(self):
        if self.at("new"):
            self.next()
            callee = self.member_only(self.primary())
            a = self.args() if self.at("(") else []
            e = ("new", callee, a)
        else:
            e = self.primary()
        while True:
            if self.eat("."):
                e = ("member", e, self.next().val)
            elif self.at("?."):
                self.next()
                e = ("member", e, self.next().val)
            elif self.at("["):
                self.next()
                k = self.expression()
                self.expect("]")
                e = ("index", e, k)
            elif self.at("("):
                e = ("call", e, self.args())
            else:
                return e

    def member_only(self, e):
        while True:
            if self.eat("."):
                e = ("member", e, self.next().val)
            elif self.at("["):
                self.next()
                k = self.expression()
                self.expect("]")
                e = ("index", e, k)
            else:
                return e

    def primary(self):
        tok = self.next()
        if tok.kind == "num":
            return ("num", tok.val)
        if tok.kind == "str":
            return ("str", tok.val)
        if tok.kind == "tpl":
            parts, subs = tok.val
            return ("tpl", tuple(parts), tuple(Parser(t).expression() for t in subs))
        if tok.kind == "id":
            v = tok.val
            if v == "this":
                return ("this",)
            if v == "true":
                return ("lit", True)
            if v == "false":
                return ("lit", False)
            if v == "null":
                return ("lit", None)
            if v == "undefined":
                return ("lit", UNDEF)
            if v == "function":
                name = self.next().val if self.peek().kind == "id" else ""
                ps = self.params()
                return ("func", name, ps, self.block(), False)
            return ("name", v)
        if tok.kind == "op":
            if tok.val == "(":
                e = self.expression()
                self.expect(")")
                return e
            if tok.val == "[":
                items = []
                while not self.eat("]"):
                    if self.eat("..."):
                        items.append(("spread", self.assign()))
                    else:
                        items.append(self.assign())
                    if not self.eat(","):
                        self.expect("]")
                        break
                return ("array", items)
            if tok.val == "{":
                props = []
                while not self.eat("}"):
                    if self.eat("..."):
                        props.append(("spread", self.assign()))
                    else:
                        kt = self.next()
                        key = kt.val if kt.kind != "num" else repr(int(kt.val))
                        if self.eat(":"):
                            props.append(("kv", key, self.assign()))
                        elif self.at("("):
                            ps = self.params()
                            props.append(("kv", key, ("func", key, ps, self.block(), False)))
                        else:
                            props.append(("kv", key, ("name", key)))
                    if not self.eat(","):
                        self.expect("}")
                        break
                return ("object", props)
        raise SyntaxError(f"unexpected {tok.val!r} at {tok.pos}")


# ---------------------------------------------------------------- runtime

BREAK = ("break",)
CONTINUE = ("continue",)


class Scope:
    __slots__ = ("vars", "parent", "this")

    def __init__(self, parent=None, this=UNDEF):
        self.vars = {}
        self.parent = parent
        self.this = this

    def lookup(self, name):
        s = self
        while s is not None:
            v = s.vars
            if name in v:
                return v[name]
            s = s.parent
        raise NameError(f"{name} is not defined")

    def assign(self, name, val):
        s = self
        while s is not None:
            if name in s.vars:
                s.vars[name] = val
                return
            s = s.parent
        raise NameError(f"assignment to undeclared {name}")


def get_member(obj, key):
    if isinstance(obj, TypedArray):
        if isinstance(key, float):
            return obj.getitem(key)
        return _typed_method(obj, key)
    if isinstance(obj, JSArray):
        if isinstance(key, float):
            i = int(key)
            return obj.items[i] if 0 <= i < len(obj.items) else UNDEF
        return _array_method(obj, key)
    if isinstance(obj, JSObject):
        return obj.get(_prop_key(key))
    if isinstance(obj, JSClass):
        return obj.props.get(key, UNDEF)
    if isinstance(obj, Fn):
        if key in obj.props:
            return obj.props[key]
        if key == "apply":  # f.apply(thisArg, argsArrayLike)
            def ap(this, a, f=obj):
                lst = a[1] if len(a) > 1 else UNDEF
                return call(f, a[0] if a else UNDEF, [] if lst is None or lst is UNDEF else iterate(lst))
            return Fn(ap)
        if key == "call":
            return Fn(lambda this, a, f=obj: call(f, a[0] if a else UNDEF, list(a[1:])))
        return UNDEF
    if isinstance(obj, JSSet):
        return _set_method(obj, key)
    if isinstance(obj, ArrayBuffer):
        if key == "byteLength":
            return float(len(obj.buf))
        return UNDEF
    if isinstance(obj, str):
        if key == "length":
            return float(len(obj))
        return UNDEF
    if obj is None or obj is UNDEF:
        raise TypeError(f"cannot read property {key!r} of {obj}")
    return UNDEF


def _prop_key(key):
    if isinstance(key, float):
        return repr(int(key)) if key == int(key) else repr(key)
    return key


def set_member(obj, key, val):
    if isinstance(obj, TypedArray):
        obj.setitem(key, val)
    elif isinstance(obj, JSArray):
        if key == "length":
            n = int(val)
            del obj.items[n:]
            return
        i = int(key)
        while len(obj.items) <= i:
            obj.items.append(UNDEF)
        obj.items[i] = val
    elif isinstance(obj, JSObject):
        obj.props[_prop_key(key)] = val
    elif isinstance(obj, Fn):
        obj.props[key] = val
    else:
        raise TypeError(f"cannot set {key!r} on {type(obj).__name__}")


def call(fn, this, args):
    if not isinstance(fn, Fn) or fn.call is None:
        raise TypeError(f"{fn!r} is not a function")
    return fn.call(this, args)


def iterate(v):
    if isinstance(v, JSArray):
        return list(v.items)
    if isinstance(v, TypedArray):
        return [v.getitem(float(i)) for i in range(v.length)]
    if isinstance(v, JSSet):
        return list(v.s)
    raise TypeError("not iterable")


def _num_arg(args, k, default=None):
    return to_number(args[k]) if len(args) > k and args[k] is not UNDEF else default


def _typed_method(a: TypedArray, key):
    if key == "length":
        return float(a.length)
    if key == "buffer":
        return a.buffer
    if key == "fill":
        def fill(this, args):
            v = args[0] if args else UNDEF
            s = int(_rel(_num_arg(args, 1, 0.0), a.length))
            e = int(_rel(_num_arg(args, 2, float(a.length)), a.length))
            cv = a._conv(v)
            for i in range(s, e):
                a.mv[i] = cv
            return a
        return Fn(fill)
    if key == "slice" or key == "subarray":
        def sl(this, args, sub=(key == "subarray")):
            s = int(_rel(_num_arg(args, 0, 0.0), a.length))
            e = int(_rel(_num_arg(args, 1, float(a.length)), a.length))
            n = max(0, e - s)
            if sub:
                return TypedArray(a.kind, a.buffer, a.offset + s * a.size, n)
            b = TypedArray(a.kind, ArrayBuffer(n * a.size))
            b.mv[:] = a.mv[s:s + n]
            return b
        return Fn(sl)
    if key == "set":
        def st(this, args):
            src = args[0]
            off = int(_num_arg(args, 1, 0.0))
            vals = iterate(src)
            for k, v in enumerate(vals):
                a.setitem(off + k, v)
            return UNDEF
        return Fn(st)
    return UNDEF


def _rel(x, n):
    x = int(x) if math.isfinite(x) else (n if x > 0 else 0)
    return max(n + x, 0) if x < 0 else min(x, n)


def _array_method(a: JSArray, key):
    if key == "length":
        return float(len(a.items))
    if key == "push":
        def push(this, args):
            a.items.extend(args)
            return float(len(a.items))
        return Fn(push)
    if key == "slice":
        def sl(this, args):
            n = len(a.items)
            s = int(_rel(_num_arg(args, 0, 0.0), n))
            e = int(_rel(_num_arg(args, 1, float(n)), n))
            return JSArray(a.items[s:e])
        return Fn(sl)
    if key == "forEach":
        def fe(this, args):
            f = args[0]
            for i, v in enumerate(list(a.items)):
                call(f, UNDEF, [v, float(i), a])
            return UNDEF
        return Fn(fe)
    if key == "map":
        def mp(this, args):
            f = args[0]
            return JSArray([call(f, UNDEF, [v, float(i), a]) for i, v in enumerate(a.items)])
        return Fn(mp)
    if key == "shift":
        return Fn(lambda this, args: a.items.pop(0) if a.items else UNDEF)
    if key == "pop":
        return Fn(lambda this, args: a.items.pop() if a.items else UNDEF)
    if key == "indexOf":
        def io(this, args):
            for i, v in enumerate(a.items):
                if strict_eq(v, args[0]):
                    return float(i)
            return -1.0
        return Fn(io)
    return UNDEF


def _set_method(s: JSSet, key):
    if key == "add":
        def add(this, args):
            s.s.add(_key(args[0]))
            return s
        return Fn(add)
    if key == "has":
        return Fn(lambda this, args: _key(args[0]) in s.s)
    if key == "delete":
        def de(this, args):
            k = _key(args[0])
            if k in s.s:
                s.s.discard(k)
                return True
            return False
        return Fn(de)
    if key == "clear":
        return Fn(lambda this, args: s.s.clear())
    if key == "size":
        return float(len(s.s))
    return UNDEF


def _math():
    def m1(f):
        def g(this, args):
            x = to_number(args[0]) if args else math.nan
            try:
                return f(x)
            except (ValueError, OverflowError):
                return math.nan
        return Fn(g)

    def floor(x):
        return x if not math.isfinite(x) else float(math.floor(x))

    def ceil(x):
        return x if not math.isfinite(x) else float(math.ceil(x))

    def sqrt(x):
        return math.sqrt(x) if x >= 0 else (math.nan if x != 0 else x)

    def sign(x):
        if x != x:
            return math.nan
        return 1.0 if x > 0 else (-1.0 if x < 0 else x)

    def rnd(x):
        return x if not math.isfinite(x) else float(math.floor(x + 0.5))

    def log2(x):
        if x != x or x < 0:
            return math.nan
        if x == 0:
            return -math.inf
        return math.log2(x)

    def cbrt(x):
        return math.copysign(abs(x) ** (1.0 / 3.0), x)

    def mmax(this, args):
        r = -math.inf
        for a in args:
            x = to_number(a)
            if x != x:
                return math.nan
            if x > r or (x == 0 and r == 0 and math.copysign(1, r) < 0):
                r = x
        return r

    def mmin(this, args):
        r = math.inf
        for a in args:
            x = to_number(a)
            if x != x:
                return math.nan
            if x < r or (x == 0 and r == 0 and math.copysign(1, x) < 0):
                r = x
        return r

    M = JSObject()
    for name, f in dict(floor=floor, ceil=ceil, sqrt=sqrt, abs=abs, sign=sign, round=rnd, log2=log2,
                        cbrt=cbrt, sin=math.sin, cos=math.cos, trunc=lambda x: x if not math.isfinite(x)
                        else float(math.trunc(x))).items():
        M.set(name, m1(f))
    M.set("max", Fn(mmax))
    M.set("min", Fn(mmin))
    M.set("PI", math.pi)
    M.set("hypot", Fn(lambda this, a: math.hypot(*[to_number(x) for x in a])))
    return M


def make_globals():
    g = Scope()
    g.vars["Math"] = _math()
    g.vars["Infinity"] = math.inf
    g.vars["NaN"] = math.nan

    def typed_ctor(kind):
        size = TypedArray.FMT[kind][1]

        def construct(args):
            a0 = args[0] if args else 0.0
            if isinstance(a0, ArrayBuffer):
                off = _num_arg(args, 1, 0.0)
                ln = _num_arg(args, 2, None)
                return TypedArray(kind, a0, off, ln)
            if isinstance(a0, (JSArray, TypedArray)):
                vals = iterate(a0)
                t = TypedArray(kind, ArrayBuffer(len(vals) * size))
                for i, v in enumerate(vals):
                    t.setitem(i, v)
                return t
            return TypedArray(kind, ArrayBuffer(int(to_number(a0)) * size))
        return JSClass(kind, None, None, native=construct)

    for kind in TypedArray.FMT:
        g.vars[kind] = typed_ctor(kind)
    g.vars["Set"] = JSClass("Set", None, None, native=lambda args: JSSet())
    arr = Fn(None, "Array")

    def from_(this, args):
        src, f = args[0], (args[1] if len(args) > 1 else None)
        if isinstance(src, JSObject):
            n = int(to_number(src.get("length")))
            vals = [UNDEF] * n
        else:
            vals = iterate(src)
        if f is not None:
            vals = [call(f, UNDEF, [v, float(i)]) for i, v in enumerate(vals)]
        return JSArray(vals)
    arr.props["from"] = Fn(from_)
    arr.props["isArray"] = Fn(lambda this, a: isinstance(a[0], JSArray))
    g.vars["Array"] = arr
    obj = Fn(None, "Object")
    obj.props["entries"] = Fn(lambda this, a: JSArray([JSArray([k, v]) for k, v in a[0].props.items()]))
    obj.props["keys"] = Fn(lambda this, a: JSArray(list(a[0].props.keys())))
    g.vars["Object"] = obj
    st = Fn(None, "String")
    st.props["fromCharCode"] = Fn(lambda this, a: "".join(chr(to_uint32(x) & 0xFFFF) for x in a))
    g.vars["String"] = st

    def btoa(this, a):
        t = a[0] if a and isinstance(a[0], str) else ""
        if any(ord(ch) > 255 for ch in t):
            raise ValueError("btoa: InvalidCharacterError (a character above U+00FF)")
        return base64.b64encode(t.encode("latin-1")).decode("ascii")
    g.vars["btoa"] = Fn(btoa)
    return g


# ---------------------------------------------------------------- compiler

def bin_op(op):
    if op == "+":
        def f(a, b):
            if isinstance(a, str) or isinstance(b, str):
                return str(a) + str(b)
            return to_number(a) + to_number(b)
        return f
    if op == "-":
        return lambda a, b: to_number(a) - to_number(b)
    if op == "*":
        return lambda a, b: to_number(a) * to_number(b)
    if op == "/":
        return js_div
    if op == "%":
        return js_mod
    if op == "**":
        def pw(a, b):
            a, b = to_number(a), to_number(b)
            try:
                return math.pow(a, b)
            except (OverflowError, ValueError):
                return math.nan if a < 0 else math.inf
        return pw
    if op == "<":
        return lambda a, b: to_number(a) < to_number(b)
    if op == ">":
        return lambda a, b: to_number(a) > to_number(b)
    if op == "<=":
        return lambda a, b: to_number(a) <= to_number(b)
    if op == ">=":
        return lambda a, b: to_number(a) >= to_number(b)
    if op in ("===", "=="):
        return strict_eq
    if op in ("!==", "!="):
        return lambda a, b: not strict_eq(a, b)
    if op == "^":
        return lambda a, b: float(to_int32(to_int32(a) ^ to_int32(b)))
    if op == "&":
        return lambda a, b: float(to_int32(to_int32(a) & to_int32(b)))
    if op == "|":
        return lambda a, b: float(to_int32(to_int32(a) | to_int32(b)))
    if op == "<<":
        return lambda a, b: float(to_int32(to_int32(a) << (to_uint32(b) & 31)))
    if op == ">>":
        return lambda a, b: float(to_int32(a) >> (to_uint32(b) & 31))
    if op == ">>>":
        return lambda a, b: float(to_uint32(a) >> (to_uint32(b) & 31))
    if op == "instanceof":
        return lambda a, b: isinstance(a, JSObject) and isinstance(b, JSClass) and a.proto is b.proto
    raise SyntaxError(f"operator {op}")


class Compiler:
    def expr(self, n):
        t = n[0]
        m = getattr(self, "e_" + t)
        return m(n)

    def e_num(self, n):
        v = float(n[1])
        return lambda env: v

    def e_str(self, n):
        v = n[1]
        return lambda env: v

    def e_lit(self, n):
        v = n[1]
        return lambda env: v

    def e_tpl(self, n):
        # template literal: the text parts with each substitution's ToString
        parts = n[1]
        subs = [self.expr(x) for x in n[2]]

        def f(env):
            out = [parts[0]]
            for k, g in enumerate(subs):
                out.append(js_to_string(g(env)))
                out.append(parts[k + 1])
            return "".join(out)
        return f

    def e_this(self, n):
        def f(env):
            s = env
            while s is not None:
                if s.this is not UNDEF:
                    return s.this
                s = s.parent
            return UNDEF
        return f

    def e_name(self, n):
        name = n[1]

        def f(env):
            s = env
            while s is not None:
                v = s.vars
                if name in v:
                    return v[name]
                s = s.parent
            raise NameError(f"{name} is not defined")
        return f

    def e_member(self, n):
        o = self.expr(n[1])
        key = n[2]
        return lambda env: get_member(o(env), key)

    def e_index(self, n):
        o = self.expr(n[1])
        k = self.expr(n[2])

        def f(env):
            obj = o(env)
            key = k(env)
            if isinstance(obj, TypedArray):
                i = int(key)
                if 0 <= i < obj.length:
                    return float(obj.mv[i])
                return UNDEF
            if isinstance(key, (int, bool)):
                key = float(key)
            return get_member(obj, key)
        return f

    def e_seq(self, n):
        fs = [self.expr(x) for x in n[1]]

        def f(env):
            v = UNDEF
            for g in fs:
                v = g(env)
            return v
        return f

    def e_cond(self, n):
        c, a, b = self.expr(n[1]), self.expr(n[2]), self.expr(n[3])
        return lambda env: a(env) if truthy(c(env)) else b(env)

    def e_logic(self, n):
        op, a, b = n[1], self.expr(n[2]), self.expr(n[3])
        if op == "&&":
            def f(env):
                x = a(env)
                return b(env) if truthy(x) else x
        elif op == "||":
            def f(env):
                x = a(env)
                return x if truthy(x) else b(env)
        else:
            def f(env):
                x = a(env)
                return b(env) if (x is None or x is UNDEF) else x
        return f

    def e_bin(self, n):
        op = bin_op(n[1])
        a, b = self.expr(n[2]), self.expr(n[3])
        return lambda env: op(a(env), b(env))

    def e_unary(self, n):
        op, a = n[1], self.expr(n[2])
        if op == "-":
            return lambda env: -to_number(a(env))
        if op == "+":
            return lambda env: to_number(a(env))
        if op == "!":
            return lambda env: not truthy(a(env))
        return lambda env: float(to_int32(~to_int32(a(env))))

    def e_typeof(self, n):
        a = self.expr(n[1])

        def f(env):
            v = a(env)
            if isinstance(v, bool):
                return "boolean"
            if isinstance(v, float):
                return "number"
            if isinstance(v, str):
                return "string"
            if v is UNDEF:
                return "undefined"
            if isinstance(v, Fn):
                return "function"
            return "object"
        return f

    def _setter(self, target):
        t = target[0]
        if t == "name":
            name = target[1]
            return lambda env, v: env.assign(name, v)
        if t == "member":
            o = self.expr(target[1])
            key = target[2]
            return lambda env, v: set_member(o(env), key, v)
        if t == "index":
            o = self.expr(target[1])
            k = self.expr(target[2])

            def f(env, v):
                obj = o(env)
                key = k(env)
                if isinstance(obj, TypedArray):
                    i = int(key)
                    if 0 <= i < obj.length:
                        obj.mv[i] = obj._conv(v)
                    return
                set_member(obj, key, v)
            return f
        raise SyntaxError(f"bad assignment target {t}")

    def _ref(self, target):
        """(getter, setter) evaluating the object/key once."""
        t = target[0]
        if t == "name":
            name = target[1]
            return (lambda env: (env,)), (lambda r: r[0].lookup(name)), (lambda r, v: r[0].assign(name, v))
        if t == "member":
            o = self.expr(target[1])
            key = target[2]
            return (lambda env: (o(env), key)), (lambda r: get_member(r[0], r[1])), \
                (lambda r, v: set_member(r[0], r[1], v))
        if t == "index":
            o = self.expr(target[1])
            k = self.expr(target[2])

            def loc(env):
                key = k(env)
                if isinstance(key, (int, bool)):
                    key = float(key)
                return (o(env), key)
            return loc, (lambda r: get_member(r[0], r[1])), (lambda r, v: set_member(r[0], r[1], v))
        raise SyntaxError("bad target")

    def e_assign(self, n):
        op, target, value = n[1], n[2], self.expr(n[3])
        if op == "=":
            if target[0] in ("object", "array"):
                pat = self._pattern_from_literal(target)
                bind = self.binder(pat, declare=False)

                def f(env):
                    v = value(env)
                    bind(env, v)
                    return v
                return f
            st = self._setter(target)

            def f(env):
                v = value(env)
                st(env, v)
                return v
            return f
        if op == "??=":
            loc, get, put = self._ref(target)

            def f(env):
                r = loc(env)
                cur = get(r)
                if cur is None or cur is UNDEF:
                    cur = value(env)
                    put(r, cur)
                return cur
            return f
        bop = bin_op(op[:-1])
        loc, get, put = self._ref(target)

        def f(env):
            r = loc(env)
            v = bop(get(r), value(env))
            put(r, v)
            return v
        return f

    def _pattern_from_literal(self, lit):
        if lit[0] == "array":
            return ("apat", [((x[0], x[1]) if x[0] == "name" else x, None) for x in lit[1]])
        raise SyntaxError("object assignment pattern")

    def e_update(self, n):
        op, prefix, target = n[1], n[2], n[3]
        d = 1.0 if op == "++" else -1.0
        loc, get, put = self._ref(target)

        def f(env):
            r = loc(env)
            old = to_number(get(r))
            new = old + d
            put(r, new)
            return new if prefix else old
        return f

    def _args(self, args):
        fs = []
        spread = False
        for a in args:
            if a[0] == "spread":
                fs.append((True, self.expr(a[1])))
                spread = True
            else:
                fs.append((False, self.expr(a)))
        if not spread:
            plain = [g for _, g in fs]
            return lambda env: [g(env) for g in plain]

        def f(env):
            out = []
            for sp, g in fs:
                if sp:
                    out.extend(iterate(g(env)))
                else:
                    out.append(g(env))
            return out
        return f

    def e_call(self, n):
        callee, args = n[1], self._args(n[2])
        if callee[0] == "member" or callee[0] == "index":
            o = self.expr(callee[1])
            if callee[0] == "member":
                key = callee[2]

                def f(env):
                    obj = o(env)
                    return call(get_member(obj, key), obj, args(env))
            else:
                kf = self.expr(callee[2])

                def f(env):
                    obj = o(env)
                    return call(get_member(obj, kf(env)), obj, args(env))
            return f
        cf = self.expr(callee)
        return lambda env: call(cf(env), UNDEF, args(env))

    def e_new(self, n):
        cf, args = self.expr(n[1]), self._args(n[2])

        def f(env):
            c = cf(env)
            if not isinstance(c, JSClass):
                raise TypeError("not a constructor")
            return c.construct(args(env))
        return f

    def e_array(self, n):
        items = self._args(n[1])
        return lambda env: JSArray(items(env))

    def e_object(self, n):
        parts = []
        for p in n[1]:
            if p[0] == "spread":
                parts.append((None, self.expr(p[1])))
            else:
                parts.append((p[1], self.expr(p[2])))

        def f(env):
            o = JSObject()
            for k, g in parts:
                if k is None:
                    src = g(env)
                    if isinstance(src, JSObject):
                        o.props.update(src.props)
                else:
                    o.props[k] = g(env)
            return o
        return f

    def e_func(self, n):
        return self.function(n[1], n[2], n[3], arrow=n[4])

    def function(self, name, params, body, arrow=False):
        binders = []
        for kind, target, default in params:
            d = self.expr(default) if default is not None else None
            binders.append((kind, self.binder(target, declare=True), d))
        run = self.stmt(body)

        def make(env):
            def call_(this, args):
                scope = Scope(env, UNDEF if arrow else this)
                if not arrow:
                    scope.vars["arguments"] = JSArray(list(args))
                for k, (kind, bind, d) in enumerate(binders):
                    if kind == "rest":
                        bind(scope, JSArray(list(args[k:])))
                        continue
                    v = args[k] if k < len(args) else UNDEF
                    if v is UNDEF and d is not None:
                        v = d(scope)
                    bind(scope, v)
                r = run(scope)
                if r is not None and r[0] == "return":
                    return r[1]
                return UNDEF
            return Fn(call_, name)
        return make

    def binder(self, target, declare=True):
        t = target[0]
        if t == "id" or t == "name":
            name = target[1]
            if declare:
                def b(env, v):
                    env.vars[name] = v
            else:
                def b(env, v):
                    env.assign(name, v)
            return b
        if t == "opat":
            parts = [(key, self.binder(tg, declare), self.expr(d) if d is not None else None)
                     for key, tg, d in target[1]]

            def b(env, v):
                for key, bind, d in parts:
                    x = get_member(v, key)
                    if x is UNDEF and d is not None:
                        x = d(env)
                    bind(env, x)
            return b
        if t == "apat":
            parts = [(self.binder(tg, declare), self.expr(d) if d is not None else None)
                     for tg, d in target[1]]

            def b(env, v):
                vals = iterate(v)
                for k, (bind, d) in enumerate(parts):
                    x = vals[k] if k < len(vals) else UNDEF
                    if x is UNDEF and d is not None:
                        x = d(env)
                    bind(env, x)
            return b
        raise SyntaxError(f"binding {t}")

    # -- statements (return None or a signal tuple)
    def stmt(self, n):
        return getattr(self, "s_" + n[0])(n)

    def s_empty(self, n):
        return lambda env: None

    def s_block(self, n):
        fs = [self.stmt(s) for s in n[1]]
        if len(fs) == 1:
            f0 = fs[0]
            return f0

        def f(env):
            for g in fs:
                r = g(env)
                if r is not None:
                    return r
            return None
        return f

    def s_expr(self, n):
        e = self.expr(n[1])

        def f(env):
            e(env)
        return f

    def s_var(self, n):
        decls = [(self.binder(t, True), self.expr(i) if i is not None else None) for t, i in n[2]]

        def f(env):
            for bind, init in decls:
                bind(env, init(env) if init is not None else UNDEF)
        return f

    def s_if(self, n):
        c, a = self.expr(n[1]), self.stmt(n[2])
        b = self.stmt(n[3]) if n[3] is not None else None
        if b is None:
            return lambda env: a(env) if truthy(c(env)) else None
        return lambda env: a(env) if truthy(c(env)) else b(env)

    def s_return(self, n):
        e = self.expr(n[1]) if n[1] is not None else None
        if e is None:
            return lambda env: ("return", UNDEF)
        return lambda env: ("return", e(env))

    def s_break(self, n):
        return lambda env: BREAK

    def s_continue(self, n):
        return lambda env: CONTINUE

    def s_for(self, n):
        init = self.stmt(n[1]) if n[1] is not None else None
        cond = self.expr(n[2]) if n[2] is not None else None
        upd = self.expr(n[3]) if n[3] is not None else None
        body = self.stmt(n[4])

        def f(env):
            scope = Scope(env)
            if init is not None:
                init(scope)
            while cond is None or truthy(cond(scope)):
                r = body(scope)
                if r is not None:
                    if r is BREAK:
                        break
                    if r is not CONTINUE:
                        return r
                if upd is not None:
                    upd(scope)
            return None
        return f

    def s_forof(self, n):
        bind = self.binder(n[2], True)
        it = self.expr(n[3])
        body = self.stmt(n[4])

        def f(env):
            for v in iterate(it(env)):
                scope = Scope(env)
                bind(scope, v)
                r = body(scope)
                if r is not None:
                    if r is BREAK:
                        break
                    if r is not CONTINUE:
                        return r
            return None
        return f

    def s_while(self, n):
        c, body = self.expr(n[1]), self.stmt(n[2])

        def f(env):
            while truthy(c(env)):
                r = body(env)
                if r is not None:
                    if r is BREAK:
                        break
                    if r is not CONTINUE:
                        return r
            return None
        return f

    def s_class(self, n):
        name, parent, methods = n[1], n[2], n[3]
        comp = [(mn, self.function(mn, ps, body), st) for mn, ps, body, st in methods]

        def f(env):
            proto = JSObject()
            cls = JSClass(name, None, proto)
            for mn, make, st in comp:
                fn = make(env)
                if mn == "constructor":
                    cls.ctor = fn
                elif st:
                    cls.props[mn] = fn
                else:
                    proto.props[mn] = fn
            env.vars[name] = cls
        return f


def run_source(src: str, scope: Scope | None = None) -> Scope:
    """Parse and execute a source file; returns its top-level scope."""
    ast = Parser(lex(src)).program()
    g = scope or make_globals()
    mod = Scope(g)
    Compiler().stmt(ast)(mod)
    return mod


# ---------------------------------------------------------------- bridges

def new(cls: JSClass, *args):
    return cls.construct([py_to_js(a) for a in args])


def method(obj, name, *args):
    return call(get_member(obj, name), obj, [py_to_js(a) for a in args])


def py_to_js(v):
    if isinstance(v, bool) or v is None or v is UNDEF or isinstance(v, (str, JSObject, JSArray,
                                                                       TypedArray, Fn)):
        return v
    if isinstance(v, (int, float)):
        return float(v)
    if isinstance(v, dict):
        return JSObject({k: py_to_js(x) for k, x in v.items()})
    if isinstance(v, (list, tuple)):
        return JSArray([py_to_js(x) for x in v])
    try:
        import numpy as np
        if isinstance(v, np.generic):
            return float(v)
    except ImportError:
        pass
    raise TypeError(type(v))


def typed_to_numpy(t: TypedArray):
    import numpy as np
    dt = {"f": np.float32, "d": np.float64, "i": np.int32, "I": np.uint32, "B": np.uint8,
          "b": np.int8, "H": np.uint16, "h": np.int16}[t.fmt]
    return np.frombuffer(bytes(t.buffer.buf[t.offset:t.offset + t.length * t.size]), dtype=dt).copy()


def numpy_into_typed(t: TypedArray, arr) -> None:
    import numpy as np
    dt = {"f": np.float32, "d": np.float64, "i": np.int32, "I": np.uint32, "B": np.uint8}[t.fmt]
    b = np.ascontiguousarray(arr, dtype=dt).tobytes()
    assert len(b) == t.length * t.size
    t.buffer.buf[t.offset:t.offset + len(b)] = b
