"""Statement and expression parser for the Fortran 77 subset UNICORN uses.

Covers what the chemistry/property routines of UNICORN are written in
(``src/lib/ckrates.f``, ``solvesp.f``, ``solveh.f``, ``spgsolv.f``,
``DATA.f`` and the set-up/property blocks of ``src/unicornd-mild-sd-5.f``):
IMPLICIT/PARAMETER/COMMON/DIMENSION/DATA declarations, assignments, labelled
and block DO loops, logical and block IF, GO TO, CONTINUE, CALL and RETURN.
I/O statements (READ/WRITE/FORMAT/OPEN/...) are kept as opaque ``io``
statements.

Expressions carry Fortran types following the standard promotion rules:
``int < real4 < real8``. A literal such as ``82.06`` is a default (single
precision) REAL constant; ``1.0D-20`` is double precision. This matters for
bit-faithful evaluation: ``RUT=82.06*TKD`` multiplies by the double nearest
to the single-precision value of 82.06.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

from .reader import RawStatement, read_fixed_form

# ----------------------------------------------------------------- lexing

DOT_OPS = {".EQ.", ".NE.", ".LT.", ".LE.", ".GT.", ".GE.", ".AND.", ".OR.",
           ".NOT.", ".TRUE.", ".FALSE.", ".EQV.", ".NEQV."}


def strip_blanks(text: str) -> str:
    """Remove blanks and upper-case everything outside quoted strings."""
    out = []
    q = None
    for ch in text:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch in " \t":
            continue
        else:
            out.append(ch.upper())
    return "".join(out)


@dataclass
class Tok:
    kind: str   # NAME INT REAL STR OP DOT
    val: str
    rkind: int = 0  # 4 or 8 for REAL literals


_num_re = re.compile(r"(\d+\.?\d*|\.\d+)([EDQ][+-]?\d+)?")


def lex(s: str) -> list[Tok]:
    toks: list[Tok] = []
    i = 0
    n = len(s)
    while i < n:
        c = s[i]
        if c.isalpha() or c == "_":
            j = i
            while j < n and (s[j].isalnum() or s[j] == "_"):
                j += 1
            toks.append(Tok("NAME", s[i:j]))
            i = j
        elif c.isdigit() or (c == "." and i + 1 < n and s[i + 1].isdigit()):
            # number; careful with "1.EQ.2"
            j = i
            while j < n and s[j].isdigit():
                j += 1
            is_real = False
            if j < n and s[j] == ".":
                # dot operator right after the integer part?
                m = re.match(r"\.[A-Z]+\.", s[j:])
                if m and m.group(0) in DOT_OPS:
                    pass
                else:
                    is_real = True
                    j += 1
                    while j < n and s[j].isdigit():
                        j += 1
            rk = 4
            if j < n and s[j] in "EDQ" and j + 1 < n and (s[j + 1].isdigit() or
                                                          (s[j + 1] in "+-" and j + 2 < n and s[j + 2].isdigit())):
                is_real = True
                if s[j] in "DQ":
                    rk = 8
                j += 1
                if s[j] in "+-":
                    j += 1
                while j < n and s[j].isdigit():
                    j += 1
            txt = s[i:j]
            if is_real:
                toks.append(Tok("REAL", txt, rk))
            else:
                toks.append(Tok("INT", txt))
            i = j
        elif c == ".":
            m = re.match(r"\.[A-Z]+\.", s[i:])
            if not m or m.group(0) not in DOT_OPS:
                raise ValueError(f"bad dot token in {s!r} at {i}")
            toks.append(Tok("DOT", m.group(0)))
            i += len(m.group(0))
        elif c in "'\"":
            j = s.index(c, i + 1)
            toks.append(Tok("STR", s[i + 1:j]))
            i = j + 1
        elif s.startswith("**", i):
            toks.append(Tok("OP", "**"))
            i += 2
        elif s.startswith("//", i):
            toks.append(Tok("OP", "//"))
            i += 2
        elif c in "+-*/(),=:":
            toks.append(Tok("OP", c))
            i += 1
        else:
            raise ValueError(f"unexpected char {c!r} in {s!r}")
    return toks


# ------------------------------------------------------------ expressions

@dataclass
class Num:
    text: str
    kind: str      # 'int' | 'real4' | 'real8'

    def value(self) -> float | int:
        if self.kind == "int":
            return int(self.text)
        return float(self.text.replace("D", "E").replace("Q", "E"))


@dataclass
class Name:
    id: str


@dataclass
class Ref:          # array element or function call
    id: str
    args: list


@dataclass
class Bin:
    op: str
    l: object
    r: object


@dataclass
class Un:
    op: str         # '-', '+', '.NOT.'
    x: object


@dataclass
class Str:
    s: str


@dataclass
class Logical:
    v: bool


class ExprParser:
    """Recursive-descent parser following Fortran operator precedence."""

    def __init__(self, toks: list[Tok]):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else None

    def take(self, kind=None, val=None):
        tk = self.peek()
        if tk is None or (kind and tk.kind != kind) or (val and tk.val != val):
            raise ValueError(f"expected {kind} {val} got {tk} in {[x.val for x in self.t]}")
        self.i += 1
        return tk

    def at(self, kind, val=None):
        tk = self.peek()
        return tk is not None and tk.kind == kind and (val is None or tk.val == val)

    def parse(self):
        e = self.p_or()
        return e

    def p_or(self):
        e = self.p_and()
        while self.at("DOT", ".OR."):
            self.i += 1
            e = Bin(".OR.", e, self.p_and())
        return e

    def p_and(self):
        e = self.p_not()
        while self.at("DOT", ".AND."):
            self.i += 1
            e = Bin(".AND.", e, self.p_not())
        return e

    def p_not(self):
        if self.at("DOT", ".NOT."):
            self.i += 1
            return Un(".NOT.", self.p_not())
        return self.p_rel()

    def p_rel(self):
        e = self.p_add()
        tk = self.peek()
        if tk is not None and tk.kind == "DOT" and tk.val in (".EQ.", ".NE.", ".LT.", ".LE.", ".GT.", ".GE."):
            self.i += 1
            e = Bin(tk.val, e, self.p_add())
        return e

    def p_add(self):
        if self.at("OP", "-") or self.at("OP", "+"):
            op = self.take().val
            e = self.p_mul()
            e = Un(op, e)
        else:
            e = self.p_mul()
        while self.at("OP", "+") or self.at("OP", "-"):
            op = self.take().val
            e = Bin(op, e, self.p_mul())
        return e

    def p_mul(self):
        e = self.p_pow()
        while self.at("OP", "*") or self.at("OP", "/"):
            op = self.take().val
            e = Bin(op, e, self.p_pow())
        return e

    def p_pow(self):
        base = self.p_prim()
        if self.at("OP", "**"):
            self.i += 1
            # right associative; exponent may carry a unary sign
            if self.at("OP", "-") or self.at("OP", "+"):
                op = self.take().val
                ex = Un(op, self.p_pow())
            else:
                ex = self.p_pow()
            return Bin("**", base, ex)
        return base

    def p_prim(self):
        tk = self.peek()
        if tk is None:
            raise ValueError("unexpected end of expression")
        if tk.kind == "OP" and tk.val == "(":
            self.i += 1
            e = self.p_or()
            self.take("OP", ")")
            return e
        if tk.kind == "INT":
            self.i += 1
            return Num(tk.val, "int")
        if tk.kind == "REAL":
            self.i += 1
            return Num(tk.val, "real8" if tk.rkind == 8 else "real4")
        if tk.kind == "STR":
            self.i += 1
            return Str(tk.val)
        if tk.kind == "DOT" and tk.val in (".TRUE.", ".FALSE."):
            self.i += 1
            return Logical(tk.val == ".TRUE.")
        if tk.kind == "NAME":
            self.i += 1
            if self.at("OP", "("):
                self.i += 1
                args = []
                if not self.at("OP", ")"):
                    args.append(self.p_or())
                    while self.at("OP", ","):
                        self.i += 1
                        args.append(self.p_or())
                self.take("OP", ")")
                return Ref(tk.val, args)
            return Name(tk.val)
        raise ValueError(f"unexpected token {tk}")


def parse_expr(text: str):
    p = ExprParser(lex(text))
    e = p.parse()
    if p.i != len(p.t):
        raise ValueError(f"trailing tokens in expression {text!r}: {[t.val for t in p.t[p.i:]]}")
    return e


def split_top(s: str, sep: str = ",") -> list[str]:
    """Split at top-level separators (outside parentheses and quotes)."""
    parts = []
    depth = 0
    q = None
    cur = []
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def match_paren(s: str, start: int) -> int:
    """Index of the parenthesis closing the one at ``start``."""
    depth = 0
    q = None
    for i in range(start, len(s)):
        ch = s[i]
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return i
    raise ValueError(f"unbalanced parentheses in {s!r}")


# ------------------------------------------------------------- statements

@dataclass
class Stmt:
    line: int
    last_line: int
    label: int | None
    kind: str
    a: dict = field(default_factory=dict)


IO_KW = ("WRITE(", "READ(", "FORMAT(", "OPEN(", "CLOSE(", "PRINT", "REWIND", "BACKSPACE", "INQUIRE(")


def classify(raw: RawStatement) -> Stmt:
    s = strip_blanks(raw.text)
    mk = lambda kind, **a: Stmt(raw.line, raw.last_line, raw.label, kind, a)
    if s.startswith("IF("):
        close = match_paren(s, 2)
        cond = s[3:close]
        rest = s[close + 1:]
        if rest == "THEN":
            return mk("ifthen", cond=parse_expr(cond))
        inner = classify(RawStatement(raw.line, raw.last_line, None, rest))
        return mk("iflog", cond=parse_expr(cond), stmt=inner)
    if s.startswith("ELSEIF("):
        close = match_paren(s, 6)
        return mk("elseif", cond=parse_expr(s[7:close]))
    if s == "ELSE":
        return mk("else")
    if s == "ENDIF":
        return mk("endif")
    if s == "ENDDO":
        return mk("enddo")
    if s == "CONTINUE":
        return mk("continue")
    if s == "RETURN":
        return mk("return")
    if s == "STOP" or s.startswith("STOP"):
        return mk("stop")
    if s == "END" or re.match(r"^END(PROGRAM|SUBROUTINE|FUNCTION|BLOCKDATA)", s):
        return mk("end")
    m = re.match(r"^GOTO(\d+)$", s)
    if m:
        return mk("goto", target=int(m.group(1)))
    m = re.match(r"^DO(\d*)([A-Z][A-Z0-9_]*)=(.*)$", s)
    if m and len(split_top(m.group(3))) in (2, 3):
        parts = split_top(m.group(3))
        return mk("do", term=int(m.group(1)) if m.group(1) else None, var=m.group(2),
                  start=parse_expr(parts[0]), end=parse_expr(parts[1]),
                  step=parse_expr(parts[2]) if len(parts) == 3 else None)
    if s.startswith("CALL"):
        m = re.match(r"^CALL([A-Z][A-Z0-9_]*)(\((.*)\))?$", s)
        args = [parse_expr(x) for x in split_top(m.group(3))] if m.group(3) else []
        return mk("call", name=m.group(1), args=args)
    if s.startswith(IO_KW):
        return mk("io", text=s)
    if s.startswith("IMPLICIT"):
        return mk("implicit", text=s[8:])
    if s.startswith("PARAMETER("):
        return mk("parameter", text=s[10:-1])
    if s.startswith("COMMON/"):
        return mk("common", text=s[6:])
    if s.startswith("DIMENSION"):
        return mk("dimension", text=s[9:])
    if s.startswith("DATA") and "/" in s and "=" not in s.split("/")[0]:
        return mk("data", text=s[4:])
    if s.startswith("SUBROUTINE"):
        m = re.match(r"^SUBROUTINE([A-Z][A-Z0-9_]*)(\((.*)\))?$", s)
        args = split_top(m.group(3)) if m.group(3) else []
        return mk("subroutine", name=m.group(1), args=args)
    if s.startswith("PROGRAM"):
        return mk("program", name=s[7:])
    if s.startswith("BLOCKDATA"):
        return mk("blockdata", name=s[9:])
    if s.startswith("INCLUDE"):
        return mk("include", text=s[7:])
    for ty in ("REAL*8", "REAL", "INTEGER", "DOUBLEPRECISION", "LOGICAL"):
        if s.startswith(ty) and "=" not in s:
            return mk("typedecl", type=ty, text=s[len(ty):])
    if s.startswith("CHARACTER") and "=" not in s:
        return mk("chardecl", text=s)
    # assignment
    depth = 0
    for i, ch in enumerate(s):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            return mk("assign", lhs=parse_expr(s[:i]), rhs=parse_expr(s[i + 1:]))
    raise ValueError(f"line {raw.line}: cannot classify statement {s!r}")


# ------------------------------------------------------------ program units

@dataclass
class Var:
    name: str
    type: str                       # 'int' | 'real8' | 'real4' | 'char' | 'logical'
    dims: list | None = None        # list of (lo, hi) int bounds
    common: str | None = None       # COMMON block name
    offset: int = 0                 # byte offset inside the COMMON block
    is_arg: bool = False

    @property
    def size(self) -> int:
        n = 1
        for lo, hi in (self.dims or []):
            n *= hi - lo + 1
        return n

    @property
    def elsize(self) -> int:
        return {"int": 4, "real8": 8, "real4": 4, "logical": 4, "char": 1}[self.type]


@dataclass
class Unit:
    kind: str                       # 'program' | 'subroutine' | 'blockdata'
    name: str
    path: str
    args: list = field(default_factory=list)
    stmts: list = field(default_factory=list)
    params: dict = field(default_factory=dict)
    vars: dict = field(default_factory=dict)
    commons: dict = field(default_factory=dict)   # block -> [var names]
    implicit: dict = field(default_factory=dict)  # letter -> type
    data: list = field(default_factory=list)      # (target expr, value expr)

    def type_of_name(self, name: str) -> str:
        if name in self.vars:
            return self.vars[name].type
        return self.implicit.get(name[0], "int" if name[0] in "IJKLMN" else "real4")


def _default_implicit() -> dict:
    return {c: ("int" if c in "IJKLMN" else "real4") for c in "ABCDEFGHIJKLMNOPQRSTUVWXYZ"}


def const_eval(e, params: dict):
    """Evaluate an integer/real constant expression (PARAMETER values)."""
    if isinstance(e, Num):
        return e.value()
    if isinstance(e, Name):
        return params[e.id]
    if isinstance(e, Un):
        v = const_eval(e.x, params)
        return -v if e.op == "-" else v
    if isinstance(e, Bin):
        a, b = const_eval(e.l, params), const_eval(e.r, params)
        if e.op == "+":
            return a + b
        if e.op == "-":
            return a - b
        if e.op == "*":
            return a * b
        if e.op == "/":
            if isinstance(a, int) and isinstance(b, int):
                q = abs(a) // abs(b)
                return q if (a >= 0) == (b >= 0) else -q
            return a / b
        if e.op == "**":
            return a ** b
    raise ValueError(f"not a constant expression: {e}")


def _parse_decl_list(text: str):
    """Parse 'A(10,LJ),B,C(2:5)' into [(name, [dim exprs] | None)]."""
    out = []
    for item in split_top(text):
        if not item:
            continue
        if "(" in item:
            k = item.index("(")
            name = item[:k]
            dims = split_top(item[k + 1:match_paren(item, k)])
            out.append((name, dims))
        else:
            out.append((item, None))
    return out


def build_units(path: str, param_override: dict | None = None) -> list[Unit]:
    """Parse a source file into program units with resolved declarations."""
    raws = read_fixed_form(path)
    units: list[Unit] = []
    cur: Unit | None = None
    for raw in raws:
        st = classify(raw)
        if st.kind in ("program", "subroutine", "blockdata"):
            cur = Unit(st.kind, st.a["name"], path, args=st.a.get("args", []))
            cur.implicit = _default_implicit()
            units.append(cur)
            continue
        if st.kind == "include":
            continue
        if cur is None:
            # statements before a unit header belong to an unnamed main program
            cur = Unit("program", "MAIN", path)
            cur.implicit = _default_implicit()
            units.append(cur)
        if st.kind == "end":
            cur.stmts.append(st)
            cur = None
            continue
        cur.stmts.append(st)
    for u in units:
        _resolve_decls(u, param_override or {})
    return units


def _dims(u: Unit, dims):
    out = []
    for d in dims:
        if ":" in d:
            lo, hi = d.split(":")
            out.append((int(const_eval(parse_expr(lo), u.params)), int(const_eval(parse_expr(hi), u.params))))
        else:
            out.append((1, int(const_eval(parse_expr(d), u.params))))
    return out


def _resolve_decls(u: Unit, override: dict):
    for a in u.args:
        pass
    for st in u.stmts:
        k = st.kind
        if k == "implicit":
            m = re.match(r"^(REAL\*8|DOUBLEPRECISION|REAL|INTEGER)\((.*)\)$", st.a["text"])
            ty = {"REAL*8": "real8", "DOUBLEPRECISION": "real8", "REAL": "real4", "INTEGER": "int"}[m.group(1)]
            for rng in m.group(2).split(","):
                if "-" in rng:
                    a, b = rng.split("-")
                    for c in range(ord(a), ord(b) + 1):
                        u.implicit[chr(c)] = ty
                else:
                    u.implicit[rng] = ty
        elif k == "parameter":
            for item in split_top(st.a["text"]):
                name, val = item.split("=", 1)
                if name in override:
                    u.params[name] = override[name]
                else:
                    u.params[name] = const_eval(parse_expr(val), u.params)
    # explicit types, dimensions, commons (in order)
    for st in u.stmts:
        k = st.kind
        if k == "typedecl":
            ty = {"REAL*8": "real8", "DOUBLEPRECISION": "real8", "REAL": "real4",
                  "INTEGER": "int", "LOGICAL": "logical"}[st.a["type"]]
            for name, dims in _parse_decl_list(st.a["text"]):
                v = u.vars.setdefault(name, Var(name, ty))
                v.type = ty
                if dims:
                    v.dims = _dims(u, dims)
        elif k == "chardecl":
            body = re.sub(r"^CHARACTER(\*\d+)?", "", st.a["text"])
            for name, dims in _parse_decl_list(body):
                name = name.split("*")[0]
                v = u.vars.setdefault(name, Var(name, "char"))
                v.type = "char"
                if dims:
                    v.dims = _dims(u, dims)
        elif k == "dimension":
            for name, dims in _parse_decl_list(st.a["text"]):
                v = u.vars.setdefault(name, Var(name, u.type_of_name(name)))
                v.dims = _dims(u, dims)
        elif k == "common":
            text = st.a["text"]
            m = re.match(r"^/([A-Z0-9_]*)/(.*)$", text)
            blk, rest = m.group(1), m.group(2)
            members = u.commons.setdefault(blk, [])
            for name, dims in _parse_decl_list(rest):
                v = u.vars.setdefault(name, Var(name, u.type_of_name(name)))
                if dims:
                    v.dims = _dims(u, dims)
                v.common = blk
                members.append(name)
    # finalize implicit types of everything referenced later on demand
    for name, v in u.vars.items():
        if v.type is None:
            v.type = u.type_of_name(name)
    for a in u.args:
        v = u.vars.setdefault(a, Var(a, u.type_of_name(a)))
        v.is_arg = True
    # common offsets (byte offsets, natural alignment)
    for blk, members in u.commons.items():
        off = 0
        for name in members:
            v = u.vars[name]
            al = v.elsize
            if off % al:
                off += al - off % al
            v.offset = off
            off += v.size * v.elsize
    # DATA statements
    for st in u.stmts:
        if st.kind == "data":
            u.data.extend(parse_data(st.a["text"]))


def parse_data(text: str):
    """Parse 'A,B(1)/1.0,2*0.0/,C/3/' into [(targets, values)] groups."""
    groups = []
    i = 0
    while i < len(text):
        j = text.index("/", i)
        targets = text[i:j]
        k = text.index("/", j + 1)
        values = text[j + 1:k]
        tl = [parse_expr(t) for t in split_top(targets) if t]
        vl = []
        for v in split_top(values):
            if not v:
                continue
            m = re.match(r"^(\d+)\*(.*)$", v)
            if m:
                vl.extend([parse_expr(m.group(2))] * int(m.group(1)))
            else:
                vl.append(parse_expr(v))
        groups.append((tl, vl))
        i = k + 1
        if i < len(text) and text[i] == ",":
            i += 1
    return groups


def expr_type(u: Unit, e) -> str:
    """Fortran type of an expression: 'int', 'real4', 'real8' or 'logical'."""
    if isinstance(e, Num):
        return e.kind
    if isinstance(e, Logical):
        return "logical"
    if isinstance(e, Str):
        return "char"
    if isinstance(e, Name):
        if e.id in u.params:
            v = u.params[e.id]
            return "int" if isinstance(v, int) else "real8"
        return u.type_of_name(e.id)
    if isinstance(e, Ref):
        if e.id in u.vars and u.vars[e.id].dims:
            return u.vars[e.id].type
        return intrinsic_type(u, e)
    if isinstance(e, Un):
        return "logical" if e.op == ".NOT." else expr_type(u, e.x)
    if isinstance(e, Bin):
        if e.op in (".EQ.", ".NE.", ".LT.", ".LE.", ".GT.", ".GE.", ".AND.", ".OR."):
            return "logical"
        a, b = expr_type(u, e.l), expr_type(u, e.r)
        if e.op == "**":
            if b == "int":
                return a
            return promote(a, b)
        return promote(a, b)
    raise ValueError(f"no type for {e}")


_RANK = {"int": 0, "real4": 1, "real8": 2}


def promote(a: str, b: str) -> str:
    return a if _RANK[a] >= _RANK[b] else b


INTRINSICS_REAL8 = {"DEXP", "DLOG", "DLOG10", "DSQRT", "DABS", "DFLOAT", "DBLE", "DSIN", "DCOS",
                    "DATAN", "DTANH", "DMAX1", "DMIN1", "DSIGN", "DATAN2"}
INTRINSICS_GENERIC = {"EXP", "LOG", "LOG10", "SQRT", "ABS", "MAX", "MIN", "SIN", "COS", "ATAN",
                      "TANH", "SIGN", "MOD", "ATAN2"}


def intrinsic_type(u: Unit, e: Ref) -> str:
    n = e.id
    if n in INTRINSICS_REAL8:
        return "real8"
    if n in ("FLOAT", "REAL", "SNGL"):
        return "real4"
    if n in ("INT", "NINT", "IFIX", "IDINT"):
        return "int"
    if n in INTRINSICS_GENERIC:
        ts = [expr_type(u, a) for a in e.args]
        t = ts[0]
        for x in ts[1:]:
            t = promote(t, x)
        return t
    raise ValueError(f"unknown function {n}")
