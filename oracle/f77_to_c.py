"""Mechanical Fortran-77 -> C translation of UNICORN's chemistry routines.

ORACLE INFRASTRUCTURE (test-only). This module is used by ``oracle/build_ref.py``
to turn the reference's own Fortran sources into C so that they can be
compiled with gcc here (there is no Fortran compiler in this image) and used
as the pin for the CPU restatement in ``oracle/unichem_oracle.c``.  Its output
goes to ``oracle/_ref/`` only (git-ignored): reference sources are never
committed.

Semantics kept from Fortran 77 (as gfortran implements them):

* storage association of COMMON blocks: every block is one byte array shared
  by all translated units; each unit sees its own declared layout on it;
* default REAL literals (``82.06``) are single precision, ``1.0D-20`` double;
  mixed-mode arithmetic promotes int < real4 < real8 operand by operand;
* ``x**n`` with an integer exponent is a product chain; with a real exponent
  it is ``pow``; DO loops use the Fortran trip count and leave the loop
  variable one step past the last value;
* local variables are static (zero-initialised) as with the F77 compilers the
  code was written for; this fixes the value of locals that the reference
  reads before writing (e.g. ``SPRF(116)`` in ``lib/ckrates.f``).
"""
from __future__ import annotations

import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from unicorn_b200.fortran.parser import (  # noqa: E402
    Bin, Logical, Name, Num, Ref, Str, Un, Unit, expr_type, promote, INTRINSICS_REAL8,
    INTRINSICS_GENERIC)

CTYPE = {"int": "int", "real8": "double", "real4": "float", "logical": "int"}


class Emitter:
    def __init__(self, unit: Unit, common_sizes: dict, global_locals: str | None = None,
                 probes: dict | None = None):
        self.u = unit
        self.common_sizes = common_sizes
        self.global_locals = global_locals   # prefix for file-scope locals (main program)
        self.used_locals: set[str] = set()
        self.lines: list[str] = []
        self.ind = 1
        self.probes = probes or {}            # line -> C statement template
        self.fragment = False
        self.used_args: set[str] = set()

    # ------------------------------------------------------------ names
    def cname(self, name: str) -> str:
        u = self.u
        v = u.vars.get(name)
        if v is not None and v.common:
            return f"(*({CTYPE[v.type]}*)(F77C_{v.common}+{v.offset}))" if not v.dims else \
                f"(({CTYPE[v.type]}*)(F77C_{v.common}+{v.offset}))"
        if v is not None and v.is_arg and not self.fragment:
            return f"(*p_{name})" if not v.dims else f"p_{name}"
        if v is not None and v.is_arg:
            # a fragment of a subroutine: its dummy arguments become globals
            self.used_args.add(name)
            return f"F77A_{self.u.name}_{name}"
        self.used_locals.add(name)
        if self.global_locals:
            return f"{self.global_locals}{name}"
        return f"L_{name}"

    def local_decls(self) -> list[str]:
        out = []
        for name in sorted(self.used_locals):
            v = self.u.vars.get(name)
            ty = v.type if v is not None else self.u.type_of_name(name)
            if ty == "char":
                continue
            n = v.size if (v is not None and v.dims) else 0
            if n:
                out.append(f"{CTYPE[ty]} {self._lname(name)}[{n}]")
            else:
                out.append(f"{CTYPE[ty]} {self._lname(name)}")
        return out

    def _lname(self, name):
        return f"{self.global_locals}{name}" if self.global_locals else f"L_{name}"

    # ------------------------------------------------------------ exprs
    def conv(self, code: str, src: str, dst: str) -> str:
        if src == dst or dst == "logical":
            return code
        return f"(({CTYPE[dst]})({code}))"

    def index(self, name: str, args) -> str:
        v = self.u.vars[name]
        terms = []
        stride = 1
        parts = []
        for (lo, hi), a in zip(v.dims, args):
            ac = self.conv(self.ex(a), expr_type(self.u, a), "int")
            parts.append(f"(({ac})-({lo}))*{stride}" if stride != 1 else f"(({ac})-({lo}))")
            stride *= hi - lo + 1
        terms = " + ".join(parts)
        return f"{self.cname(name)}[{terms}]"

    def ex(self, e) -> str:
        u = self.u
        if isinstance(e, Num):
            if e.kind == "int":
                return str(int(e.text))
            t = e.text.replace("D", "E").replace("Q", "E")
            if "." not in t and "E" not in t:
                t += ".0"
            if t.startswith("."):
                t = "0" + t
            t = t.replace(".E", ".0E")
            if t.endswith("."):
                t += "0"
            return f"{t}f" if e.kind == "real4" else t
        if isinstance(e, Logical):
            return "1" if e.v else "0"
        if isinstance(e, Str):
            return '""'
        if isinstance(e, Name):
            if e.id in u.params:
                v = u.params[e.id]
                return repr(v) if isinstance(v, int) else f"{v!r}"
            return self.cname(e.id)
        if isinstance(e, Ref):
            v = u.vars.get(e.id)
            if v is not None and v.dims:
                return self.index(e.id, e.args)
            return self.intrinsic(e)
        if isinstance(e, Un):
            if e.op == ".NOT.":
                return f"(!{self.ex(e.x)})"
            return f"({e.op}{self.ex(e.x)})"
        if isinstance(e, Bin):
            lt, rt = expr_type(u, e.l), expr_type(u, e.r)
            if e.op in (".AND.", ".OR."):
                op = "&&" if e.op == ".AND." else "||"
                return f"({self.ex(e.l)} {op} {self.ex(e.r)})"
            if e.op in (".EQ.", ".NE.", ".LT.", ".LE.", ".GT.", ".GE."):
                t = promote(lt, rt)
                op = {".EQ.": "==", ".NE.": "!=", ".LT.": "<", ".LE.": "<=", ".GT.": ">", ".GE.": ">="}[e.op]
                return f"({self.conv(self.ex(e.l), lt, t)} {op} {self.conv(self.ex(e.r), rt, t)})"
            if e.op == "**":
                if rt == "int":
                    fn = {"int": "f77_ipow", "real4": "f77_powi_f", "real8": "f77_powi_d"}[lt]
                    return f"{fn}({self.ex(e.l)}, {self.ex(e.r)})"
                t = promote(lt, rt)
                fn = "powf" if t == "real4" else "pow"
                return f"{fn}({self.conv(self.ex(e.l), lt, t)}, {self.conv(self.ex(e.r), rt, t)})"
            t = promote(lt, rt)
            return f"({self.conv(self.ex(e.l), lt, t)} {e.op} {self.conv(self.ex(e.r), rt, t)})"
        raise ValueError(f"cannot emit {e}")

    def intrinsic(self, e: Ref) -> str:
        n = e.id
        args = e.args
        u = self.u
        if n in ("DFLOAT", "DBLE"):
            return f"((double)({self.ex(args[0])}))"
        if n in ("FLOAT", "REAL", "SNGL"):
            return f"((float)({self.ex(args[0])}))"
        if n in ("INT", "IFIX", "IDINT"):
            return f"((int)({self.ex(args[0])}))"
        d8 = {"DEXP": "exp", "DLOG": "log", "DLOG10": "log10", "DSQRT": "sqrt", "DABS": "fabs",
              "DSIN": "sin", "DCOS": "cos", "DATAN": "atan", "DTANH": "tanh"}
        if n in d8:
            return f"{d8[n]}({self.conv(self.ex(args[0]), expr_type(u, args[0]), 'real8')})"
        if n in INTRINSICS_GENERIC:
            t = expr_type(u, e)
            base = {"EXP": "exp", "LOG": "log", "LOG10": "log10", "SQRT": "sqrt", "ABS": "fabs",
                    "SIN": "sin", "COS": "cos", "ATAN": "atan", "TANH": "tanh"}
            if n in base:
                if t == "int" and n == "ABS":
                    return f"abs({self.ex(args[0])})"
                f = base[n] + ("f" if t == "real4" else "")
                return f"{f}({self.conv(self.ex(args[0]), expr_type(u, args[0]), t)})"
            if n in ("MAX", "MIN"):
                cs = [self.conv(self.ex(a), expr_type(u, a), t) for a in args]
                fn = {"MAX": "f77_max", "MIN": "f77_min"}[n] + {"int": "_i", "real4": "_f", "real8": "_d"}[t]
                acc = cs[0]
                for c in cs[1:]:
                    acc = f"{fn}({acc}, {c})"
                return acc
        raise ValueError(f"unsupported intrinsic {n}")

    # ------------------------------------------------------------ statements
    def w(self, s: str):
        self.lines.append("    " * self.ind + s)

    def emit_stmt(self, st):
        k = st.kind
        a = st.a
        if k == "assign":
            lt = expr_type(self.u, a["lhs"])
            rt = expr_type(self.u, a["rhs"])
            self.w(f"{self.ex(a['lhs'])} = {self.conv(self.ex(a['rhs']), rt, lt)};")
            if st.line in self.probes:
                self.w(self.probes[st.line])
        elif k == "iflog":
            inner = Emitter(self.u, self.common_sizes, self.global_locals, self.probes)
            inner.fragment = self.fragment
            inner.ind = 0
            inner.emit_stmt(a["stmt"])
            self.used_locals |= inner.used_locals
            self.used_args |= inner.used_args
            body = " ".join(x.strip() for x in inner.lines)
            self.w(f"if ({self.ex(a['cond'])}) {{ {body} }}")
        elif k == "ifthen":
            self.w(f"if ({self.ex(a['cond'])}) {{")
            self.ind += 1
        elif k == "elseif":
            self.ind -= 1
            self.w(f"}} else if ({self.ex(a['cond'])}) {{")
            self.ind += 1
        elif k == "else":
            self.ind -= 1
            self.w("} else {")
            self.ind += 1
        elif k == "endif":
            self.ind -= 1
            self.w("}")
        elif k == "goto":
            self.w(f"goto L{a['target']};")
        elif k == "continue":
            self.w(";")
        elif k in ("return", "stop"):
            self.w("return;")
        elif k == "call":
            args = ", ".join(f"&({self.ex(x)})" for x in a["args"])
            self.w(f"f77_{a['name'].lower()}({args});")
        elif k in ("io", "implicit", "parameter", "common", "dimension", "data", "typedecl",
                   "chardecl", "end"):
            pass
        else:
            raise ValueError(f"line {st.line}: cannot emit {k}")

    def emit_body(self, stmts):
        open_do = []   # stack of (term_label or None)
        for st in stmts:
            if st.label is not None:
                self.w(f"L{st.label}: ;")
            if st.kind == "do":
                a = st.a
                var = self.ex(Name(a["var"]))
                s = self.conv(self.ex(a["start"]), expr_type(self.u, a["start"]), "int")
                e = self.conv(self.ex(a["end"]), expr_type(self.u, a["end"]), "int")
                stp = self.conv(self.ex(a["step"]), expr_type(self.u, a["step"]), "int") if a["step"] else "1"
                d = len(open_do)
                self.w(f"{{ int s_{d} = {s}, e_{d} = {e}, st_{d} = {stp}; {var} = s_{d};")
                self.w(f"  for (int tc_{d} = (e_{d} - s_{d} + st_{d}) / st_{d}; tc_{d} > 0; --tc_{d}, {var} += st_{d}) {{")
                self.ind += 1
                open_do.append(a["term"])
                continue
            if st.kind == "enddo":
                self.emit_stmt(Stmt_continue(st))
                open_do.pop()
                self.ind -= 1
                self.w("} }")
                continue
            self.emit_stmt(st)
            while open_do and st.label is not None and open_do[-1] == st.label:
                open_do.pop()
                self.ind -= 1
                self.w("} }")
        if open_do:
            raise ValueError(f"unterminated DO loops {open_do} in {self.u.name}")


class Stmt_continue:
    def __init__(self, st):
        self.kind = "continue"
        self.a = {}
        self.line = st.line
        self.label = None


PRELUDE = r"""
#include <math.h>
#include <string.h>
static inline int f77_ipow(int b, int e) { int r = 1; while (e-- > 0) r *= b; return r; }
/* x**n for integer n: the product chain gcc builds for constant exponents */
static inline double f77_powi_d(double x, int n) {
    if (n < 0) return 1.0 / f77_powi_d(x, -n);
    if (n == 0) return 1.0;
    if (n == 1) return x;
    if (n == 2) return x * x;
    if (n == 3) { double t = x * x; return t * x; }
    if (n == 4) { double t = x * x; return t * t; }
    if (n == 5) { double t = x * x; double u = t * x; return u * t; }
    { double h = f77_powi_d(x, n / 2); double r = h * h; return (n & 1) ? r * x : r; }
}
static inline float f77_powi_f(float x, int n) {
    if (n == 2) return x * x;
    float r = 1.0f; while (n-- > 0) r *= x; return r;
}
static inline double f77_max_d(double a, double b) { return a > b ? a : b; }
static inline double f77_min_d(double a, double b) { return a < b ? a : b; }
static inline int f77_max_i(int a, int b) { return a > b ? a : b; }
static inline int f77_min_i(int a, int b) { return a < b ? a : b; }
"""


def common_sizes_of(units) -> dict:
    sizes: dict[str, int] = {}
    for u in units:
        for blk, members in u.commons.items():
            end = 0
            for name in members:
                v = u.vars[name]
                end = max(end, v.offset + v.size * v.elsize)
            sizes[blk] = max(sizes.get(blk, 0), end)
    return sizes


def data_init(u: Unit, em: Emitter) -> list[str]:
    """C assignments implementing the DATA statements of a unit."""
    out = []
    for targets, values in u.data:
        if any(isinstance(t, (Name, Ref)) and u.type_of_name(t.id) == "char" for t in targets):
            continue
        flat = []
        for t in targets:
            v = u.vars.get(t.id if isinstance(t, (Name, Ref)) else None)
            if isinstance(t, Name) and v is not None and v.dims:
                for k in range(v.size):
                    flat.append((f"{em.cname(t.id)}[{k}]", v.type))
            else:
                ty = expr_type(u, t)
                flat.append((em.ex(t), ty))
        if len(flat) != len(values):
            raise ValueError(f"DATA count mismatch in {u.name}: {len(flat)} targets, {len(values)} values")
        for (lhs, ty), val in zip(flat, values):
            vt = expr_type(u, val)
            out.append(f"    {lhs} = {em.conv(em.ex(val), vt, ty)};")
    return out


def translate(units_frags, common_units) -> str:
    """units_frags: list of (unit, func_name, line_ranges|None, global_prefix|None, probes).

    Returns one C translation unit."""
    sizes = common_sizes_of(common_units)
    out = [PRELUDE]
    for blk, n in sorted(sizes.items()):
        out.append(f"unsigned char F77C_{blk}[{(n + 63) // 64 * 64}] __attribute__((aligned(64)));")
        out.append(f"const long F77C_{blk}_size = {n};")
    glob_decls: dict[str, str] = {}
    funcs = []
    for unit, fname, ranges, gprefix, probes in units_frags:
        em = Emitter(unit, sizes, gprefix, probes)
        em.fragment = ranges is not None
        if ranges == "data":
            body = data_init(unit, em)
        else:
            stmts = [s for s in unit.stmts
                     if ranges is None or any(lo <= s.line <= hi for lo, hi in ranges)]
            em.emit_body(stmts)
            body = em.lines
        params = []
        for a in (unit.args if ranges is None else []):
            v = unit.vars[a]
            params.append(f"{CTYPE[v.type]} *p_{a}")
        sig = f"void {fname}({', '.join(params) if params else 'void'})"
        decls = em.local_decls()
        for a in sorted(em.used_args):
            v = unit.vars[a]
            glob_decls[f"{CTYPE[v.type]} F77A_{unit.name}_{a}"] = 1
        if gprefix:
            for d in decls:
                glob_decls[d] = 1
            funcs.append(sig + " {\n" + "\n".join(body) + "\n}\n")
        else:
            funcs.append(sig + " {\n" + "".join(f"    static {d};\n" for d in decls) + "\n".join(body) + "\n}\n")
    out.extend(f"{d};" for d in glob_decls)
    out.extend(funcs)
    return "\n".join(out) + "\n"
