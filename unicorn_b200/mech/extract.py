"""Mechanism extractor: UNICORN Fortran sources -> ``sandiego52.json``.

Build-time tool. Reads the reference's Fortran *sources* (never executes
them) and writes the 52-species / 544-reaction San Diego mechanism exactly as
the reference encodes it, so that nothing is transcribed by hand:

* species names, NASA polynomials and Omega(2,2) fits ... ``src/lib/DATA.f:24-666``
* Arrhenius / fall-off / Troe parameters .................. ``src/lib/DATA.f:667-1306``
* molar masses, sigma, eps/k, Omega(1,1) fit CI11 ......... ``src/unicornd-mild-sd-5.f:76-113``
* reverse-rate equilibrium formulas (per even slot) ....... ``src/lib/ckrates.f:116-642``
* third-body sums TBODY, TB001..TB010 ..................... ``src/lib/ckrates.f:645-731``
* per-reaction third body of the fall-off blend ........... ``src/lib/ckrates.f:743-759``
* rate-coefficient assembly RC = C*rho^n*[TB]*k/prod(W) ... ``src/lib/ckrates.f:796-1333``
* point-implicit species update program .................... ``src/lib/solvesp.f:85-2806``
* reaction rates RA and production lists PRD .............. ``src/lib/solveh.f:116-676``

Numbers keep their Fortran kinds: a default-REAL literal in a DATA statement
(``/5.75D+19, -1.4, 0.0/``) is rounded to single precision before it is
stored in the REAL*8 table, as the Fortran compiler does.

Every product is a left-to-right chain of factors and every sum a
left-to-right list of signed terms, in the reference's statement order, so
that evaluators can reproduce the reference's rounding.

Usage: python -m unicorn_b200.mech.extract [--ref <reference checkout>]
(default: $UNICORN_REF, else ``reference`` beside this repository)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
from pathlib import Path

import numpy as np

from unicorn_b200.fortran.parser import Bin, Name, Num, Ref, Un, build_units
from unicorn_b200.refsrc import reference_root

LSP, LRX = 52, 544
HERE = Path(__file__).resolve().parent
OUT = HERE / "sandiego52.json"

# Fortran name of the species plane k (1-based) in lib/ckrates.f (FA0..FCB),
# lib/solvesp.f (SA0..SCB for current values, EA0/WA0/PA0/QA0 face coefficients)
_DIG = "0123456789ABCDEFGHIJ"


def plane_index(name: str) -> int:
    """'FA0' -> 1, 'SAJ' -> 20, 'SB0' -> 21, 'FCB' -> 52 (1-based species)."""
    grp = "ABC".index(name[1])
    return grp * 20 + _DIG.index(name[2]) + 1


def fval(e) -> float:
    """Value of a numeric literal expression with its Fortran kind."""
    if isinstance(e, Un):
        v = fval(e.x)
        return -v if e.op == "-" else v
    if isinstance(e, Num):
        v = e.value()
        if e.kind == "real4":
            return float(np.float32(v))
        return float(v)
    raise ValueError(f"not a literal: {e}")


def chain(e, ops=("*", "/")):
    """Flatten a left-assoc chain a op b op c into [(None,a),(op,b),(op,c)]."""
    out = []
    while isinstance(e, Bin) and e.op in ops:
        out.append((e.op, e.r))
        e = e.l
    out.append((None, e))
    return out[::-1]


def terms_of(e):
    """Flatten a left-assoc +/- sum into [(sign, term_expr)]."""
    out = []
    while isinstance(e, Bin) and e.op in ("+", "-"):
        out.append((+1 if e.op == "+" else -1, e.r))
        e = e.l
    if isinstance(e, Un) and e.op in ("+", "-"):
        out.append((+1 if e.op == "+" else -1, e.x))
    else:
        out.append((+1, e))
    return out[::-1]


def sha(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()[:16]


# ------------------------------------------------------------------ DATA.f

def species_names(data_path: Path) -> list[str]:
    names = []
    for line in data_path.read_text(encoding="latin-1").splitlines():
        m = re.match(r"^C-{10,}\s+(\S+)\s+-{10,}\s*$", line)
        if m:
            names.append(m.group(1))
    if len(names) != LSP:
        raise ValueError(f"found {len(names)} species names in DATA.f")
    return names


def data_tables(unit) -> dict:
    store: dict[str, dict] = {}
    for targets, values in unit.data:
        if any(unit.type_of_name(t.id) == "char" for t in targets):
            continue
        flat = []
        for t in targets:
            if isinstance(t, Name):
                v = unit.vars.get(t.id)
                if v is not None and v.dims:
                    flat.extend((t.id, k) for k in range(v.size))
                else:
                    flat.append((t.id, 0))
            elif isinstance(t, Ref):
                v = unit.vars[t.id]
                idx = [int(fval(a)) for a in t.args]
                lin = 0
                stride = 1
                for (lo, hi), i in zip(v.dims, idx):
                    lin += (i - lo) * stride
                    stride *= hi - lo + 1
                flat.append((t.id, lin))
        assert len(flat) == len(values), (targets, len(values))
        for (name, k), val in zip(flat, values):
            store.setdefault(name, {})[k] = fval(val)
    return store


# ------------------------------------------------------------------ ckrates.f

def factor(e):
    """Classify one factor of a product in the species-update / rate code."""
    if isinstance(e, Num) or (isinstance(e, Un) and isinstance(e.x, Num)):
        return ["num", fval(e)]
    if isinstance(e, Name):
        m = re.match(r"^A(\d{4})$", e.id)
        if m:
            return ["A", int(m.group(1))]
        if e.id == "FNEW":
            return ["FNEW"]
        return ["var", e.id]
    if isinstance(e, Ref):
        if e.id in ("RC",):
            return ["RC", int(fval(e.args[-1]))]
        if e.id == "RA":
            return ["RA", int(fval(e.args[0]))]
        if e.id == "SRA":
            return ["SRA", int(fval(e.args[0]))]
        if e.id == "SOUR":
            return ["SOUR", int(fval(e.args[-1]))]
        if e.id == "SSP":
            return ["Y", int(fval(e.args[-1]))]
        if re.match(r"^S[ABC][0-9A-J]$", e.id):
            return ["Y", plane_index(e.id)]
        if re.match(r"^F[ABC][0-9A-J]$", e.id):
            return ["Y0", plane_index(e.id)]
        if e.id in ("WM", "GSP", "SPRF", "AKF"):
            return [e.id, int(fval(e.args[0]))]
    raise ValueError(f"unexpected factor {e}")


def product(e):
    """A product chain -> list of factors (all '*' operators)."""
    ch = chain(e, ("*",))
    return [factor(x) for _, x in ch]


def signed_sum(e):
    """A +/- sum of products -> [[sign, [factors...]], ...]."""
    return [[s, product(t)] for s, t in terms_of(e)]


def parse_ckrates(u) -> dict:
    rev = {}
    tb = {}
    dmole = {}
    rc = {}
    for st in u.stmts:
        if st.kind == "iflog" and st.a["stmt"].kind == "assign":
            inner = st.a["stmt"]
            lhs = inner.a["lhs"]
            if isinstance(lhs, Name) and lhs.id == "DMOLE":
                c = st.a["cond"]
                ir = int(fval(c.r))
                grp = chain(inner.a["rhs"])[0][1].id
                dmole[ir] = grp
            continue
        if st.kind != "assign":
            continue
        lhs, rhs = st.a["lhs"], st.a["rhs"]
        if isinstance(lhs, Ref) and lhs.id == "SPRF" and isinstance(lhs.args[0], Num):
            r = int(lhs.args[0].text)
            # AKF(r)*SPRF(r-1) [ /RUT | *RUT ] / ( GSP chain )
            ch = chain(rhs)
            assert ch[0][1].id == "AKF" and int(fval(ch[0][1].args[0])) == r
            assert ch[1][0] == "*" and ch[1][1].id == "SPRF" and int(fval(ch[1][1].args[0])) == r - 1
            rut = 0
            rest = ch[2:]
            if rest[0][1] == Name("RUT") or (isinstance(rest[0][1], Name) and rest[0][1].id == "RUT"):
                rut = -1 if rest[0][0] == "/" else +1
                rest = rest[1:]
            assert len(rest) == 1 and rest[0][0] == "/", st.line
            q = chain(rest[0][1])
            qchain = [[op or "*", int(fval(x.args[0]))] for op, x in q]
            assert all(isinstance(x, Ref) and x.id == "GSP" for _, x in q)
            rev[r] = {"rut": rut, "q": qchain, "line": st.line}
        elif isinstance(lhs, Name) and re.match(r"^TB(ODY|\d{3})$", lhs.id):
            name = lhs.id
            terms = []
            for s, t in terms_of(rhs):
                if isinstance(t, Name) and t.id == "TBODY":
                    terms.append([s, "TBODY"])
                    continue
                ch = chain(t)
                # [coef *] FAx / WM(k)
                f = [(op, x) for op, x in ch]
                if len(f) == 2:
                    coef = None
                    y, w = f[0][1], f[1][1]
                else:
                    coef = fval(f[0][1])
                    y, w = f[1][1], f[2][1]
                    assert f[1][0] == "*"
                assert f[-1][0] == "/" and w.id == "WM"
                k = plane_index(y.id)
                assert int(fval(w.args[0])) == k
                terms.append([s, k, coef])
            if name in tb and name == "TBODY":
                tb[name].extend(terms[1:])      # TBODY=TBODY+FAx/WM(k)
            else:
                tb[name] = terms
        elif isinstance(lhs, Ref) and lhs.id == "RC":
            r = int(fval(lhs.args[1]))
            ch = chain(rhs)
            c = ch[0][1].id
            order = {"C1ST": 1, "C2ND": 2, "C3RD": 3}[c]
            assert ch[1][1].id == f"RHO{order}"
            idx = 2
            tbn = None
            if isinstance(ch[idx][1], Name) and ch[idx][1].id.startswith("TB"):
                tbn = ch[idx][1].id
                idx += 1
            assert ch[idx][1].id == "SPRF" and int(fval(ch[idx][1].args[0])) == r
            post = []   # ["/", "W", k] divide by WM(k); ["*", "Y", k] multiply by Y_k
            for op, x in ch[idx + 1:]:
                if x.id == "WM":
                    assert op == "/"
                    post.append(["/", "W", int(fval(x.args[0]))])
                else:
                    assert op == "*" and re.match(r"^F[ABC][0-9A-J]$", x.id), st.line
                    post.append(["*", "Y", plane_index(x.id)])
            rc[r] = {"order": order, "tb": tbn, "post": post, "line": st.line}
    return {"reverse": rev, "tb": tb, "dmole": dmole, "rc": rc}


# ------------------------------------------------------------------ solvesp.f

def parse_solvesp(u) -> dict:
    """Structured form of the per-cell point-implicit update program."""
    body = []
    in_cell = False
    for st in u.stmts:
        if st.kind == "iflog" and isinstance(st.a["cond"], Bin) and \
                isinstance(st.a["cond"].l, Ref) and st.a["cond"].l.id == "ISKIP":
            in_cell = True
            continue
        if in_cell:
            if st.label == 305:
                break
            body.append(st)
    blocks = []
    pending = []          # A-term (re)computations since the last species update
    cur = None
    phase = "pre"         # pre: before an equation, eq: inside it, post: after Y_k update
    for st in body:
        if st.kind == "iflog":
            inner = st.a["stmt"]
            assert inner.kind == "assign" and inner.a["lhs"] == Name("FNEW"), st.line
            continue
        assert st.kind == "assign", (st.line, st.kind)
        lhs, rhs = st.a["lhs"], st.a["rhs"]
        ln = lhs.id
        if re.match(r"^A\d{4}$", ln):
            r = int(ln[1:])
            fac = product(rhs) if not isinstance(rhs, Num) else [["num", fval(rhs)]]
            if fac[0][0] == "FNEW":
                assert phase == "post" and fac[1] == ["A", r], st.line
                cur["multiply"].append(r)
                continue
            assert phase != "eq", st.line
            phase = "pre"
            pending.append([r, fac])
            continue
        if ln in ("RHS1A", "RHS1B") and phase != "eq":
            cur = {"recompute": pending, "multiply": [], "prod": None, "line": st.line}
            pending = []
            blocks.append(cur)
            phase = "eq"
        if ln == "RHS1A":
            cur["prod"] = signed_sum(rhs)
        elif ln == "RHS1B":
            cur["extra"] = signed_sum(rhs) if not isinstance(rhs, Num) else [[1, [["num", fval(rhs)]]]]
        elif ln == "RHS1":
            if phase != "eq":
                break          # the two soot equations (lib/solvesp.f:2807-2830) follow
            y0 = chain(rhs.l)[1][1]
            cur["species"] = plane_index(y0.id)
        elif ln == "RHS2":
            if isinstance(rhs, Num):
                cur["loss"] = None
            else:
                assert isinstance(rhs, Un) and rhs.op == "-" and rhs.x.op == "*"
                dtw = chain(rhs.x.l, ("*",))
                assert [x.id for _, x in dtw] == ["DT", "WM"], st.line
                cur["loss"] = signed_sum(rhs.x.r)
        elif ln in ("PPP", "FNEW", "RSD"):
            pass
        elif re.match(r"^S[ABC][0-9A-J]$", ln):
            assert plane_index(ln) == cur["species"], st.line
            phase = "post"
        else:
            raise ValueError(f"line {st.line}: unexpected statement {ln}")
    sp = [b.get("species") for b in blocks]
    assert sp == list(range(1, 52)), sp
    assert not pending
    return {"blocks": blocks}


# ------------------------------------------------------------------ solveh.f

def parse_solveh(u) -> dict:
    ra = {}
    prd = {}
    for st in u.stmts:
        if st.kind != "assign":
            continue
        lhs, rhs = st.a["lhs"], st.a["rhs"]
        if isinstance(lhs, Ref) and lhs.id == "RA":
            r = int(fval(lhs.args[0]))
            if isinstance(rhs, Num):
                ra[r] = None      # RA(r)=0.0 (slots never written by CKRATES)
                continue
            fac = product(rhs)
            assert fac[0] == ["RC", r]
            ra[r] = [f[1] for f in fac[1:]]
            assert all(f[0] == "Y" for f in fac[1:])
        elif isinstance(lhs, Ref) and lhs.id == "PRD" and isinstance(lhs.args[0], Num):
            k = int(fval(lhs.args[0]))
            if isinstance(rhs, Num):
                prd[k] = None
                continue
            ch = chain(rhs, ("*",))
            assert ch[0][1].id == "WM" and ch[1][1].id == "HFO"
            prd[k] = signed_sum(ch[2][1])
    return {"ra": ra, "prd": prd}


# ------------------------------------------------------------------ driver

def extract(ref: Path) -> dict:
    src = ref / "src"
    data_u = build_units(str(src / "lib/DATA.f"))[0]
    main_u = [u for u in build_units(str(src / "unicornd-mild-sd-5.f")) if u.kind == "program"][0]
    ck = build_units(str(src / "lib/ckrates.f"))[0]
    sp = build_units(str(src / "lib/solvesp.f"))[0]
    sh = build_units(str(src / "lib/solveh.f"))[0]
    d = data_tables(data_u)
    m = data_tables(main_u)
    names = species_names(src / "lib/DATA.f")
    poly = [[d[f"P{k:03d}"][i] for i in range(14)] for k in range(1, LSP + 1)]
    ci = [[d[f"C{k:03d}"][i] for i in range(12)] for k in range(1, LSP + 1)]
    g = lambda nm, r: d.get(nm, {}).get(r - 1, 0.0)
    reac = []
    for r in range(1, LRX + 1):
        reac.append({
            "akf": g("AKF", r), "alf": g("ALF", r), "exaf": g("EXAF", r),
            "aklow": g("AKLOW", r), "allow": g("ALLOW", r), "ealow": g("EALOW", r),
            "troe": [d.get("TROE", {}).get((r - 1) + LRX * c, 0.0) for c in range(4)],
        })
    ci11 = [[m["CI11"][(k - 1) + 4 * (c - 1)] for c in range(1, 6)] for k in range(1, 5)]
    mech = {
        "name": "San Diego mechanism as encoded in UNICORN (52 species, 544 reaction slots)",
        "provenance": {p: sha(src / p) for p in ("lib/DATA.f", "lib/ckrates.f", "lib/solvesp.f",
                                                   "lib/solveh.f", "unicornd-mild-sd-5.f")},
        "lsp": LSP, "lrx": LRX,
        "lrev": int(d["LREV"][0]),
        "tpol": [d["TPOL1"][0], d["TPOL2"][0]],
        "species": names,
        "wsp": [m["WSP"][k] for k in range(LSP)],
        "cdia": [m["CDIA"][k] for k in range(LSP)],
        "tlj": [m["TLJ"][k] for k in range(LSP)],
        "ci11": ci11,
        "poly": poly,
        "omega22": ci,
        "reactions": reac,
    }
    mech.update(parse_ckrates(ck))
    mech["update"] = parse_solvesp(sp)
    mech.update(parse_solveh(sh))
    # JSON keys must be strings; keep reaction/species numbers 1-based
    for key in ("reverse", "dmole", "rc", "ra", "prd"):
        mech[key] = {str(k): v for k, v in sorted(mech[key].items())}
    return mech


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=str(reference_root()))
    ap.add_argument("--out", default=str(OUT))
    a = ap.parse_args()
    mech = extract(Path(a.ref))
    Path(a.out).write_text(json.dumps(mech, indent=None, separators=(",", ":")))
    print(f"wrote {a.out}: {len(mech['reverse'])} reverse formulas, {len(mech['rc'])} RC slots, "
          f"{len(mech['update']['blocks'])} update blocks, {len(mech['ra'])} RA, "
          f"{sum(1 for v in mech['prd'].values() if v)} PRD lists")


if __name__ == "__main__":
    main()
