"""Generate the device-side mechanism tables and the species-update program.

Build-time tool: reads ``sandiego52.json`` (written by ``extract.py``) and
writes ``unicorn_b200/csrc/generated/mech_tables.h`` and
``unicorn_b200/csrc/generated/update_program.cuh``.

The species update of the reference (``src/lib/solvesp.f:85-2806``) keeps
544 scalar "A-terms" per cell that are recomputed with one species factored
out, multiplied by the freshly updated mass fraction, and reused by later
species. On a GPU, 544 doubles per cell do not fit on chip, so the generator
executes that statement sequence symbolically: every A-term becomes an
expression tree over three kinds of leaves, RC(r), Y_j as it was at the
start of the pass (``yo``) and Y_j after its own update in this pass
(``yn``). Each production and loss term of each species is then emitted as
that tree, with the reference's operand order, so the device code needs only
RC, the old and the new Y of the cell.
"""
from __future__ import annotations

import json
from pathlib import Path

LSP, LRX = 52, 544
HERE = Path(__file__).resolve().parent
MECH = HERE / "sandiego52.json"
GEN = HERE.parent / "csrc" / "generated"


# ------------------------------------------------------------------ symbolic update

class Leaf:
    __slots__ = ("kind", "idx", "val")

    def __init__(self, kind, idx=0, val=0.0):
        self.kind, self.idx, self.val = kind, idx, val

    def c(self, ctx) -> str:
        if self.kind == "RC":
            return ctx.rc(self.idx)
        if self.kind == "yo":
            return ctx.yo(self.idx) if hasattr(ctx, "yo") else f"YO({self.idx})"
        if self.kind == "yn":
            return f"YN({self.idx})"
        if self.kind == "y0":
            return f"Y0({self.idx})"
        if self.kind == "SOUR":
            return f"SOUR({self.idx})"
        if self.kind == "num":
            return repr(float(self.val))
        raise ValueError(self.kind)


class Mul:
    __slots__ = ("a", "b")

    def __init__(self, a, b):
        self.a, self.b = a, b

    def c(self, ctx) -> str:
        return f"({self.a.c(ctx)} * {self.b.c(ctx)})"


def leaves(e, out):
    if isinstance(e, Mul):
        leaves(e.a, out)
        leaves(e.b, out)
    else:
        out.append(e)
    return out


def resolve_update(mech: dict) -> list[dict]:
    """Symbolic execution of the per-cell update program.

    Returns one dict per species block k (0-based) with expression trees for
    the production sum (list of (sign, tree) or None = reuse the previous
    block's value), the extra sum, and the loss sum (None = 0)."""
    A: dict[int, object] = {}
    updated: set[int] = set()

    def yleaf(k0):
        return Leaf("yn" if k0 in updated else "yo", k0)

    def chain_tree(factors):
        t = None
        for f in factors:
            kind = f[0]
            if kind == "num":
                x = Leaf("num", val=f[1])
            elif kind == "Y":
                x = yleaf(f[1] - 1)
            elif kind == "Y0":
                x = Leaf("y0", f[1] - 1)
            elif kind == "RC":
                x = Leaf("RC", f[1] - 1)
            elif kind == "SOUR":
                x = Leaf("SOUR", f[1] - 1)
            elif kind == "A":
                x = A[f[1]]
            else:
                raise ValueError(kind)
            t = x if t is None else Mul(t, x)
        return t

    out = []
    for b in mech["update"]["blocks"]:
        k0 = b["species"] - 1
        for r, fac in b["recompute"]:
            A[r] = chain_tree(fac)
        blk = {"species": k0}
        blk["prod"] = None if b["prod"] is None else [(s, chain_tree(f)) for s, f in b["prod"]]
        blk["extra"] = [(s, chain_tree(f)) for s, f in b["extra"]]
        blk["loss"] = None if b["loss"] is None else [(s, chain_tree(f)) for s, f in b["loss"]]
        out.append(blk)
        updated.add(k0)
        for r in b["multiply"]:
            A[r] = Mul(Leaf("yn", k0), A[r])
    return out


def emit_sum(terms, ctx, acc: str) -> list[str]:
    lines = []
    for i, (s, t) in enumerate(terms):
        v = t.c(ctx)
        if i == 0:
            lines.append(f"{acc} = {'' if s > 0 else '-'}{v};")
        else:
            lines.append(f"{acc} = {acc} {'+' if s > 0 else '-'} {v};")
    return lines


class _Ctx:
    """Emission context: the last use of each RC(r) in a pass is emitted as
    RC_LAST(r), so the device code can tell L2 that the line will not be
    needed again this pass."""

    def __init__(self, last_use: dict | None = None):
        self.last_use = last_use or {}
        self.count: dict[int, int] = {}

    def rc(self, r0: int) -> str:
        self.count[r0] = self.count.get(r0, 0) + 1
        if self.last_use.get(r0) == self.count[r0]:
            return f"RC_LAST({r0})"
        return f"RC({r0})"


def gen_update_program(mech: dict) -> str:
    blocks = resolve_update(mech)
    uses: dict[int, int] = {}
    for b in blocks:
        for key in ("prod", "extra", "loss"):
            for _, t in (b[key] or []):
                for leaf in leaves(t, []):
                    if leaf.kind == "RC":
                        uses[leaf.idx] = uses.get(leaf.idx, 0) + 1
    ctx = _Ctx(uses)
    # RC rows each species block reads, in first-use order (for L2 prefetch)
    rows, offs = [], []
    for b in blocks:
        offs.append(len(rows))
        seen = []
        for key in ("prod", "extra", "loss"):
            for _, t in (b[key] or []):
                for leaf in leaves(t, []):
                    if leaf.kind == "RC" and leaf.idx not in seen:
                        seen.append(leaf.idx)
        rows.extend(seen)
    offs.append(len(rows))
    L = ["// Generated by unicorn_b200/mech/codegen.py from the update program of",
         "// src/lib/solvesp.f:85-2806 (one block per species, in the reference's order).",
         "// Requires accessor macros RC(r) (0-based reaction slot; RC_LAST(r) marks its",
         "// last use in a pass), YO(k) (Y at the",
         "// start of the pass), YN(k) (Y after its own update), Y0(k) (old time level),",
         "// SOUR(m), WM(k), FACE_SUM(k), FACE_NBR(k); scalars rho, dt, sor1, sor2, rsd;",
         "// and UC_UPDATE_TAIL(k), which clips fnew and stores it as YN(k);",
         "// UC_UPDATE_SYNC() runs after every species (a barrier, or nothing);",
         "// UC_UPDATE_BLOCK_BEGIN(b) runs before species block b (e.g. to prefetch).",
         "#pragma once",
         "#define UC_UPDATE_PROGRAM() do { \\",
         "    double prod = 0.0, extra, loss, rhs1, rhs2, ppp, fnew; \\"]
    nterms = 0
    for bi, b in enumerate(blocks):
        k = b["species"]
        body = [f"UC_UPDATE_BLOCK_BEGIN({bi});"]
        if b["prod"] is not None:
            body += emit_sum(b["prod"], ctx, "prod")
            nterms += len(b["prod"])
        body += emit_sum(b["extra"], ctx, "extra")
        nterms += len(b["extra"])
        body.append(f"rhs1 = rho * Y0({k}) + dt * WM({k}) * (prod + extra);")
        if b["loss"] is None:
            body.append("rhs2 = 0.0;")
        else:
            body += emit_sum(b["loss"], ctx, "loss")
            nterms += len(b["loss"])
            body.append(f"rhs2 = -(dt * WM({k}) * loss);")
        body.append(f"ppp = rho - FACE_SUM({k});")
        body.append(f"fnew = sor2 * YO({k}) + (rhs1 - FACE_NBR({k})) * sor1 / (ppp - rhs2);")
        body.append(f"rsd += fabs(YO({k}) - fnew);")
        body.append(f"UC_UPDATE_TAIL({k});")
        body.append("UC_UPDATE_SYNC();")
        L.append(f"    /* species {k + 1} */ \\")
        L.extend("    " + x + " \\" for x in body)
    L.append("} while (0)")
    L.insert(6, f"// {nterms} production/extra/loss terms per cell and pass")
    L.append("")
    L.append(f"#define UC_UPD_NBLOCKS {len(blocks)}")
    L.append("#ifdef __CUDACC__")
    L.append("// RC rows read by each species block (first-use order): rows [off[b], off[b+1]).")
    L.append(f"static __device__ const int16_t uc_upd_row_off[{len(offs)}] = {{{', '.join(map(str, offs))}}};")
    L.append(f"static __device__ const int16_t uc_upd_rows[{len(rows)}] = {{{', '.join(map(str, rows))}}};")
    L.append("#endif")
    return "\n".join(L) + "\n\n" + gen_inplace_program(blocks, uses)


# ------------------------------------------------------------------ in-place form

class _InPlaceCtx(_Ctx):
    """Emission context of the in-place program: one Y array per tile, each
    species overwritten by its own update. A species' start-of-pass value read
    after its update (through an A-term built before it) comes from a shadow
    copy YOS(m) the tile keeps for those few species."""

    def __init__(self, last_use: dict):
        super().__init__(last_use)
        self.updated: set[int] = set()
        self.shadow: list[int] = []

    def yo(self, k: int) -> str:
        if k not in self.updated:
            return f"YO({k})"
        if k not in self.shadow:
            self.shadow.append(k)
        return f"YOS({self.shadow.index(k)})"


def gen_inplace_program(blocks, uses: dict) -> str:
    ctx = _InPlaceCtx(uses)
    body = []
    for b in blocks:
        k = b["species"]
        if b["prod"] is not None:
            body += emit_sum(b["prod"], ctx, "prod")
        body += emit_sum(b["extra"], ctx, "extra")
        body.append(f"rhs1 = rho * Y0({k}) + dt * WM({k}) * (prod + extra);")
        if b["loss"] is None:
            body.append("rhs2 = 0.0;")
        else:
            body += emit_sum(b["loss"], ctx, "loss")
            body.append(f"rhs2 = -(dt * WM({k}) * loss);")
        body.append(f"ppp = rho - FACE_SUM({k});")
        body.append(f"fnew = sor2 * YO({k}) + (rhs1 - FACE_NBR({k})) * sor1 / (ppp - rhs2);")
        body.append(f"rsd += fabs(YO({k}) - fnew);")
        body.append(f"UC_UPDATE_TAIL({k});")
        ctx.updated.add(k)
    L = ["// In-place form of the same program: YO(k) and YN(k) name one array; YOS(m)",
         "// is the start-of-pass value of species uc_ip_shadow[m], read after that",
         "// species' own update.",
         f"#define UC_IP_NSHADOW {len(ctx.shadow)}",
         f"#define UC_IP_SHADOW_LIST {{{', '.join(map(str, ctx.shadow or [0]))}}}",
         "#define UC_UPDATE_PROGRAM_IP() do { \\",
         "    double prod = 0.0, extra, loss, rhs1, rhs2, ppp, fnew; \\"]
    L.extend("    " + x + " \\" for x in body)
    L.append("} while (0)")
    L.append("#ifdef __CUDACC__")
    L.append(f"static __constant__ int8_t uc_ip_shadow[{max(1, len(ctx.shadow))}] = UC_IP_SHADOW_LIST;")
    L.append("#endif")
    gen_inplace_program.shadow = list(ctx.shadow)
    return "\n".join(L) + "\n"


# ------------------------------------------------------------------ tile-resident form

TR_NTMEM, TR_SEG = 256, 12


class _TRCtx(_InPlaceCtx):
    """Emission context of the tile-resident program: RC(r) becomes a token
    that is later bound to a shared-memory row or a tensor-memory register."""

    def rc(self, r0: int) -> str:
        return f"@{r0}@"


def gen_tr_program(blocks, uses: dict, shadow: list[int]) -> str:
    """The in-place program for a tile whose RC block lives on chip: the RC rows
    used least often (TR_NTMEM of them) in tensor memory, two 32-bit columns
    each, the others in shared memory. Tensor-memory operands are loaded into
    registers ahead of use in segments of at most TR_SEG values, alternating
    between two register banks: the loads of segment s+1 are issued before the
    statements of segment s run and waited for after them, so their latency is
    hidden behind segment s. The arithmetic, its operands and their order are
    those of the in-place program."""
    import re
    ctx = _TRCtx(uses)
    body = [f"UC_TR_PF(0, {blocks[0]['species']});"]
    for bi, b in enumerate(blocks):
        k = b["species"]
        slot = bi % 2
        if bi + 1 < len(blocks):
            # old time level and face terms of the next species, one block ahead of their use
            body.append(f"UC_TR_PF({(bi + 1) % 2}, {blocks[bi + 1]['species']});")
        # the production, extra and loss sums are independent of each other: their statements are
        # interleaved (each sum keeps its own order) so that two or three chains are in flight
        sums = [emit_sum(b["prod"], ctx, "prod") if b["prod"] is not None else [],
                emit_sum(b["extra"], ctx, "extra"),
                emit_sum(b["loss"], ctx, "loss") if b["loss"] is not None else []]
        for i in range(max(len(x) for x in sums)):
            body += [x[i] for x in sums if i < len(x)]
        body.append(f"rhs1 = rho * Y0S({slot}) + dt * WM({k}) * (prod + extra);")
        body.append("rhs2 = 0.0;" if b["loss"] is None else f"rhs2 = -(dt * WM({k}) * loss);")
        body.append(f"ppp = rho - FSS({slot});")
        body.append(f"fnew = sor2 * YO({k}) + (rhs1 - FNS({slot})) * sor1 / (ppp - rhs2);")
        body.append(f"rsd += fabs(YO({k}) - fnew);")
        body.append(f"UC_UPDATE_TAIL({k});")
        body.append("UC_TR_SYNC();")
        ctx.updated.add(k)
    assert ctx.shadow == shadow, "the tile-resident and in-place programs must shadow the same species"
    tok = re.compile(r"@(\d+)@")
    # by slot number: slots [0, TR_NTMEM) in tensor memory, the rest in shared memory, so that each
    # part is one contiguous range of the RC plane's rows and is staged by a few tiled bulk copies
    trow = list(range(TR_NTMEM))
    srow = list(range(TR_NTMEM, LRX))
    tcol = {r: i for i, r in enumerate(trow)}
    scol = {r: i for i, r in enumerate(srow)}
    # segments: runs of statements with at most TR_SEG distinct tensor-memory rows
    segs = []          # (statements, tensor-memory rows in first-use order)
    cur, cur_rows = [], []
    for st in body:
        need = [int(x) for x in tok.findall(st) if int(x) in tcol]
        new = [r for r in dict.fromkeys(need) if r not in cur_rows]
        if cur and len(cur_rows) + len(new) > TR_SEG:
            segs.append((cur, cur_rows))
            cur, cur_rows = [], []
            new = list(dict.fromkeys(need))
        cur.append(st)
        cur_rows += new
    segs.append((cur, cur_rows))
    out = []

    def loads(si):
        bank = si % 2
        return [f"TM_LD({bank}, {q}, {2 * tcol[r]});" for q, r in enumerate(segs[si][1])]

    out += loads(0)
    out.append("TM_WAIT(0);")
    for si, (stmts, trs) in enumerate(segs):
        bank = si % 2
        slot = {r: q for q, r in enumerate(trs)}
        if si + 1 < len(segs):
            out += loads(si + 1)

        def bind(m, slot=slot, bank=bank):
            r = int(m.group(1))
            return f"RCT({bank}, {slot[r]})" if r in tcol else f"RCS({scol[r]})"
        out += [tok.sub(bind, st) for st in stmts]
        if si + 1 < len(segs):
            out.append(f"TM_WAIT({(si + 1) % 2});")
    nld = sum(len(t) for _, t in segs)

    def muls(t):
        return 1 + muls(t.a) + muls(t.b) if isinstance(t, Mul) else 0
    # floating-point operations per cell and pass: the multiplications of each term and its addition
    # into the sum, and the 16 of each species' closing statements (rhs1 5, rhs2 2, ppp 1, fnew 6 with
    # the division as one, the residual 2); the two soot scalars 19
    flops = sum(muls(t) + 1 for b in blocks for key in ("prod", "extra", "loss") for _, t in (b[key] or [])) + \
        16 * len(blocks) + 19
    L = ["// Generated by unicorn_b200/mech/codegen.py: the in-place species-update program",
         "// (src/lib/solvesp.f:85-2806) for a tile whose RC block is held on chip.",
         f"// RC slots 0..{len(trow) - 1} in tensor memory (slot i in columns 2i, 2i+1: low and high",
         f"// word), slots {len(trow)}..{LRX - 1} in shared memory. Requires RCS(i) (shared-memory row i of the",
         "// cell), TM_LD(bank, q, col) (load the double at column col into slot q of a",
         "// register bank), TM_WAIT(bank) (wait for the loads of that bank), RCT(bank, q),",
         "// UC_TR_PF(slot, k) (fetch Y0, FACE_SUM and FACE_NBR of species k into register slot 0",
         "// or 1; read as Y0S, FSS, FNS), UC_TR_SYNC() (after every species: a barrier or nothing)",
         "// and the accessors of the in-place program (YO, YN, YOS, SOUR, WM, UC_UPDATE_TAIL;",
         "// scalars rho, dt, sor1, sor2, rsd). The production, extra and loss statements of a",
         "// species are interleaved; each sum keeps the reference's order.",
         f"// {len(segs)} segments and {nld} tensor-memory loads per cell and pass.",
         "#pragma once",
         f"#define UC_TR_NT {len(trow)}",
         f"#define UC_TR_NS {len(srow)}",
         f"#define UC_TR_SEG {TR_SEG}",
         f"#define UC_UPDATE_FLOPS_PER_CELL_PASS {flops}",
         "#define UC_TR_SHADOW_SAVE() do { " + " ".join(f"YOS({m}) = YO({k});" for m, k in enumerate(shadow)) + " } while (0)",
         "#define UC_UPDATE_PROGRAM_TR() do { \\",
         "    double prod = 0.0, extra, loss, rhs1, rhs2, ppp, fnew; \\"]
    L.extend("    " + x + " \\" for x in out)
    L.append("} while (0)")
    L.append("#ifdef __CUDACC__")
    L.append(f"static __constant__ int16_t uc_tr_trow[{len(trow)}] = {{{', '.join(map(str, trow))}}};")
    L.append(f"static __constant__ int16_t uc_tr_srow[{len(srow)}] = {{{', '.join(map(str, srow))}}};")
    L.append("#else")
    L.append(f"static const short uc_tr_trow[{len(trow)}] = {{{', '.join(map(str, trow))}}};")
    L.append(f"static const short uc_tr_srow[{len(srow)}] = {{{', '.join(map(str, srow))}}};")
    L.append("#endif")
    return "\n".join(L) + "\n"


# ------------------------------------------------------------------ tables

def fmt(v: float) -> str:
    return repr(float(v)) if v == v else "0.0"


def arr(name, ctype, vals, per_line=8) -> str:
    vals = list(vals)
    rows = []
    for i in range(0, len(vals), per_line):
        rows.append("    " + ", ".join(vals[i:i + per_line]))
    return f"static const {ctype} {name}[{len(vals)}] = {{\n" + ",\n".join(rows) + "\n};\n"


def element_counts(names) -> list[list[int]]:
    import re
    out = []
    for nm in names:
        base = re.sub(r"^[A-Z]-", "", nm)
        c = {"C": 0, "H": 0, "O": 0}
        if base not in ("AR", "HE", "N2"):
            assert re.fullmatch(r"([CHO]\d*)+", base), nm
            for el, cnt in re.findall(r"([CHO])(\d*)", base):
                c[el] += int(cnt) if cnt else 1
        out.append([c["C"], c["H"], c["O"]])
    return out


def gen_tables(mech: dict) -> str:
    R = mech["reactions"]
    out = ["// Generated by unicorn_b200/mech/codegen.py from sandiego52.json (the",
           "// San Diego mechanism as UNICORN encodes it: src/lib/DATA.f, src/lib/ckrates.f,",
           "// src/lib/solveh.f, src/unicornd-mild-sd-5.f:76-113). Do not edit.",
           "#pragma once", "#include <stdint.h>",
           f"#define UC_LSP {LSP}", f"#define UC_LRX {LRX}", f"#define UC_NPAIR {LRX // 2}",
           f"#define UC_TPOL1 {fmt(mech['tpol'][0])}", f"#define UC_TPOL2 {fmt(mech['tpol'][1])}"]
    out.append(arr("uc_wsp", "double", map(fmt, mech["wsp"])))
    # atoms of C, H and O per species, read from the species names (T-, S-, I-, N- are isomer prefixes;
    # AR, HE and N2 carry none of the three): every reaction conserves them, so the exact omega does
    out.append(arr("uc_elem_cho", "int8_t", (str(v) for row in element_counts(mech["species"]) for v in row), 3))
    out.append(arr("uc_cdia", "double", map(fmt, mech["cdia"])))
    out.append(arr("uc_tlj", "double", map(fmt, mech["tlj"])))
    out.append(arr("uc_poly", "double", (fmt(v) for row in mech["poly"] for v in row)))
    out.append(arr("uc_om22", "double", (fmt(v) for row in mech["omega22"] for v in row)))
    out.append(arr("uc_ci11", "double", (fmt(v) for row in mech["ci11"] for v in row)))
    for k in ("akf", "alf", "exaf", "aklow", "allow", "ealow"):
        out.append(arr(f"uc_raw_{k}", "double", (fmt(x[k]) for x in R)))
    out.append(arr("uc_raw_troe", "double", (fmt(v) for x in R for v in x["troe"])))
    # reverse formulas: per even slot (0-based odd index r0), rut and q chain (<= 6 factors)
    QMAX = max(len(v["q"]) for v in mech["reverse"].values())
    rev_has, rev_rut, rev_len = [0] * LRX, [0] * LRX, [0] * LRX
    rev_sp = [0] * (LRX * QMAX)
    rev_div = [0] * (LRX * QMAX)
    for key, rv in mech["reverse"].items():
        r0 = int(key) - 1
        rev_has[r0], rev_rut[r0], rev_len[r0] = 1, rv["rut"], len(rv["q"])
        for t, (op, sp) in enumerate(rv["q"]):
            rev_sp[r0 * QMAX + t] = sp - 1
            rev_div[r0 * QMAX + t] = 1 if op == "/" else 0
    out.append(f"#define UC_QMAX {QMAX}")
    out.append(arr("uc_rev_has", "int8_t", map(str, rev_has), 32))
    out.append(arr("uc_rev_rut", "int8_t", map(str, rev_rut), 32))
    out.append(arr("uc_rev_len", "int8_t", map(str, rev_len), 32))
    out.append(arr("uc_rev_sp", "int8_t", map(str, rev_sp), 32))
    out.append(arr("uc_rev_div", "int8_t", map(str, rev_div), 32))
    # third-body groups 1..10: TBODY + sum sign*coef*Y/W
    tbn = [0] * 11
    tbo = [0] * 11
    tsp, tsg, tco, thc = [], [], [], []
    for g in range(1, 11):
        terms = mech["tb"][f"TB{g:03d}"][1:]
        tbo[g], tbn[g] = len(tsp), len(terms)
        for s, k, c in terms:
            tsp.append(k - 1)
            tsg.append(s)
            tco.append(0.0 if c is None else c)
            thc.append(0 if c is None else 1)
    out.append(arr("uc_tb_off", "int16_t", map(str, tbo), 16))
    out.append(arr("uc_tb_len", "int16_t", map(str, tbn), 16))
    out.append(arr("uc_tb_sp", "int8_t", map(str, tsp), 32))
    out.append(arr("uc_tb_sign", "int8_t", map(str, tsg), 32))
    out.append(arr("uc_tb_coef", "double", map(fmt, tco)))
    out.append(arr("uc_tb_hascoef", "int8_t", map(str, thc), 32))
    dm = [0] * LRX
    for key, g in mech["dmole"].items():
        dm[int(key) - 1] = int(g[2:])
    out.append(arr("uc_dmole_grp", "int8_t", map(str, dm), 32))
    # RC assembly: order (0 = never written), tb (-1 none, 0 TBODY, g), post ops <= 4
    PMAX = max(len(v["post"]) for v in mech["rc"].values())
    rc_order, rc_tb, rc_len = [0] * LRX, [-1] * LRX, [0] * LRX
    rc_kind = [0] * (LRX * PMAX)
    rc_idx = [0] * (LRX * PMAX)
    for key, rc in mech["rc"].items():
        r0 = int(key) - 1
        rc_order[r0] = rc["order"]
        rc_tb[r0] = -1 if rc["tb"] is None else (0 if rc["tb"] == "TBODY" else int(rc["tb"][2:]))
        rc_len[r0] = len(rc["post"])
        for t, (op, kind, idx) in enumerate(rc["post"]):
            rc_kind[r0 * PMAX + t] = 1 if kind == "Y" else 0   # 1: *Y_idx, 0: /W_idx
            rc_idx[r0 * PMAX + t] = idx - 1
    out.append(f"#define UC_PMAX {PMAX}")
    out.append(arr("uc_rc_order", "int8_t", map(str, rc_order), 32))
    out.append(arr("uc_rc_tb", "int8_t", map(str, rc_tb), 32))
    out.append(arr("uc_rc_len", "int8_t", map(str, rc_len), 32))
    out.append(arr("uc_rc_kind", "int8_t", map(str, rc_kind), 32))
    out.append(arr("uc_rc_idx", "int8_t", map(str, rc_idx), 32))
    # RA reactant lists (<= 3), 0 = slot never written
    ra_len = [0] * LRX
    ra_sp = [0] * (LRX * 3)
    for key, sps in mech["ra"].items():
        r0 = int(key) - 1
        if sps is None:
            continue
        ra_len[r0] = len(sps)
        for t, s in enumerate(sps):
            ra_sp[r0 * 3 + t] = s - 1
    out.append(arr("uc_ra_len", "int8_t", map(str, ra_len), 32))
    out.append(arr("uc_ra_sp", "int8_t", map(str, ra_sp), 32))
    # PRD term lists per species: packed (r0 | sign<<15 | coef_flag<<14), coef is 1.000 or SRA(0)
    prd_off, prd_len, prd_term, prd_coef = [0] * LSP, [0] * LSP, [], []
    loss_off, loss_len, loss_term = [0] * LSP, [0] * LSP, []
    for key, terms in mech["prd"].items():
        k0 = int(key) - 1
        if not terms:
            continue
        prd_off[k0] = len(prd_term)
        loss_off[k0] = len(loss_term)
        for s, fac in terms:
            kinds = [f[0] for f in fac]
            if kinds == ["SRA"]:
                # SRA(i) = 0.0 (src/lib/solveh.f:671-676): a zero term
                prd_term.append((LRX) | ((1 if s < 0 else 0) << 15) | (1 << 13))
                prd_coef.append(0.0)
                continue
            if kinds == ["RA"]:
                coef, r = None, fac[0][1]
            else:
                assert kinds == ["num", "RA"], fac
                coef, r = fac[0][1], fac[1][1]
            prd_term.append((r - 1) | ((1 if s < 0 else 0) << 15) | ((1 if coef is not None else 0) << 14))
            prd_coef.append(0.0 if coef is None else coef)
            if s < 0:
                assert coef is None, "loss terms carry no coefficient in this mechanism"
                loss_term.append(r - 1)
        prd_len[k0] = len(prd_term) - prd_off[k0]
        loss_len[k0] = len(loss_term) - loss_off[k0]
    out.append(arr("uc_prd_off", "int16_t", map(str, prd_off), 16))
    out.append(arr("uc_prd_len", "int16_t", map(str, prd_len), 16))
    out.append(arr("uc_prd_term", "uint16_t", map(str, prd_term), 16))
    out.append(arr("uc_prd_coef", "double", map(fmt, prd_coef)))
    out.append(arr("uc_loss_off", "int16_t", map(str, loss_off), 16))
    out.append(arr("uc_loss_len", "int16_t", map(str, loss_len), 16))
    out.append(arr("uc_loss_term", "uint16_t", map(str, loss_term), 16))
    out.append(f"#define UC_NPRD_TERMS {len(prd_term)}")
    out.append(f"#define UC_NLOSS_TERMS {len(loss_term)}")
    return "\n".join(out) + "\n"


def main():
    mech = json.loads(MECH.read_text())
    GEN.mkdir(parents=True, exist_ok=True)
    (GEN / "mech_tables.h").write_text(gen_tables(mech))
    (GEN / "update_program.cuh").write_text(gen_update_program(mech))
    blocks = resolve_update(mech)
    uses: dict[int, int] = {}
    for b in blocks:
        for key in ("prod", "extra", "loss"):
            for _, t in (b[key] or []):
                for leaf in leaves(t, []):
                    if leaf.kind == "RC":
                        uses[leaf.idx] = uses.get(leaf.idx, 0) + 1
    (GEN / "update_program_tr.cuh").write_text(gen_tr_program(blocks, uses, gen_inplace_program.shadow))
    print(f"wrote {GEN / 'mech_tables.h'}, {GEN / 'update_program.cuh'} and {GEN / 'update_program_tr.cuh'}")


if __name__ == "__main__":
    main()
