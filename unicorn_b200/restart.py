"""Restart files of the reference (FLAMEA / FLAME.DATA) for device-resident runs.

The layout is that of SUBROUTINE PRNTDK (src/lib/prntdk.f:17-33), which
READFF (src/lib/readff.f:20-60) reads back:

  IFLAME = 200000 (swirl) + 100*LSP + INFUEL + 400000 (soot) [+ 100000 with bodies],
           FORMAT (I6,2('-'),'FLAME DATA FROM UNICOND-HEPT-SD(',
                   ' 52 SPECIES & 544 REACTIONS OF SANDIEGO MECH) DATA',2('-'))
  LI,LJ,ISYM,IFLOW,ISWRL,ITHRM,ICHEM,IGRAV,INERT,ITR  (10I6) and DT (F12.10)
  the 20 scales ALSTR .. REI                          (8(1PE14.7,1X))
  [NBODY and the body corners                        (21I6)]
  X, Y, RHO, FSP(.,1..51), U, V, W, P, QDOT, TK       (one record, 8(1PE14.7,1X))
  STMF, STND                                          (a new record)
  [AK, EPS when IFLOW = 2]
Arrays are the reference's non-dimensional fields over the LJ x LI grid, J
fastest. N2 is not written; the reader closes it as 1 - sum of the others.
"""
from __future__ import annotations

import numpy as np

SCALES = ["ALSTR", "VSTR", "RSTR", "PSTR", "TSTR", "TMSTR", "AMSTR", "ACSTR", "DSTR", "HSTR", "CPSTR", "AKSTR",
          "EPSTR", "WMSTR", "GASC", "BETA1", "BETA2", "BETA3", "BETA4", "REI"]
TITLE = "FLAME DATA FROM UNICOND-HEPT-SD( 52 SPECIES & 544 REACTIONS OF SANDIEGO MECH) DATA"


def pe14_7(v: float) -> str:
    """Fortran 1PE14.7: [-]d.dddddddE+dd (exponents beyond two digits as +ddd, without the E)."""
    if v == 0.0:
        return " 0.0000000E+00"
    s = f"{abs(v):.7e}"
    mant, ex = s.split("e")
    e = int(ex)
    tail = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    return (("-" if v < 0 else "") + mant + tail).rjust(14)


def _records(values) -> list[str]:
    vals = [pe14_7(float(v)) + " " for v in values]
    return ["".join(vals[i:i + 8]) for i in range(0, len(vals), 8)]


def write_restart(path, f: dict, scales: dict, lj: int, li: int, infuel: int = 11, isym: int = 1, iflow: int = 1,
                  iswrl: int = 1, ithrm: int = 1, ichem: int = 1, igrav: int = 0, itr: int = 1, dt: float = 1e-3,
                  bodies=None):
    """f: X, Y, RHO, U, V, W, P, QDOT, TK, STMF, STND [n] and FSP [52 or 51, n] (and AK, EPS if iflow == 2)."""
    n = lj * li
    iflame = 200000 + 52 * 100 + infuel + 400000 + (100000 if bodies else 0)
    lines = [f"{iflame:6d}--{TITLE}--",
             "".join(f"{v:6d}" for v in (li, lj, isym, iflow, iswrl, ithrm, ichem, igrav, 0, itr)) + f"{dt:12.10f}"]
    lines += _records([scales[k] for k in SCALES])
    if bodies:
        ints = [len(bodies)] + [c for b in bodies for c in b]
        # FORMAT(21I6): 21 integers per record, the list continues on further records
        lines += ["".join(f"{v:6d}" for v in ints[i:i + 21]) for i in range(0, len(ints), 21)]
    body = [f["X"], f["Y"], f["RHO"]] + [f["FSP"][k] for k in range(51)] + [f["U"], f["V"], f["W"], f["P"],
                                                                           f["QDOT"], f["TK"]]
    lines += _records(np.concatenate([np.asarray(a, dtype=np.float64).reshape(n) for a in body]))
    lines += _records(np.concatenate([np.asarray(f["STMF"]).reshape(n), np.asarray(f["STND"]).reshape(n)]))
    if iflow == 2:
        lines += _records(np.concatenate([np.asarray(f["AK"]).reshape(n), np.asarray(f["EPS"]).reshape(n)]))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def _parse_e(field: str) -> float:
    t = field.strip()
    if "E" not in t.upper():            # d.ddddddd+ddd
        k = max(t.rfind("+"), t.rfind("-"))
        t = t[:k] + "E" + t[k:]
    return float(t)


def read_restart(path) -> tuple[dict, dict]:
    """(header, fields) as READFF decodes them (readff.f:20-60)."""
    lines = open(path).read().splitlines()
    iflame = int(lines[0][:6])
    h = {"IFLAME": iflame}
    nsoot = iflame > 400000
    if nsoot:
        iflame -= 400000
    nswrl = iflame > 200000
    if nswrl:
        iflame -= 200000
    ints = [int(lines[1][6 * i:6 * i + 6]) for i in range(10 if nswrl else 9)]
    names = ["LI", "LJ", "ISYM", "IFLOW"] + (["ISWRL"] if nswrl else []) + ["ITHRM", "ICHEM", "IGRAV", "INERT", "ITR"]
    h.update(dict(zip(names, ints)))
    h["DT"] = float(lines[1][6 * len(ints):6 * len(ints) + 12])
    pos = 2

    def read_values(count):
        nonlocal pos
        out = []
        while len(out) < count:
            l = lines[pos]
            pos += 1
            out += [_parse_e(l[15 * i:15 * i + 14]) for i in range(min(8, (len(l) + 1) // 15))]
        return np.array(out[:count])

    sc = read_values(20)
    h["scales"] = dict(zip(SCALES, sc))
    if iflame >= 100000:
        iflame -= 100000
        # NBODY and the corners of each body under FORMAT(21I6): 21 per record
        nn = int(lines[pos][:6])
        ints = []
        while len(ints) < 1 + 4 * nn:
            l = lines[pos]
            pos += 1
            ints += [int(l[6 * i:6 * i + 6]) for i in range(min(21, len(l) // 6))]
        h["bodies"] = [ints[1 + 4 * b:5 + 4 * b] for b in range(nn)]
    lsp = iflame // 100
    h["INFUEL"] = iflame % 100
    n = h["LI"] * h["LJ"]
    data = read_values(n * (lsp + 7) + (n if nswrl else 0)).reshape(-1, n)
    names = ["X", "Y", "RHO"] + [f"FSP{k}" for k in range(lsp - 1)] + ["U", "V"] + (["W"] if nswrl else []) + \
            ["P", "QDOT", "TK"]
    f = {nm: data[i] for i, nm in enumerate(names)}
    f["FSP"] = np.vstack([f.pop(f"FSP{k}") for k in range(lsp - 1)] + [np.zeros(n)])
    f["FSP"][lsp - 1] = 1.0 - f["FSP"][:lsp - 1].sum(axis=0)
    if nsoot:
        s = read_values(2 * n).reshape(2, n)
        f["STMF"], f["STND"] = s[0], s[1]
    if h["IFLOW"] == 2:
        s = read_values(2 * n).reshape(2, n)
        f["AK"], f["EPS"] = s[0], s[1]
    return h, f
