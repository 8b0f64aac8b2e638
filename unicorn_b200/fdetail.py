"""The FDETAIL file of the reference (SUBROUTINE STDATA, src/lib/stdata.f:120-175)
written from the fields that uc_fdetail computes on the device.

Layout: a line ' ITR TTIME' (FORMAT 1X,I6,F15.10), the Tecplot variable line
(FORMAT 105), then one record per grid point, I outer and J inner,
'I,J,' followed by 218 values in E15.7E3 separated by commas (FORMAT 104).
The variable line keeps the reference's spelling: "x-CH2CO" in the Y and h
groups, and no comma between the D, QDSP and h groups.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

MECH = Path(__file__).resolve().parent / "mech" / "sandiego52.json"


def variables_line(species: list[str]) -> str:
    def group(prefix, quirk):
        out = []
        for s in species:
            p = "x" if (quirk and s == "CH2CO") else prefix
            out.append(f'"{p}-{s}"')
        return ",".join(out)
    head = '"i","j","z","r","RHO","v","u","T","QDOT","VMU","VTC","CP",'
    return ("VARIABLES=" + head + group("Y", True) + "," + group("VDF", False) + group("PRD", False) +
            group("H", True))


def e15_7e3(v: float) -> str:
    """Fortran E15.7E3: [-]0.dddddddE+ddd, right-aligned in 15 columns."""
    if v == 0.0 or not np.isfinite(v):
        body = "0.0000000E+000" if v == 0.0 else "***************"[:14]
        return body.rjust(15)
    s = f"{abs(v):.6e}"                      # d.dddddde+XX, correctly rounded to 7 digits
    mant, ex = s.split("e")
    digits = mant.replace(".", "")
    e = int(ex) + 1
    body = f"0.{digits}E{'+' if e >= 0 else '-'}{abs(e):03d}"
    return ("-" + body if v < 0 else body).rjust(15)


def write_fdetail(path, fields: np.ndarray, lj: int, li: int, itr: int = 0, ttime: float = 0.0,
                  species: list[str] | None = None):
    """fields [218, lj*li] from UniChem.fdetail (J fastest)."""
    if species is None:
        species = json.loads(MECH.read_text())["species"]
    with open(path, "w") as fh:
        fh.write(f" {itr:6d}{ttime:15.10f}\n")
        fh.write(variables_line(species) + "\n")
        for i in range(li):
            for j in range(lj):
                c = i * lj + j
                vals = ",".join(e15_7e3(float(x)) for x in fields[:, c])
                fh.write(f"{i + 1:4d},{j + 1:4d},{vals}\n")


def read_fdetail(path):
    """(itr, ttime, variables line, fields [218, n]) of an FDETAIL file."""
    lines = Path(path).read_text().splitlines()
    itr, ttime = int(lines[0][1:7]), float(lines[0][7:22])
    recs = [l.split(",") for l in lines[2:]]
    data = np.array([[float(x.replace("E", "e")) for x in r[2:]] for r in recs]).T
    return itr, ttime, lines[1], data
