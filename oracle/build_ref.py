"""Recipe: build the reference's own chemistry routines as a C shared library.

ORACLE INFRASTRUCTURE (test-only). There is no Fortran compiler in this
image, so the reference Fortran is translated mechanically to C by
``oracle/f77_to_c.py`` from the files where they lie under the reference
checkout and compiled with gcc. Output goes to ``oracle/_ref/`` only
(git-ignored; it travels with the repository snapshot to the GPU host, where
no reference checkout exists).

Translated pieces (reference paths relative to the UNICORN checkout):

* ``src/lib/DATA.f``            BLOCK DATA THERMO (all)          -> f77_blockdata
* ``src/lib/ckrates.f``         SUBROUTINE CKRATES (all)         -> f77_ckrates
* ``src/lib/solvesp.f``         SUBROUTINE SOLVESP (all)         -> f77_solvesp
* ``src/lib/solveh.f:34-57,116-1145``  h_k, RA, PRD, QDSP, QDOT  -> f77_solveh_omega
* ``src/lib/solveh.f:34-38,1170-1234`` T from h by Newton        -> f77_solveh_temperature
* ``src/lib/spgsolv.f:98-232``  mixture cp (TCP probed per cell) -> f77_spgsolv_cp
* ``src/lib/spgsolv.f:98-1290`` cp, EKT/EMU, face conductances and the
  E/W/N/S coefficients of the species equations    -> f77_spgsolv_coef
* ``src/lib/stdata.f:26-118``   regular-grid fields, cp and h_k of FDETAIL -> f77_stdata_rg
* ``src/lib/solveh.f:34-1145``  enthalpy-equation right-hand side (species
  enthalpy diffusion, radiation, heat release)     -> f77_solveh_rhs
* ``src/lib/solveh.f:34-1234``  the whole of SOLVEH: right-hand side, point
  relaxation of FPZ and the temperature from it   -> f77_solveh_full
* ``src/unicornd-mild-sd-5.f:1056-1068`` density from the gas law at PBACK -> f77_main_density
* ``src/unicornd-mild-sd-5.f:84-113`` DATA WSP/CDIA/TLJ/CI11      -> f77_main_data
* ``src/unicornd-mild-sd-5.f:327-483`` set-up of tables/scales    -> f77_main_setup
* ``src/unicornd-mild-sd-5.f:821-1006`` Y clip + transport props   -> f77_main_props

The grid size is a compile-time PARAMETER in the reference (LI=711, LJ=131,
``src/unicornd-mild-sd-5.f:3``); the recipe overrides it (default LJ=34,
LI=66: a 32x64 = 2048-cell interior) and the driver in ``oracle/ref.py``
processes larger fields in chunks of that size.

Usage: python oracle/build_ref.py [--ref <reference checkout>] [--lj 34 --li 66]
(default: $UNICORN_REF, else ``reference`` beside this repository)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))

from unicorn_b200.fortran.parser import build_units  # noqa: E402
from f77_to_c import translate  # noqa: E402

OUT = HERE / "_ref"


def build(ref: str, lj: int, li: int, out: Path = OUT) -> Path:
    src = Path(ref) / "src"
    ov = {"LJ": lj, "LI": li}
    ov_main = dict(ov)
    # main computes derived PARAMETERs from LI/LJ; keep them consistent
    data = build_units(str(src / "lib/DATA.f"), ov)[0]
    ckr = build_units(str(src / "lib/ckrates.f"), ov)[0]
    ssp = build_units(str(src / "lib/solvesp.f"), ov)[0]
    sh = build_units(str(src / "lib/solveh.f"), ov)[0]
    spg = build_units(str(src / "lib/spgsolv.f"), ov)[0]
    std = build_units(str(src / "lib/stdata.f"), ov)[0]
    main = [u for u in build_units(str(src / "unicornd-mild-sd-5.f"), ov_main) if u.kind == "program"][0]
    ncell = lj * li
    probe_cp = {173: f"F77P_TCP[(L_I-1)*{lj} + (L_J-1)] = L_TCP;"}
    frags = [
        (data, "f77_blockdata", "data", None, None),
        (main, "f77_main_data", "data", "MAIN_", None),
        (main, "f77_main_setup", [(327, 483)], "MAIN_", None),
        (main, "f77_main_props", [(821, 1006)], "MAIN_", None),
        (ckr, "f77_ckrates", None, None, None),
        (ssp, "f77_solvesp", None, None, None),
        (sh, "f77_solveh_omega", [(34, 57), (116, 1145)], None, None),
        (sh, "f77_solveh_temperature", [(34, 38), (1170, 1234)], None, None),
        (spg, "f77_spgsolv_cp", [(98, 232)], None, probe_cp),
        (spg, "f77_spgsolv_coef", [(98, 1290)], None, None),
        (std, "f77_stdata_rg", [(26, 118)], None, None),
        (sh, "f77_solveh_rhs", [(34, 1145)], None, None),
        (sh, "f77_solveh_full", [(34, 1234)], None, None),
        (main, "f77_main_density", [(1056, 1068)], "MAIN_", None),
    ]
    code = translate(frags, [data, ckr, ssp, sh, spg, std, main])
    code = code.replace("#include <string.h>", f"#include <string.h>\ndouble F77P_TCP[{ncell}];", 1)
    out.mkdir(parents=True, exist_ok=True)
    cfile = out / "unicorn_ref.c"
    cfile.write_text(code)
    # layout of COMMON variables (main program's view) and main locals for the driver
    layout = {"LJ": lj, "LI": li, "units": {}, "main_locals": {}, "args": {}}
    for u in (main, ckr, ssp, sh, spg, std, data):
        layout["units"][u.name] = {
            name: {"block": v.common, "offset": v.offset, "type": v.type, "dims": v.dims}
            for name, v in u.vars.items() if v.common}
        layout["args"][u.name] = {a: u.vars[a].type for a in u.args}
    import re
    for name in sorted(set(re.findall(r"\bMAIN_([A-Z0-9_]+)", code))):
        v = main.vars.get(name)
        ty = v.type if v is not None else main.type_of_name(name)
        if ty != "char":
            layout["main_locals"][name] = {"type": ty, "dims": v.dims if v is not None else None}
    (out / "layout.json").write_text(json.dumps(layout, indent=1))
    so = out / "libunicorn_ref.so"
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-w", "-o", str(so), str(cfile), "-lm"]
    subprocess.run(cmd, check=True)
    return so


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    from unicorn_b200.refsrc import reference_root
    ap.add_argument("--ref", default=str(reference_root()))
    ap.add_argument("--lj", type=int, default=34)
    ap.add_argument("--li", type=int, default=66)
    a = ap.parse_args()
    print(build(a.ref, a.lj, a.li))
