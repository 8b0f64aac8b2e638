"""Generate the golden fixtures of this directory from the reference's own
routines (``oracle/_ref``: the reference Fortran translated to C and compiled
from the sources by ``oracle/build_ref.py``).

Run in a checkout that has the reference sources next to it:

    python tests/golden/make_golden.py [--ref-src DIR]

Each fixture is a compressed ``.npz`` of inputs and the reference's outputs,
non-dimensional in the reference's own units:

  rates_omega.npz   48 cells, 300..2600 K, with soot: RC[544], SOUR[6],
                    QDSP[52], QDOT, HENTH[52] (lib/ckrates.f, lib/solveh.f)
  cp_props.npz      48 cells with some negative minors: TCP
                    (lib/spgsolv.f:102-173), clipped Y, VMU, VTC, VDFSP
                    (main program 821-1006)
  update.npz        a 12x16 heptane jet slice: SOLVESP with 4 passes and tol 0,
                    and with 100 passes and tol 1e-8 (pass count included)
  temperature.npz   64 cells: T from the sensible enthalpy by Newton
                    (lib/solveh.f:1170-1234)
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
from unicorn_b200.refsrc import reference_root  # noqa: E402


def states(scales, wm, n, seed, tlo, thi):
    rng = np.random.default_rng(seed)
    y = 10 ** rng.uniform(-10, -3, (52, n))
    y[1] = rng.uniform(0.05, 0.23, n)
    y[51] = 0.7
    y[12] = rng.uniform(0.0, 0.1, n)
    y[46] = rng.uniform(0.0, 0.05, n)
    y /= y.sum(0)
    T = rng.uniform(tlo, thi, n)
    tk = T / scales["TSTR"]
    rho = scales["PBACK"] / (scales["BETA1"] * tk * (y / wm[:, None]).sum(0))
    return tk, rho, y


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-src", default=str(reference_root()))
    args = ap.parse_args()
    from oracle import ref as R
    if not R.available():
        from oracle.build_ref import build
        build(args.ref_src, 34, 66)
    ref = R.RefUnicorn()
    from unicorn_b200.fields import jet_field, nondimensional, sensible_enthalpy
    from oracle.oracle import Oracle
    sc, wm = ref.scales, ref.wm

    tk, rho, y = states(sc, wm, 48, 101, 300.0, 2600.0)
    rng = np.random.default_rng(101)
    stmf = np.where(np.arange(48) % 3 == 0, rng.uniform(0, 1e-4, 48), 0.0)
    stnd = np.where(np.arange(48) % 3 == 0, 10 ** rng.uniform(-1, 12, 48), 0.0)
    rc, sour = ref.ckrates(tk, rho, y, stmf, stnd)
    qdsp, qdot, henth = ref.omega(tk, rho, y, stmf, stnd)
    np.savez_compressed(HERE / "rates_omega.npz", tk=tk, rho=rho, y=y, stmf=stmf, stnd=stnd,
                        rc=rc, sour=sour, qdsp=qdsp, qdot=qdot, henth=henth)

    tk, rho, y = states(sc, wm, 48, 102, 300.0, 3000.0)
    y[3, ::4] = -1e-6
    tcp = ref.cp(tk, y)
    yc, vmu, vtc, vdf = ref.props(tk, y)
    np.savez_compressed(HERE / "cp_props.npz", tk=tk, y=y, tcp=tcp, yc=yc, vmu=vmu, vtc=vtc, vdf=vdf)

    f = jet_field(12, 16, fuel=11, t_peak=2300.0, seed=4)
    tk, rho = nondimensional(f, sc, wm)
    out = dict(tk=tk, rho=rho, y=f.y, dt=1e-3, relx=0.99, spnorm=float(ref.LE * 51))
    for isor, tol, tag in ((4, 0.0, "a"), (100, 1e-8, "b")):
        yn, s1, s2, passes = ref.species_update(tk, rho, f.y, 1e-3, isor=isor, relx=0.99, tol=tol)
        out.update({f"isor_{tag}": isor, f"tol_{tag}": tol, f"y_{tag}": yn, f"stmf_{tag}": s1,
                    f"stnd_{tag}": s2, f"passes_{tag}": passes})
    np.savez_compressed(HERE / "update.npz", **out)

    tk, rho, y = states(sc, wm, 64, 103, 300.0, 2900.0)
    T = tk * sc["TSTR"]
    poly = np.array(Oracle().mech["poly"])
    ht = sensible_enthalpy(T, y, poly, wm, ref.hfo, sc)
    guess = np.random.default_rng(103).uniform(300, 2500, 64) / sc["TSTR"]
    np.savez_compressed(HERE / "temperature.npz", guess=guess, y=y, ht=ht, tk=ref.temperature(guess, y, ht))
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
