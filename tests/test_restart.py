"""Restart files in the layout of the reference's PRNTDK / READFF
(unicorn_b200/restart.py): edit descriptors, record structure, round trip."""
import numpy as np
import pytest

from unicorn_b200.restart import pe14_7, read_restart, write_restart, SCALES


@pytest.mark.parametrize("v,s", [(0.0, " 0.0000000E+00"), (1.0, " 1.0000000E+00"), (-123.45678912, "-1.2345679E+02"),
                                 (1e-120, " 1.0000000-120"), (6.02e23, " 6.0200000E+23")])
def test_pe14_7(v, s):
    assert pe14_7(v) == s and len(s) == 14


def sample(lj, li, seed=0):
    rng = np.random.default_rng(seed)
    n = lj * li
    f = {k: rng.standard_normal(n) * 10.0 ** rng.integers(-20, 20, n) for k in
         ("X", "Y", "RHO", "U", "V", "W", "P", "QDOT", "TK", "STMF", "STND", "AK", "EPS")}
    y = 10 ** rng.uniform(-12, -1, (52, n))
    y[51] = 0.0
    y[51] = 1.0 - y[:51].sum(axis=0)
    f["FSP"] = y
    return f


@pytest.mark.parametrize("iflow,bodies", [(1, None), (2, [[3, 4, 6, 8]]),
                                          (1, [[b + 1, b + 2, b + 3, b + 4] for b in range(7)])])
def test_round_trip(tmp_path, iflow, bodies):
    lj, li = 7, 5
    f = sample(lj, li)
    sc = {k: float(i + 1) * 0.37 for i, k in enumerate(SCALES)}
    p = tmp_path / "FLAME.DATA"
    write_restart(p, f, sc, lj, li, infuel=11, iflow=iflow, itr=42, dt=1e-3, bodies=bodies)
    h, g = read_restart(p)
    assert h["IFLAME"] == 605211 + (100000 if bodies else 0)
    assert (h["LI"], h["LJ"], h["ITR"], h["INFUEL"], h["IFLOW"]) == (li, lj, 42, 11, iflow)
    assert abs(h["DT"] - 1e-3) < 1e-15
    assert all(abs(h["scales"][k] - sc[k]) <= 5e-8 * abs(sc[k]) for k in SCALES)
    for k in ("X", "Y", "RHO", "U", "V", "W", "P", "QDOT", "TK", "STMF", "STND") + (("AK", "EPS") if iflow == 2 else ()):
        assert np.allclose(g[k], f[k], rtol=5.1e-8, atol=0), k
    assert np.allclose(g["FSP"][:51], f["FSP"][:51], rtol=5.1e-8, atol=0)
    assert np.allclose(g["FSP"][51], f["FSP"][51], rtol=0, atol=5e-8)     # closed from the 51 8-digit values
    if bodies:
        assert h["bodies"] == bodies
    lines = p.read_text().splitlines()
    assert lines[0].startswith("605211--FLAME DATA") if not bodies else lines[0].startswith("705211--")
    assert len(lines[1]) == 72 and all(len(l) == 120 for l in lines[2:4])
