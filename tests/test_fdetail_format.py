"""The FDETAIL writer (unicorn_b200/fdetail.py): the Fortran edit descriptors
of stdata.f:120-175 and the variable line of its FORMAT 105."""
import re
from pathlib import Path

import numpy as np
import pytest

from unicorn_b200.fdetail import e15_7e3, read_fdetail, variables_line, write_fdetail
from unicorn_b200.refsrc import reference_root

REF = reference_root()


@pytest.mark.parametrize("v,s", [(0.0, " 0.0000000E+000"), (1.0, " 0.1000000E+001"), (-123.4567, "-0.1234567E+003"),
                                 (2.5e-310, " 0.2500000E-309"), (9.99999996e-5, " 0.1000000E-003"),
                                 (6.02e23, " 0.6020000E+024")])
def test_e15_7e3(v, s):
    assert e15_7e3(v) == s and len(s) == 15


def test_variables_line_is_the_references():
    src = REF / "src" / "lib" / "stdata.f"
    if not src.exists():
        pytest.skip("reference sources not present")
    lines = src.read_text().splitlines()
    start = next(i for i, l in enumerate(lines) if re.match(r"\s*105\s+FORMAT", l))
    stop = next(i for i in range(start, len(lines)) if lines[i].strip() == "RETURN")
    ref = "".join(re.findall(r"'([^']*)'", "\n".join(lines[start:stop])))
    import json
    from unicorn_b200.fdetail import MECH
    assert variables_line(json.loads(MECH.read_text())["species"]) == ref


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    lj, li = 5, 4
    f = rng.standard_normal((218, lj * li)) * 10.0 ** rng.integers(-30, 30, (218, lj * li))
    p = tmp_path / "FDETAIL"
    write_fdetail(p, f, lj, li, itr=12, ttime=0.0125)
    itr, t, var, g = read_fdetail(p)
    assert itr == 12 and abs(t - 0.0125) < 1e-12 and var.startswith("VARIABLES=")
    assert np.allclose(g, f, rtol=5.1e-7, atol=0)          # 7 digits of a 0.d mantissa
    first = p.read_text().splitlines()[2]
    assert first.startswith("   1,   1,") and len(first) == 10 + 218 * 16 - 1
