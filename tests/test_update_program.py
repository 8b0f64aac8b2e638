"""The generated species-update program (unicorn_b200/csrc/generated/
update_program.cuh) against the oracle, on the host: compiles
tests/update_program_harness.cpp with g++ (no FMA contraction). The program
keeps the reference's operation order, so it must match the oracle bit for
bit -- this checks the symbolic resolution of the reference's A-terms.
The soot sources are zero here (the soot equations live outside the program)."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import random_state

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    so = tmp_path_factory.mktemp("h") / "harness.so"
    subprocess.run(["g++", "-O1", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(so),
                    str(ROOT / "tests" / "update_program_harness.cpp")], check=True)
    return ctypes.CDLL(str(so))


def _closure(y):
    y = y.copy()
    for c in range(y.shape[1]):
        ft = y[0, c]
        for k in range(1, 51):
            ft = ft + y[k, c]
        n2 = 1.0 - ft
        if ft > 1.0:
            y[:51, c] = y[:51, c] / ft
            n2 = 0.0
        y[51, c] = n2
    return y


@pytest.mark.parametrize("isor", [1, 3])
def test_generated_programs_match_oracle(oracle, harness, isor):
    tk, rho, y = random_state(oracle, 300, 21)
    rc, sour = oracle.rates(tk, rho, y)
    sour[:] = 0.0
    P = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    yo, _, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=isor)
    args = lambda yy: (len(tk), P(rho), P(y), P(yy), P(rc), P(sour), P(oracle.wm), ctypes.c_double(1e-3), isor,
                       ctypes.c_double(0.99), ctypes.c_double(1e-8), ctypes.c_double(len(tk) * 51.0))
    y1 = np.ascontiguousarray(y.copy())
    p1 = harness.harness_update(*args(y1))
    assert p1 == po and np.array_equal(_closure(y1), yo)


@pytest.mark.parametrize("isor", [1, 3])
def test_inplace_program_equals_two_set_program(oracle, harness, isor):
    """The in-place form of the program (one Y array, eight species read at their start-of-pass
    value from the cell's Y row) gives bit for bit what the two-array form gives."""
    tk, rho, y = random_state(oracle, 300, 22)
    rc, sour = oracle.rates(tk, rho, y)
    sour[:] = 0.0
    P = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    args = lambda yy: (len(tk), P(rho), P(y), P(yy), P(rc), P(sour), P(oracle.wm), ctypes.c_double(1e-3), isor,
                       ctypes.c_double(0.99), ctypes.c_double(1e-8), ctypes.c_double(len(tk) * 51.0))
    y1, y2 = np.ascontiguousarray(y.copy()), np.ascontiguousarray(y.copy())
    p1 = harness.harness_update(*args(y1))
    p2 = harness.harness_update_ip(*args(y2))
    assert p1 == p2 and np.array_equal(y1, y2)
    assert np.abs(y1 - y).max() > 1e-8            # the update moved Y


@pytest.mark.parametrize("isor", [1, 3])
def test_tile_resident_program_equals_two_set_program(oracle, harness, isor):
    """The tile-resident form (RC rows split between shared and tensor memory, tensor-memory
    operands loaded into two register banks segment by segment) gives bit for bit what the
    two-array form gives."""
    tk, rho, y = random_state(oracle, 300, 23)
    rc, sour = oracle.rates(tk, rho, y)
    sour[:] = 0.0
    P = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    args = lambda yy: (len(tk), P(rho), P(y), P(yy), P(rc), P(sour), P(oracle.wm), ctypes.c_double(1e-3), isor,
                       ctypes.c_double(0.99), ctypes.c_double(1e-8), ctypes.c_double(len(tk) * 51.0))
    y1, y2 = np.ascontiguousarray(y.copy()), np.ascontiguousarray(y.copy())
    p1 = harness.harness_update(*args(y1))
    p2 = harness.harness_update_tr(*args(y2))
    assert p1 == p2 and np.array_equal(y1, y2)
