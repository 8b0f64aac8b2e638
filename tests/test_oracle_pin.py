"""The CPU restatement (oracle/unichem_oracle.c) against the reference's own
routines (oracle/_ref: the reference Fortran translated to C), bit for bit."""
import numpy as np
import pytest

from conftest import random_state
from unicorn_b200.fields import jet_field, nondimensional


def test_setup_tables_bitwise(oracle, ref):
    for k, v in ref.scales.items():
        if k in oracle.scales:
            assert oracle.scales[k] == v, k
    assert np.array_equal(oracle.wm, ref.wm)
    assert np.array_equal(oracle.hfo, ref.hfo)


@pytest.mark.parametrize("seed,tlo,thi", [(0, 300, 2600), (1, 900, 1100), (2, 1500, 3000)])
def test_rates_omega_props_bitwise(oracle, ref, seed, tlo, thi):
    tk, rho, y = random_state(oracle, 700, seed, tlo, thi)
    rc_r, s_r = ref.ckrates(tk, rho, y)
    rc_o, s_o = oracle.rates(tk, rho, y)
    assert np.array_equal(rc_r, rc_o)
    assert np.array_equal(s_r, s_o)
    q_r, qd_r, h_r = ref.omega(tk, rho, y)
    q_o, qd_o, h_o, _ = oracle.omega(tk, rho, y)
    assert np.array_equal(q_r, q_o) and np.array_equal(qd_r, qd_o) and np.array_equal(h_r, h_o)
    assert np.array_equal(ref.cp(tk, y), oracle.cp(tk, y))
    yc_r, mu_r, la_r, d_r = ref.props(tk, y)
    yc_o, mu_o, la_o, d_o, _ = oracle.props(tk, y)
    for a, b in ((yc_r, yc_o), (mu_r, mu_o), (la_r, la_o), (d_r, d_o)):
        assert np.array_equal(a, b)


def test_soot_and_negative_inputs_bitwise(oracle, ref):
    """Soot sources with non-zero soot, and negative mass fractions (clipped by the property block)."""
    tk, rho, y = random_state(oracle, 300, 7)
    rng = np.random.default_rng(7)
    stmf = rng.uniform(0, 1e-4, 300)
    stnd = 10 ** rng.uniform(-1, 12, 300)
    rc_r, s_r = ref.ckrates(tk, rho, y, stmf, stnd)
    rc_o, s_o = oracle.rates(tk, rho, y, stmf, stnd)
    assert np.array_equal(rc_r, rc_o) and np.array_equal(s_r, s_o)
    y2 = y.copy()
    y2[3, ::3] = -1e-6
    assert all(np.array_equal(a, b) for a, b in zip(ref.props(tk, y2), oracle.props(tk, y2)[:4]))


@pytest.mark.parametrize("isor,tol", [(1, 1e-8), (4, 0.0), (100, 1e-8)])
def test_species_update_bitwise(oracle, ref, isor, tol):
    f = jet_field(40, 50, fuel=11, t_peak=2300.0, seed=3)      # 2000 cells: one reference chunk
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    y = f.y
    yr, s1, s2, pr = ref.species_update(tk, rho, y, 1e-3, isor=isor, relx=0.99, tol=tol)
    rc, sour = oracle.rates(tk, rho, y)
    yo, so, po = oracle.species_update(rho, y, rc, sour, 1e-3, isor=isor, tol=tol, spnorm=float(ref.LE * 51))
    assert pr == po
    assert np.array_equal(yr, yo)
    assert np.array_equal(s1, so[0]) and np.array_equal(s2, so[1])


def test_temperature_bitwise(oracle, ref):
    from unicorn_b200.fields import sensible_enthalpy
    tk, rho, y = random_state(oracle, 900, 11, 300, 2900)
    T = tk * oracle.scales["TSTR"]
    ht = sensible_enthalpy(T, y, np.array(oracle.mech["poly"]), oracle.wm, oracle.hfo, oracle.scales)
    guess = np.random.default_rng(1).uniform(300, 2500, 900) / oracle.scales["TSTR"]
    t_r = ref.temperature(guess, y, ht)
    t_o = oracle.temperature(guess, y, ht)
    assert np.array_equal(t_r, t_o)
    assert np.abs(t_o * oracle.scales["TSTR"] - T).max() < 2e-3


@pytest.mark.parametrize("isor,tol", [(3, 0.0), (100, 1e-8)])
def test_iskip_bitwise(oracle, ref, isor, tol):
    """ISKIP (lib/skipdf.f: 3 injection cells, 10 and 11 body cells; 1 and 2 skip nothing here) in
    CKRATES (ckrates.f:94), SOLVEH's rates (solveh.f:119) and SOLVESP (solvesp.f:89,2842), starting
    from the zero arrays of a fresh run: the oracle's wrappers give the translated reference's
    results bit for bit, and skipped cells keep their state."""
    f = jet_field(40, 50, fuel=11, t_peak=2300.0, seed=3)      # 2000 cells: one reference chunk
    tk, rho = nondimensional(f, oracle.scales, oracle.wm)
    y = f.y
    iskip = np.zeros(f.n, dtype=np.int32)
    iskip[100:180] = 3
    iskip[500:520] = 10
    iskip[900:905] = 11
    iskip[1200:1210] = 1
    iskip[1300:1310] = 2
    rc_r, s_r = ref.ckrates(tk, rho, y, iskip=iskip)
    rc_o, s_o = oracle.rates_iskip(tk, rho, y, iskip)
    assert np.array_equal(rc_r, rc_o) and np.array_equal(s_r, s_o)
    assert not rc_o[:, 100:180].any() and rc_o[:, 1200:1210].any()
    q_r, qd_r, _ = ref.omega(tk, rho, y, iskip=iskip)
    q_o, qd_o, _, _ = oracle.omega_iskip(tk, rho, y, iskip)
    assert np.array_equal(q_r, q_o) and np.array_equal(qd_r, qd_o)
    yr, s1, s2, pr = ref.species_update(tk, rho, y, 1e-3, isor=isor, relx=0.99, tol=tol, iskip=iskip)
    yo, so, po = oracle.species_update_iskip(rho, y, rc_o, s_o, 1e-3, iskip, isor=isor, tol=tol,
                                             spnorm=float(ref.LE * 51))
    assert pr == po
    assert np.array_equal(yr, yo)
    assert np.array_equal(s1, so[0]) and np.array_equal(s2, so[1])
    skipped = iskip >= 3
    assert np.array_equal(yo[:, skipped], y[:, skipped])
